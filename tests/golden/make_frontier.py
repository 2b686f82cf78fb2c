#!/usr/bin/env python3
"""Frontier fixtures: eight 5e9-wide blocks spread over the reference's two raw evidence
archives (exhaustive/evidence/exhaustive-2026-09-18.tar.gz and -09-19.tar.gz, S ~ 1.95e12 to
3.5e12) -- their sorted-output sha256, M lines and TOTAL counters -- into frontier.json.

    python tests/golden/make_frontier.py REFERENCE_TREE
"""
from __future__ import annotations

import json
import re
import sys
import tarfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import parse_stderr, sha  # noqa: E402


def main() -> int:
    if len(sys.argv) != 2:
        print(__doc__, file=sys.stderr)
        return 2
    ref = Path(sys.argv[1])
    blocks = []
    for arch, picks in (("exhaustive-2026-09-18", (40, 80, 120, 155)), ("exhaustive-2026-09-19", (1, 60, 110, 159))):
        with tarfile.open(ref / "exhaustive" / "evidence" / f"{arch}.tar.gz") as tar:
            for k in picks:
                name = f"{arch}/block-{k:04d}"
                err = tar.extractfile(name + ".err").read().decode()
                out = tar.extractfile(name + ".out").read().decode().splitlines(keepends=True)
                hdr = re.search(r"s4: S in \[(\d+),\s*(\d+)\)", err)
                blocks.append({"block": name, "lo": int(hdr.group(1)), "hi": int(hdr.group(2)), "sha256": sha(out),
                               "n_lines": len(out), "m_lines": sorted(x for x in out if x.startswith("M:")),
                               **{kk: v for kk, v in parse_stderr(err).items() if kk != "hist5"}})
    (HERE / "frontier.json").write_text(json.dumps(blocks, indent=1, sort_keys=True) + "\n")
    print("wrote", HERE / "frontier.json", len(blocks), "blocks")
    return 0


if __name__ == "__main__":
    sys.exit(main())
