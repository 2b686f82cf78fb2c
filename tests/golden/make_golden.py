#!/usr/bin/env python3
"""Regenerate the golden fixtures in tests/golden/ from the reference engine itself.

Runs oracle/_ref/s4 -- the reference's exhaustive/s4.c compiled unmodified by
`make -C oracle ref` -- and reads the reference's own logs and unit-test vectors from the
reference tree.  Needs the reference tree (--ref); the fixtures it writes
are committed, so the tests never need the reference at run time.

    python tests/golden/make_golden.py --ref REFERENCE_TREE [--reuse DIR] [--skip-1e10]

--reuse DIR takes s4_1e9.{out,err} / s4_1e10.{out,err} already produced by
`s4 1 1000000000 8 20` / `s4 1 10000000000 8 20` in DIR instead of re-running them
(the 1e10 run takes about four minutes on eight cores).
"""
from __future__ import annotations

import argparse
import gzip
import hashlib
import json
import random
import re
import subprocess
import sys
import tarfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
S4 = REPO / "oracle" / "_ref" / "s4"

TOTAL_RE = re.compile(r"^TOTAL: (.*)$", re.M)
CAP_RE = re.compile(r"^CAPACITY: reps=(\d+)/\d+ divisors=(\d+)/\d+ extensions=(\d+)/\d+", re.M)
HIST_RE = re.compile(r"^5-sets by log2\(largest element\)[^:]*:(.*)$", re.M)
KEYMAP = {"S_done": "S_done", "pairs": "pairs", "S_ge3": "S_ge3", "triples": "triples", "4-sets": "sets4",
          "5-sets": "sets5", "6-sets": "sets6", "multi-ext-4sets": "multi", "ext_cand": "ext_cand",
          "ext_sqrt": "ext_sqrt"}


def parse_stderr(text: str) -> dict:
    tot = TOTAL_RE.search(text).group(1)
    d = {KEYMAP[k]: int(v) for k, v in re.findall(r"([\w-]+)=(\d+)", tot) if k in KEYMAP}
    h = HIST_RE.search(text)
    d["hist5"] = {int(a): int(b) for a, b in re.findall(r"(\d+):(\d+)", h.group(1))} if h else {}
    c = CAP_RE.search(text)
    if c:
        d["max_reps"], d["max_divisors"], d["max_extensions"] = map(int, c.groups())
    return d


def sha(lines) -> str:
    return hashlib.sha256("".join(sorted(lines)).encode()).hexdigest()


def run_s4(lo: int, hi: int, threads: int = 1, extra=()):
    p = subprocess.run([str(S4), str(lo), str(hi), str(threads), "20", *extra], capture_output=True, text=True,
                       check=True)
    return p.stdout.splitlines(keepends=True), p.stderr


def random_subranges(seed: int, n: int):
    """Seeded subranges: widths log-uniform in [1e3, 1e6], offsets uniform up to 1e11 (plus a few
    up to 1e12), the shapes of the batched and serving workloads at test scale."""
    rng = random.Random(seed)
    out = []
    for i in range(n):
        width = int(10 ** rng.uniform(3, 6))
        top = 10 ** 12 if i % 8 == 7 else 10 ** 11
        lo = rng.randint(1, top)
        out.append((lo, lo + width))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference source tree")
    ap.add_argument("--reuse", default=None)
    ap.add_argument("--skip-1e10", action="store_true")
    args = ap.parse_args()
    ref = Path(args.ref)
    if not S4.exists():
        subprocess.run(["make", "-C", str(REPO / "oracle"), "ref", f"REF_DIR={ref}"], check=True)
    golden = {"source": "oracle/_ref/s4 (reference exhaustive/s4.c, unmodified); reference logs and tests",
              "runs": {}}

    # [1,1e7): full sorted output (the README's small validation run, README.md:156-159)
    lines, err = run_s4(1, 10 ** 7, 4, ["--verify"])
    (HERE / "s4_1e7.sorted.txt").write_text("".join(sorted(lines)))
    golden["runs"]["1e7"] = {"lo": 1, "hi": 10 ** 7, "sha256": sha(lines), "n_lines": len(lines), **parse_stderr(err)}
    # --dump4: every 4-set below 1e7 (4-set enumeration parity); only hash + count committed
    lines, err = run_s4(1, 10 ** 7, 1, ["--dump4", "100000000", "--noext"])
    quads = [x for x in lines if x.startswith("4:")]
    golden["runs"]["dump4_1e7"] = {"lo": 1, "hi": 10 ** 7, "sha256": sha(quads), "n_lines": len(quads),
                                   **parse_stderr(err)}
    # a small dump4 slice kept verbatim (first 2000 4-sets below 1e7, reference order)
    lines, _ = run_s4(1, 10 ** 7, 1, ["--dump4", "2000", "--noext"])
    (HERE / "dump4_first2000.txt").write_text("".join(x for x in lines if x.startswith("4:")))

    # [1,1e9) and [1,1e10): hashes, counters, all M lines; 1e9 output kept gzipped
    for tag, hi in (("1e9", 10 ** 9), ("1e10", 10 ** 10)):
        if tag == "1e10" and args.skip_1e10:
            continue
        if args.reuse and (Path(args.reuse) / f"s4_{tag}.out").exists():
            lines = (Path(args.reuse) / f"s4_{tag}.out").read_text().splitlines(keepends=True)
            err = (Path(args.reuse) / f"s4_{tag}.err").read_text()
        else:
            lines, err = run_s4(1, hi, 8)
        golden["runs"][tag] = {"lo": 1, "hi": hi, "sha256": sha(lines), "n_lines": len(lines), **parse_stderr(err)}
        (HERE / f"m_lines_{tag}.txt").write_text("".join(sorted(x for x in lines if x.startswith("M:"))))
        if tag == "1e9":
            with gzip.open(HERE / "s4_1e9.sorted.txt.gz", "wt") as f:
                f.write("".join(sorted(lines)))

    # singleton S known answers: exhaustive/test_verify.py:13 and :31-32,
    # bruteforce-scratchpad/dotnet/test1.txt, and the boundary repairs logs/boundary_{1..9}.err
    singles = {}
    for S in [362141, 885125, 50578642000] + [k * 10 ** 11 for k in range(1, 10)]:
        lines, err = run_s4(S, S + 1, 1, ["--verify"])
        singles[str(S)] = {"lines": lines, **parse_stderr(err)}
    golden["singletons"] = singles
    boundary = {}
    for k in range(1, 10):
        text = (ref / "exhaustive" / "logs" / f"boundary_{k}.err").read_text()
        boundary[str(k * 10 ** 11)] = {kk: v for kk, v in parse_stderr(text).items() if kk != "hist5"}
    golden["boundary_logs"] = boundary
    # the valid records of exhaustive/test_verify.py: the known five-set (:13) and the
    # three-extension M record (:31-32); the deliberately broken lines of :20-21 are skipped
    tv = (ref / "exhaustive" / "test_verify.py").read_text()
    joined, cur = [], ""
    for lit in re.findall(r"b'([^']*)'", tv):
        cur += lit
        if cur.endswith("\\n"):
            joined.append(cur[:-2])
            cur = ""
    fives = [x for x in joined if x.startswith("5:")]
    golden["test_verify_lines"] = fives[:1] + [x for x in joined if x.startswith("M:")]

    # seeded random subranges (batched / serving workload shapes at test scale)
    subs = []
    for lo, hi in random_subranges(20261203, 48):
        lines, err = run_s4(lo, hi, 1)
        subs.append({"lo": lo, "hi": hi, "lines": sorted(lines), **parse_stderr(err)})
    golden["subranges"] = subs

    # frontier blocks from the reference's archived raw evidence (two 5e9-wide blocks at S~2e12)
    tb = ref / "exhaustive" / "evidence" / "exhaustive-2026-09-18.tar.gz"
    frontier = []
    if tb.exists():
        with tarfile.open(tb) as tar:
            for name in ("exhaustive-2026-09-18/block-0001", "exhaustive-2026-09-18/block-0002"):
                err = tar.extractfile(name + ".err").read().decode()
                out = tar.extractfile(name + ".out").read().decode().splitlines(keepends=True)
                hdr = re.search(r"s4: S in \[(\d+),\s*(\d+)\)", err)
                frontier.append({"block": name, "lo": int(hdr.group(1)), "hi": int(hdr.group(2)),
                                 "sha256": sha(out), "n_lines": len(out), "m_lines": sorted(x for x in out if x.startswith("M:")),
                                 **{k: v for k, v in parse_stderr(err).items() if k != "hist5"}})
    golden["frontier_blocks"] = frontier
    (HERE / "golden.json").write_text(json.dumps(golden, indent=1, sort_keys=True) + "\n")
    print("wrote", HERE / "golden.json")


if __name__ == "__main__":
    sys.exit(main())
