#!/usr/bin/env python3
"""Fixtures of the drop-in CLI (bin/s4gpu) for tests/test_controller.py, made on a B200.

* The two blocks the reference's archived block controller requests in that test
  (run_exhaustive.py Search.run, with its clock stood in so that every block takes 2 s): the
  controller's own command line, `s4gpu lo hi 16 20 --verify --out F --ckpt C`, its stdout
  file, stderr and checkpoint, as <lo>-<hi>.out / .err / .ckpt.
* The "M:" lines of `s4gpu 1 10000000000 16 20`, the multi-extension 4-sets below 1e10, for the
  near-miss classification test (s4gpu_m_lines_1e10.txt).

    python tests/golden/make_controller_blocks.py [OUTDIR]      (default tests/golden/controller_blocks)
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "controller_blocks"
S4GPU = HERE.parent.parent / "pairwise-square-sums_b200" / "bin" / "s4gpu"
START = 10 ** 12
BLOCKS = [(START, START + 2 * 10 ** 8), (START + 2 * 10 ** 8, START + 7 * 10 ** 8)]


def main() -> int:
    out_dir = (Path(sys.argv[1]) if len(sys.argv) > 1 else OUT).resolve()
    out_dir.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        for lo, hi in BLOCKS:
            stem = out_dir / f"{lo}-{hi}"
            with open(stem.with_suffix(".err"), "w") as err:
                subprocess.run([str(S4GPU), str(lo), str(hi), "16", "20", "--verify", "--out",
                                str(stem.with_suffix(".out")), "--ckpt", str(stem.with_suffix(".ckpt"))],
                               cwd=tmp, stderr=err, stdout=subprocess.DEVNULL, check=True)
        out = Path(tmp) / "all.out"
        subprocess.run([str(S4GPU), "1", str(10 ** 10), "16", "20", "--out", str(out)], cwd=tmp,
                       stderr=subprocess.DEVNULL, stdout=subprocess.DEVNULL, check=True)
        m = [line for line in out.read_text().splitlines(keepends=True) if line.startswith("M:")]
        (out_dir / "s4gpu_m_lines_1e10.txt").write_text("".join(sorted(m)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
