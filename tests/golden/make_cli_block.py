"""Write one block of the drop-in CLI's output as a fixture: `bin/s4gpu 1 10000000 16 20
--verify --out block-0001.out --ckpt block-0001.ckpt`, started the way the block controller
starts `s4` (run_exhaustive.py:207-215: run directory as cwd, stdout discarded, stderr into
block-0001.err), plus block.json with the interval and the run parameters.

Needs a B200.  Usage: python tests/golden/make_cli_block.py [OUTDIR] (default
tests/golden/cli_block).  tests/test_consumers.py hands the block to the reference's own
consumers (controller, packer, verifier) and to their restatements in tests/consumers.py.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

import consumers  # noqa: E402

CLI = HERE.parent.parent / "pairwise-square-sums_b200" / "bin" / "s4gpu"
LO, HI, THREADS, CHUNK_LOG2 = 1, 10 ** 7, 16, 20


def main():
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "cli_block"
    out.mkdir(parents=True, exist_ok=True)
    for ext in ("out", "err", "ckpt"):
        (out / ("block-0001." + ext)).unlink(missing_ok=True)
    rc, _ = consumers.run_block(CLI, out.resolve(), "block-0001", LO, HI, THREADS)
    if rc != 0:
        sys.exit(f"s4gpu exited {rc}: " + (out / "block-0001.err").read_text())
    (out / "block.json").write_text(json.dumps({"id": "block-0001", "lo": LO, "hi": HI, "threads": THREADS,
                                                "chunk_log2": CHUNK_LOG2}, indent=1) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
