#!/usr/bin/env python3
"""Stand-in for the search binary under the reference's block controller, on a machine without
a GPU: replays blocks that bin/s4gpu wrote on a B200 (tests/golden/controller_blocks), given the
controller's own command line `lo hi threads log2_chunk --verify --out F --ckpt C`.  The
recorded stdout file and checkpoint are copied to F and C and the recorded stderr is written to
stderr, as s4gpu wrote them; a block that was not recorded exits 3."""
import os
import shutil
import sys
import time
from pathlib import Path


def main() -> int:
    a = sys.argv[1:]
    lo, hi = a[0], a[1]
    stem = Path(os.environ["PS4_REPLAY_DIR"]) / f"{lo}-{hi}"
    if not stem.with_suffix(".err").exists():
        sys.stderr.write(f"no recorded block for [{lo}, {hi})\n")
        return 3
    time.sleep(0.3)          # a block is never over before the controller first polls it
    shutil.copyfile(stem.with_suffix(".out"), a[a.index("--out") + 1])
    shutil.copyfile(stem.with_suffix(".ckpt"), a[a.index("--ckpt") + 1])
    sys.stderr.write(stem.with_suffix(".err").read_text())
    return 0


if __name__ == "__main__":
    sys.exit(main())
