"""Oracle vs the reference binary itself (oracle/_ref/s4, built from the reference's own
exhaustive/s4.c by `make -C oracle ref`) on fresh seeded ranges.  Skipped where that
binary was not built (it needs the reference tree at build time)."""
from __future__ import annotations

import random
import subprocess

import pytest

from conftest import REPO, assert_stats_equal
from oracle import orc
from golden.make_golden import parse_stderr

S4 = REPO / "oracle" / "_ref" / "s4"
pytestmark = pytest.mark.skipif(not S4.exists(), reason="reference binary oracle/_ref/s4 not built")


def ref_run(lo, hi, threads=2, extra=()):
    p = subprocess.run([str(S4), str(lo), str(hi), str(threads), "16", *extra], capture_output=True, text=True,
                       check=True)
    return p.stdout.splitlines(keepends=True), parse_stderr(p.stderr)


@pytest.mark.parametrize("seed", range(6))
def test_oracle_equals_reference_binary(seed):
    rng = random.Random(1000 + seed)
    width = int(10 ** rng.uniform(3, 5.5))
    lo = rng.randint(1, 10 ** rng.choice([6, 9, 11, 12]))
    lines, want = ref_run(lo, lo + width)
    rc, got, olines, err = orc.search(lo, lo + width)
    assert rc == 0, err
    assert sorted(olines) == sorted(lines)
    assert_stats_equal(got, want, label=f"[{lo},{lo + width})")


def test_oracle_equals_reference_binary_dump4():
    lines, want = ref_run(3 * 10 ** 6, 3 * 10 ** 6 + 50000, threads=1, extra=["--dump4", "100000000", "--noext"])
    rc, got, olines, err = orc.search(3 * 10 ** 6, 3 * 10 ** 6 + 50000, dump4=10 ** 8, flags=orc.NOEXT)
    assert olines == lines            # same lines in the same order (one region)
    assert_stats_equal(got, want, label="dump4")
