"""PS4_KERNEL_PERSIST: a whole call as one persistent launch over a device ring of 4-sets.

CTAs switch between producing tiles' 4-sets into the ring and extending them from it, so a call
of any number of subranges is one launch (after a ring-initialising one).  Bar: bit-exact, as
for every kernel -- the reference's fixtures (tests/golden, from the reference's own s4) at
1e7, 1e9, 1e10, its 48 seeded subranges and an archived frontier block, dump4 and verify; the
config-3 workload's per-item results against the two-kernel pipeline are in test_gpu_batch.py.
Its bounded waits are checked by making one run out on a flag that nothing sets.
"""
from __future__ import annotations

import ctypes as C

import pytest

from conftest import GOLDEN_DIR, assert_stats_equal, sha_sorted
from ps4b200 import Search, _abi

pytestmark = pytest.mark.gpu


def test_1e7_lines_and_counters_one_launch(golden, golden_1e7_lines):
    with Search(10 ** 7, kernel="persist", verify=True) as s:
        r = s.range(1, 10 ** 7)
        assert s.last_launches == 2                     # ring initialisation + the persistent kernel
    assert sorted(r.lines) == golden_1e7_lines
    assert_stats_equal(r.stats, golden["runs"]["1e7"], label="persist 1e7")


def test_dump4_1e7_every_4set(golden):
    with Search(10 ** 7, kernel="persist", dump4=True, noext=True) as s:
        r = s.range(1, 10 ** 7)
    g = golden["runs"]["dump4_1e7"]
    assert len(r.quads) == g["n_lines"] == 325094 == r.stats["sets4"]
    assert sha_sorted(r.quads) == g["sha256"]


def test_1e9(golden, golden_1e9_lines):
    with Search(10 ** 9, kernel="persist") as s:
        r = s.range(1, 10 ** 9)
    assert sorted(r.lines) == golden_1e9_lines
    assert_stats_equal(r.stats, golden["runs"]["1e9"], label="persist 1e9")


def test_1e10(golden):
    with Search(10 ** 10, kernel="persist") as s:
        r = s.range(1, 10 ** 10)
    g = golden["runs"]["1e10"]
    assert sha_sorted(r.lines) == g["sha256"]
    assert_stats_equal(r.stats, g, label="persist 1e10")
    want_m = (GOLDEN_DIR / "m_lines_1e10.txt").read_text().splitlines(keepends=True)
    assert sorted(x for x in r.lines if x.startswith("M:")) == want_m


def test_golden_subranges_one_launch(golden):
    subs = golden["subranges"]
    with Search(2 * 10 ** 12, kernel="persist") as s:
        stats, r = s.batch([x["lo"] for x in subs], [x["hi"] for x in subs])
        assert s.last_launches == 2
    got = {}
    for line, item in zip(r.lines, r.items):
        got.setdefault(item, []).append(line)
    for i, sub in enumerate(subs):
        assert sorted(got.get(i, [])) == sub["lines"], i
        assert_stats_equal(stats[i], sub, label=f"persist item {i}")


def test_frontier_block(golden):
    blk = golden["frontier_blocks"][0]
    with Search(blk["hi"], kernel="persist") as s:
        r = s.range(blk["lo"], blk["hi"])
    assert sha_sorted(r.lines) == blk["sha256"]
    assert_stats_equal(r.stats, blk, hist=False, label=blk["block"])


def test_bounded_wait_gives_up_and_the_device_stays_usable(golden_1e7_lines):
    lib = _abi.load()
    waited = C.c_uint64()
    assert lib.ps4_check_ring_wait(0, C.byref(waited)) == _abi.PS4_ERR_TIMEOUT
    assert 2e9 <= waited.value < 2e10, waited.value
    with Search(10 ** 7, kernel="persist") as s:
        r = s.range(1, 10 ** 7)
    assert sorted(r.lines) == golden_1e7_lines
