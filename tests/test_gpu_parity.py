"""Parity of the sm_100a search with the reference, through the C-ABI (lib/libps4.so).

Bar: bit-exact.  Result lines equal the reference's after canonical sorting (LC_ALL=C sort,
test_preflight.py:30-31), every TOTAL counter, the 5-set histogram and the CAPACITY maxima
equal.  Fixtures come from the reference binary (tests/golden/make_golden.py); small fresh
ranges are checked against the CPU restatement (oracle/) run on the same box.
"""
from __future__ import annotations

import os
import random
import subprocess

import pytest

from conftest import GOLDEN_DIR, REPO, assert_stats_equal, sha_sorted
from golden.make_golden import parse_stderr
from oracle import orc
from ps4b200 import Ps4Error, Search, _abi

pytestmark = pytest.mark.gpu

KERNELS = ("batched", "plain", "fused")
S4 = REPO / "oracle" / "_ref" / "s4"


@pytest.fixture(scope="module")
def big():
    with Search(2 * 10 ** 12) as s:
        yield s


@pytest.mark.parametrize("kernel", KERNELS)
def test_1e7_lines_and_counters(golden, golden_1e7_lines, kernel):
    with Search(10 ** 7, kernel=kernel, verify=True) as s:
        r = s.range(1, 10 ** 7)
    assert sorted(r.lines) == golden_1e7_lines
    assert_stats_equal(r.stats, golden["runs"]["1e7"], label=kernel)


@pytest.mark.parametrize("kernel", KERNELS)
def test_dump4_1e7_every_4set(golden, kernel):
    with Search(10 ** 7, kernel=kernel, dump4=True, noext=True) as s:
        r = s.range(1, 10 ** 7)
    g = golden["runs"]["dump4_1e7"]
    assert len(r.quads) == g["n_lines"] == 325094 == r.stats["sets4"]
    assert sha_sorted(r.quads) == g["sha256"]
    assert r.stats["ext_cand"] == 0 and r.stats["ext_sqrt"] == 0


def test_dump4_reference_order(golden):
    """Sorting the dump records by the emission key gives the reference's own order."""
    import ctypes as C
    want = (GOLDEN_DIR / "dump4_first2000.txt").read_text().splitlines(keepends=True)
    with Search(10 ** 7, dump4=True, noext=True) as s:
        s.range(1, 400000)
        lib, res = s.lib, s._res
        keyed = []
        for i in range(res.n_quads):
            S, v, o = C.c_uint64(), (C.c_uint64 * 4)(), (C.c_uint32 * 4)()
            lib.ps4_quad_values(C.byref(s._quads[i]), C.byref(S), v, o)
            buf = C.create_string_buffer(256)
            lib.ps4_format_quad(C.byref(s._quads[i]), buf, 256)
            keyed.append(((S.value, tuple(o)), buf.value.decode()))
    got = [line for _, line in sorted(keyed)]
    assert len(got) > len(want) == 2000
    assert got[:len(want)] == want


def test_singletons_and_boundary_logs(golden, big):
    for S, g in golden["singletons"].items():
        S = int(S)
        r = big.range(S, S + 1)
        assert r.lines == g["lines"], S
        assert_stats_equal(r.stats, g, label=str(S))
    for S, g in golden["boundary_logs"].items():
        r = big.range(int(S), int(S) + 1)
        assert r.lines == []
        assert_stats_equal(r.stats, g, hist=False, label=f"boundary {S}")


def test_subranges_one_call_each(golden, big):
    for sub in golden["subranges"]:
        r = big.range(sub["lo"], sub["hi"])
        assert sorted(r.lines) == sub["lines"], (sub["lo"], sub["hi"])
        assert_stats_equal(r.stats, sub, label=f"[{sub['lo']},{sub['hi']})")


def test_subranges_batched_in_one_launch(golden, big):
    subs = golden["subranges"]
    stats, r = big.batch([s["lo"] for s in subs], [s["hi"] for s in subs])
    assert big.last_launches == 2          # one batch: the tile kernel, then the extension engine
    by_item = {}
    for line, item in zip(r.lines, r.items):
        by_item.setdefault(item, []).append(line)
    for i, sub in enumerate(subs):
        assert sorted(by_item.get(i, [])) == sub["lines"], i
        assert_stats_equal(stats[i], sub, label=f"item {i}")


def test_1e9(golden, golden_1e9_lines):
    with Search(10 ** 9) as s:
        r = s.range(1, 10 ** 9)
    assert sorted(r.lines) == golden_1e9_lines
    assert sha_sorted(r.lines) == golden["runs"]["1e9"]["sha256"]
    assert_stats_equal(r.stats, golden["runs"]["1e9"], label="1e9")


@pytest.mark.parametrize("kernel", KERNELS)
def test_1e10(golden, kernel):
    """The headline workload, S < 1e10: sorted-output hash, counters, every M line."""
    with Search(10 ** 10, kernel=kernel) as s:
        r = s.range(1, 10 ** 10)
    g = golden["runs"]["1e10"]
    assert sha_sorted(r.lines) == g["sha256"] == "33292b86eb0c9dda87dcb93830e0c5117f9e079b2726eccabb566a24d7b34838"
    assert len(r.lines) == g["n_lines"] == 54477
    assert_stats_equal(r.stats, g, label=f"1e10 {kernel}")
    want_m = (GOLDEN_DIR / "m_lines_1e10.txt").read_text().splitlines(keepends=True)
    assert sorted(x for x in r.lines if x.startswith("M:")) == want_m


def test_frontier_blocks(golden, big):
    """Two 5e9-wide blocks at S ~ 1.95e12 from the reference's archived raw evidence
    (exhaustive/evidence/exhaustive-2026-09-18.tar.gz, block-0001/0002)."""
    for blk in golden["frontier_blocks"]:
        r = big.range(blk["lo"], blk["hi"])
        assert sha_sorted(r.lines) == blk["sha256"], blk["block"]
        assert sorted(x for x in r.lines if x.startswith("M:")) == blk["m_lines"]
        assert_stats_equal(r.stats, blk, hist=False, label=blk["block"])


def test_frontier_blocks_wide():
    """Eight more archived blocks spread over S ~ 2.15e12 .. 3.51e12 (exhaustive-2026-09-18 and
    -09-19 raw evidence; tests/golden/make_frontier.py), where the tile kernel scans groups of
    tiles into per-tile lists: sorted-output hash, every M line, every TOTAL counter."""
    import json
    blocks = json.loads((GOLDEN_DIR / "frontier.json").read_text())
    with Search(max(b["hi"] for b in blocks) + 1) as s:
        for blk in blocks:
            r = s.range(blk["lo"], blk["hi"])
            assert sha_sorted(r.lines) == blk["sha256"], blk["block"]
            assert len(r.lines) == blk["n_lines"]
            assert sorted(x for x in r.lines if x.startswith("M:")) == blk["m_lines"], blk["block"]
            assert_stats_equal(r.stats, blk, hist=False, label=blk["block"])


@pytest.mark.skipif(not S4.exists(), reason="reference binary oracle/_ref/s4 not built")
@pytest.mark.parametrize("lo,width", [(12 * 10 ** 12, 2 * 10 ** 7), (17_500_000_000_000, 10 ** 7)])
def test_top_of_range_vs_reference_s4(lo, width):
    """At the reference's own frontier (S ~ 1.2e13) and just below the library's bound 2^44
    (1.759e13), where roots approach 2^22 and the factor tables 8.4e6 entries: the reference's
    s4 on every host thread over the same range -- sorted lines, all ten counters, the 5-set
    histogram and the CAPACITY maxima."""
    hi = lo + width
    with Search(hi) as s:
        r = s.range(lo, hi)
    p = subprocess.run([str(S4), str(lo), str(hi), str(os.cpu_count() or 1), "20"], capture_output=True, text=True,
                       check=True)
    assert sorted(r.lines) == sorted(p.stdout.splitlines(keepends=True))
    assert_stats_equal(r.stats, parse_stderr(p.stderr), label=f"s4 [{lo},{hi})")


@pytest.mark.parametrize("seed", range(8))
def test_fresh_ranges_against_oracle(big, seed):
    rng = random.Random(77 + seed)
    width = int(10 ** rng.uniform(3, 5.3))
    lo = rng.randint(1, 10 ** rng.choice([5, 8, 10, 11, 12]))
    r = big.range(lo, lo + width)
    rc, ost, olines, err = orc.search(lo, lo + width)
    assert rc == 0, err
    assert sorted(r.lines) == sorted(olines)
    assert_stats_equal(r.stats, ost, label=f"[{lo},{lo + width})")


def test_empty_and_tiny_ranges(big):
    for lo, hi in [(5, 5), (10, 3), (0, 1), (0, 2), (1, 2), (2, 3), (1, 10), (16383, 16385), (65, 130)]:
        r = big.range(lo, hi)
        rc, ost, olines, _ = orc.search(lo, hi)
        assert r.lines == olines
        assert_stats_equal(r.stats, ost, label=f"[{lo},{hi})")


def test_tile_size_and_split_independence():
    lo, hi = 10 ** 9, 10 ** 9 + 3 * 10 ** 7
    ref = None
    for tl in (12, 13, 14):
        with Search(hi, log2_tile=tl) as s:
            r = s.range(lo, hi)
        key = (sorted(r.lines), {k: r.stats[k] for k in orc.COUNTERS})
        ref = ref or key
        assert key == ref, tl
    with Search(hi) as s:
        mid = lo + 12345677
        a, b = s.range(lo, mid), s.range(mid, hi)
    assert sorted(a.lines + b.lines) == ref[0]
    assert {k: a.stats[k] + b.stats[k] for k in orc.COUNTERS} == ref[1]


def test_plain_equals_batched_mid_range():
    lo, hi = 3 * 10 ** 10, 3 * 10 ** 10 + 2 * 10 ** 7
    out = {}
    for k in KERNELS:
        with Search(hi, kernel=k) as s:
            r = s.range(lo, hi)
        out[k] = (sorted(r.lines), r.stats)
    assert out["batched"][0] == out["plain"][0]
    assert_stats_equal(out["batched"][1], out["plain"][1])


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("caps,code,msg", [
    (dict(cap_reps=2), _abi.PS4_ERR_CAP_REPS, "representation capacity exceeded"),
    (dict(cap_divs=1), _abi.PS4_ERR_CAP_DIVS, "divisor capacity exceeded"),
    (dict(cap_ext=1), _abi.PS4_ERR_CAP_EXT, "extension capacity exceeded"),
])
def test_capacity_failures(kernel, caps, code, msg):
    """test_preflight.py's injected capacity failures (-DS4_MAX_REPS=2 / _DIVS=1 / _EXT=1)."""
    with Search(10 ** 7, kernel=kernel, **caps) as s:
        with pytest.raises(Ps4Error) as e:
            s.range(1, 10 ** 7)
    assert e.value.code == code
    assert e.value.message == f"FATAL: {msg}; this interval is NOT certified complete"


def test_noext_counters(golden):
    with Search(10 ** 7, noext=True) as s:
        r = s.range(1, 10 ** 7)
    g = golden["runs"]["dump4_1e7"]
    assert r.lines == []
    for k in ("S_done", "pairs", "S_ge3", "triples", "sets4"):
        assert r.stats[k] == g[k]
    assert r.stats["ext_cand"] == r.stats["ext_sqrt"] == r.stats["sets5"] == 0


def test_context_reuse_is_stateless(big):
    a = big.range(10 ** 11, 10 ** 11 + 10 ** 6)
    big.range(10 ** 7, 2 * 10 ** 7)
    b = big.range(10 ** 11, 10 ** 11 + 10 ** 6)
    assert a.lines == b.lines and a.stats == b.stats
