"""Batched uneven subranges: many items in one call, the call's launch sequence captured as
one CUDA graph, batches cost-ordered, launch shapes from the autotuner.

Bar: bit-exact -- every item's lines and counters equal the same subrange searched alone,
and equal the reference's (golden fixtures) or the oracle's where those are affordable.
"""
from __future__ import annotations

import random

import pytest

from conftest import assert_stats_equal
from oracle import orc
from ps4b200 import Search, workloads

pytestmark = pytest.mark.gpu

SMALL_QUEUE = {"log2_tile": 14, "gen_ctas": 2, "ext_ctas": 3, "log2_jobs": 20}   # ~3.8e6 S per batch


def _by_item(r):
    out = {}
    for line, item in zip(r.lines, r.items):
        out.setdefault(item, []).append(line)
    return out


def test_golden_subranges_many_batches_one_graph(golden):
    """The reference's 48 subranges cut into many small batches: one graph, replayed."""
    subs = golden["subranges"]
    los, his = [s["lo"] for s in subs], [s["hi"] for s in subs]
    with Search(2 * 10 ** 12) as s:
        s.tuning = SMALL_QUEUE
        stats, r = s.batch(los, his)
        assert s.last_launches >= 4 and s.graph_counts() == (1, 0)
        stats2, r2 = s.batch(los, his)
        assert s.graph_counts() == (1, 1)                 # the second call replays the graph
    assert r2.lines == r.lines and stats2 == stats
    got = _by_item(r)
    for i, sub in enumerate(subs):
        assert sorted(got.get(i, [])) == sub["lines"], i
        assert_stats_equal(stats[i], sub, label=f"item {i}")


@pytest.mark.parametrize("graph", ["always", "never"])
def test_graph_and_direct_launches_agree(graph):
    lo, hi = 10 ** 9, 10 ** 9 + 3 * 10 ** 7
    with Search(hi, graph=graph) as s:
        s.tuning = SMALL_QUEUE
        a = s.range(lo, hi)
        caps, _ = s.graph_counts()
        assert caps == (1 if graph == "always" else 0)
    with Search(hi, graph="never") as s:
        b = s.range(lo, hi)
    assert a.lines == b.lines
    assert_stats_equal(a.stats, b.stats)


def test_autotune_keeps_results():
    los, his = workloads.subranges(64, seed=5, wmax=1e8)
    with Search(int(his.max()) + 1) as s:
        base = s.batch(los.tolist(), his.tolist())
        t = s.autotune(los.tolist(), his.tolist(), budget_s=3.0)
        assert 12 <= t["log2_tile"] <= 14 and 1 <= t["gen_ctas"] <= 2 and 1 <= t["ext_ctas"] <= 3 and t["rate"] > 0
        assert s.tuning["log2_tile"] == t["log2_tile"]
        again = s.batch(los.tolist(), his.tolist())
    assert again[1].lines == base[1].lines and again[0] == base[0]


def test_4096_uneven_subranges():
    """The full batched workload: 4096 subranges, widths log-uniform in [1e5, 1e9], offsets
    uniform in [1, 1e11], seed 20261203, autotuned, in one call.  Checked item by item against
    single-subrange calls on a random sample, and against the oracle on narrow items."""
    los, his = workloads.subranges(4096, seed=20261203)
    los, his = los.tolist(), his.tolist()
    with Search(max(his) + 1) as s:
        s.autotune(los, his, budget_s=4.0)
        stats, r = s.batch(los, his)
        assert s.graph_counts()[0] == 1
        got = _by_item(r)
        rng = random.Random(7)
        for i in rng.sample(range(4096), 24):
            one = s.range(los[i], his[i])
            assert sorted(got.get(i, [])) == sorted(one.lines), i
            assert_stats_equal(stats[i], one.stats, label=f"item {i}")
    narrow = [i for i in range(4096) if his[i] - los[i] < 150000]
    assert len(narrow) > 100
    for i in rng.sample(narrow, 12):
        rc, ost, olines, err = orc.search(los[i], his[i])
        assert rc == 0, err
        assert sorted(got.get(i, [])) == sorted(olines), i
        assert_stats_equal(stats[i], ost, label=f"oracle item {i}")
    assert sum(st["S_done"] for st in stats) == sum(h - l for l, h in zip(los, his))
