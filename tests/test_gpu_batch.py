"""Batched uneven subranges: many items in one call, the call's launch sequence captured as
one CUDA graph, batches cost-ordered, launch shapes from the autotuner.

Bar: bit-exact -- every item's lines and counters equal the same subrange searched alone,
and equal the reference's (golden fixtures) or the oracle's where those are affordable.
"""
from __future__ import annotations

import os
import random
import subprocess

import pytest

from conftest import REPO, assert_stats_equal
from golden.make_golden import parse_stderr
from oracle import orc
from ps4b200 import Search, workloads

S4 = REPO / "oracle" / "_ref" / "s4"

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


CONFIG3_SEED = 20261203


@pytest.fixture(scope="module")
def config3():
    """The full batched workload: 4096 subranges, widths log-uniform in [1e5, 1e9], offsets
    uniform in [1, 1e11], seed 20261203, autotuned, in one call (one CUDA graph)."""
    los, his = workloads.subranges(4096, seed=CONFIG3_SEED)
    los, his = los.tolist(), his.tolist()
    s = Search(max(his) + 1)
    s.autotune(los, his, budget_s=4.0)
    stats, r = s.batch(los, his)
    assert s.graph_counts()[0] == 1
    yield s, los, his, stats, _by_item(r)
    s.close()


def test_4096_uneven_subranges_vs_single_calls_and_oracle(config3):
    """Item by item against single-subrange calls on a random sample, and against the oracle
    (the CPU restatement) on narrow items."""
    s, los, his, stats, got = config3
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


@pytest.mark.skipif(not S4.exists(), reason="reference binary oracle/_ref/s4 not built")
def test_4096_uneven_subranges_wide_high_items_vs_reference(config3):
    """Wide items (>= 1e8 S) at high offsets (>= 5e10), where the batch cutter splits an item
    across batches, against the reference's own s4 on every host thread:
    sorted lines, all ten counters, the 5-set histogram and the CAPACITY maxima."""
    s, los, his, stats, got = config3
    threads = str(os.cpu_count() or 1)
    wide = [i for i in range(4096) if his[i] - los[i] >= 10 ** 8 and los[i] >= 5 * 10 ** 10]
    assert len(wide) > 50
    rng = random.Random(11)
    pick = sorted(rng.sample([i for i in wide if his[i] - los[i] < 3 * 10 ** 8], 3))
    pick.append(min((i for i in wide if his[i] - los[i] >= 5 * 10 ** 8), key=lambda i: his[i] - los[i]))
    for i in pick:
        p = subprocess.run([str(S4), str(los[i]), str(his[i]), threads, "20"], capture_output=True, text=True,
                           check=True)
        want = parse_stderr(p.stderr)
        assert sorted(got.get(i, [])) == sorted(p.stdout.splitlines(keepends=True)), i
        assert_stats_equal(stats[i], want, label=f"s4 item {i} [{los[i]},{his[i]})")


def test_4096_uneven_subranges_union_vs_fused_kernel(config3):
    """The whole 4096-item union against the fused kernel -- tiles, staging and a per-lane
    divisor odometer in one kernel, a different extension route from the batched engine --
    run over the same list: every item's lines and counters equal."""
    _, los, his, stats, got = config3
    with Search(max(his) + 1, kernel="fused") as f:
        fstats, fr = f.batch(los, his)
    fgot = _by_item(fr)
    assert sum(len(v) for v in fgot.values()) == sum(len(v) for v in got.values())
    for i in range(4096):
        assert sorted(got.get(i, [])) == sorted(fgot.get(i, [])), i
        assert_stats_equal(stats[i], fstats[i], label=f"fused item {i}")


def test_4096_uneven_subranges_persistent_kernel_one_launch(config3):
    """The same 4096 items through PS4_KERNEL_PERSIST -- the whole call as one persistent launch
    over a ring of 4-sets -- equal the two-kernel pipeline's item by item."""
    _, los, his, stats, got = config3
    with Search(max(his) + 1, kernel="persist") as p:
        pstats, pr = p.batch(los, his)
        assert p.last_launches == 2                       # ring initialisation + the persistent kernel
    pgot = _by_item(pr)
    for i in range(4096):
        assert sorted(got.get(i, [])) == sorted(pgot.get(i, [])), i
        assert_stats_equal(stats[i], pstats[i], label=f"persist item {i}")
