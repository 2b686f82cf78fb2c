"""One range on several devices, host logic on CPU.

ps4_plan_shards cuts [lo, hi) into contiguous shards of about equal search cost; two gloo
ranks each search their shard -- here with the oracle, the search being a function of S alone
-- and ps4b200.shards.search_sharded gathers and merges the shards' results: the merged lines
equal one search of the whole range line for line (same order), the counters equal, and the
job time is the slowest rank's (bench.aggregate)."""
from __future__ import annotations

import os
import sys

import pytest
import torch.multiprocessing as mp

from conftest import REPO, assert_stats_equal

BOUND = 500000                     # the first 5-set is at S = 362141 (test_verify.py:13)


def _oracle_range(a: int, b: int):
    from oracle import orc
    from ps4b200 import RangeResult
    rc, st, lines, err = orc.search(a, b)
    assert rc == 0, err
    return RangeResult(stats=st, lines=lines)


def _rank(rank: int, world: int, port: int, q):
    import torch.distributed as dist
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "pairwise-square-sums_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from ps4b200 import shards
        merged, (lo, hi) = shards.search_sharded(1, BOUND, rank=rank, world=world, dist=dist,
                                                 search_fn=_oracle_range)
        assert (lo, hi) == bench.shard(rank, world, BOUND)
        times, totals = bench.aggregate(dist, world, [float(rank + 1)], [float(hi - lo)], "cpu")
        if rank == 0:
            q.put((times, totals, merged.lines, merged.stats, (lo, hi)))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_equal_one_search():
    from oracle import orc
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    times, totals, lines, stats, first = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert first[0] == 1 and 1 < first[1] < BOUND
    assert times == [2.0]                                   # the slowest rank's time
    assert totals == [float(BOUND - 1)]                     # the shards cover the range once
    rc, want_stats, want, _ = orc.search(1, BOUND)
    assert rc == 0
    assert lines == want and len(lines) > 0                 # same lines, same order
    assert_stats_equal(stats, want_stats, label="merged shards")


def _cost(a: int, b: int) -> float:
    return b ** 1.16 - a ** 1.16


@pytest.mark.parametrize("lo,hi,n", [(1, 10 ** 10, 2), (1, 10 ** 10, 8), (5 * 10 ** 10, 10 ** 12, 7),
                                     (10 ** 9, 10 ** 9 + 10 ** 6, 4)])
def test_plan_shards_balances_cost(lo, hi, n):
    from ps4b200 import shards
    b = shards.plan(lo, hi, n)
    assert len(b) == n + 1 and b[0] == max(lo, 1) and b[-1] == hi
    assert all(x <= y for x, y in zip(b, b[1:]))
    assert all(x % (1 << 14) == 0 for x in b[1:-1])
    costs = [_cost(x, y) for x, y in zip(b, b[1:])]
    mean = _cost(b[0], b[-1]) / n
    assert max(abs(c - mean) for c in costs) <= 0.01 * mean + _cost(hi - (1 << 14), hi)
    if hi >= 2 * max(lo, 1) and hi > 10 * (1 << 14) * n:
        widths = [y - x for x, y in zip(b, b[1:])]
        assert widths[0] > widths[-1]                       # cost per S grows with S


def test_plan_shards_edges():
    from ps4b200 import shards
    assert shards.plan(0, 100, 1) == [1, 100]
    assert shards.plan(5, 5, 3) == [5, 5, 5, 5]
    b = shards.plan(1, 1000, 4)                             # narrower than one tile a shard
    assert b[0] == 1 and b[-1] == 1000 and all(x <= y for x, y in zip(b, b[1:]))
    m = shards.merge_stats([{"S_done": 1, "pairs": 2, "S_ge3": 0, "triples": 0, "sets4": 3, "sets5": 1, "sets6": 0,
                             "multi": 0, "ext_cand": 5, "ext_sqrt": 1, "hist5": {20: 1}, "max_reps": 4,
                             "max_divisors": 9, "max_extensions": 1},
                            {"S_done": 2, "pairs": 1, "S_ge3": 1, "triples": 1, "sets4": 1, "sets5": 2, "sets6": 0,
                             "multi": 1, "ext_cand": 7, "ext_sqrt": 2, "hist5": {20: 1, 22: 1}, "max_reps": 6,
                             "max_divisors": 3, "max_extensions": 2}])
    assert m["S_done"] == 3 and m["ext_cand"] == 12 and m["hist5"] == {20: 2, 22: 1}
    assert (m["max_reps"], m["max_divisors"], m["max_extensions"]) == (6, 9, 2)
