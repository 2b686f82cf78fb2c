"""The multi-GPU path's host logic on CPU, two gloo ranks: each rank searches its own S shard
(bench.shard) -- here with the oracle, the search being a function of S alone -- and the
ranks combine only their figures (bench.aggregate).  The union equals one search of the whole
range, and the job time is the slowest rank's."""
from __future__ import annotations

import os
import sys

import pytest
import torch.multiprocessing as mp

from conftest import REPO

BOUND = 250000                     # the first 5-set is at S = 362141 (test_verify.py:13)


def _rank(rank: int, world: int, port: int, q):
    import torch.distributed as dist
    sys.path.insert(0, str(REPO))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from oracle import orc
        lo, hi = bench.shard(rank, BOUND)
        rc, st, lines, err = orc.search(lo, hi)
        assert rc == 0, err
        keys = ("S_done", "sets4", "sets5", "ext_cand", "ext_sqrt", "multi")
        times, totals = bench.aggregate(dist, world, [float(rank + 1)], [float(st[k]) for k in keys], "cpu")
        gathered = [None] * world
        dist.all_gather_object(gathered, lines)
        if rank == 0:
            q.put((times, dict(zip(keys, totals)), sorted(sum(gathered, [])), (lo, hi)))
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
    times, totals, lines, first = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert first == (1, BOUND)
    assert times == [2.0]                                   # the slowest rank's time
    rc, st, want, _ = orc.search(1, 2 * BOUND)
    assert rc == 0
    assert lines == sorted(want) and len(lines) > 0
    for k, v in totals.items():
        assert v == st[k], k
