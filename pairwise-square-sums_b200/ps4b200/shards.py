"""One search range on several devices, one process per device.

The reference splits [S_lo, S_hi) into equal-width regions, one per CPU thread
(exhaustive/s4.c:452-456), and sums the threads' counters at the end (s4.c:488-495).  Here the
range is cut into contiguous shards of about equal search cost (``plan``, the library's
ps4_plan_shards), each process searches its shard on its own GPU (``Search.range``), and the
shards' results meet on the host: every result line and counter is a function of S alone
(s4.c:313-341), so the lines concatenate in shard order into the whole range's canonical order
and the counters add (the CAPACITY maxima take the maximum).  Nothing crosses NVLink during the
search; the only collective is one gather of each shard's results (torch.distributed, any
backend) after it.
"""
from __future__ import annotations

import ctypes as C

from . import _abi
from .search import RangeResult

ADDITIVE = _abi.COUNTER_NAMES
MAXIMA = ("max_reps", "max_divisors", "max_extensions")


def plan(lo: int, hi: int, n: int) -> list[int]:
    """n + 1 bounds: shard i is [b[i], b[i+1]), of about equal search cost (ps4_plan_shards)."""
    lib = _abi.load()
    b = (C.c_uint64 * (n + 1))()
    rc = lib.ps4_plan_shards(lo, hi, n, b)
    if rc != _abi.PS4_OK:
        raise ValueError(f"ps4_plan_shards({lo}, {hi}, {n}) failed: {rc}")
    return [int(x) for x in b]


def merge_stats(parts: list[dict]) -> dict:
    """Counters of consecutive shards as one range's: sums, histogram sums, maxima."""
    out = {k: sum(p[k] for p in parts) for k in ADDITIVE}
    hist: dict[int, int] = {}
    for p in parts:
        for k, v in p.get("hist5", {}).items():
            hist[int(k)] = hist.get(int(k), 0) + int(v)
    out["hist5"] = dict(sorted(hist.items()))
    for k in MAXIMA:
        out[k] = max((p.get(k, 0) for p in parts), default=0)
    return out


def merge(results: list[RangeResult]) -> RangeResult:
    """The shards' results, in shard order, as one range's result."""
    out = RangeResult(stats=merge_stats([r.stats for r in results]))
    for r in results:
        out.lines.extend(r.lines)
        out.six_lines.extend(r.six_lines)
        out.quads.extend(r.quads)
        out.kernel_ms = max(out.kernel_ms, r.kernel_ms)
    return out


def search_sharded(lo: int, hi: int, *, rank: int, world: int, dist=None, search_fn=None, search=None):
    """Search [lo, hi) across `world` processes; this process searches shard `rank`.

    search_fn(a, b) -> RangeResult does one shard (default: ``search.range``).  With world > 1,
    `dist` is an initialised torch.distributed module; every rank receives the merged result.
    Returns (merged result, this rank's shard bounds)."""
    bounds = plan(lo, hi, world)
    a, b = bounds[rank], bounds[rank + 1]
    if search_fn is None:
        search_fn = search.range
    mine = search_fn(a, b)
    if world == 1:
        return mine, (a, b)
    payload = (mine.stats, mine.lines, mine.six_lines, mine.quads, mine.kernel_ms)
    got = [None] * world
    dist.all_gather_object(got, payload)
    parts = [RangeResult(stats=s, lines=l, six_lines=x, quads=q, kernel_ms=k) for s, l, x, q, k in got]
    return merge(parts), (a, b)
