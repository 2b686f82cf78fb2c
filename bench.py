#!/usr/bin/env python3
"""Benchmark: the exhaustive square-sum search over S in [1, 1e10) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--kernel batched|plain]

One step = one complete search of S in [1, 1e10) (the reference's `s4 1 10000000000`): every
4-set with S below the bound, every extension, every counter.  N > 1 runs under torchrun, one
process per GPU; the same range is cut into N contiguous shards of about equal search cost
(ps4b200.shards.plan, the library's ps4_plan_shards), each rank searches its shard (strong
scaling, no data-path collective; the time is the max over ranks; the e2e leg gathers the
shards' results on the host).  Rank 0 prints one JSON line.

value      S covered per second with the work enqueued on the device (CUDA events on the
           launch stream around each step; a 256 MiB write flushes L2 between steps,
           outside the events)
e2e        the same through the public C-ABI call with host result buffers
           (ps4_search_range: input copy, search, result copies, host collection)
roofline   integer-issue roofline: algorithmic int32 lane-ops per launch (ps4b200/opmodel.py,
           frozen) / kernel time, against 4 warp-instructions x 32 lanes per SM per clock
cpu_baseline  the reference's own s4 (oracle/_ref/s4, all host threads) on a stratified
           sample of the same range (4 slices of --ref-slice S), timed on this host
--impl reference  that CPU reference alone over the same slices, as the reference arm
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "pairwise-square-sums_b200"))

BOUND = 10 ** 10
METRIC = "range_per_s"
UNIT = "S/s"


def shard(rank: int, world: int, bound: int = BOUND) -> tuple[int, int]:
    """Rank r's shard of S in [1, bound): contiguous, about equal search cost per rank."""
    from ps4b200 import shards
    b = shards.plan(1, bound, world)
    return b[rank], b[rank + 1]


def aggregate(dist, world: int, times: list, totals: list, device) -> tuple[list, list]:
    """The job's figures from every rank's: the slowest rank's times (max), the summed totals.
    The only collectives of a multi-GPU run; the search itself exchanges nothing."""
    import torch
    vals = torch.tensor(times, dtype=torch.float64, device=device)
    tot = torch.tensor(totals, dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return vals.tolist(), tot.tolist()


# ------------------------------------------------------------------ CPU reference (s4)

def _s4_binary():
    ref = REPO / "oracle" / "_ref" / "s4"
    if ref.exists():
        return ref, "reference"
    port = REPO / "oracle" / "ps4_oracle"
    return port, "port"


def _run_s4(binary: Path, kind: str, lo: int, hi: int, threads: int) -> float:
    """Seconds of search work for one s4 run: the slowest region thread's own timer (the
    process wall time adds s4's 1 s polling granularity, s4.c:470-474)."""
    if kind == "reference":
        t0 = time.perf_counter()
        p = subprocess.run([str(binary), str(lo), str(hi), str(threads), "20"], capture_output=True, text=True,
                           check=True)
        wall = time.perf_counter() - t0
        secs = [float(x) for x in re.findall(r"^\s+thread\s+\d+: .*?\s([\d.]+)s$", p.stderr, re.M)]
        return max(secs) if secs and max(secs) > 0 else wall
    t0 = time.perf_counter()
    subprocess.run([str(binary), str(lo), str(hi)], capture_output=True, text=True, check=True)
    return time.perf_counter() - t0


def _strata(width: int, lo: int, hi: int, k: int = 4):
    """k slices of `width` centred at the midpoints of k equal parts of [lo, hi)."""
    span = hi - lo
    return [(lo + span * (2 * j + 1) // (2 * k) - width // 2, lo + span * (2 * j + 1) // (2 * k) - width // 2 + width)
            for j in range(k)]


def cpu_sample_plan(lo: int, hi: int, budget_s: float, slice_w: int):
    """The CPU sample: the reference's s4 on all host threads over 4 fixed slices of slice_w S (the
    bench line's cpu_baseline and the reference arm time the same slices); the single-thread oracle
    port, where s4 is not built, over slices sized to budget_s from a probe."""
    binary, kind = _s4_binary()
    threads = (os.cpu_count() or 1) if kind == "reference" else 1
    if kind == "reference":
        return binary, kind, threads, _strata(min(slice_w, max((hi - lo) // 8, 1)), lo, hi)
    w0 = 2 * 10 ** 7
    mid = (lo + hi) // 2
    t = _run_s4(binary, kind, mid, mid + w0, threads)
    rate = w0 / max(t, 1e-3)
    width = int(max(10 ** 6, min((hi - lo) // 8, rate * budget_s / 4)))
    return binary, kind, threads, _strata(width, lo, hi)


def cpu_sample_run(binary, kind, threads, slices) -> tuple[float, int]:
    secs = sum(_run_s4(binary, kind, a, b, threads) for a, b in slices)
    return secs, sum(b - a for a, b in slices)


def run_reference(args, rank: int):
    """The reference arm: s4 itself on this host's cores, on a bounded sample of the workload."""
    if rank != 0:
        return
    lo, hi = 1, BOUND
    binary, kind, threads, slices = cpu_sample_plan(lo, hi, budget_s=args.ref_budget, slice_w=args.ref_slice)
    for _ in range(args.warmup):
        cpu_sample_run(binary, kind, threads, slices)
    total_s, total_S = 0.0, 0
    for _ in range(args.steps):
        s, n = cpu_sample_run(binary, kind, threads, slices)
        total_s += s
        total_S += n
    value = total_S / total_s
    sample = f"{len(slices)} slices of {slices[0][1] - slices[0][0]} S at the midpoints of 4 equal parts of [1,1e10)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total_s / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "exhaustive",
            "config": {"workload": "exhaustive square-sum search, S in [1,1e10) (s4 bound 1e10), sampled",
                       "bound": BOUND, "sample": sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    Q = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9 and (not self.uuid or self.uuid in f[0]):
                self.rows.append(f)

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(self.rows[0][2]) if self.rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------ side workloads

TRIPLE_SEED = 20261203


def measure_triples(local: int, stream, n: int = 10 ** 5, dmax: int = 10 ** 12, steps: int = 5, warmup: int = 3,
                    cpu: bool = True) -> dict:
    """Batched triple extension: n seeded triples (x, y, z uniform in [1, 1e5]), every d <= dmax.
    value = triples/s of the kernel (CUDA events on the launch stream); e2e through
    ps4_extend_triples with the triples in pinned host memory and sorted records back."""
    import numpy as np
    import torch
    from ps4b200 import Search, workloads
    abc = workloads.triples(n, seed=TRIPLE_SEED)
    pinned = torch.empty((n, 3), dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    pinned[:] = abc
    with Search(2 * 10 ** 12, device=local, stream=stream.cuda_stream) as s:
        for _ in range(warmup):
            s.extend_triples(pinned, dmax, as_lists=False)
        torch.cuda.synchronize()
        kms, wall, st = 0.0, 0.0, None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            recs, state, st = s.extend_triples(pinned, dmax, as_lists=False)
            kms += s.last_kernel_ms
        e1.record(stream)
        torch.cuda.synchronize()
        wall = e0.elapsed_time(e1)
        h2d, d2h = s.transfer_bytes()
    out = {"workload": f"{n} seeded triples (x,y,z uniform in [1,1e5]), every d <= {dmax:.0e}",
           "value": n * steps / (kms / 1e3), "unit": "triples/s",
           "candidates_per_s": st["ext_cand"] * steps / (kms / 1e3), "kernel_ms": kms / steps,
           "exts": st["exts"],
           "e2e": {"value": n * steps / (wall / 1e3), "unit": "triples/s", "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h}}
    if cpu:
        from oracle import orc
        k = 20000
        t0 = time.perf_counter()
        for a, b, c in abc[:k].tolist():
            orc.extend_triple(a, b, c, dmax)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": k / t, "unit": "triples/s", "cores": 1, "kind": "port",
                               "sample": f"first {k} of the same triples, oracle/ps4_oracle.c orc_extend_triple"}
    return out


def measure_serve(local: int, n_req: int, rates, seed: int = 20261204, budget: int = 8 << 30) -> dict:
    """The serving loop on a seeded Poisson stream (70 % subranges, width log-uniform in
    [1e4, 1e9], offset uniform in [1, 1e12]; 30 % triples, d <= 1e12), replayed in real time
    once per arrival rate (the same requests each time: the seed fixes their contents, the rate
    only scales the gaps); then the same requests in the offline batched form (one batch call,
    one triple call), with every result of every stream compared with it."""
    from ps4b200 import Search, workloads
    from ps4b200.serve import Server, run_stream
    streams, reps = [], []
    with Search(10 ** 12 + 10 ** 9 + 1, device=local) as s:
        for rate in rates:
            reqs = workloads.requests(n_req, seed=seed, rate=rate)
            with Server(s, hbm_budget=budget) as srv:
                run_stream(srv, workloads.requests(20, seed=seed + 7, rate=1000.0, wmax=1e7))     # warm-up
                reps.append(run_stream(srv, reqs))
        ranges = [r for r in reqs if r.kind == "range"]
        tris = [r for r in reqs if r.kind == "triple"]
        t0 = time.monotonic()
        stats, res = s.batch([r.lo for r in ranges], [r.hi for r in ranges])
        ext, state, tst = s.extend_triples([r.abc for r in tris], 10 ** 12)
        off_s = time.monotonic() - t0
    by_item = {}
    for line, item in zip(res.lines, res.items):
        by_item.setdefault(item, []).append(line)
    S_total = sum(r.hi - r.lo for r in ranges)
    all_same = True
    for rate, rep in zip(rates, reps):
        same = True
        for i, r in enumerate(ranges):
            g = rep.results[r.rid]
            same &= (not isinstance(g, Exception)) and g.lines == by_item.get(i, []) and g.stats == stats[i]
        for i, r in enumerate(tris):
            g = rep.results[r.rid]
            same &= (not isinstance(g, Exception)) and g[0] == ext[i] and g[1] == int(state[i])
        all_same &= same
        lat = sorted(rep.latency_s.values())
        streams.append({"rate_per_s": rate, "p50_ms": 1e3 * rep.percentile(50), "p90_ms": 1e3 * rep.percentile(90),
                        "p99_ms": 1e3 * rep.percentile(99), "max_ms": 1e3 * lat[-1],
                        "requests_per_s": n_req / rep.wall_s, "S_per_s": S_total / rep.wall_s,
                        "wall_s": rep.wall_s, "steps": rep.info["steps"], "step_reruns": rep.info["step_reruns"],
                        "gpu_busy_frac": rep.info["gpu_ms"] / 1e3 / rep.wall_s,
                        "arena_peak_bytes": rep.info["arena_peak"], "identical_to_offline": bool(same)})
    return {"workload": f"{n_req} requests, Poisson arrivals, seed {seed}: 70% subranges (width "
                        f"log-uniform [1e4,1e9], offset uniform [1,1e12]), 30% triples (d <= 1e12); the same "
                        f"requests at each rate",
            "streams": streams, "S_total": S_total, "offline_S_per_s": S_total / off_s, "offline_s": off_s,
            "identical_to_offline": bool(all_same), "hbm_budget_bytes": budget}


CONFIG3_SEED = 20261203


def config3_cpu_sample(los, his, budget_s: float = 12.0, seed: int = 5):
    """The reference's s4 on all host threads over a seeded sample of the 4096 items, each
    clipped to a centred slice of at most 4e7 S, about budget_s seconds of work in all."""
    import random
    binary, kind = _s4_binary()
    threads = (os.cpu_count() or 1) if kind == "reference" else 1
    rng = random.Random(seed)
    order = rng.sample(range(len(los)), len(los))
    secs, S, n = 0.0, 0, 0
    for i in order:
        w = min(his[i] - los[i], 4 * 10 ** 7)
        a = los[i] + (his[i] - los[i] - w) // 2
        secs += _run_s4(binary, kind, a, a + w, threads)
        S += w
        n += 1
        if secs >= budget_s:
            break
    return {"value": S / secs, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{n} seeded items of the 4096, each a centred slice of at most 4e7 S ({S} S in all), "
                      f"slowest region thread's own timer per s4 run"}


def measure_subranges(local: int, stream, steps: int, warmup: int, cpu: bool = True, kernel: str = "batched",
                      compare: str | None = "persist") -> dict:
    """The batched uneven-subrange workload: 4096 subranges (seed 20261203, widths log-uniform
    in [1e5, 1e9], offsets uniform in [1, 1e11]) in one call: on the two-kernel pipeline,
    autotuned, its launches captured as one CUDA graph, or on the persistent kernel, one launch
    over a ring of 4-sets.  value: S/s from the
    library's CUDA events around each call's launches; e2e: the same calls timed from the host
    (pinned inputs copied in, results copied out and formatted).  `compare`: the other kernel,
    one step, its rate and whether every item's counters and lines equal."""
    import torch
    from ps4b200 import Search, workloads
    los, his = workloads.subranges(4096, seed=CONFIG3_SEED)
    los, his = los.tolist(), his.tolist()
    props = torch.cuda.get_device_properties(local)
    with Search(max(his) + 1, device=local, stream=stream.cuda_stream, kernel=kernel) as s:
        tune = s.autotune(los, his, budget_s=4.0) if kernel == "batched" else None
        for _ in range(warmup):
            s.batch(los, his, want_lines=False)
        clocks = ClockSampler(str(getattr(props, "uuid", "")))
        clocks.start()
        torch.cuda.synchronize()
        kms, launches, h2d, d2h = 0.0, 0, 0, 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            stats, res = s.batch(los, his, want_lines=True)
            kms += s.last_kernel_ms
            launches += s.last_launches
            a_, b_ = s.transfer_bytes()
            h2d += a_
            d2h += b_
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop()
        caps, replays = s.graph_counts()
    S = sum(h - l for l, h in zip(los, his))
    out = {"workload": "4096 uneven subranges, seed 20261203, widths log-uniform in [1e5,1e9], offsets uniform in "
                       "[1,1e11], one call = one CUDA graph", "S_total": S, "kernel": kernel,
           "value": S * steps / (kms / 1e3), "unit": UNIT, "steps": steps, "warmup": warmup,
           "ms_per_step": kms / steps, "candidates_per_s": sum(st["ext_cand"] for st in stats) * steps / (kms / 1e3),
           "result_lines": len(res.lines),
           "e2e": {"value": S * steps / (e0.elapsed_time(e1) / 1e3), "unit": UNIT,
                   "h2d_bytes_per_step": h2d // steps, "d2h_bytes_per_step": d2h // steps},
           "tuning": tune, "graphs_captured": caps, "graph_replays": replays,
           "gpu_launches_per_step": launches // steps, "clocks": clk}
    if compare:
        with Search(max(his) + 1, device=local, stream=stream.cuda_stream, kernel=compare) as o:
            otune = o.autotune(los, his, budget_s=4.0) if compare == "batched" else None
            ostats, ores = o.batch(los, his, want_lines=True)
            out["compare"] = {"kernel": compare, "value": S / (o.last_kernel_ms / 1e3), "unit": UNIT,
                              "ms_per_step": o.last_kernel_ms, "gpu_launches_per_step": o.last_launches,
                              "tuning": otune,
                              "identical": ostats == stats and sorted(zip(ores.items, ores.lines)) ==
                              sorted(zip(res.items, res.lines))}
    if cpu:
        out["cpu_baseline"] = config3_cpu_sample(los, his)
    return out


def run_subranges(args, local: int):
    """The batched uneven-subrange workload as its own line."""
    import torch
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    out = measure_subranges(local, stream, args.steps, args.warmup, cpu=not args.no_cpu_baseline)
    line = {"metric": METRIC, "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64", "data": "synthetic", **out}
    print(json.dumps(line), flush=True)


def run_serve(args, local: int):
    import torch
    torch.cuda.set_device(local)
    out = measure_serve(local, args.serve_requests, args.serve_rates)
    print(json.dumps({"metric": "serve_latency_p50_p99", **out}), flush=True)


# ------------------------------------------------------------------ our arm

def read_traffic_per_S(kernel: str):
    """DRAM bytes per S of one kernel, from its committed ncu summary."""
    p = REPO / "profiles" / f"ncu_{kernel}_5e9.txt"
    if not p.exists():
        return None
    m = re.search(r"^dram_bytes_per_S:\s*([\d.eE+-]+)", p.read_text(), re.M)
    return float(m.group(1)) if m else None


def read_issue_active(kernel: str):
    """Fraction of issue slots busy (smsp__issue_active) of one kernel, from its ncu summary."""
    p = REPO / "profiles" / f"ncu_{kernel}_5e9.txt"
    if not p.exists():
        return None
    m = re.search(r"issue slots busy \(smsp__issue_active\)\s+([\d.]+) %", p.read_text())
    return float(m.group(1)) / 100 if m else None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--kernel", choices=["batched", "plain", "fused", "persist"], default="batched")
    ap.add_argument("--ref-budget", type=float, default=12.0,
                    help="seconds of work per reference step when only the single-thread oracle port is built")
    ap.add_argument("--ref-slice", type=int, default=3 * 10 ** 8,
                    help="S per slice of the reference's s4 (4 slices, the same in the reference arm and the "
                         "bench line's cpu_baseline)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--workload", choices=["exhaustive", "subranges", "triples", "serve"], default="exhaustive",
                    help="exhaustive: the headline line (S < 1e10); the others print their own line")
    ap.add_argument("--serve-requests", type=int, default=10000)
    ap.add_argument("--serve-rates", type=lambda x: [float(v) for v in x.split(",")], default=[50.0, 120.0],
                    help="arrival rates (requests/s), comma-separated; the same requests at each")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-subranges", action="store_true")
    ap.add_argument("--subrange-steps", type=int, default=1)
    ap.add_argument("--no-triples", action="store_true")
    ap.add_argument("--range", type=int, nargs=2, default=None, metavar=("LO", "HI"),
                    help="search [LO, HI) instead of the rank's shard (a smaller case for ncu captures)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.workload != "exhaustive":
        import torch
        torch.cuda.set_device(local)
        if rank != 0:
            return
        if args.workload == "subranges":
            return run_subranges(args, local)
        if args.workload == "serve":
            return run_serve(args, local)
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        out = measure_triples(local, stream, steps=args.steps, warmup=args.warmup)
        print(json.dumps({"metric": "triples_per_s", **out}), flush=True)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from ps4b200 import Search, opmodel, shards

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    lo, hi = shard(rank, world) if args.range is None else tuple(args.range)
    # one dedicated stream carries the library's launches, the L2 flush and the timing events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    s = Search(hi, device=local, kernel=args.kernel, stream=stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    props = torch.cuda.get_device_properties(local)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        s.enqueue(lo, hi)
        s.finish(want_lines=False)
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(str(getattr(props, "uuid", "")))
    clocks.start()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kernel_ms, stats, launches = [], None, 0
    for i in range(args.steps):
        flush.zero_()                                  # L2 flush, outside the timed events
        ev[i][0].record(stream)
        s.enqueue(lo, hi)
        ev[i][1].record(stream)
        r = s.finish(want_lines=False)
        kernel_ms.append(r.kernel_ms)
        launches += s.last_launches
        stats = r.stats
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    dev_s = sum(a.elapsed_time(b) for a, b in ev) / 1000.0
    kern_s = sum(kernel_ms) / 1000.0
    S_rank = (hi - lo) * args.steps
    cand_rank = stats["ext_cand"] * args.steps
    ops_launch = opmodel.ops(stats)

    # e2e: the public C-ABI call with host buffers, input copy + result copies inside
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h2d = d2h = 0
    e2e_lines = 0
    for _ in range(args.steps):
        if args.range is None:             # the whole range: this rank's shard, results gathered
            rr, _ = shards.search_sharded(1, BOUND, rank=rank, world=world, dist=dist, search=s)
        else:
            rr = s.range(lo, hi)
        a_, b_ = s.transfer_bytes()
        h2d += a_
        d2h += b_
        e2e_lines = len(rr.lines)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_s = e0.elapsed_time(e1) / 1000.0

    # per-kernel split of one step (events around every launch, direct launches)
    with Search(hi, device=local, kernel=args.kernel, stream=stream.cuda_stream, time_kernels=True) as sk:
        sk.enqueue(lo, hi)
        sk.finish(want_lines=False)
        flush.zero_()
        sk.enqueue(lo, hi)
        sk.finish(want_lines=False)
        gen_ms, ext_ms = sk.last_kernel_split

    (dev_s, e2e_s, kern_s), (S_all, cand_all) = aggregate(dist, world, [dev_s, e2e_s, kern_s],
                                                          [S_rank, cand_rank], "cuda")

    def other_kernel(kernel: str, warm: bool) -> dict:
        """One timed step of [lo, hi) on another kernel choice, results checked against ours."""
        with Search(hi, device=local, kernel=kernel, stream=stream.cuda_stream) as sp:
            if warm:
                sp.enqueue(lo, hi)
                sp.finish(want_lines=False)
            flush.zero_()
            pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            pe0.record(stream)
            sp.enqueue(lo, hi)
            pe1.record(stream)
            pr = sp.finish(want_lines=False)
            torch.cuda.synchronize()
            assert pr.stats == stats, f"{kernel} and batched kernels disagree"
            pt = pe0.elapsed_time(pe1) / 1000.0
        return {"value": (hi - lo) / pt, "unit": UNIT, "ms_per_step": 1000 * pt,
                "batched_over_" + kernel: ((hi - lo) / (dev_s / args.steps)) / ((hi - lo) / pt)}

    plain = fused = None
    if world == 1 and args.kernel == "batched" and not args.no_plain:
        plain = other_kernel("plain", warm=False)       # one thread per S: 28 s, no warm-up needed
        fused = other_kernel("fused", warm=True)        # tiles, staging and per-lane extension in one kernel

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        binary, kind, threads, slices = cpu_sample_plan(lo, hi, budget_s=4.0, slice_w=args.ref_slice)
        secs, n = cpu_sample_run(binary, kind, threads, slices)
        cpu = {"value": n / secs, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{len(slices)} slices of {slices[0][1] - slices[0][0]} S at the midpoints of 4 equal "
                         f"parts of [1,1e10), slowest region thread's own timer"}

    triples = serving = subranges = None
    if rank == 0 and world == 1 and args.range is None:
        if not args.no_triples:
            triples = measure_triples(local, stream)
        if not args.no_subranges:
            subranges = measure_subranges(local, stream, args.subrange_steps, 1, cpu=not args.no_cpu_baseline)
        if not args.no_serve:
            serving = measure_serve(local, args.serve_requests, args.serve_rates)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    sm_hz = (clk["sm_mhz"] or 1965.0) * 1e6
    peak = opmodel.issue_peak_lane_ops(props.multi_processor_count, sm_hz)
    achieved_step = ops_launch / (kern_s / args.steps)
    ops_gen, ops_ext = opmodel.ops_split(stats)
    kernels = {
        "gen_jobs": {"ms_per_step": gen_ms, "ops_per_step": ops_gen,
                     "achieved": ops_gen / (gen_ms / 1e3) if gen_ms else None,
                     "traffic_per_step": (read_traffic_per_S("gen_jobs") or 0) * (hi - lo) or None},
        "extend_jobs": {"ms_per_step": ext_ms, "ops_per_step": ops_ext,
                        "achieved": ops_ext / (ext_ms / 1e3) if ext_ms else None,
                        "traffic_per_step": (read_traffic_per_S("extend_jobs") or 0) * (hi - lo) or None},
    }
    for name, k in kernels.items():
        k["frac"] = k["achieved"] / peak if k["achieved"] else None
        k["issue_active_ncu"] = read_issue_active(name)
    dom = "extend_jobs" if ext_ms >= gen_ms else "gen_jobs"
    line = {
        "metric": METRIC, "value": S_all / dev_s, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * dev_s / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "exhaustive",
        "config": {"workload": "exhaustive square-sum 4-set search + extension, S in [1,1e10) (s4 bound 1e10)"
                               + (f", {world} cost-balanced contiguous S shards, one per GPU" if world > 1 else ""),
                   "bound": BOUND, "shard": [lo, hi], "kernel": args.kernel,
                   "l2": "256 MiB write between timed steps", "parallelism": f"S shards x{world}"},
        "candidates_per_s": cand_all / dev_s,
        "sets4_per_s": stats["sets4"] * world * args.steps / dev_s,
        "kernel_ms_per_step": 1000 * kern_s / args.steps,
        "roofline": {"bound": "int_issue", "kernel": dom, "achieved": kernels[dom]["achieved"], "peak": peak,
                     "unit": "lane-op/s", "frac": kernels[dom]["frac"],
                     "peak_source": f"{props.multi_processor_count} SMs x 128 lanes x median SM clock under load "
                                    f"({sm_hz / 1e6:.0f} MHz sampled); " +
                                    ("MEASURED_PEAKS.json has no integer peak" if (REPO / "MEASURED_PEAKS.json").exists()
                                     else "no MEASURED_PEAKS.json on this box"),
                     "per": "step (all launches of the kernel in one search of the range; a step is "
                            f"{launches // max(args.steps, 1) // 2} batches)",
                     "ops": kernels[dom]["ops_per_step"], "traffic": kernels[dom]["traffic_per_step"],
                     "issue_active_ncu": kernels[dom]["issue_active_ncu"],
                     "issue_active_source": f"profiles/ncu_{dom}_5e9.txt (5e8-S capture at S = 5e9)",
                     "step_achieved": achieved_step, "step_frac": achieved_step / peak,
                     "kernels": kernels},
        "e2e": {"value": S_all / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps, "result_lines": e2e_lines},
        "gpu_launches": launches,
        "clocks": clk,
        "plain_gpu": plain,
        "fused_gpu": fused,
        "cpu_baseline": cpu,
        "triples": triples,
        "subranges": subranges,
        "serving": serving,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
