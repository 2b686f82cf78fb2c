"""Python face of the serving loop (ps4_serve_* in include/ps4.h).

``Server(search)`` wraps a device server on a ``Search`` context; ``run_stream`` replays a
request stream (``workloads.requests``) against it in real time -- each request submitted at
its arrival time, the server driven in between -- and reports per-request latency.  All
scheduling, admission and device work happen in the library; this module only feeds requests
and collects results.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .search import Ps4Error, RangeResult, Search, _alloc


class ServeConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_uint64), ("max_slots", C.c_uint32), ("max_step_items", C.c_uint32),
                ("step_S", C.c_uint64), ("max_step_triples", C.c_uint32), ("hits_floor", C.c_uint32),
                ("hits_per_1e6_S", C.c_uint32), ("reserved", C.c_uint32)]


class ServeDone(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int32), ("kind", C.c_uint32), ("n_records", C.c_uint64),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double), ("steps", C.c_uint32),
                ("reruns", C.c_uint32), ("message", C.c_char * 160)]


class ServeInfo(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "waiting", "active", "finished", "steps", "step_reruns",
                                          "arena_bytes", "arena_used", "arena_peak", "device_bytes")] + [
        ("gpu_ms", C.c_double)]


_declared = False


def _declare(lib):
    global _declared
    if _declared:
        return
    P = C.POINTER
    sig = {
        "ps4_serve_create": (C.c_int, [C.c_void_p, P(ServeConfig), P(C.c_void_p)]),
        "ps4_serve_destroy": (None, [C.c_void_p]),
        "ps4_serve_last_error": (C.c_char_p, [C.c_void_p]),
        "ps4_serve_submit_range": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64]),
        "ps4_serve_submit_triple": (C.c_int, [C.c_void_p, C.c_uint64, P(C.c_uint64), C.c_uint64]),
        "ps4_serve_progress": (C.c_int, [C.c_void_p, C.c_uint32, P(ServeDone), C.c_uint32, P(C.c_uint32)]),
        "ps4_serve_take_range": (C.c_int, [C.c_void_p, C.c_uint64, P(_abi.Stats), P(_abi.Results)]),
        "ps4_serve_take_triple": (C.c_int, [C.c_void_p, C.c_uint64, P(C.c_uint8), P(_abi.TriExt), C.c_uint64,
                                            P(C.c_uint64), P(_abi.TriStats)]),
        "ps4_serve_get_info": (None, [C.c_void_p, P(ServeInfo)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _declared = True


class Server:
    """A device server on the tables of ``search`` (which must outlive it)."""

    def __init__(self, search: Search, *, hbm_budget: int = 0, max_slots: int = 0, max_step_items: int = 0,
                 step_S: int = 0, max_step_triples: int = 0, hits_floor: int = 0, hits_per_1e6_S: int = 0):
        self.search = search
        self.lib = search.lib
        _declare(self.lib)
        cfg = ServeConfig(hbm_budget, max_slots, max_step_items, step_S, max_step_triples, hits_floor,
                          hits_per_1e6_S, 0)
        self.srv = C.c_void_p()
        rc = self.lib.ps4_serve_create(search.ctx, C.byref(cfg), C.byref(self.srv))
        if rc != _abi.PS4_OK:
            msg = self.lib.ps4_serve_last_error(self.srv).decode()
            self.close()
            raise Ps4Error(rc, msg)
        self._done = (ServeDone * 256)()
        self._tri_out = (_abi.TriExt * 64)()

    def close(self):
        if getattr(self, "srv", None):
            self.lib.ps4_serve_destroy(self.srv)
            self.srv = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != _abi.PS4_OK:
            raise Ps4Error(rc, self.lib.ps4_serve_last_error(self.srv).decode())

    def submit_range(self, tag: int, lo: int, hi: int) -> None:
        self._check(self.lib.ps4_serve_submit_range(self.srv, tag, lo, hi))

    def submit_triple(self, tag: int, abc, dmax: int) -> None:
        arr = (C.c_uint64 * 3)(*[int(v) for v in abc])
        self._check(self.lib.ps4_serve_submit_triple(self.srv, tag, arr, int(dmax)))

    def progress(self, wait_us: int = 0) -> list[dict]:
        """Drive the server; returns the queries that finished (tag, status, times ...)."""
        n = C.c_uint32()
        self._check(self.lib.ps4_serve_progress(self.srv, int(wait_us), self._done, len(self._done), C.byref(n)))
        out = []
        for i in range(n.value):
            d = self._done[i]
            out.append({"tag": int(d.tag), "status": int(d.status), "kind": int(d.kind),
                        "n_records": int(d.n_records), "t_submit": d.t_submit, "t_admit": d.t_admit,
                        "t_done": d.t_done, "steps": int(d.steps), "reruns": int(d.reruns),
                        "message": d.message.decode()})
        return out

    def take_range(self, tag: int) -> RangeResult:
        """Counters and result lines of a finished subrange query (as ``Search.range``)."""
        s = self.search
        st = _abi.Stats()
        while True:
            rc = self.lib.ps4_serve_take_range(self.srv, tag, C.byref(st), C.byref(s._res))
            if rc == _abi.PS4_ERR_OUTPUT_FULL:
                s._grow()
                continue
            self._check(rc)
            break
        out = RangeResult(stats=st.as_dict())
        s._collect(out)
        return out

    def take_triple(self, tag: int):
        """(sorted extensions, state, stats) of a finished triple query (as ``Search.extend_triples``)."""
        st = _abi.TriStats()
        state = C.c_uint8()
        n = C.c_uint64()
        while True:
            rc = self.lib.ps4_serve_take_triple(self.srv, tag, C.byref(state), self._tri_out, len(self._tri_out),
                                                C.byref(n), C.byref(st))
            if rc == _abi.PS4_ERR_OUTPUT_FULL:
                self._tri_out = (_abi.TriExt * (int(n.value) * 2))()
                continue
            self._check(rc)
            break
        return [int(self._tri_out[i].d) for i in range(n.value)], int(state.value), st.as_dict()

    def info(self) -> dict:
        i = ServeInfo()
        self.lib.ps4_serve_get_info(self.srv, C.byref(i))
        return {n: (float(getattr(i, n)) if n == "gpu_ms" else int(getattr(i, n))) for n, _ in i._fields_}


@dataclass
class StreamReport:
    latency_s: dict = field(default_factory=dict)     # rid -> seconds from arrival to finish
    done: dict = field(default_factory=dict)          # rid -> the finish record (steps, reruns, times)
    results: dict = field(default_factory=dict)       # rid -> RangeResult / (exts, state, stats) / Ps4Error
    wall_s: float = 0.0
    info: dict = field(default_factory=dict)

    def percentile(self, p: float) -> float:
        return float(np.percentile(np.array(list(self.latency_s.values())), p))


def run_stream(server: Server, reqs, *, collect: bool = True, max_wait_us: int = 2000) -> StreamReport:
    """Replay ``reqs`` (sorted by arrival) in real time: submit each at t0 + t_arrive, drive the
    server in between, take every result as it finishes.  Latency is finish time minus the
    scheduled arrival (CLOCK_MONOTONIC on both sides), so time the loop spends elsewhere counts."""
    rep = StreamReport()
    by_tag = {r.rid: r for r in reqs}
    n = len(reqs)
    i = 0
    finished = 0
    t0 = time.monotonic()
    while finished < n:
        now = time.monotonic() - t0
        while i < n and reqs[i].t_arrive <= now:
            r = reqs[i]
            if r.kind == "range":
                server.submit_range(r.rid, r.lo, r.hi)
            else:
                server.submit_triple(r.rid, r.abc, r.dmax)
            i += 1
        wait = max_wait_us
        if i < n:
            wait = int(max(0.0, min(max_wait_us * 1e-6, reqs[i].t_arrive - (time.monotonic() - t0))) * 1e6)
        for d in server.progress(wait):
            r = by_tag[d["tag"]]
            rep.latency_s[r.rid] = d["t_done"] - (t0 + r.t_arrive)
            rep.done[r.rid] = d
            finished += 1
            if d["status"] != _abi.PS4_OK:
                try:
                    (server.take_range if r.kind == "range" else server.take_triple)(r.rid)
                except Ps4Error as e:
                    rep.results[r.rid] = e
                continue
            if r.kind == "range":
                res = server.take_range(r.rid)
                rep.results[r.rid] = res if collect else res.stats
            else:
                rep.results[r.rid] = server.take_triple(r.rid)
        if i < n and not server.info()["active"] and not server.info()["waiting"]:
            gap = reqs[i].t_arrive - (time.monotonic() - t0)
            if gap > 0:
                time.sleep(min(gap, 0.002))
    rep.wall_s = time.monotonic() - t0
    rep.info = server.info()
    return rep
