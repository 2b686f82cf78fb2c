"""Python face of the search: one object per device context, mirroring the reference's
process interface (exhaustive/s4.c) as calls.

``Search(s_hi_max).range(lo, hi)`` returns what one ``s4 lo hi`` invocation reports: the
counters of its TOTAL / CAPACITY lines (s4.c:498-506) and its result lines (s4.c:24-27),
byte-identical in text.  Every call goes through the C-ABI of lib/libps4.so; the numbers
are computed on the GPU only.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

from . import _abi

_LINE_CAP = 1 << 16


class Ps4Error(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


@dataclass
class RangeResult:
    stats: dict
    lines: list = field(default_factory=list)      # "M:" and "5:" lines, reference order
    six_lines: list = field(default_factory=list)  # "!!!!!!!! FOUND 6-SET:" alert lines
    quads: list = field(default_factory=list)      # "4:" lines (dump4 mode)
    items: list = field(default_factory=list)      # item index of each entry of `lines`
    kernel_ms: float = 0.0


def _alloc(kind, n):
    n = max(int(n), 1)
    return (kind * n)(), n


class Search:
    """A device context (tables for S < s_hi_max) and its search calls."""

    def __init__(self, s_hi_max: int, device: int = 0, *, noext: bool = False, verify: bool = False,
                 dump4: bool = False, kernel: str = "batched", cap_reps: int = 0, cap_divs: int = 0,
                 cap_ext: int = 0, log2_tile: int = 0, ctas_per_sm: int = 0, stream: int | None = None,
                 graph: str = "auto", time_kernels: bool = False):
        self.lib = _abi.load()
        cfg = _abi.Config()
        cfg.device = device
        cfg.s_hi_max = int(s_hi_max)
        cfg.cap_reps, cfg.cap_divs, cfg.cap_ext = cap_reps, cap_divs, cap_ext
        cfg.flags = ((_abi.PS4_F_NOEXT if noext else 0) | (_abi.PS4_F_VERIFY if verify else 0)
                     | (_abi.PS4_F_DUMP4 if dump4 else 0))
        cfg.kernel = {"batched": _abi.PS4_KERNEL_BATCHED, "plain": _abi.PS4_KERNEL_PLAIN,
                      "fused": _abi.PS4_KERNEL_FUSED, "persist": _abi.PS4_KERNEL_PERSIST}[kernel]
        cfg.log2_tile = log2_tile
        cfg.ctas_per_sm = ctas_per_sm
        cfg.stream = stream
        cfg.use_graph = {"auto": _abi.PS4_GRAPH_AUTO, "always": _abi.PS4_GRAPH_ALWAYS,
                         "never": _abi.PS4_GRAPH_NEVER}[graph]
        cfg.time_kernels = 1 if time_kernels else 0
        self.dump4 = dump4
        self.ctx = C.c_void_p()
        rc = self.lib.ps4_create(C.byref(cfg), C.byref(self.ctx))
        if rc != _abi.PS4_OK:
            msg = self.lib.ps4_last_error(self.ctx).decode() if self.ctx else "ps4_create failed"
            self.close()
            raise Ps4Error(rc, msg)
        self._res = _abi.Results()
        self._hits, self._res.hits_cap = _alloc(_abi.Hit, 1 << 12)
        self._exts, self._res.exts_cap = _alloc(_abi.Ext, 1 << 13)
        self._sixes, self._res.sixes_cap = _alloc(_abi.Six, 64)
        self._quads, self._res.quads_cap = _alloc(_abi.Quad, (1 << 16) if dump4 else 1)
        self._bind()

    def _bind(self):
        r = self._res
        r.hits = C.cast(self._hits, C.POINTER(_abi.Hit))
        r.exts = C.cast(self._exts, C.POINTER(_abi.Ext))
        r.sixes = C.cast(self._sixes, C.POINTER(_abi.Six))
        r.quads = C.cast(self._quads, C.POINTER(_abi.Quad))
        if not self.dump4:
            r.quads_cap = 0

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.ps4_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def last_kernel_ms(self) -> float:
        return float(self.lib.ps4_last_kernel_ms(self.ctx))

    @property
    def last_launches(self) -> int:
        return int(self.lib.ps4_last_launches(self.ctx))

    def _grow(self):
        r = self._res
        if r.n_hits > r.hits_cap:
            self._hits, r.hits_cap = _alloc(_abi.Hit, r.n_hits * 3 // 2)
        if r.n_exts > r.exts_cap:
            self._exts, r.exts_cap = _alloc(_abi.Ext, r.n_exts * 3 // 2)
        if r.n_sixes > r.sixes_cap:
            self._sixes, r.sixes_cap = _alloc(_abi.Six, r.n_sixes * 3 // 2)
        if self.dump4 and r.n_quads > r.quads_cap:
            self._quads, r.quads_cap = _alloc(_abi.Quad, r.n_quads * 3 // 2)
        self._bind()

    def _reserve(self, width: int):
        """Host result buffers for a call of this many S (as the library sizes its own)."""
        need = 1024 + int(2e-5 * width)
        r = self._res
        if need > r.hits_cap:
            self._hits, r.hits_cap = _alloc(_abi.Hit, need)
        if 2 * need > r.exts_cap:
            self._exts, r.exts_cap = _alloc(_abi.Ext, 2 * need)
        self._bind()

    def _call(self, fn):
        while True:
            rc = fn()
            if rc == _abi.PS4_ERR_OUTPUT_FULL:
                self._grow()
                continue
            if rc != _abi.PS4_OK:
                raise Ps4Error(rc, self.lib.ps4_last_error(self.ctx).decode())
            return

    def range(self, lo: int, hi: int, *, want_lines: bool = True) -> RangeResult:
        """Every S in [lo, hi): counters and result lines (one reference invocation)."""
        self._reserve(max(hi - lo, 0))
        st = _abi.Stats()
        self._call(lambda: self.lib.ps4_search_range(self.ctx, lo, hi, C.byref(st), C.byref(self._res)))
        out = RangeResult(stats=st.as_dict(), kernel_ms=self.last_kernel_ms)
        if want_lines:
            self._collect(out)
        return out

    def enqueue(self, lo: int, hi: int) -> None:
        """Start a search of [lo, hi) on the context's stream and return at once."""
        rc = self.lib.ps4_search_enqueue(self.ctx, lo, hi)
        if rc != _abi.PS4_OK:
            raise Ps4Error(rc, self.lib.ps4_last_error(self.ctx).decode())

    def finish(self, *, want_lines: bool = True) -> RangeResult:
        """Wait for the enqueued search and collect it like ``range``."""
        st = _abi.Stats()
        self._call(lambda: self.lib.ps4_search_finish(self.ctx, C.byref(st), C.byref(self._res)))
        out = RangeResult(stats=st.as_dict(), kernel_ms=self.last_kernel_ms)
        if want_lines:
            self._collect(out)
        return out

    def autotune(self, los, his, budget_s: float = 2.0) -> dict:
        """Time launch shapes on a sample of the workload; the fastest stays on the context."""
        n = len(los)
        lo_arr = (C.c_uint64 * n)(*los)
        hi_arr = (C.c_uint64 * n)(*his)
        t = _abi.Tuning()
        self._call(lambda: self.lib.ps4_autotune(self.ctx, lo_arr, hi_arr, n, budget_s, C.byref(t)))
        return t.as_dict()

    @property
    def tuning(self) -> dict:
        t = _abi.Tuning()
        self.lib.ps4_get_tuning(self.ctx, C.byref(t))
        return t.as_dict()

    @tuning.setter
    def tuning(self, d: dict) -> None:
        t = _abi.Tuning(d["log2_tile"], d["gen_ctas"], d["ext_ctas"], d["log2_jobs"], d.get("rate", 0.0))
        self._call(lambda: self.lib.ps4_set_tuning(self.ctx, C.byref(t)))

    @property
    def last_kernel_split(self) -> tuple[float, float]:
        """(tile kernel ms, extension engine ms) of the last call (needs time_kernels=True)."""
        g, x = C.c_double(), C.c_double()
        self.lib.ps4_last_kernel_split(self.ctx, C.byref(g), C.byref(x))
        return float(g.value), float(x.value)

    def graph_counts(self) -> tuple[int, int]:
        """(CUDA graphs captured, graph replays) on this context so far."""
        a, b = C.c_uint64(), C.c_uint64()
        self.lib.ps4_graph_counts(self.ctx, C.byref(a), C.byref(b))
        return int(a.value), int(b.value)

    def transfer_bytes(self) -> tuple[int, int]:
        h2d, d2h = C.c_uint64(), C.c_uint64()
        self.lib.ps4_last_transfer_bytes(self.ctx, C.byref(h2d), C.byref(d2h))
        return int(h2d.value), int(d2h.value)

    def batch(self, los, his, *, want_lines: bool = True):
        """Many subranges in one launch: (per-item stats list, RangeResult with item tags)."""
        n = len(los)
        lo_arr = (C.c_uint64 * n)(*los)
        hi_arr = (C.c_uint64 * n)(*his)
        self._reserve(sum(max(int(b) - int(a), 0) for a, b in zip(los, his)))
        st = (_abi.Stats * n)()
        self._call(lambda: self.lib.ps4_search_batch(self.ctx, lo_arr, hi_arr, n, st, C.byref(self._res)))
        out = RangeResult(stats={}, kernel_ms=self.last_kernel_ms)
        if want_lines:
            self._collect(out)
        return [s.as_dict() for s in st], out

    def extend_triples(self, abc, dmax: int, *, as_lists: bool = True):
        """Every d <= dmax extending each square-sum triple (rows of ``abc``) to a 4-set.

        Returns (exts, state, stats): exts[i] the sorted extensions of triple i, state[i] 0 for
        a searched triple and 1 for a row that is not a square-sum triple of distinct positive
        integers, stats the call's counters.  With as_lists=False exts is the record array
        (fields d, item) sorted by (item, d) instead of per-triple lists."""
        import numpy as np
        a = abc if (isinstance(abc, np.ndarray) and abc.dtype == np.uint64 and abc.flags.c_contiguous
                    and abc.ndim == 2) else np.ascontiguousarray(np.asarray(abc, dtype=np.uint64).reshape(-1, 3))
        n = a.shape[0]
        state = np.zeros(max(n, 1), dtype=np.uint8)
        cap = max(self._tri_cap, 1024) if hasattr(self, "_tri_cap") else 1 << 16
        st = _abi.TriStats()
        while True:
            out = self._tri_buf if getattr(self, "_tri_buf", None) is not None and len(self._tri_buf) >= cap \
                else (_abi.TriExt * cap)()
            self._tri_buf = out
            cap = len(out)
            n_out = C.c_uint64()
            rc = self.lib.ps4_extend_triples(self.ctx, a.ctypes.data, n, int(dmax), state.ctypes.data, out, cap,
                                             C.byref(n_out), C.byref(st))
            if rc == _abi.PS4_ERR_OUTPUT_FULL:
                cap = int(n_out.value) * 3 // 2 + 1024
                continue
            if rc != _abi.PS4_OK:
                raise Ps4Error(rc, self.lib.ps4_last_error(self.ctx).decode())
            break
        self._tri_cap = cap
        recs = np.frombuffer(out, dtype=np.dtype([("d", "<u8"), ("item", "<u4"), ("reserved", "<u4")]),
                             count=int(n_out.value))
        if not as_lists:
            return recs.copy(), state[:n], st.as_dict()
        exts = [[] for _ in range(n)]
        for d, item in zip(recs["d"].tolist(), recs["item"].tolist()):
            exts[item].append(d)
        return exts, state[:n], st.as_dict()

    def _collect(self, out: RangeResult):
        r = self._res
        buf = C.create_string_buffer(_LINE_CAP)
        if r.n_hits:
            # every hit's lines in one call (ps4_format_hits), grown once if the estimate is short
            # (the text buffer is kept between calls and only the bytes written are copied out)
            cap = max(1 << 16, 160 * r.n_hits + 48 * r.n_exts)
            items = (C.c_uint32 * (r.n_hits + r.n_exts))()
            nl = C.c_uint64()
            for _ in range(2):
                if getattr(self, "_fmt_cap", 0) < cap:
                    self._fmt_buf, self._fmt_cap = C.create_string_buffer(cap), cap
                n = self.lib.ps4_format_hits(self._hits, r.n_hits, self._exts, self._fmt_buf, self._fmt_cap, items,
                                             C.byref(nl))
                if n >= 0:
                    break
                if n == -1:
                    raise Ps4Error(_abi.PS4_ERR_ARG, "a hit formats to more than 8 KB")
                cap = -n
            out.lines.extend(C.string_at(self._fmt_buf, n).decode().splitlines(keepends=True))
            out.items.extend(items[:nl.value])
        for s in range(r.n_sixes):
            six = self._sixes[s]
            n = self.lib.ps4_format_six(C.byref(self._hits[six.hit]), self._exts, C.byref(six), buf, _LINE_CAP)
            if n > 0:
                out.six_lines.append(buf.value.decode())
        if self.dump4:
            for q in range(r.n_quads):
                n = self.lib.ps4_format_quad(C.byref(self._quads[q]), buf, _LINE_CAP)
                if n > 0:
                    out.quads.append(buf.value.decode())
