"""ctypes wrapper of the CPU restatement (oracle/libps4oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg as the checker.  Never imported by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "libps4oracle.so"
REF_S4 = HERE / "_ref" / "s4"

COUNTERS = ("S_done", "pairs", "S_ge3", "triples", "sets4", "sets5", "sets6", "multi", "ext_cand", "ext_sqrt")
NOEXT, VERIFY, TEST6 = 1, 2, 4


class _Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in COUNTERS] + [
        ("hist5", C.c_uint64 * 100), ("max_reps", C.c_uint64), ("max_divisors", C.c_uint64),
        ("max_extensions", C.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"{LIB} missing: run `make -C {HERE}`")
        _lib = C.CDLL(str(LIB))
        _lib.orc_search.restype = C.c_int
        _lib.orc_search.argtypes = [C.c_uint64, C.c_uint64, C.c_uint, C.c_long, C.c_int, C.c_uint, C.c_uint,
                                    C.c_uint, C.c_char_p, C.POINTER(_Stats), C.c_char_p, C.c_size_t]
        _lib.orc_isqrt128.restype = C.c_uint64
        _lib.orc_isqrt128.argtypes = [C.c_uint64, C.c_uint64]
        _lib.orc_is_square128.restype = C.c_int
        _lib.orc_is_square128.argtypes = [C.c_uint64, C.c_uint64]
        _lib.orc_extend_triple.restype = C.c_long
        _lib.orc_extend_triple.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                           C.POINTER(C.c_uint64), C.c_long]
    return _lib


def stats_dict(st: _Stats) -> dict:
    d = {n: int(getattr(st, n)) for n in COUNTERS}
    d["hist5"] = {i: int(v) for i, v in enumerate(st.hist5) if v}
    d["max_reps"] = int(st.max_reps)
    d["max_divisors"] = int(st.max_divisors)
    d["max_extensions"] = int(st.max_extensions)
    return d


def search(lo: int, hi: int, *, dump4: int = 0, flags: int = 0, chunk_log2: int = 20,
           cap_reps: int = 0, cap_divs: int = 0, cap_ext: int = 0):
    """(rc, stats, lines, err): the oracle's run over [lo, hi)."""
    st = _Stats()
    err = C.create_string_buffer(512)
    fd, path = tempfile.mkstemp(prefix="orc_", suffix=".out")
    os.close(fd)
    try:
        rc = lib().orc_search(lo, hi, chunk_log2, dump4, flags, cap_reps, cap_divs, cap_ext,
                              path.encode(), C.byref(st), err, 512)
        lines = Path(path).read_text().splitlines(keepends=True)
    finally:
        os.unlink(path)
    return rc, stats_dict(st), lines, err.value.decode()


def isqrt128(n: int) -> int:
    return int(lib().orc_isqrt128(n >> 64, n & (2**64 - 1)))


def is_square128(n: int) -> bool:
    return bool(lib().orc_is_square128(n >> 64, n & (2**64 - 1)))


def extend_triple(a: int, b: int, c: int, dmax: int, cap: int = 4096) -> list[int]:
    out = (C.c_uint64 * cap)()
    n = lib().orc_extend_triple(a, b, c, dmax, out, cap)
    if n < 0:
        raise ValueError("not a square-sum triple")
    if n > cap:
        return extend_triple(a, b, c, dmax, n)
    return [int(out[i]) for i in range(n)]
