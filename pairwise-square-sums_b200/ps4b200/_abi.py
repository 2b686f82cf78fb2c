"""ctypes mirror of include/ps4.h (the C-ABI of lib/libps4.so).

The library is built in-tree (``make -C pairwise-square-sums_b200``).  Loading fails loudly
when it is missing: there is no CPU implementation behind this package.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent.parent          # pairwise-square-sums_b200/
LIB_PATH = PKG_ROOT / "lib" / "libps4.so"
CLI_PATH = PKG_ROOT / "bin" / "s4gpu"
HEADER_PATH = PKG_ROOT.parent / "include" / "ps4.h"

PS4_OK = 0
PS4_ERR_ARG = 1
PS4_ERR_CUDA = 3
PS4_ERR_CAP_REPS = 10
PS4_ERR_CAP_DIVS = 11
PS4_ERR_CAP_EXT = 12
PS4_ERR_VERIFY = 13
PS4_ERR_CAP_INTERNAL = 14
PS4_ERR_OUTPUT_FULL = 20
PS4_ERR_TIMEOUT = 21

# fixed result buffers of ps4_search_range_noalloc
PS4_NOALLOC_MAX_HITS = 65536
PS4_NOALLOC_MAX_EXTS = 131072
PS4_NOALLOC_MAX_SIXES = 256

PS4_F_NOEXT = 1
PS4_F_VERIFY = 2
PS4_F_DUMP4 = 4

PS4_KERNEL_BATCHED = 0
PS4_KERNEL_PLAIN = 1
PS4_KERNEL_FUSED = 2
PS4_KERNEL_PERSIST = 3

PS4_GRAPH_AUTO = 0
PS4_GRAPH_ALWAYS = 1
PS4_GRAPH_NEVER = 2

PS4_HIT_MULTI = 1
PS4_HIT_DRILL_OK = 2
PS4_EXT_FIVE = 1
PS4_EXT_FIVE_OK = 2

COUNTER_NAMES = ("S_done", "pairs", "S_ge3", "triples", "sets4", "sets5", "sets6", "multi",
                 "ext_cand", "ext_sqrt")


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("s_hi_max", C.c_uint64), ("cap_reps", C.c_uint32),
                ("cap_divs", C.c_uint32), ("cap_ext", C.c_uint32), ("flags", C.c_uint32),
                ("kernel", C.c_uint32), ("log2_tile", C.c_uint32), ("ctas_per_sm", C.c_uint32),
                ("stream", C.c_void_p), ("use_graph", C.c_uint32), ("time_kernels", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("log2_tile", C.c_uint32), ("gen_ctas", C.c_uint32), ("ext_ctas", C.c_uint32),
                ("log2_jobs", C.c_uint32), ("rate", C.c_double)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in COUNTER_NAMES] + [
        ("hist5", C.c_uint64 * 100), ("max_reps", C.c_uint64), ("max_divisors", C.c_uint64),
        ("max_extensions", C.c_uint64)]

    def as_dict(self) -> dict:
        d = {n: int(getattr(self, n)) for n in COUNTER_NAMES}
        d["hist5"] = {i: int(v) for i, v in enumerate(self.hist5) if v}
        d["max_reps"] = int(self.max_reps)
        d["max_divisors"] = int(self.max_divisors)
        d["max_extensions"] = int(self.max_extensions)
        return d


class Hit(C.Structure):
    _fields_ = [("S", C.c_uint64), ("v", C.c_uint64 * 4), ("n_ext", C.c_uint32), ("first_ext", C.c_uint32),
                ("flags", C.c_uint32), ("item", C.c_uint32), ("order", C.c_uint32 * 4)]


class Ext(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_uint64), ("key", C.c_uint32), ("flags", C.c_uint32)]


class Six(C.Structure):
    _fields_ = [("hit", C.c_uint32), ("t", C.c_uint32), ("s", C.c_uint32), ("flags", C.c_uint32)]


class Quad(C.Structure):
    _fields_ = [("r_ab", C.c_uint32), ("r_ac", C.c_uint32), ("r_ad", C.c_uint32), ("r_bc", C.c_uint32),
                ("r_bd", C.c_uint32), ("r_cd", C.c_uint32)]


class TriExt(C.Structure):
    _fields_ = [("d", C.c_uint64), ("item", C.c_uint32), ("reserved", C.c_uint32)]


class TriStats(C.Structure):
    _fields_ = [("triples", C.c_uint64), ("invalid", C.c_uint64), ("ext_cand", C.c_uint64),
                ("ext_sqrt", C.c_uint64), ("exts", C.c_uint64)]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class Results(C.Structure):
    _fields_ = [("hits", C.POINTER(Hit)), ("hits_cap", C.c_uint64), ("n_hits", C.c_uint64),
                ("exts", C.POINTER(Ext)), ("exts_cap", C.c_uint64), ("n_exts", C.c_uint64),
                ("sixes", C.POINTER(Six)), ("sixes_cap", C.c_uint64), ("n_sixes", C.c_uint64),
                ("quads", C.POINTER(Quad)), ("quads_cap", C.c_uint64), ("n_quads", C.c_uint64)]


_lib = None


def load() -> C.CDLL:
    """Load lib/libps4.so once and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_ROOT}` "
                           "(the search has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    P = C.POINTER
    sig = {
        "ps4_abi_version": (C.c_int, []),
        "ps4_create": (C.c_int, [P(Config), P(C.c_void_p)]),
        "ps4_destroy": (None, [C.c_void_p]),
        "ps4_last_error": (C.c_char_p, [C.c_void_p]),
        "ps4_last_kernel_ms": (C.c_double, [C.c_void_p]),
        "ps4_last_launches": (C.c_uint64, [C.c_void_p]),
        "ps4_search_range": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, P(Stats), P(Results)]),
        "ps4_search_batch": (C.c_int, [C.c_void_p, P(C.c_uint64), P(C.c_uint64), C.c_uint32, P(Stats),
                                       P(Results)]),
        "ps4_search_range_noalloc": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, P(Stats), P(Results)]),
        "ps4_search_enqueue": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64]),
        "ps4_plan_shards": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint32, P(C.c_uint64)]),
        "ps4_check_ring_wait": (C.c_int, [C.c_int, P(C.c_uint64)]),
        "ps4_check_roots": (C.c_int, [C.c_int, P(C.c_uint64), P(C.c_uint64), C.c_uint32, P(C.c_uint64),
                                      P(C.c_uint32)]),
        "ps4_search_finish": (C.c_int, [C.c_void_p, P(Stats), P(Results)]),
        "ps4_last_transfer_bytes": (None, [C.c_void_p, P(C.c_uint64), P(C.c_uint64)]),
        "ps4_extend_triples": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p,
                                         C.c_uint64, P(C.c_uint64), P(TriStats)]),
        "ps4_autotune": (C.c_int, [C.c_void_p, P(C.c_uint64), P(C.c_uint64), C.c_uint32, C.c_double, P(Tuning)]),
        "ps4_set_tuning": (C.c_int, [C.c_void_p, P(Tuning)]),
        "ps4_get_tuning": (None, [C.c_void_p, P(Tuning)]),
        "ps4_graph_counts": (None, [C.c_void_p, P(C.c_uint64), P(C.c_uint64)]),
        "ps4_last_kernel_split": (None, [C.c_void_p, P(C.c_double), P(C.c_double)]),
        "ps4_format_hit": (C.c_long, [P(Hit), P(Ext), C.c_char_p, C.c_size_t]),
        "ps4_format_hits": (C.c_long, [P(Hit), C.c_uint64, P(Ext), C.c_char_p, C.c_size_t, P(C.c_uint32),
                                       P(C.c_uint64)]),
        "ps4_format_six": (C.c_long, [P(Hit), P(Ext), P(Six), C.c_char_p, C.c_size_t]),
        "ps4_format_drill": (C.c_long, [P(Hit), P(Ext), C.c_char_p, C.c_size_t]),
        "ps4_format_quad": (C.c_long, [P(Quad), C.c_char_p, C.c_size_t]),
        "ps4_quad_values": (None, [P(Quad), P(C.c_uint64), P(C.c_uint64), P(C.c_uint32)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def header_symbols() -> list[str]:
    """Every function the public header declares (for the export check)."""
    import re
    text = HEADER_PATH.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ps4_[a-z0-9_]+)\s*\(", text)))


os.environ.setdefault("CUDA_MODULE_LOADING", "LAZY")
