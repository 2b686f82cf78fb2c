"""The device's exact square roots, called directly on their edge values.

Every square test and every tile scan of the search rests on these routines: a floating-point
estimate followed by an exact integer correction, restating isqrt64 / isqrt128 / is_sq128
(exhaustive/s4.c:95-108).  ps4_check_roots runs them on the GPU over values a float estimate
gets wrong most easily -- r^2 - 1, r^2, r^2 + 1 around powers of two up to 2^64 - 1, and
2^128 - 1 -- and this test compares every result with Python's exact integer arithmetic.
Bar: bit-exact.
"""
from __future__ import annotations

import ctypes as C
import math
import random

import pytest

from ps4b200 import _abi

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def edge_values() -> list[int]:
    vals = {0, 1, 2, 3, 4, 5, (1 << 128) - 1, (1 << 128) - 2, (1 << 100) - 1, 1 << 100, (1 << 64) - 1, 1 << 64,
            (1 << 64) + 1, (1 << 46) - 1, 1 << 46}
    for b in (8, 16, 22, 23, 24, 26, 31, 32, 33, 44, 46, 48, 50, 52, 53, 54, 60, 63, 64):
        for d in range(-3, 4):
            r = (1 << b) + d
            if r < 0 or r > M64:
                continue
            for n in (r * r - 1, r * r, r * r + 1):
                if 0 <= n < (1 << 128):
                    vals.add(n)
    rng = random.Random(20261204)
    for bits in (20, 40, 46, 64, 88, 99, 100, 127, 128):
        for _ in range(64):
            r = rng.getrandbits(bits // 2 + (bits & 1)) | 1
            r = min(r, M64)
            for n in (r * r - 1, r * r, r * r + 1, rng.getrandbits(bits)):
                if 0 <= n < (1 << 128):
                    vals.add(n)
    return sorted(vals)


def test_device_roots_on_edge_values():
    lib = _abi.load()
    vals = edge_values()
    n = len(vals)
    lo = (C.c_uint64 * n)(*[v & M64 for v in vals])
    hi = (C.c_uint64 * n)(*[v >> 64 for v in vals])
    roots = (C.c_uint64 * (4 * n))()
    flags = (C.c_uint32 * n)()
    assert lib.ps4_check_roots(0, lo, hi, n, roots, flags) == _abi.PS4_OK
    fast_checked = 0
    for i, v in enumerate(vals):
        r = math.isqrt(v)
        low = v & M64
        assert roots[4 * i] == r, f"isqrt128({v})"
        assert roots[4 * i + 1] == math.isqrt(low), f"isqrt64({low})"
        c = math.isqrt(low)
        assert roots[4 * i + 2] == (c if c * c == low else c + 1), f"ceil_sqrt64({low})"
        assert roots[4 * i + 3] == (math.isqrt(low) if low < (1 << 46) else 0), f"isqrt_lt2p46({low})"
        assert bool(flags[i] & 1) == (r * r == v), f"is_square_exact({v})"
        if v < (1 << 100):
            assert bool(flags[i] & 2) == (r * r == v), f"is_square_fast({v})"
            fast_checked += 1
        else:
            assert not flags[i] & 2
    assert n > 1500 and fast_checked > 1000
