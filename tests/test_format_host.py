"""Host line formatting (ps4_format_*, csrc/ps4_format.c): the batch formatter equals the
per-hit one, line for line, on synthetic records (no GPU)."""
from __future__ import annotations

import ctypes as C
import random

from ps4b200 import _abi


def _records(n, seed):
    rng = random.Random(seed)
    hits = (_abi.Hit * n)()
    exts = []
    for i in range(n):
        h = hits[i]
        h.S = rng.randrange(10 ** 6, 10 ** 12)
        for j in range(4):
            h.v[j] = rng.randrange(1, h.S)
        k = rng.choice([1, 1, 2, 3])
        h.n_ext, h.first_ext, h.item = k, len(exts), rng.randrange(0, 50)
        h.flags = _abi.PS4_HIT_MULTI if k >= 2 else 0
        for _ in range(k):
            e = _abi.Ext()
            e.lo = rng.randrange(1, 2 ** 64)
            e.hi = rng.choice([0, 0, 0, rng.randrange(1, 2 ** 20)])
            e.flags = rng.choice([0, _abi.PS4_EXT_FIVE, _abi.PS4_EXT_FIVE | _abi.PS4_EXT_FIVE_OK])
            exts.append(e)
    earr = (_abi.Ext * max(len(exts), 1))(*exts)
    return hits, earr, len(exts)


def test_batch_formatter_matches_per_hit():
    lib = _abi.load()
    hits, exts, ne = _records(500, 3)
    want_lines, want_items = [], []
    buf = C.create_string_buffer(1 << 14)
    for i in range(len(hits)):
        n = lib.ps4_format_hit(C.byref(hits[i]), exts, buf, len(buf))
        assert n >= 0
        for line in buf.value.decode().splitlines(keepends=True):
            want_lines.append(line)
            want_items.append(hits[i].item)
    assert len(want_lines) > 300
    cap = 1 << 20
    big = C.create_string_buffer(cap)
    items = (C.c_uint32 * (len(hits) + ne))()
    nl = C.c_uint64()
    n = lib.ps4_format_hits(hits, len(hits), exts, big, cap, items, C.byref(nl))
    assert n == sum(len(x) for x in want_lines)
    assert big.raw[:n].decode().splitlines(keepends=True) == want_lines
    assert nl.value == len(want_lines) and list(items[:nl.value]) == want_items
    # too small: the needed length comes back, the buffer ends at a complete hit
    small = C.create_string_buffer(1000)
    n2 = lib.ps4_format_hits(hits, len(hits), exts, small, 1000, None, C.byref(nl))
    assert n2 == -(n + 1) and nl.value == len(want_lines)
    got = small.value.decode()
    assert got == "".join(want_lines)[:len(got)] and got.endswith("\n") and len(got) < 1000


def test_decimal_text_of_edge_values():
    """Members, S and extensions print as Python's str(int) does: powers of ten, 2^64 -/+ 1,
    128-bit values whose 19-digit blocks are zero or start with zeros, up to 2^128 - 1."""
    lib = _abi.load()
    edge = [1, 9, 10, 99, 100, 10 ** 18, 10 ** 19 - 1, 10 ** 19, 10 ** 19 + 1, 2 ** 64 - 1, 2 ** 64, 2 ** 64 + 1,
            10 ** 20, 123 * 10 ** 19 + 5, 10 ** 38, 10 ** 38 - 1, 3 * 10 ** 38 + 7, 2 ** 127, 2 ** 128 - 1]
    u64 = [x for x in edge if x < 2 ** 64]
    buf = C.create_string_buffer(1 << 12)
    for i, x in enumerate(edge):
        h = _abi.Hit()
        h.S = u64[i % len(u64)]
        vs = [u64[(i + k) % len(u64)] for k in range(1, 5)]
        for j in range(4):
            h.v[j] = vs[j]
        e = (_abi.Ext * 2)()
        y = edge[(i + 7) % len(edge)]
        for k, val in enumerate((x, y)):
            e[k].lo, e[k].hi, e[k].flags = val & (2 ** 64 - 1), val >> 64, 0
        h.n_ext, h.first_ext, h.flags = 2, 0, _abi.PS4_HIT_MULTI
        n = lib.ps4_format_hit(C.byref(h), e, buf, len(buf))
        want = f"M: [{','.join(map(str, vs))}] ext=[{x},{y}] S={h.S}\n"
        assert n == len(want) and buf.value.decode() == want


def test_decimal_text_of_random_values():
    """2,000 extensions of log-uniform bit length (1..128) and members and S of 1..64 bits print
    as Python's str(int) does."""
    lib = _abi.load()
    rng = random.Random(2026)
    buf = C.create_string_buffer(1 << 12)
    for _ in range(1000):
        h = _abi.Hit()
        vs = [rng.getrandbits(rng.randint(1, 64)) or 1 for _ in range(4)]
        for j in range(4):
            h.v[j] = vs[j]
        h.S = rng.getrandbits(rng.randint(1, 64))
        xs = [rng.getrandbits(rng.randint(1, 128)) for _ in range(2)]
        e = (_abi.Ext * 2)()
        for k, val in enumerate(xs):
            e[k].lo, e[k].hi, e[k].flags = val & (2 ** 64 - 1), val >> 64, 0
        h.n_ext, h.first_ext, h.flags = 2, 0, _abi.PS4_HIT_MULTI
        n = lib.ps4_format_hit(C.byref(h), e, buf, len(buf))
        want = f"M: [{','.join(map(str, vs))}] ext=[{xs[0]},{xs[1]}] S={h.S}\n"
        assert n == len(want) and buf.value.decode() == want
