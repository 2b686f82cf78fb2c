"""ps4_search_range_noalloc: the search with no device allocation during the call.

Who needs it: callers that cannot call cudaMalloc when they search -- programs that work in
a fixed device-memory budget or hand all device memory out from their own pool, and serving
loops that cannot take cudaMalloc/cudaFree on the request path (both block the host, and
cudaFree also waits for the whole device).  The entry point keeps its 4-set staging and its
device-side result buffers in one static array inside the library instead.

Checked through the C-ABI against the regular entry point, ps4_search_range, on two calls in
a row over different ranges (so the second call cannot pass on the first call's leftovers in
the shared array), then on a repeat of the first range; then at S = 1e10 and 5e11, where the
tile scan costs most (the regular entry point scans groups of 16 tiles into lists, this one scans
each of its own tiles); then the fixed
result buffers overflowing.  The bar is bit-exact: counters and result lines equal.  The
file is named to be collected last.
"""
from __future__ import annotations

import ctypes as C

import pytest

from ps4b200 import Ps4Error, RangeResult, Search, _abi

pytestmark = pytest.mark.gpu

# A kernel launched for the first time may have its code loaded then (lazy module loading),
# which can take a little device memory; the entry point's own buffers are 65.5 MB.
CODE_LOAD_SLACK = 8 << 20


def search_noalloc(s: Search, lo: int, hi: int) -> RangeResult:
    """One ps4_search_range_noalloc call on the context of `s`, results into its host buffers."""
    lib = s.lib
    while True:
        st = _abi.Stats()
        rc = lib.ps4_search_range_noalloc(s.ctx, lo, hi, C.byref(st), C.byref(s._res))
        r = s._res
        fixed_full = (r.n_hits > _abi.PS4_NOALLOC_MAX_HITS or r.n_exts > _abi.PS4_NOALLOC_MAX_EXTS
                      or r.n_sixes > _abi.PS4_NOALLOC_MAX_SIXES)
        if rc == _abi.PS4_ERR_OUTPUT_FULL and not fixed_full and (
                r.n_hits > r.hits_cap or r.n_exts > r.exts_cap or r.n_sixes > r.sixes_cap):
            s._grow()                       # our host buffers were short: grow and repeat
            continue
        if rc != _abi.PS4_OK:
            raise Ps4Error(rc, lib.ps4_last_error(s.ctx).decode())
        out = RangeResult(stats=st.as_dict())
        s._collect(out)
        return out


def free_device_bytes() -> int:
    import torch
    return torch.cuda.mem_get_info(0)[0]


def test_noalloc_matches_search_range_on_two_calls_in_a_row():
    ranges = [(10 ** 9, 10 ** 9 + 3 * 10 ** 7), (1, 10 ** 7)]
    with Search(2 * 10 ** 9) as s:
        want = [s.range(lo, hi) for lo, hi in ranges]
        free0 = free_device_bytes()                                       # before the first call
        got = [search_noalloc(s, lo, hi) for lo, hi in ranges]          # two calls in a row
        free1 = free_device_bytes()
        assert free0 - free1 <= CODE_LOAD_SLACK, (free0, free1)
        for (lo, hi), g, w in zip(ranges, got, want):
            assert g.stats == w.stats, (lo, hi)
            assert sorted(g.lines) == sorted(w.lines), (lo, hi)
            assert g.six_lines == w.six_lines == []
        assert len(want[1].lines) == 125                                  # S < 1e7: 123 five-sets + 2 M
        # a repeat of the first range, after the second call left its own data in the array,
        # allocates nothing on the device and gives the same answer again
        again = search_noalloc(s, *ranges[0])
        assert free_device_bytes() == free1
        assert again.stats == want[0].stats and sorted(again.lines) == sorted(want[0].lines)


@pytest.mark.parametrize("lo", [10 ** 10, 5 * 10 ** 11])
def test_noalloc_matches_search_range_above_1e10(lo):
    """High S, where each tile's own scan (this entry point) and the regular entry point's scan of
    16-tile groups into lists differ most in cost."""
    hi = lo + 10 ** 7
    with Search(hi) as s:
        want = s.range(lo, hi)
        got = search_noalloc(s, lo, hi)
    assert got.stats == want.stats
    assert sorted(got.lines) == sorted(want.lines)
    assert want.stats["sets4"] > 0


def test_noalloc_fixed_result_buffers_overflow():
    """S < 2e10 holds about 9e4 hits, more than the 65,536 the fixed buffer keeps: the call
    says which buffer overflowed and by how much, copies nothing, and the next call works."""
    with Search(2 * 10 ** 10) as s:
        st = _abi.Stats()
        rc = s.lib.ps4_search_range_noalloc(s.ctx, 1, 2 * 10 ** 10, C.byref(st), C.byref(s._res))
        msg = s.lib.ps4_last_error(s.ctx).decode()
        assert rc == _abi.PS4_ERR_OUTPUT_FULL, msg
        assert s._res.n_hits > _abi.PS4_NOALLOC_MAX_HITS, s._res.n_hits
        assert "hits" in msg and str(s._res.n_hits) in msg and "shorter range" in msg
        assert st.S_done == 0                                            # counters untouched
        want = s.range(10 ** 9, 10 ** 9 + 10 ** 7)
        got = search_noalloc(s, 10 ** 9, 10 ** 9 + 10 ** 7)
    assert got.stats == want.stats and sorted(got.lines) == sorted(want.lines)


def test_noalloc_rejects_what_its_fixed_array_cannot_hold():
    with Search(10 ** 7, dump4=True) as s:
        st = _abi.Stats()
        rc = s.lib.ps4_search_range_noalloc(s.ctx, 1, 10 ** 6, C.byref(st), C.byref(s._res))
        assert rc == _abi.PS4_ERR_ARG
        assert "dump4" in s.lib.ps4_last_error(s.ctx).decode()
    with Search(10 ** 7, cap_reps=600) as s:
        rc = s.lib.ps4_search_range_noalloc(s.ctx, 1, 10 ** 6, C.byref(_abi.Stats()), C.byref(s._res))
        assert rc == _abi.PS4_ERR_ARG
        assert "cap_reps <= 512" in s.lib.ps4_last_error(s.ctx).decode()
    with Search(10 ** 7) as s:
        rc = s.lib.ps4_search_range_noalloc(s.ctx, 1, 10 ** 8, C.byref(_abi.Stats()), C.byref(s._res))
        assert rc == _abi.PS4_ERR_ARG
        assert "s_hi_max" in s.lib.ps4_last_error(s.ctx).decode()
