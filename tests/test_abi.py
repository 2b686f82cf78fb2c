"""The C-ABI boundary without a GPU: the library loads, exports every symbol include/ps4.h
declares, refuses to run without an sm_100 device (no CPU fallback), and formats records
into the reference's exact line text (exhaustive/s4.c:24-27,214-220,239,250-253)."""
from __future__ import annotations

import ctypes as C
import math
import subprocess

import pytest

from conftest import GOLDEN_DIR, PKG
from ps4b200 import _abi


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    declared = _abi.header_symbols()
    assert "ps4_search_range" in declared and "ps4_create" in declared
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/ps4.h but not exported"
    nm = subprocess.run(["nm", "-D", "--defined-only", str(_abi.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in nm.splitlines() if " T " in line}
    assert set(declared) <= exported


def test_abi_version():
    assert _abi.load().ps4_abi_version() == 1


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU refusal")
def test_create_without_gpu_fails_loudly():
    from ps4b200 import Ps4Error, Search
    with pytest.raises(Ps4Error) as e:
        Search(10 ** 6)
    assert e.value.code == _abi.PS4_ERR_CUDA
    assert "no CPU path" in e.value.message or "device" in e.value.message


def _ext(value: int, key: int, flags: int) -> _abi.Ext:
    e = _abi.Ext()
    e.lo, e.hi, e.key, e.flags = value & (2**64 - 1), value >> 64, key, flags
    return e


def _hit(S, v, n_ext, flags=0) -> _abi.Hit:
    h = _abi.Hit()
    h.S = S
    for i in range(4):
        h.v[i] = v[i]
    h.n_ext, h.first_ext, h.flags = n_ext, 0, flags
    return h


def _fmt(fn, *args) -> str:
    buf = C.create_string_buffer(1 << 14)
    n = fn(*args, buf, 1 << 14)
    assert n >= 0
    return buf.value.decode()


def test_format_five_line():
    lib = _abi.load()
    exts = (_abi.Ext * 1)(_ext(763442, 3, _abi.PS4_EXT_FIVE | _abi.PS4_EXT_FIVE_OK))
    h = _hit(362141, [148583, 7442, 177458, 28658], 1)
    assert _fmt(lib.ps4_format_hit, C.byref(h), exts) == "5: [763442,177458,148583,28658,7442] S=362141\n"
    exts[0].flags = _abi.PS4_EXT_FIVE                         # verify flag off -> the reference's marker
    assert _fmt(lib.ps4_format_hit, C.byref(h), exts).endswith("S=362141  *** VERIFY FAILED ***\n")


def test_format_m_lines_match_golden():
    """Every M line at S < 1e10, rebuilt from its numbers, formats identically."""
    lib = _abi.load()
    for line in (GOLDEN_DIR / "m_lines_1e10.txt").read_text().splitlines(keepends=True):
        quad = list(map(int, line.split("M: [")[1].split("]")[0].split(",")))
        ext = list(map(int, line.split("ext=[")[1].split("]")[0].split(",")))
        S = int(line.rsplit("S=", 1)[1])
        exts = (_abi.Ext * len(ext))(*[_ext(e, i, 0) for i, e in enumerate(ext)])
        h = _hit(S, quad, len(ext), _abi.PS4_HIT_MULTI)
        assert _fmt(lib.ps4_format_hit, C.byref(h), exts) == line


def test_format_u128_and_six_and_drill():
    lib = _abi.load()
    big = 2**64 * 12345 + 678
    exts = (_abi.Ext * 2)(_ext(big, 0, _abi.PS4_EXT_FIVE | _abi.PS4_EXT_FIVE_OK), _ext(5, 1, 0))
    h = _hit(10, [4, 3, 2, 1], 2, _abi.PS4_HIT_MULTI)
    text = _fmt(lib.ps4_format_hit, C.byref(h), exts)
    assert text.splitlines()[0] == f"M: [4,3,2,1] ext=[{big},5] S=10"
    assert text.splitlines()[1] == f"5: [{big},4,3,2,1] S=10"
    six = _abi.Six(0, 0, 1, 0)
    assert _fmt(lib.ps4_format_six, C.byref(h), exts, C.byref(six)) == \
        f"!!!!!!!! FOUND 6-SET: [{big},5,4,3,2,1] S=10  *** VERIFY FAILED ***\n"
    assert _fmt(lib.ps4_format_drill, C.byref(h), exts) == \
        f"TEST-6SET (NOT A SOLUTION, --test-sixset drill): [{big},5,4,3,2,1] S=10  *** VERIFY FAILED ***\n"


def test_format_quad_lines_match_golden_dump():
    lib = _abi.load()
    for line in (GOLDEN_DIR / "dump4_first2000.txt").read_text().splitlines(keepends=True)[:300]:
        a, b, c, d = map(int, line.split("[")[1].split("]")[0].split(","))
        q = _abi.Quad(*(math.isqrt(x) for x in (a + b, a + c, a + d, b + c, b + d, c + d)))
        assert _fmt(lib.ps4_format_quad, C.byref(q)) == line
