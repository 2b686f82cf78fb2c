"""Batched triple extension on the GPU (ps4_extend_triples) against the oracle's restatement
of the extension step (oracle/ps4_oracle.c orc_extend_triple, after exhaustive/s4.c:160-207).

Bar: bit-exact -- for every triple the same sorted list of d.
"""
from __future__ import annotations

import ctypes as C
import random

import numpy as np
import pytest

from oracle import orc
from ps4b200 import Ps4Error, Search, _abi, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with Search(2 * 10 ** 12) as s:
        yield s


def _oracle(abc, dmax):
    return [orc.extend_triple(int(a), int(b), int(c), dmax) for a, b, c in abc]


def test_seeded_triples_d_le_1e12(ctx):
    """The batched workload's triples (x, y, z uniform in [1, 1e5]), d <= 1e12."""
    abc = workloads.triples(20000, seed=20261203)
    got, state, st = ctx.extend_triples(abc, 10 ** 12)
    assert not state.any()
    want = _oracle(abc, 10 ** 12)
    assert got == want
    assert st["triples"] == 20000 and st["invalid"] == 0
    assert st["exts"] == sum(len(w) for w in want) > 0
    assert st["ext_cand"] >= st["ext_sqrt"] >= st["exts"]


def test_reference_4sets_close_their_triples(ctx):
    """Every 4-set the reference prints (--dump4 fixture): each 3-subset extends to the
    missing member."""
    from conftest import GOLDEN_DIR
    quads = []
    for line in (GOLDEN_DIR / "dump4_first2000.txt").read_text().splitlines()[:500]:
        quads.append(tuple(map(int, line.split("[")[1].split("]")[0].split(","))))
    tri, miss = [], []
    for q in quads:
        for drop in range(4):
            tri.append([x for i, x in enumerate(q) if i != drop])
            miss.append(q[drop])
    got, state, _ = ctx.extend_triples(tri, 10 ** 7)
    assert not state.any()
    for t, m, g in zip(tri, miss, got):
        assert m in g, (t, m)
    assert got == _oracle(tri, 10 ** 7)


def test_member_order_and_small_dmax(ctx):
    rng = random.Random(5)
    abc = workloads.triples(2000, seed=7, xmax=3000)
    perm = np.array([rng.sample(list(row), 3) for row in abc.tolist()], dtype=np.uint64)
    for dmax in (0, 1, 10 ** 4, 10 ** 8, 2 ** 62):
        got, _, _ = ctx.extend_triples(perm, dmax)
        assert got == _oracle(abc, dmax), dmax


def test_invalid_inputs_are_flagged(ctx):
    rows = [(0, 1, 3), (5, 5, 11), (1, 3, 5), (2, 7, 9), (6, 19, 30)]   # the last is a square-sum triple
    got, state, st = ctx.extend_triples(rows, 10 ** 6)
    assert state.tolist() == [1, 1, 1, 1, 0]
    assert st["invalid"] == 4 and st["triples"] == 1
    assert got[:4] == [[], [], [], []]
    assert got[4] == orc.extend_triple(6, 19, 30, 10 ** 6)


def test_beyond_tables_is_an_error():
    """Pairwise-sum roots past the context's factor tables give PS4_ERR_ARG, not a silent miss."""
    with Search(10 ** 6) as s:             # tables for roots summing below 2064
        with pytest.raises(Ps4Error) as e:
            s.extend_triples([(960000, 1290000, 1600000)], 10 ** 9)   # sums 1500^2, 1600^2, 1700^2
        assert e.value.code == _abi.PS4_ERR_ARG and "factor tables" in e.value.message
        got, state, _ = s.extend_triples([(6, 19, 30)], 10 ** 6)     # the context stays usable
        assert state.tolist() == [0]


def test_output_full_reports_needed(ctx):
    abc = workloads.triples(3000, seed=9)
    a = np.ascontiguousarray(abc)
    out = (_abi.TriExt * 1)()
    n_out = C.c_uint64()
    rc = ctx.lib.ps4_extend_triples(ctx.ctx, a.ctypes.data, a.shape[0], 10 ** 12, None, out, 1, C.byref(n_out), None)
    want = sum(len(w) for w in _oracle(abc, 10 ** 12))
    assert rc == _abi.PS4_ERR_OUTPUT_FULL and n_out.value == want > 1
    got, _, _ = ctx.extend_triples(abc, 10 ** 12)
    assert sum(map(len, got)) == want


def test_empty_call(ctx):
    got, state, st = ctx.extend_triples(np.zeros((0, 3), dtype=np.uint64), 10 ** 12)
    assert got == [] and st["triples"] == 0
