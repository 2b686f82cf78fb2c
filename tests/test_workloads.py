"""The seeded query generators (ps4b200.workloads): deterministic and shaped as specified."""
from __future__ import annotations

import math

import numpy as np

from ps4b200 import workloads


def test_triples_are_square_sum_triples():
    abc = workloads.triples(5000, seed=1)
    assert abc.shape == (5000, 3) and abc.dtype == np.uint64
    for a, b, c in abc.tolist()[:2000]:
        assert min(a, b, c) > 0 and len({a, b, c}) == 3
        for s in (a + b, a + c, b + c):
            assert math.isqrt(s) ** 2 == s
        assert max(a, b, c) < 10 ** 10
    assert (workloads.triples(5000, seed=1) == abc).all()
    assert not (workloads.triples(5000, seed=2) == abc).all()


def test_subranges_shape():
    lo, hi = workloads.subranges(4096, seed=3)
    w = (hi - lo).astype(np.float64)
    assert w.min() >= 1e5 and w.max() <= 1e9 and lo.min() >= 1 and lo.max() <= 1e11
    # log-uniform: about a quarter of the widths in each of the four decades
    dec = np.floor(np.log10(w)).astype(int)
    assert all(800 < (dec == d).sum() < 1250 for d in (5, 6, 7, 8))


def test_request_stream():
    reqs = workloads.requests(10000, seed=4, rate=100.0)
    assert len(reqs) == 10000
    t = [r.t_arrive for r in reqs]
    assert t == sorted(t) and abs(t[-1] / 10000 - 0.01) < 0.001
    n_range = sum(r.kind == "range" for r in reqs)
    assert 6700 < n_range < 7300
    for r in reqs[:200]:
        if r.kind == "range":
            assert 1e4 <= r.hi - r.lo <= 1e9 and 1 <= r.lo <= 1e12
        else:
            a, b, c = r.abc
            assert all(math.isqrt(s) ** 2 == s for s in (a + b, a + c, b + c)) and r.dmax == 10 ** 12
