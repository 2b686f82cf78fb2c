"""Seeded synthetic query streams for the batched, triple-extension and serving workloads.

The reference drives its search as one ``s4 lo hi`` process per block (run_exhaustive.py:
200-238) and has no triple or serving front end; these generators produce the query mixes the
GPU build is measured and tested on, deterministically from a seed (numpy PCG64):

* ``subranges``: uneven [lo, hi) work items, widths log-uniform, offsets uniform;
* ``triples``: square-sum triples a, b, c from x, y, z uniform in [1, xmax], kept when
  x^2 + y^2 + z^2 is even and a = (x^2+y^2-z^2)/2, b = (x^2-y^2+z^2)/2, c = (-x^2+y^2+z^2)/2
  are distinct positive integers (then a+b = x^2, a+c = y^2, b+c = z^2);
* ``requests``: a Poisson arrival stream mixing the two kinds.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def subranges(n: int, seed: int, *, wmin: float = 1e5, wmax: float = 1e9, omax: float = 1e11):
    """n items [lo, hi): width 10^U(log10 wmin, log10 wmax), lo uniform in [1, omax]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = np.floor(10.0 ** rng.uniform(np.log10(wmin), np.log10(wmax), n)).astype(np.uint64)
    lo = rng.integers(1, int(omax), n, endpoint=True, dtype=np.uint64)
    return lo, lo + w


def triples(n: int, seed: int, *, xmax: int = 10 ** 5) -> np.ndarray:
    """n square-sum triples (rows a, b, c) drawn as described in the module docstring."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.empty((0, 3), dtype=np.uint64)
    while out.shape[0] < n:
        m = max(4 * (n - out.shape[0]), 1024)
        x, y, z = (rng.integers(1, xmax, m, endpoint=True, dtype=np.int64) for _ in range(3))
        x2, y2, z2 = x * x, y * y, z * z
        ok = (x2 + y2 + z2) % 2 == 0
        a, b, c = (x2 + y2 - z2) // 2, (x2 - y2 + z2) // 2, (-x2 + y2 + z2) // 2
        ok &= (a > 0) & (b > 0) & (c > 0) & (a != b) & (a != c) & (b != c)
        out = np.concatenate([out, np.stack([a[ok], b[ok], c[ok]], axis=1).astype(np.uint64)])
    return out[:n]


@dataclass
class Request:
    """One query of the serving stream: a subrange [lo, hi) or a triple to extend by d <= dmax."""
    rid: int
    t_arrive: float            # seconds from the start of the stream
    kind: str                  # "range" or "triple"
    lo: int = 0
    hi: int = 0
    abc: tuple = ()
    dmax: int = 0


def requests(n: int, seed: int, *, rate: float, frac_range: float = 0.7, wmin: float = 1e4, wmax: float = 1e9,
             omax: float = 1e12, xmax: int = 10 ** 5, dmax: int = 10 ** 12) -> list[Request]:
    """n requests with exponential inter-arrival times (rate per second): a fraction
    frac_range of subrange queries (width log-uniform in [wmin, wmax], lo uniform in
    [1, omax]), the rest triple-extension queries built like ``triples``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    is_range = rng.uniform(0, 1, n) < frac_range
    lo, hi = subranges(n, seed + 1, wmin=wmin, wmax=wmax, omax=omax)
    tri = triples(n, seed + 2, xmax=xmax)
    out = []
    for i in range(n):
        if is_range[i]:
            out.append(Request(i, float(t[i]), "range", lo=int(lo[i]), hi=int(hi[i])))
        else:
            out.append(Request(i, float(t[i]), "triple", abc=tuple(int(v) for v in tri[i]), dmax=dmax))
    return out
