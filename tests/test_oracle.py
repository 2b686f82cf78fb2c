"""The CPU restatement (oracle/) pinned to the reference's golden vectors.

Golden vectors (tests/golden/, made by make_golden.py from the reference itself):
sorted-output sha256 and every TOTAL / histogram / CAPACITY value at S < 1e7 and for the
--dump4 4-set list, the singleton-S known answers (exhaustive/test_verify.py:13,31-32,
bruteforce-scratchpad/dotnet/test1.txt, exhaustive/logs/boundary_*.err) and 48 seeded
subranges up to S ~ 1e12.
"""
from __future__ import annotations

import random

import pytest

from conftest import assert_stats_equal, sha_sorted
from oracle import orc


def test_oracle_1e7_matches_reference(golden, golden_1e7_lines):
    rc, st, lines, err = orc.search(1, 10 ** 7, flags=orc.VERIFY)
    assert rc == 0, err
    g = golden["runs"]["1e7"]
    assert sorted(lines) == golden_1e7_lines
    assert sha_sorted(lines) == g["sha256"] == "657d64f2ffbf2d9e848f82acb5362c79ebfd05b9a61a6e4171b6a7f659709e14"
    assert_stats_equal(st, g, label="1e7")
    # README.md:158 expectation
    assert (st["sets5"], st["multi"], st["sets6"]) == (123, 2, 0)


def test_oracle_dump4_1e7(golden):
    rc, st, lines, err = orc.search(1, 10 ** 7, dump4=10 ** 8, flags=orc.NOEXT)
    assert rc == 0, err
    g = golden["runs"]["dump4_1e7"]
    assert len(lines) == g["n_lines"] == 325094
    assert sha_sorted(lines) == g["sha256"]


def test_oracle_dump4_order_is_reference_order():
    """First 2000 4-sets in the reference's own processing order, verbatim."""
    from conftest import GOLDEN_DIR
    want = (GOLDEN_DIR / "dump4_first2000.txt").read_text().splitlines(keepends=True)
    rc, _, lines, err = orc.search(1, 10 ** 7, dump4=2000, flags=orc.NOEXT)
    assert rc == 0, err
    assert lines == want


@pytest.mark.parametrize("S", [362141, 885125, 50578642000] + [k * 10 ** 11 for k in range(1, 10)])
def test_oracle_singletons(golden, S):
    g = golden["singletons"][str(S)]
    rc, st, lines, err = orc.search(S, S + 1, flags=orc.VERIFY)
    assert rc == 0, err
    assert lines == g["lines"]
    assert_stats_equal(st, g, label=str(S))


def test_oracle_boundary_logs(golden):
    """exhaustive/logs/boundary_{1..9}.err: the reference's own singleton repairs."""
    for S, want in golden["boundary_logs"].items():
        S = int(S)
        rc, st, lines, err = orc.search(S, S + 1)
        assert rc == 0 and lines == []
        assert_stats_equal(st, want, hist=False, label=f"boundary {S}")


def test_oracle_known_vectors(golden):
    """exhaustive/test_verify.py records: the 5-set line verbatim; the M record as a set
    (the reference's current build prints its extensions in a different order than the
    test file, which was written against an earlier build)."""
    five, multi = golden["test_verify_lines"]
    _, _, lines, _ = orc.search(362141, 362142)
    assert [x.rstrip("\n") for x in lines] == [five]
    _, _, lines, _ = orc.search(50578642000, 50578642001)
    assert len(lines) == 1
    got = lines[0].strip()
    assert got.split(" ext=")[0] == multi.split(" ext=")[0]
    ext = lambda s: set(s.split("ext=[")[1].split("]")[0].split(","))
    assert ext(got) == ext(multi)


def test_oracle_subranges(golden):
    for sub in golden["subranges"][:24]:
        rc, st, lines, err = orc.search(sub["lo"], sub["hi"])
        assert rc == 0, err
        assert sorted(lines) == sub["lines"]
        assert_stats_equal(st, sub, label=f"[{sub['lo']},{sub['hi']})")


def test_oracle_chunk_size_does_not_change_results():
    a = orc.search(10 ** 6, 3 * 10 ** 6, chunk_log2=20)
    b = orc.search(10 ** 6, 3 * 10 ** 6, chunk_log2=13)
    assert a[1] == b[1] and sorted(a[2]) == sorted(b[2])


@pytest.mark.parametrize("cap,kw,msg", [
    ("reps", dict(cap_reps=2), "representation capacity exceeded"),
    ("divs", dict(cap_divs=1), "divisor capacity exceeded"),
    ("ext", dict(cap_ext=1), "extension capacity exceeded"),
])
def test_oracle_capacity_failures(cap, kw, msg):
    """test_preflight.py's injected capacity failures (-DS4_MAX_*), as runtime caps."""
    rc, _, _, err = orc.search(1, 10 ** 7, **kw)
    assert rc == 2
    assert err == f"FATAL: {msg}; this interval is NOT certified complete"


def test_isqrt_edges():
    vals = [0, 1, 2, 3, 4, 2**32 - 1, 2**32, (2**32 - 1) ** 2, 2**64 - 1, 2**64, (2**40 + 7) ** 2,
            (2**40 + 7) ** 2 - 1, (2**50 - 3) ** 2 + 1, 2**100, 2**126 - 1]
    rng = random.Random(5)
    vals += [rng.randrange(2**k) for k in range(1, 127) for _ in range(3)]
    for n in vals:
        import math
        r = math.isqrt(n)
        assert orc.isqrt128(n) == r, n
        assert orc.is_square128(n) == (r * r == n), n


def _quads_below(limit):
    _, _, lines, _ = orc.search(1, limit, dump4=10 ** 9, flags=orc.NOEXT)
    for line in lines:
        a, b, c, d = map(int, line.split("[")[1].split("]")[0].split(","))
        yield a, b, c, d


def test_triple_extension_oracle_cross_pinned():
    """No reference function extends a triple.  Pin the restatement on the reference's
    4-sets: for every 4-set below S=2e5, each of its four 3-subsets must extend to the
    missing member (with d bound above it)."""
    n = 0
    for q in _quads_below(200000):
        for drop in range(4):
            tri = [x for i, x in enumerate(q) if i != drop]
            got = orc.extend_triple(*tri, dmax=max(q) + 10)
            assert q[drop] in got, (q, drop, got)
            n += 1
    assert n > 1000


def test_triple_extension_brute_force():
    """Small triples against a direct search over d."""
    import math
    rng = random.Random(11)
    done = 0
    while done < 60:
        x, y, z = (rng.randint(2, 400) for _ in range(3))
        if (x * x + y * y + z * z) % 2:
            continue
        a, b, c = (x * x + y * y - z * z) // 2, (x * x - y * y + z * z) // 2, (-x * x + y * y + z * z) // 2
        if min(a, b, c) <= 0 or len({a, b, c}) < 3:
            continue
        dmax = 200000
        sq = lambda v: math.isqrt(v) ** 2 == v
        want = [d for d in range(1, dmax + 1) if d not in (a, b, c) and sq(d + a) and sq(d + b) and sq(d + c)]
        assert orc.extend_triple(a, b, c, dmax) == want, (a, b, c)
        done += 1
