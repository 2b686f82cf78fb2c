"""What the reference's consumers of one `s4` block require of it, restated for tests that
drive the drop-in CLI (bin/s4gpu) the way those consumers drive `s4`.

A block is one process run `s4 lo hi T 20 --verify --out B.out --ckpt B.ckpt` with its stderr
in B.err.  The archived block controller starts it and reads it back
(sources/exhaustive/run_exhaustive.py:200-238, parse_result :74-94, width rule :244-248); the
evidence packer re-checks its checkpoint (exhaustive/compact.py:29-45); the verifier scans
every result line (exhaustive/verify.py:140-164), reducing each `M:` record to its primitive
near misses (exhaustive/evidence/verify_continuation.original.py:42-58).
tests/test_consumers.py runs those consumers' own code on a committed CLI block beside these
restatements, where the reference tree is at hand.
"""
from __future__ import annotations

import ast
import itertools
import math
import re
import subprocess
import time
from functools import reduce
from pathlib import Path

# the ten additive counters, in checkpoint column order (s4.c:81, compact.py:19-20)
COUNTERS = ("S_done", "pairs", "S_ge3", "triples", "4-sets", "5-sets", "6-sets", "multi-ext-4sets",
            "ext_cand", "ext_sqrt")
FAILURE_MARKERS = ("FATAL:", "VERIFY FAILED", "BAD 4-set")
FIVE = re.compile(r"5: \[([\d,]+)\] S=(\d+)")
MULTI = re.compile(r"M: \[([\d,]+)\] ext=\[([\d,]+)\] S=(\d+)")
CAPACITY = re.compile(r"CAPACITY: reps=(\d+)/(\d+) divisors=(\d+)/(\d+) extensions=(\d+)/(\d+)")


def square(n: int) -> bool:
    return n >= 0 and math.isqrt(n) ** 2 == n


def largest_square_divisor(n: int) -> int:
    """The largest square dividing n > 0 (trial division; the values here are < 2^64)."""
    out, d = 1, 2
    while d * d <= n:
        while n % (d * d) == 0:
            n //= d * d
            out *= d * d
        d += 1
    return out


def region_end(lo: int, hi: int, threads: int, i: int) -> int:
    """End of region i of the reference's equal split (s4.c:452-456)."""
    return lo + (hi - lo) * (i + 1) // threads


def parse_block(err_text: str, ckpt_text: str, lo: int, hi: int):
    """The controller's acceptance of a finished block (run_exhaustive.py:74-94): no failure
    marker, one TOTAL line covering hi - lo, a CAPACITY line within its limits, and a DONE
    checkpoint of the same interval whose regions all reached their ends."""
    assert not any(m in err_text for m in FAILURE_MARKERS), "failure marker in stderr"
    totals_lines = [x for x in err_text.splitlines() if x.startswith("TOTAL:")]
    assert len(totals_lines) == 1, "expected one TOTAL line"
    totals = {k: int(v) for k, v in re.findall(r"([\w-]+)=(\d+)", totals_lines[0])}
    assert totals["S_done"] == hi - lo
    cap = CAPACITY.search(err_text)
    assert cap is not None, "no CAPACITY line"
    maxima = {key: (int(cap[2 * i + 1]), int(cap[2 * i + 2]))
              for i, key in enumerate(("representations", "divisors", "extensions"))}
    assert all(used <= limit for used, limit in maxima.values())
    cp = ckpt_text.splitlines()
    assert cp[0] == "s4ckpt v1" and cp[-1] == "DONE"
    a, b, threads, _chunk = map(int, cp[1].split())
    assert (a, b) == (lo, hi) and len(cp) == threads + 3
    for i, line in enumerate(cp[2:-1]):
        vals = list(map(int, line.split()))
        assert vals[0] == i and vals[1] == vals[2] == region_end(lo, hi, threads, i)
    return totals, maxima


def check_checkpoint(ckpt_text: str, lo: int, hi: int, threads: int, chunk_log2: int, totals: dict):
    """The packer's checkpoint audit (compact.py:29-45): the run's parameters, one 13-column
    row per region covering exactly that region, and column sums equal to the TOTAL line."""
    lines = ckpt_text.splitlines()
    assert lines[0] == "s4ckpt v1" and lines[-1] == "DONE", "incomplete checkpoint"
    assert tuple(map(int, lines[1].split())) == (lo, hi, threads, 1 << chunk_log2), "checkpoint parameters"
    assert len(lines) == threads + 3, "checkpoint thread count"
    rows = [list(map(int, x.split())) for x in lines[2:-1]]
    for i, row in enumerate(rows):
        start, end = lo + (hi - lo) * i // threads, region_end(lo, hi, threads, i)
        assert len(row) == 13 and row[:3] == [i, end, end], "incomplete thread range"
        assert row[3] == end - start and min(row) >= 0, "thread coverage count"
    for j, key in enumerate(COUNTERS):
        assert sum(row[3 + j] for row in rows) == totals[key], "checkpoint counter mismatch: " + key
    return rows


def parse_multi(line: str):
    """An `M:` record reduced to its primitive near misses (verify_continuation.original.py:
    42-58): the four members and >= 2 extensions are distinct and positive, every member-member
    and member-extension sum is square; each pair of extensions whose sum is not square, divided
    by the largest square dividing the gcd of the six values, is a 6-set with exactly 14 of its
    15 sums square.  Returns (S, {primitive 6-set: its two extensions}, {6-sets found})."""
    four, ext = (list(ast.literal_eval(g)) for g in re.findall(r"\[[^]]*\]", line))
    assert len(four) == 4 and len(ext) >= 2
    allv = four + ext
    assert len(set(allv)) == len(allv) and min(allv) > 0
    assert all(square(a + b) for a, b in itertools.combinations(four, 2))
    assert all(square(a + b) for a in four for b in ext)
    near, sixes = {}, set()
    for a, b in itertools.combinations(ext, 2):
        vals = four + [a, b]
        if square(a + b):
            sixes.add(tuple(sorted(vals)))
            continue
        k = largest_square_divisor(reduce(math.gcd, vals))
        prim = tuple(sorted(v // k for v in vals))
        assert sum(square(x + y) for x, y in itertools.combinations(prim, 2)) == 14
        near[prim] = tuple(sorted((a // k, b // k)))
    return sum(four), near, sixes


def scan(lines, lo: int, hi: int):
    """The verifier's pass over a block's result lines (verify.py:140-164): every line is a
    5-set or an `M:` record of an S in [lo, hi); 5-sets are exact; `M:` records hold no 6-set.
    Returns (counts, five-sets, near misses, largest extension count)."""
    counts = {"five": 0, "multi": 0}
    five, near, max_ext = set(), {}, 0
    for raw in lines:
        line = raw.rstrip("\r\n")
        m = FIVE.fullmatch(line)
        if m:
            values = tuple(sorted(map(int, m[1].split(","))))
            total = int(m[2])
            assert len(values) == len(set(values)) == 5 and values[0] > 0, "invalid five-set"
            assert sum(values[:4]) == total and lo <= total < hi, "five-set outside interval"
            assert all(square(a + b) for a, b in itertools.combinations(values, 2)), "nonsquare five-set sum"
            five.add(values)
            counts["five"] += 1
            continue
        m = MULTI.fullmatch(line)
        assert m is not None, f"unexpected result line: {line[:150]}"
        total, partial, sixes = parse_multi(line)
        assert total == int(m[3]) and lo <= total < hi, "multi-extension record outside interval"
        assert not sixes, "6-set in a multi-extension record"
        max_ext = max(max_ext, len(m[2].split(",")))
        near.update(partial)
        counts["multi"] += 1
    return counts, five, near, max_ext


def next_width(done_blocks: list[dict], available_s: float) -> int:
    """The controller's adaptive block width (run_exhaustive.py:244-247): the seconds per S of
    the last five blocks (36 ns before any), 15 % margin, whole 1e8, at most 5e9."""
    last = done_blocks[-5:]
    rate = sum(b["elapsed"] for b in last) / sum(b["hi"] - b["lo"] for b in last) if last else 36e-9
    return min(5 * 10 ** 9, int(available_s / (rate * 1.15)) // 10 ** 8 * 10 ** 8)


def run_block(binary: Path, directory: Path, name: str, lo: int, hi: int, threads: int = 16,
              timeout: float = 600.0):
    """One block started the way the controller starts `s4` (run_exhaustive.py:207-215): in the
    run directory, stdout discarded, stderr into <name>.err.  Returns (returncode, seconds)."""
    args = [str(binary), str(lo), str(hi), str(threads), "20", "--verify",
            "--out", str(directory / (name + ".out")), "--ckpt", str(directory / (name + ".ckpt"))]
    began = time.monotonic()
    with (directory / (name + ".err")).open("w") as log:
        p = subprocess.Popen(args, cwd=directory, stdout=subprocess.DEVNULL, stderr=log)
        rc = p.wait(timeout=timeout)
    return rc, time.monotonic() - began
