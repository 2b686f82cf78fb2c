"""The drop-in CLI (bin/s4gpu) on the GPU, checked the way the reference's own preflight
test checks s4 (archived test_preflight.py): small census equality as sorted line lists,
injected capacity failures with exit 2, and kill/resume equivalence; plus the stderr and
checkpoint formats its consumers parse (verify.py:102-136, compact.py:29-45), consecutive blocks
driven as the archived block controller drives s4 (run_exhaustive.py:200-248), and the stop on
the controller's SIGTERM with its resume."""
from __future__ import annotations

import re
import signal
import subprocess
import time

import pytest

import consumers
from conftest import PKG, assert_stats_equal, sha_sorted
from golden.make_golden import parse_stderr
from oracle import orc
from ps4b200 import Search

pytestmark = pytest.mark.gpu
CLI = PKG / "bin" / "s4gpu"


def run(args, cwd, env=None, check_rc=0):
    import os
    e = dict(os.environ)
    e.update(env or {})
    p = subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, cwd=cwd, env=e, timeout=600)
    if check_rc is not None:
        assert p.returncode == check_rc, p.stderr
    return p


def test_cli_1e7_census(tmp_path, golden, golden_1e7_lines):
    p = run([1, 10 ** 7, 4, 20, "--verify", "--out", "r.out", "--ckpt", "r.ckpt"], tmp_path)
    lines = (tmp_path / "r.out").read_text().splitlines(keepends=True)
    assert sorted(lines) == golden_1e7_lines
    st = parse_stderr(p.stderr)
    assert_stats_equal(st, golden["runs"]["1e7"], label="cli")
    # the header and per-thread coverage lines exactly as verify.py:historical_coverage reads them
    hdr = re.search(r"s4: S in \[(\d+),\s*(\d+)\), (\d+) threads", p.stderr)
    assert hdr.groups() == ("1", "10000000", "4")
    rows = re.findall(r"^\s+thread\s+(\d+): S \[(\d+),(\d+)\)", p.stderr, re.M)
    lo, hi, nt = 1, 10 ** 7, 4
    assert [tuple(map(int, r)) for r in rows] == [(i, lo + (hi - lo) * i // nt, lo + (hi - lo) * (i + 1) // nt)
                                                  for i in range(nt)]
    ck = (tmp_path / "r.ckpt").read_text().splitlines()
    assert ck[0] == "s4ckpt v1" and ck[1] == "1 10000000 4 1048576" and ck[-1] == "DONE"
    rows = [list(map(int, x.split())) for x in ck[2:-1]]
    assert [r[0] for r in rows] == [0, 1, 2, 3] and all(r[1] == r[2] for r in rows)
    assert sum(r[3] for r in rows) == 10 ** 7 - 1                       # S_done per region sums up
    assert sum(r[7] for r in rows) == golden["runs"]["1e7"]["sets4"]


def test_cli_capacity_failures_exit_2(tmp_path):
    for var, msg in (("S4_MAX_REPS", "representation"), ("S4_MAX_DIVS", "divisor"), ("S4_MAX_EXT", "extension")):
        p = run([1, 10 ** 7, 2, 20], tmp_path, env={var: "2" if var == "S4_MAX_REPS" else "1"}, check_rc=2)
        assert f"FATAL: {msg} capacity exceeded; this interval is NOT certified complete" in p.stderr


def test_cli_resume_equivalence(tmp_path):
    """A run 'killed' after its first chunks, then resumed, reports the same census.
    The interrupted state is written the way the CLI writes it: region 0 stopped at a
    chunk boundary with its counters so far, region 1 not started, partial output kept."""
    lo, hi, T, W = 1, 2 * 10 ** 7, 2, 1 << 20
    full = run([lo, hi, T, 20, "--out", "full.out"], tmp_path)
    stop = lo + 5 * W
    with Search(hi) as s:
        part = s.range(lo, stop)
    (tmp_path / "res.out").write_text("".join(part.lines))
    st = part.stats
    mid = lo + (hi - lo) // 2
    (tmp_path / "res.ckpt").write_text(
        f"s4ckpt v1\n{lo} {hi} {T} {W}\n"
        f"0 {stop} {mid} {st['S_done']} {st['pairs']} {st['S_ge3']} {st['triples']} {st['sets4']} {st['sets5']} "
        f"{st['sets6']} {st['multi']} {st['ext_cand']} {st['ext_sqrt']}\n"
        f"1 {mid} {hi} 0 0 0 0 0 0 0 0 0 0\n")
    res = run([lo, hi, 0, 20, "--out", "res.out", "--ckpt", "res.ckpt", "--resume"], tmp_path)
    assert "RESUMED from checkpoint" in res.stderr
    assert "  thread  0 resumes at S=%d (region end %d)" % (stop, mid) in res.stderr
    a, b = parse_stderr(full.stderr), parse_stderr(res.stderr)
    assert_stats_equal(b, a, hist=False, maxima=False)
    assert sorted(set((tmp_path / "res.out").read_text().splitlines())) == \
        sorted(set((tmp_path / "full.out").read_text().splitlines()))
    assert (tmp_path / "res.ckpt").read_text().endswith("DONE\n")
    again = run([lo, hi, 0, 20, "--out", "res.out", "--ckpt", "res.ckpt", "--resume"], tmp_path)
    assert "nothing to do" in again.stderr


def test_cli_sixset_drill(tmp_path):
    """--test-sixset fires the durable 6-set alert path once with a non-solution (s4.c:255-260)."""
    p = run([1, 10 ** 7, 1, 20, "--test-sixset", "--out", "d.out"], tmp_path)
    alert = (tmp_path / "SIXSET_FOUND.txt").read_text()
    rc, _, olines, _ = orc.search(1, 10 ** 7, flags=orc.TEST6)
    drill = [x for x in olines if x.startswith("TEST-6SET")]
    assert alert == drill[0]
    assert drill[0] in p.stderr and drill[0] in (tmp_path / "d.out").read_text()
    assert alert.rstrip().endswith("*** VERIFY FAILED ***")


def test_cli_dump4_per_region_limit(tmp_path):
    """--dump4 N prints the first N 4-sets of each region in processing order (s4.c:237-241)."""
    lo, hi, T, N = 1, 3 * 10 ** 6, 3, 500
    p = run([lo, hi, T, 16, "--dump4", N, "--noext", "--out", "q.out"], tmp_path)
    got = sorted((tmp_path / "q.out").read_text().splitlines(keepends=True))
    want = []
    for t in range(T):
        a, b = lo + (hi - lo) * t // T, lo + (hi - lo) * (t + 1) // T
        _, _, lines, _ = orc.search(a, b, dump4=N, flags=orc.NOEXT)
        want += lines
    assert got == sorted(want)


def test_cli_matches_reference_order_single_region(tmp_path):
    """With one region the CLI's result file equals the oracle's byte for byte (same order)."""
    run([10 ** 8, 10 ** 8 + 3 * 10 ** 6, 1, 18, "--out", "o.out"], tmp_path)
    _, _, olines, _ = orc.search(10 ** 8, 10 ** 8 + 3 * 10 ** 6)
    assert (tmp_path / "o.out").read_text() == "".join(olines)


def test_cli_block_controller_contract(tmp_path):
    """Three consecutive blocks from the controller's default frontier, each started, read back
    and sized as the archived block controller does (run_exhaustive.py:200-248), then audited as
    the packer and the verifier audit a block (compact.py:29-45, verify.py:140-164)."""
    frontier, done = 1_001_000_000_000, []
    for k in range(3):
        width = consumers.next_width(done, available_s=6.0)
        assert width >= 10 ** 8
        name = "block-%04d" % (k + 1)
        lo, hi = frontier, frontier + width
        rc, secs = consumers.run_block(CLI, tmp_path, name, lo, hi)
        assert rc == 0, (tmp_path / (name + ".err")).read_text()
        err = (tmp_path / (name + ".err")).read_text()
        ckpt = (tmp_path / (name + ".ckpt")).read_text()
        totals, maxima = consumers.parse_block(err, ckpt, lo, hi)
        consumers.check_checkpoint(ckpt, lo, hi, 16, 20, totals)
        lines = (tmp_path / (name + ".out")).read_text().splitlines(keepends=True)
        counts, five, near, max_ext = consumers.scan(lines, lo, hi)
        assert counts["multi"] == totals["multi-ext-4sets"] and totals["6-sets"] == 0
        assert max_ext <= maxima["extensions"][0]
        done.append({"lo": lo, "hi": hi, "elapsed": secs})
        frontier = hi
    assert not (tmp_path / "SIXSET_FOUND.txt").exists()
    assert [b["lo"] for b in done[1:]] == [b["hi"] for b in done[:-1]]       # contiguous frontier


def test_cli_sigterm_stops_at_a_batch_and_resumes(tmp_path):
    """The controller's deadline (run_exhaustive.py:221-224: SIGTERM, SIGKILL 10 s later): the
    CLI stops at the next batch boundary with the reference's exit status (killed by SIGTERM),
    prints no TOTAL line, leaves a checkpoint of the positions reached, and --resume completes
    the interval with the counters and result lines, none repeated, of one uninterrupted run."""
    lo, hi, T = 10 ** 11, 10 ** 11 + 3 * 10 ** 10, 16
    whole, part = tmp_path / "whole", tmp_path / "part"
    whole.mkdir()
    part.mkdir()
    ref = run([lo, hi, T, 20, "--out", "w.out", "--ckpt", "w.ckpt"], whole)
    args = [str(CLI), str(lo), str(hi), str(T), "20", "--out", "p.out", "--ckpt", "p.ckpt"]
    with (part / "p.err").open("w") as log:
        p = subprocess.Popen(args, cwd=part, stdout=subprocess.DEVNULL, stderr=log)
        t0 = time.monotonic()
        while not (part / "p.ckpt").exists() and p.poll() is None and time.monotonic() - t0 < 120:
            time.sleep(0.005)               # the first checkpoint follows the first batch
        p.send_signal(signal.SIGTERM)
        rc = p.wait(timeout=60)
    err = (part / "p.err").read_text()
    assert rc == -signal.SIGTERM, err
    assert "TOTAL:" not in err and "stopped by signal 15" in err
    ck = (part / "p.ckpt").read_text().splitlines()
    assert ck[0] == "s4ckpt v1" and ck[-1] != "DONE" and len(ck) == T + 2
    rows = [list(map(int, x.split())) for x in ck[2:]]
    assert any(r[1] < r[2] for r in rows)                                    # stopped part-way
    assert all(r[3] == r[1] - (lo + (hi - lo) * r[0] // T) for r in rows)    # S_done = positions reached
    res = run([lo, hi, T, 20, "--out", "p.out", "--ckpt", "p.ckpt", "--resume"], part)
    assert "RESUMED from checkpoint" in res.stderr
    assert (part / "p.ckpt").read_text().endswith("DONE\n")
    assert_stats_equal(parse_stderr(res.stderr), parse_stderr(ref.stderr), hist=False, maxima=False,
                       label="stopped + resumed")
    got = (part / "p.out").read_text().splitlines()
    want = (whole / "w.out").read_text().splitlines()
    assert len(got) == len(set(got)) and sorted(got) == sorted(want)
