"""The reference's archived block controller and near-miss classifiers, run on bin/s4gpu output.

The reference runs its census as blocks: run_exhaustive.py's Search.run (archived in
exhaustive/evidence/exhaustive-2026-10-13-8h-compact.tar.gz, sources/exhaustive/run_exhaustive.py
:200-260) picks each block's width from the measured time of the last blocks, starts the search
binary on it with a deadline, watches SIXSET_FOUND.txt, and accepts a block through parse_result
(:74-94) into manifest.json.  Here that controller, unchanged, drives bin/s4gpu's blocks: the
blocks were written by s4gpu on a B200 (tests/golden/make_controller_blocks.py) and are replayed
by tests/controller_replay.py, since this machine has no GPU.  Two stand-ins keep the run short
and exact: the controller's clock (each block takes 2 s of it, so the adaptive widths are
known: 2e8, then 5e8 S) and its final audit subprocess (the archived audit reads the 1e12-census
output that is not part of the reference tree).  The archived independent verifier then checks
the run directory (verify_continuation.original.py check_blocks :78-108 and its line checks),
and the near-miss classifiers -- the verifier's euler_count (:61-74) and the audit's classify.py
Euler test -- classify the multi-extension records s4gpu found below 1e10 exactly as they
classify the reference's own.
"""
from __future__ import annotations

import importlib.util
import itertools
import json
import os
import shutil
import subprocess
import sys
import tarfile
import types
from pathlib import Path

import pytest

from conftest import GOLDEN_DIR, REPO, reference_tree

REF = reference_tree()
needs_ref = pytest.mark.skipif(REF is None, reason="the reference tree is not present")
FIX = Path(os.environ.get("PS4_CONTROLLER_BLOCKS", GOLDEN_DIR / "controller_blocks"))
ARCHIVE = "exhaustive-2026-10-13-8h-compact.tar.gz"
START = 10 ** 12
BLOCKS = [(START, START + 2 * 10 ** 8), (START + 2 * 10 ** 8, START + 7 * 10 ** 8)]


def _load(name: str, path: Path, extra_path=()):
    sys.path[:0] = [str(p) for p in extra_path]
    try:
        spec = importlib.util.spec_from_file_location(name, path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        for p in extra_path:
            sys.path.remove(str(p))
    return mod


@pytest.fixture(scope="module")
def archived(tmp_path_factory):
    """The archive's snapshot of the controller's source tree (its sources/ directory: s4.c,
    exhaustive/*.py, noneuler/classify.py), extracted without writing into the reference tree."""
    sys.dont_write_bytecode = True
    root = tmp_path_factory.mktemp("archived") / "root"
    with tarfile.open(REF / "exhaustive" / "evidence" / ARCHIVE) as tar:
        for m in tar.getmembers():
            if m.isfile() and "/sources/" in m.name:
                dest = root / m.name.split("/sources/", 1)[1]
                dest.parent.mkdir(parents=True, exist_ok=True)
                dest.write_bytes(tar.extractfile(m).read())
    return root


@pytest.fixture(scope="module")
def verifier():
    return _load("ref_verify_continuation", REF / "exhaustive" / "evidence" / "verify_continuation.original.py")


class Clock:
    """The controller's time module: time(), monotonic() and sleep() on one stand-in clock.
    sleep() waits for the running block to end and then advances the clock by its argument, so
    the controller's one poll per block sees it take exactly 2 s."""

    def __init__(self, t0: float):
        self.t = t0
        self.search = None

    def time(self):
        return self.t

    def monotonic(self):
        return self.t

    def sleep(self, s):
        if self.search is not None and self.search.child is not None:
            self.search.child.wait(timeout=120)
        self.t += s


@needs_ref
def test_archived_controller_drives_s4gpu_blocks(archived, verifier, tmp_path, monkeypatch):
    rx = _load("ref_run_exhaustive", archived / "exhaustive" / "run_exhaustive.py", [archived / "exhaustive"])
    t0 = 1.8e9
    clock = Clock(t0)
    audits = []
    rx.time = clock
    rx.subprocess = types.SimpleNamespace(
        Popen=subprocess.Popen, DEVNULL=subprocess.DEVNULL, TimeoutExpired=subprocess.TimeoutExpired,
        check_output=subprocess.check_output,
        run=lambda args, **kw: audits.append(args) or subprocess.CompletedProcess(args, 0))
    monkeypatch.setenv("PS4_REPLAY_DIR", str(FIX))
    out = tmp_path / "run"
    (out / "preflight").mkdir(parents=True)
    shutil.copy2(REPO / "tests" / "controller_replay.py", out / "preflight" / "s4")
    (out / "preflight" / "summary.json").write_text(json.dumps(
        {"passed": True, "source_sha256": rx.sha(archived / "s4.c"), "binary_sha256": rx.sha(out / "preflight" / "s4")}))
    # a 23.5 s search budget: the first block gets 8.5 s at the controller's default 36 ns per S (2e8 S),
    # the second 6.5 s at the first block's 2 s per 2e8 S (5e8 S); then the budget is spent
    search = rx.Search(out, t0, 23.5 / 3600, 0, 16, START)
    clock.search = search
    search.run()

    m = json.loads((out / "manifest.json").read_text())
    status = json.loads((out / "status.json").read_text())
    done = [(b["lo"], b["hi"]) for b in m["completed_blocks"]]
    assert done == BLOCKS
    assert [a["command"][1:] for a in m["attempts"]] == [
        [str(lo), str(hi), "16", "20", "--verify", "--out", str(out / f"block-{i + 1:04d}.out"), "--ckpt",
         str(out / f"block-{i + 1:04d}.ckpt")] for i, (lo, hi) in enumerate(BLOCKS)]
    assert all(b["complete"] and b["returncode"] == 0 and b["elapsed_seconds"] == 2.0 for b in m["completed_blocks"])
    assert status["status"] == "budget_exhausted" and status["audit_passed"]
    assert status["frontier"] == BLOCKS[-1][1] and status["six_sets"] == 0
    assert status["five_sets"] == sum(b["totals"]["5-sets"] for b in m["completed_blocks"]) > 0
    assert len(audits) == 1 and audits[0][1].endswith("exhaustive/audit_exhaustive.py")
    for b in m["completed_blocks"]:
        assert b["totals"]["S_done"] == b["hi"] - b["lo"]
        assert b["capacity_maxima"]["representations"]["limit"] == 512

    # the archived independent verifier on the run directory
    frontier, files, maxima = verifier.check_blocks(out, m)
    assert frontier == BLOCKS[-1][1] and len(files) == 2
    for path, lo, hi, stats in files:
        five = multi = 0
        for line in path.read_text().splitlines():
            s = int(line.rsplit("S=", 1)[1])
            assert lo <= s < hi
            if line.startswith("5:"):
                vals = tuple(sorted(map(int, line[4:line.index("]")].split(","))))
                assert len(set(vals)) == 5 and sum(vals[:4]) == s
                assert all(verifier.square(a + b) for a, b in itertools.combinations(vals, 2))
                five += 1
            else:
                total, near, hits = verifier.parse_multi(line)
                assert total == s and not hits
                multi += 1
        assert (five, multi, 0) == (stats["5-sets"], stats["multi-ext-4sets"], stats["6-sets"])


def _classify(lines, verifier, classify):
    """near-miss primitive 6-set -> (non-square pair, Euler squares by the verifier's euler_count,
    Euler squares by the audit's classify.py test), over the records' M lines."""
    out = {}
    for line in lines:
        _, near, hits = verifier.parse_multi(line)
        assert not hits
        for vals, bad in near.items():
            by_audit = 0
            for a in (v for v in vals if v not in bad):
                x = bad + (a,)
                y = tuple(v for v in vals if v not in x)
                _, roots = classify.latin_square(x, y)
                by_audit += classify.euler_signs(roots) is not None
            out[vals] = (bad, verifier.euler_count(vals, bad), by_audit)
    return out


@needs_ref
def test_near_miss_classification_of_s4gpu_records(archived, verifier):
    classify = _load("ref_classify", archived / "noneuler" / "classify.py")
    gpu = (FIX / "s4gpu_m_lines_1e10.txt").read_text().splitlines()
    ref = (GOLDEN_DIR / "m_lines_1e10.txt").read_text().splitlines()
    assert len(gpu) == 268 and sorted(gpu) == sorted(ref)
    got = _classify(gpu, verifier, classify)
    want = _classify(ref, verifier, classify)
    assert got == want and len(got) > 60                              # 268 records, 68 primitive near misses
    assert all(e1 == e2 for _, e1, e2 in got.values())             # the two Euler tests agree
    assert classify.load(str(FIX / "s4gpu_m_lines_1e10.txt")) == classify.load(str(GOLDEN_DIR / "m_lines_1e10.txt"))
    assert max(e for _, e, _ in got.values()) <= 4                    # four choices of the third member
