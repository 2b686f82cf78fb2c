"""Shared test set-up.

Marker `gpu`: the test needs a B200 (sm_100a).  CPU runs use `-m "not gpu"`; the GPU
tests are the parity tests proper and always go through the C-ABI of lib/libps4.so.
"""
from __future__ import annotations

import gzip
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
PKG = REPO / "pairwise-square-sums_b200"
GOLDEN_DIR = REPO / "tests" / "golden"
sys.path.insert(0, str(PKG))
sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (run with -m gpu)")


def _ensure_built():
    """Build the oracle and the library in-tree if a fresh checkout lacks them."""
    if not (REPO / "oracle" / "libps4oracle.so").exists():
        subprocess.run(["make", "-C", str(REPO / "oracle")], check=True, capture_output=True)
    if not (PKG / "lib" / "libps4.so").exists() or not (PKG / "bin" / "s4gpu").exists():
        subprocess.run(["make", "-C", str(PKG)], check=True, capture_output=True)


_ensure_built()


def reference_tree():
    """The reference's source tree, where tests read its own modules and evidence: the
    PS4_REFERENCE_TREE environment variable, else the directory `make -C oracle ref` recorded in
    oracle/_ref/REF_DIR when it built the reference binary; None when neither names one that
    exists (on a GPU box the tree is absent and those tests skip)."""
    env = os.environ.get("PS4_REFERENCE_TREE")
    cand = Path(env) if env else None
    rec = REPO / "oracle" / "_ref" / "REF_DIR"
    if cand is None and rec.exists():
        cand = Path(rec.read_text().strip())
    return cand if cand is not None and (cand / "exhaustive").is_dir() else None


@pytest.fixture(scope="session")
def golden() -> dict:
    return json.loads((GOLDEN_DIR / "golden.json").read_text())


@pytest.fixture(scope="session")
def golden_1e7_lines() -> list[str]:
    return (GOLDEN_DIR / "s4_1e7.sorted.txt").read_text().splitlines(keepends=True)


@pytest.fixture(scope="session")
def golden_1e9_lines() -> list[str]:
    with gzip.open(GOLDEN_DIR / "s4_1e9.sorted.txt.gz", "rt") as f:
        return f.read().splitlines(keepends=True)


COUNTERS = ("S_done", "pairs", "S_ge3", "triples", "sets4", "sets5", "sets6", "multi", "ext_cand", "ext_sqrt")
MAXIMA = ("max_reps", "max_divisors", "max_extensions")


def assert_stats_equal(got: dict, want: dict, *, hist: bool = True, maxima: bool = True, label: str = ""):
    for k in COUNTERS:
        assert got[k] == want[k], f"{label} counter {k}: got {got[k]} want {want[k]}"
    if maxima:
        for k in MAXIMA:
            if k in want:
                assert got[k] == want[k], f"{label} {k}: got {got[k]} want {want[k]}"
    if hist and "hist5" in want:
        g = {int(a): int(b) for a, b in got["hist5"].items()}
        w = {int(a): int(b) for a, b in want["hist5"].items()}
        assert g == w, f"{label} hist5 differs"


def sha_sorted(lines) -> str:
    import hashlib
    return hashlib.sha256("".join(sorted(lines)).encode()).hexdigest()
