"""A block of the drop-in CLI's output (tests/golden/cli_block, written by make_cli_block.py on
a B200) handed to the consumers of `s4` blocks: the restatements in tests/consumers.py always,
and the reference's own code unchanged where the reference tree is at hand -- the archived
block controller's parse_result (run_exhaustive.py:74-94, read from an evidence archive), the
packer's checkpoint audit (compact.py:29-45) and the verifier's line scan with the archived
M-record reduction (verify.py:102-164, verify_continuation.original.py:42-58).  Mistakes are
planted in copies of the fixture, on the CPU, to show both sides reject them."""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import tarfile
from pathlib import Path

import pytest

import consumers
from conftest import GOLDEN_DIR, reference_tree
from golden.make_golden import parse_stderr

BLOCK = GOLDEN_DIR / "cli_block"
REF_TREE = reference_tree()
HAVE_REF = REF_TREE is not None and (REF_TREE / "exhaustive" / "verify.py").is_file()
CONTROLLER_ARCHIVE = "exhaustive-2026-10-13-8h-compact.tar.gz"
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="the reference tree is not present")


@pytest.fixture(scope="module")
def block():
    meta = json.loads((BLOCK / "block.json").read_text())
    files = {ext: (BLOCK / (meta["id"] + "." + ext)).read_text() for ext in ("out", "err", "ckpt")}
    return meta, files


class Audit:
    """The validator object the packer's checks report to (compact.py:29-45): raises."""

    def require(self, cond, message):
        if not cond:
            raise AssertionError(message)


def _load(name: str, path: Path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def ref(tmp_path_factory):
    """The reference's consumer modules, imported from its tree without writing into it."""
    sys.dont_write_bytecode = True
    ex = REF_TREE / "exhaustive"
    tmp = tmp_path_factory.mktemp("controller")
    with tarfile.open(ex / "evidence" / CONTROLLER_ARCHIVE) as tar:
        for m in tar.getmembers():
            if m.name.endswith(("/sources/exhaustive/run_exhaustive.py", "/sources/exhaustive/cpu_budget.py")):
                (tmp / Path(m.name).name).write_bytes(tar.extractfile(m).read())
    sys.path[:0] = [str(ex), str(tmp)]
    try:
        verify = _load("ref_verify", ex / "verify.py")           # imports compact and the archived verifier
        controller = _load("ref_run_exhaustive", tmp / "run_exhaustive.py")
    finally:
        sys.path.remove(str(ex))
        sys.path.remove(str(tmp))
    return {"verify": verify, "compact": verify.compact, "original": verify.original, "controller": controller}


# ------------------------------------------------------------------ restatements, always

def test_block_is_the_reference_census(block, golden, golden_1e7_lines):
    """The fixture block is s4's census of [1, 1e7): the same sorted lines and counters."""
    meta, f = block
    assert (meta["lo"], meta["hi"], meta["threads"], meta["chunk_log2"]) == (1, 10 ** 7, 16, 20)
    assert sorted(f["out"].splitlines(keepends=True)) == golden_1e7_lines
    st = parse_stderr(f["err"])
    for k in ("S_done", "pairs", "S_ge3", "triples", "sets4", "sets5", "sets6", "multi", "ext_cand", "ext_sqrt"):
        assert st[k] == golden["runs"]["1e7"][k], k


def test_restated_consumers_accept_block(block):
    meta, f = block
    lo, hi = meta["lo"], meta["hi"]
    totals, maxima = consumers.parse_block(f["err"], f["ckpt"], lo, hi)
    consumers.check_checkpoint(f["ckpt"], lo, hi, meta["threads"], meta["chunk_log2"], totals)
    counts, five, near, max_ext = consumers.scan(f["out"].splitlines(keepends=True), lo, hi)
    assert counts == {"five": 123, "multi": 2} and totals["multi-ext-4sets"] == 2
    assert len(near) >= 1 and max_ext <= maxima["extensions"][0]


def _planted(f: dict):
    """Copies of the block, each with one mistake a consumer must catch."""
    ck = f["ckpt"].splitlines(keepends=True)
    row = ck[3].split()
    row[3] = str(int(row[3]) - 1)
    out = f["out"].splitlines(keepends=True)
    five = next(i for i, x in enumerate(out) if x.startswith("5: "))
    bad_five = out[five].replace("[", "[1", 1)
    return {
        "ckpt_not_done": (f["err"], "".join(ck[:-1]), f["out"]),
        "ckpt_row_count": (f["err"], "".join(ck[:3] + [" ".join(row) + "\n"] + ck[4:]), f["out"]),
        "ckpt_region_missing": (f["err"], "".join(ck[:2] + ck[3:]), f["out"]),
        "stderr_fatal": (f["err"] + "FATAL: divisor capacity exceeded; this interval is NOT certified complete\n",
                         f["ckpt"], f["out"]),
        "stderr_two_totals": (f["err"] + [x for x in f["err"].splitlines(keepends=True)
                                          if x.startswith("TOTAL:")][0], f["ckpt"], f["out"]),
        "out_bad_five": (f["err"], f["ckpt"], "".join(out[:five] + [bad_five] + out[five + 1:])),
        "out_foreign_line": (f["err"], f["ckpt"], f["out"] + "4: [1,2,3,4] S=10\n"),
    }


def _restated_accepts(meta, err, ckpt, out) -> bool:
    lo, hi = meta["lo"], meta["hi"]
    try:
        totals, _ = consumers.parse_block(err, ckpt, lo, hi)
        consumers.check_checkpoint(ckpt, lo, hi, meta["threads"], meta["chunk_log2"], totals)
        consumers.scan(out.splitlines(keepends=True), lo, hi)
    except (AssertionError, ValueError, KeyError, IndexError):
        return False
    return True


def test_restated_consumers_reject_planted_mistakes(block):
    meta, f = block
    for name, (err, ckpt, out) in _planted(f).items():
        assert not _restated_accepts(meta, err, ckpt, out), name


def test_restated_parse_multi_on_archived_records():
    """parse_multi's reduction on the M records of s4's [1, 1e10) census: 6-set free, every
    record reduces to primitive 14-of-15 near misses, 68 distinct ones (most records are square
    multiples of another's six values)."""
    lines = (GOLDEN_DIR / "m_lines_1e10.txt").read_text().splitlines()
    near = {}
    for line in lines:
        S, partial, sixes = consumers.parse_multi(line)
        assert not sixes and S < 10 ** 10
        near.update(partial)
    assert len(lines) == 268 and len(near) == 68


# ------------------------------------------------------------------ the reference's own code

def _ref_accepts(ref, meta, err, ckpt, out, tmp: Path) -> bool:
    lo, hi = meta["lo"], meta["hi"]
    (tmp / "b.err").write_text(err)
    (tmp / "b.ckpt").write_text(ckpt)
    (tmp / "b.out").write_text(out)
    try:
        totals, _ = ref["controller"].parse_result(tmp / "b.err", lo, hi, tmp / "b.ckpt")
        ref["verify"].read_stats(err)
        ref["compact"].check_checkpoint(Audit(), ckpt, {"lo": lo, "hi": hi, "totals": totals},
                                        {"threads": meta["threads"], "chunk_log2": meta["chunk_log2"]})
        with (tmp / "b.out").open("rb") as s:
            ref["verify"].scan(s, lo, hi, set(), {})
    except (AssertionError, ValueError, KeyError, IndexError, TypeError, RuntimeError):
        return False
    return True


@needs_ref
def test_reference_consumers_accept_block(ref, block, tmp_path):
    meta, f = block
    lo, hi = meta["lo"], meta["hi"]
    assert _ref_accepts(ref, meta, f["err"], f["ckpt"], f["out"], tmp_path)
    (tmp_path / "b.err").write_text(f["err"])
    (tmp_path / "b.ckpt").write_text(f["ckpt"])
    (tmp_path / "b.out").write_text(f["out"])
    totals, maxima = ref["controller"].parse_result(tmp_path / "b.err", lo, hi, tmp_path / "b.ckpt")
    mine_totals, mine_maxima = consumers.parse_block(f["err"], f["ckpt"], lo, hi)
    assert totals == mine_totals
    assert {k: (v["used"], v["limit"]) for k, v in maxima.items()} == mine_maxima
    five, near = set(), {}
    with (tmp_path / "b.out").open("rb") as s:
        counts, _digest, max_ext = ref["verify"].scan(s, lo, hi, five, near)
    mc, mfive, mnear, mmax = consumers.scan(f["out"].splitlines(keepends=True), lo, hi)
    assert (counts["five"], counts["multi"], max_ext) == (mc["five"], mc["multi"], mmax)
    assert five == mfive and near == mnear


@needs_ref
def test_reference_consumers_reject_planted_mistakes(ref, block, tmp_path):
    meta, f = block
    for name, (err, ckpt, out) in _planted(f).items():
        assert not _ref_accepts(ref, meta, err, ckpt, out, tmp_path), name


@needs_ref
def test_reference_parse_multi_equals_restatement(ref):
    for line in (GOLDEN_DIR / "m_lines_1e10.txt").read_text().splitlines():
        assert ref["original"].parse_multi(line) == consumers.parse_multi(line)
