"""Host logic of the drop-in CLI that runs before any device work: argv grammar,
checkpoint guards and the s4ckpt v1 parameter checks (exhaustive/s4.c:394-433)."""
from __future__ import annotations

import subprocess

import pytest

from conftest import PKG

CLI = PKG / "bin" / "s4gpu"


def run(args, cwd):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=120)


def test_existing_checkpoint_needs_resume(tmp_path):
    (tmp_path / "c.ckpt").write_text("s4ckpt v1\n1 100 1 1048576\n0 100 100 0 0 0 0 0 0 0 0 0 0\nDONE\n")
    p = run([1, 100, 1, 20, "--ckpt", "c.ckpt"], tmp_path)
    assert p.returncode == 1
    assert "checkpoint c.ckpt exists: add --resume to continue it, or delete it to start over" in p.stderr


def test_resume_of_done_checkpoint_is_a_no_op(tmp_path):
    (tmp_path / "c.ckpt").write_text("s4ckpt v1\n1 100 2 1048576\n0 50 50 49 0 0 0 0 0 0 0 0 0\n"
                                     "1 100 100 50 0 0 0 0 0 0 0 0 0\nDONE\n")
    p = run([1, 100, 0, 20, "--ckpt", "c.ckpt", "--resume"], tmp_path)   # threads from the checkpoint
    assert p.returncode == 0
    assert "checkpoint c.ckpt marks S in [1, 100) as complete; nothing to do" in p.stderr


@pytest.mark.parametrize("args", [[1, 101, 2, 20], [1, 100, 3, 20], [1, 100, 2, 19]])
def test_resume_parameter_mismatch(tmp_path, args):
    (tmp_path / "c.ckpt").write_text("s4ckpt v1\n1 100 2 1048576\n0 50 50 49 0 0 0 0 0 0 0 0 0\n"
                                     "1 100 100 50 0 0 0 0 0 0 0 0 0\n")
    p = run([*args, "--ckpt", "c.ckpt", "--resume"], tmp_path)
    assert p.returncode == 1
    assert "current parameters differ" in p.stderr


def test_bad_checkpoint_header(tmp_path):
    (tmp_path / "c.ckpt").write_text("something else\n")
    p = run([1, 100, 1, 20, "--ckpt", "c.ckpt", "--resume"], tmp_path)
    assert p.returncode == 1 and "bad header" in p.stderr


def test_bad_thread_line(tmp_path):
    (tmp_path / "c.ckpt").write_text("s4ckpt v1\n1 100 2 1048576\n0 50 50 49 0 0 0 0 0 0 0 0 0\n"
                                     "1 100 99 50 0 0 0 0 0 0 0 0 0\n")
    p = run([1, 100, 2, 20, "--ckpt", "c.ckpt", "--resume"], tmp_path)
    assert p.returncode == 1 and "bad line for thread 1" in p.stderr


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU refusal")
def test_cli_without_gpu_exits_1(tmp_path):
    p = run([1, 1000, 1, 20], tmp_path)
    assert p.returncode == 1 and p.stderr.startswith("s4gpu: ")
