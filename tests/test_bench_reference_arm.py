"""bench.py's reference arm on the CPU: `--impl reference` times the reference's own s4 (or the
oracle port where s4 is not built) on a bounded sample of [1,1e10) and prints one JSON line
with the keys the bench contract asks for; under a launcher every rank but 0 exits quietly."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

S4 = REPO / "oracle" / "_ref" / "s4"
PORT = REPO / "oracle" / "ps4_oracle"


def _run(env_extra: dict) -> subprocess.CompletedProcess:
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0", "--ref-budget", "0.4", "--ref-slice", "2000000"],
                          capture_output=True, text=True, env=env, timeout=600, cwd=REPO)


@pytest.mark.skipif(not S4.exists() and not PORT.exists(), reason="neither oracle/_ref/s4 nor the oracle port is built")
def test_reference_arm_line():
    p = _run({})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] and d["unit"] == "S/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["kind"] == ("reference" if S4.exists() else "port")
    if S4.exists():
        assert "slices of 2000000 S" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
