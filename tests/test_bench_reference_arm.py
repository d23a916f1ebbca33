"""bench.py's reference arm on the CPU (it times the reference's own compiled
routines, oracle/_ref, on the host cores): one JSON line with the benchmark's
contract keys at a small size, and under a multi-rank launch only rank 0
prints it.  Skipped where the reference build is absent."""
import json
import os
import subprocess
import sys

import pytest

from oracle.oracle import ref_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref (the reference build) is not built here")

CMD = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nxy", "64", "--steps", "1",
       "--warmup", "1"]


def run(env_extra):
    env = dict(os.environ, **env_extra)
    p = subprocess.run(CMD, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return [l for l in p.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    lines = run({"RANK": "0", "WORLD_SIZE": "1"})
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "voxel-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("plain3d_64x64")


def test_reference_arm_other_ranks_print_nothing():
    assert run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
