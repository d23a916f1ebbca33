"""The drop-in boundary end to end: bin/XT_Engine run with the launcher's
command line in a directory holding the launcher's input files, against the
reference XT_Engine's output files for the same command (tests/golden/
engine_*.npz, made by tests/golden/make_engine_golden.py).

Tolerances:
  * --gpu_sequential (the reference's visiting order and random draws): the
    object within 1e-4 of its range, every per-iteration cost within 1e-4
    relative, the variance estimate within 1e-4 relative, the offset and the
    magnitude-update map within 1e-3 (they are sums of the object's changes);
  * the default parallel schedule: the same output files with the same sizes,
    a cost that never increases, and the reference's cost after the same
    number of iterations reached within 1e-2 relative or bettered.
"""
import os
import subprocess

import numpy as np
import pytest

import common

pytestmark = pytest.mark.gpu

ENGINE = os.path.join(common.ROOT, "timbir-python_b200", "bin", "XT_Engine")
# engine_launcher: the launcher's physical lengths (delta_t = 0.65) and its
# positivity-off build
NAMES = ["engine_plain", "engine_counts_multires", "engine_launcher"]


def run_engine(name, tmp_path, extra):
    g = dict(np.load(os.path.join(common.GOLDEN, name + ".npz")))
    for k, v in g.items():
        if k.startswith("in:"):
            (tmp_path / k[3:]).write_bytes(v.tobytes())
    # the reference binary's compile-time POSITIVITY_CONSTRAINT as this
    # engine's runtime switch (older fixtures: compiled with it)
    pos = int(g["positivity"]) if "positivity" in g else 1
    args = [str(s) for s in g["args"]] + ["--positivity", str(pos)]
    r = subprocess.run([ENGINE] + args + extra, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    want = {k[4:]: np.frombuffer(v.tobytes(), np.float32) for k, v in g.items() if k.startswith("out:")}
    got = {f: np.fromfile(tmp_path / f, np.float32) for f in want if (tmp_path / f).exists()}
    assert set(got) == set(want)
    for f in want:
        assert got[f].size == want[f].size, f
    return got, want


@pytest.mark.parametrize("name", NAMES)
def test_engine_sequential_matches_reference_files(name, tmp_path):
    got, want = run_engine(name, tmp_path, ["--gpu_sequential", "--quiet"])
    ref = want["object_n0_time_0.bin"]
    scale = float(np.abs(ref).max())
    assert np.max(np.abs(got["object_n0_time_0.bin"] - ref)) / scale < 1e-4
    np.testing.assert_allclose(got["cost_n0.bin"], want["cost_n0.bin"], rtol=1e-4)
    np.testing.assert_allclose(got["variance_estimate_n0.bin"], want["variance_estimate_n0.bin"], rtol=1e-4)
    d = want["proj_offset_n0.bin"]
    np.testing.assert_allclose(got["proj_offset_n0.bin"], d, rtol=1e-3, atol=1e-3 * max(float(np.abs(d).max()), 1e-6))
    m = want["mag_update_map_n0.bin"]
    np.testing.assert_allclose(got["mag_update_map_n0.bin"], m, rtol=1e-3, atol=1e-3 * float(np.abs(m).max()))


@pytest.mark.parametrize("name", NAMES)
def test_engine_parallel_schedule_files_and_cost(name, tmp_path):
    got, want = run_engine(name, tmp_path, ["--quiet"])
    c = got["cost_n0.bin"].astype(np.float64)
    assert np.all(np.diff(c) <= 1e-6 * np.abs(c[:-1]))
    assert c[-1] <= float(want["cost_n0.bin"][-1]) * (1 + 1e-2)


@pytest.mark.parametrize("start", [["--gpu_fbp_start"], ["--gpu_multires_start", "10"]])
def test_engine_warm_start_switches(start, tmp_path):
    """The launcher's command plus a warm-start switch runs end to end: the
    same output files, and a cost that never increases after the start (what
    the starts gain is measured by bench.py and tests/test_learned_start.py;
    on this 36-view toy case the FBP image itself costs more than zero)."""
    got, want = run_engine("engine_plain", tmp_path, ["--quiet"] + start)
    c = got["cost_n0.bin"].astype(np.float64)
    assert np.all(np.isfinite(c)) and c.size == want["cost_n0.bin"].size
    assert np.all(np.diff(c) <= 1e-6 * np.abs(c[:-1]))
