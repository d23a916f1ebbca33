"""Failure handling of bin/XT_Engine on the host, injected through its input
files (nothing here faults a GPU).

As in the reference program (Source_Code_4D_Fast), a configuration or
input error ends the run with exit status 1 and an ERROR line in
DEBUG_n0_delta_xy_<a>_delta_z_<b>.log:
  * view_info.txt missing or not in the "time - angle," grammar
    (initSparseAnglesfrmFile, XT_Init.c:130-156), or holding another number
    of views than --num_projections (XT_Init.c:158-161);
  * an unknown --sinobin or --initICD (XT_Engine.c computeWriteSinogram,
    XT_ICD_update.c initObject);
  * a missing input .bin file (Read4mBin, XT_IOMisc.c:89-90).
A .bin file shorter than its array is logged with the reference's message
(XT_IOMisc.c:92-94) and the run goes on, the unread rest taken as zero.

The cases that fail before the device is set up run on the CPU; the missing
and short sinogram files are read after it, so those cases need the GPU.
"""
import os
import subprocess

import numpy as np
import pytest

import common
import xtg

ENGINE = os.path.join(common.ROOT, "timbir-python_b200", "bin", "XT_Engine")
LOG = "DEBUG_n0_delta_xy_1_delta_z_1.log"

pytestmark = pytest.mark.skipif(not os.path.exists(ENGINE), reason="bin/XT_Engine not built")


def setup_run(tmp_path, NP=36, write_views=True, with_sino=True):
    p = common.params(N=32, NT=4, NP=NP)
    t, a = common.views(p)
    if write_views:
        xtg.write_view_file(str(tmp_path / "view_info.txt"), t, a)
    if with_sino:
        x, ax, y, w = common.data(p, t, a, seed=3)
        (tmp_path / "projection_n0.bin").write_bytes(y.tobytes())
        (tmp_path / "weight_n0.bin").write_bytes(w.tobytes())
    return p


def run(tmp_path, p, extra=()):
    r = subprocess.run([ENGINE] + p.cli() + ["--quiet"] + list(extra), cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    log = (tmp_path / LOG).read_text() if (tmp_path / LOG).exists() else ""
    return r.returncode, log, r.stderr


def test_missing_view_file(tmp_path):
    p = setup_run(tmp_path, write_views=False)
    rc, log, _ = run(tmp_path, p)
    assert rc == 1 and "ERROR: Error in reading file view_info.txt" in log


def test_malformed_view_file(tmp_path):
    p = setup_run(tmp_path)
    text = (tmp_path / "view_info.txt").read_text()
    (tmp_path / "view_info.txt").write_text(text.replace(",", ";", 3))
    rc, log, _ = run(tmp_path, p)
    assert rc == 1 and "is not correctly formatted to be read" in log


def test_view_count_mismatch(tmp_path):
    p = setup_run(tmp_path)
    p.num_projections = 40
    rc, log, _ = run(tmp_path, p)
    assert rc == 1 and "Number of projections read is 36 and expected is 40" in log


@pytest.mark.parametrize("opt,val,msg", [("sinobin", 2, "Cannot recognize sinobin value"),
                                         ("initICD", 5, "initICD value not recognized")])
def test_unknown_option_values(tmp_path, opt, val, msg):
    p = setup_run(tmp_path)
    setattr(p, opt, val)
    rc, log, _ = run(tmp_path, p)
    assert rc == 1 and msg in log


def test_missing_previous_stage_variance(tmp_path):
    """--initICD 1 reads the previous stage's variance_estimate_n0.bin first."""
    p = setup_run(tmp_path)
    p.initICD = 1
    rc, log, _ = run(tmp_path, p)
    assert rc == 1 and "ERROR: error in reading file variance_estimate_n0.bin" in log


@pytest.mark.gpu
def test_missing_sinogram_file(tmp_path):
    p = setup_run(tmp_path)
    os.unlink(tmp_path / "weight_n0.bin")
    rc, log, _ = run(tmp_path, p)
    assert rc == 1 and "ERROR: error in reading file weight_n0.bin" in log


@pytest.mark.gpu
def test_short_sinogram_file_is_logged_and_run_continues(tmp_path):
    p = setup_run(tmp_path)
    w = np.fromfile(tmp_path / "weight_n0.bin", np.float32)
    (tmp_path / "weight_n0.bin").write_bytes(w[: w.size - 100].tobytes())
    rc, log, err = run(tmp_path, p)
    assert rc == 0, log + err
    assert f"Number of elements read does not match required, required = {w.size}, read = {w.size - 100}" in log
    x = np.fromfile(tmp_path / "object_n0_time_0.bin", np.float32)
    assert x.size == 32 * 32 * 4 and np.all(np.isfinite(x))
