"""CPU tests of the product's host side: the C-ABI libraries load and export
every symbol their headers declare (no GPU call), the host geometry / H_r /
A-matrix match the reference's (golden fixtures, bit for bit), the CLI
parser accepts the launcher's command line, and the data generator is
deterministic."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import common
import xtg

ROOT = common.ROOT
PKG = os.path.join(ROOT, "timbir-python_b200")


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:xtg(?:en)?|xtc)_[a-z0-9_]+)\s*\(", txt)))


def test_headers_match_binding_lists():
    assert declared("xtg.h") == sorted(xtg.XTG_SYMBOLS)
    assert declared("xt_gen.h") == sorted(xtg.XTGEN_SYMBOLS)
    assert declared("xtg_cnn.h") == sorted(xtg.XTC_SYMBOLS)


@pytest.mark.parametrize("lib,names", [("libxtgpu.so", "XTG_SYMBOLS"), ("libxtgen.so", "XTGEN_SYMBOLS"),
                                       ("libxtgpu.so", "XTC_SYMBOLS")])
def test_libraries_export_declared_symbols(lib, names):
    L = C.CDLL(os.path.join(PKG, "lib", lib))
    for s in getattr(xtg, names):
        assert hasattr(L, s), s
    nm = subprocess.run(["nm", "-D", "--defined-only", os.path.join(PKG, "lib", lib)], capture_output=True,
                        text=True).stdout
    for s in getattr(xtg, names):
        assert re.search(rf"\bT {s}\b", nm), s


def test_abi_version_without_gpu():
    assert xtg.gpu_lib().xtg_abi_version() == 1


def test_create_fails_loudly_without_gpu():
    """No CPU fallback: without an sm_100 device xtg_create reports an error."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    p = common.params()
    t, a = common.views(p)
    with pytest.raises(RuntimeError, match="xtg_create"):
        xtg.Context(p, t, a)


GOLD = {
    "plain3d": dict(N=32, NT=4, NP=36),
    "timbir4d": dict(N=16, NT=2, NP=48, n_time=3),
    "coarse_xy2": dict(N=32, NT=4, NP=30, dxy=2.0, dz=2.0),
    "zinger_nhicd": dict(N=24, NT=4, NP=30, zinger=True, nhicd=True, offset=2, var=1),
}


@pytest.mark.parametrize("name", sorted(GOLD))
def test_host_geometry_matches_reference(name):
    g = dict(np.load(os.path.join(common.GOLDEN, name + ".npz")))
    p = common.params(**GOLD[name])
    geo, cs, sn, fov, hr = xtg.host_geometry(p, g["times"], g["angles"])
    assert np.array_equal(hr, g["hr"])
    assert np.array_equal(cs, g["cosv"]) and np.array_equal(sn, g["sinv"])
    d = g["derived"]
    for k, name_ in enumerate(("delta_r", None, "R0", "RMax", "x0", "y0", "delta_xy", "OffsetR", "Sigma_S_Q",
                               "Sigma_S_Q_P", "Sigma_T_Q", "Sigma_T_Q_P", "TF")):
        if name_:
            assert np.float32(getattr(geo, name_)) == np.float32(d[k]), name_
    assert np.array_equal(np.array(geo.SF[:], np.float32), d[13:40].astype(np.float32))
    # frame of each view, initSparseAnglesOfObject
    pn, pi = g["proj_num"], g["proj_idx"]
    want = np.repeat(np.arange(len(pn)), pn)
    assert np.array_equal(fov[pi], want)


@pytest.mark.parametrize("name", ["plain3d", "coarse_xy2"])
def test_host_amatrix_matches_reference(name):
    g = dict(np.load(os.path.join(common.GOLDEN, name + ".npz")))
    p = common.params(**GOLD[name])
    for q, (row, col, view) in enumerate(g["a_trip"][:120]):
        v, i = xtg.host_amatrix(p, g["times"], g["angles"], int(row), int(col), int(view))
        n = int((g["a_idx"][q] >= 0).sum())
        assert np.array_equal(v, g["a_vals"][q, :n]) and np.array_equal(i, g["a_idx"][q, :n])


def test_generator_forward_matches_reference():
    g = dict(np.load(os.path.join(common.GOLDEN, "timbir4d.npz")))
    p = common.params(**GOLD["timbir4d"])
    assert np.array_equal(xtg.forward_cpu(p, g["times"], g["angles"], g["x_true"]), g["ax"])


def test_generator_deterministic():
    ax = np.random.default_rng(0).random((7, 9, 4)).astype(np.float32)
    y1, w1 = xtg.measure(ax, 1e4, 5, zinger_frac=0.1)
    y2, w2 = xtg.measure(ax, 1e4, 5, zinger_frac=0.1)
    assert np.array_equal(y1, y2) and np.array_equal(w1, w2)
    assert (w1 >= 1).all() and np.all(np.abs(np.log(1e4 / w1) - y1) >= 0)
    x1 = xtg.phantom((2, 3, 16, 16), 4, 0.01, 9, n_moving=2, max_shift=1.0, growing=1)
    x2 = xtg.phantom((2, 3, 16, 16), 4, 0.01, 9, n_moving=2, max_shift=1.0, growing=1)
    assert np.array_equal(x1, x2) and x1.max() > 0


def test_interlaced_views_follow_launcher():
    """gen_interlaced_views_0_to_Inf (XT_Interlaced_Angles.py:107-139), K=8, N_theta=256."""
    t, a = xtg.views_interlaced(8, 256, 64)
    i = np.arange(64)
    L = 256 // 8
    br = np.array([int(format(int(v), "03b")[::-1], 2) for v in (i // L) % 8])
    v = i * 8 + br
    assert np.allclose(t, v / 8.0) and np.allclose(a, v * 180.0 / 256)


def test_view_file_roundtrip(tmp_path):
    t, a = xtg.views_interlaced(4, 16, 12)
    f = str(tmp_path / "view_info.txt")
    t2, a2 = xtg.write_view_file(f, t, a)
    txt = open(f).read().strip().splitlines()
    assert len(txt) == 12 and all(re.fullmatch(r"[0-9.]+ - [0-9.]+,", s) for s in txt)
    assert np.allclose(t2, t) and np.allclose(a2, a)


def test_engine_cli_rejects_hdf_and_parses_launcher_line(tmp_path):
    """The launcher's command string (XT_MBIR_Reconstruction.py:124) parses; an
    unknown option is reported and skipped like the reference; --readSino4mHDF
    exits 1 with a message (no libhdf5 here)."""
    eng = os.path.join(PKG, "bin", "XT_Engine")
    line = ("--p 1.2 --sigma_s 200000 --sigma_t 200000 --c_s 1e-06 --c_t 1e-06 --delta_xy 1 --delta_z 1 "
            "--length_r 32 --length_t 4 --voxel_thresh 0 --cost_thresh 100 --iter 2 --rotation_center 16 "
            "--alpha 1.5 --sinobin 1 --initICD 0 --Rtime0 0 --Rtime_delta 36 --Rtime_num 1 --num_projections 36 "
            "--x_start 0 --x_width 32 --N_r 32 --N_t 4 --detector_slice_begin 0 --detector_slice_num 4 "
            "--num_threads 1 --radius_obj 32 --updateProjOffset 0 --writeTiff 0 --zingerT 100000 --zingerDel 0 "
            "--Est_of_Var 1 --phantom_N_xy 32 --phantom_N_z 4 --no_NHICD --readSino4mHDF --bogus_option")
    r = subprocess.run([eng] + line.split(), cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1
    assert "Cannot recognize argument" in r.stdout
    assert os.path.exists(tmp_path / "DEBUG_HDF_Read_n0.log")
