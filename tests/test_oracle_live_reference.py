"""The CPU oracle restatement (oracle/xt_oracle.c) against the reference's own
routines compiled from its sources (oracle/_ref), live, on seeded random
geometries beyond the committed fixtures: detector sizes, view counts,
delta_xy / delta_z of 1 and 2, rotation centres off the middle, zinger
correction and NHICD on and off, offset re-estimation; the launcher's
physical detector pitch (delta_r = delta_t = 0.65) with positivity on and
off; and 4D cases of 2-3 frames of interlaced views with moving objects.  Skipped where the
reference build is absent (the committed fixtures pin the oracle there).

Single-threaded, so everything is compared bit for bit: the geometry
derivation, the detector response H_r, the view tables, A-matrix columns,
the forward projection and e = y - Ax - d, the FP32 MAP cost, and the object,
cost, offset, variance and magnitude map after each of three iterations from
the reference's RNG seed.
"""
import os

import numpy as np
import pytest

import common
import xtg
from oracle.oracle import Oracle, Reference, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref (the reference build) is not built here")


def random_case(seed):
    rng = np.random.default_rng(seed)
    dxy = float(rng.choice([1.0, 2.0]))
    dz = float(rng.choice([1.0, 2.0]))
    n_vox = int(rng.choice([8, 10, 12]))
    N = int(n_vox * dxy)
    NT = int(rng.choice([2, 4]) * dz)
    NP = int(rng.choice([18, 24, 30]))
    zinger = bool(rng.integers(0, 2))
    nhicd = bool(rng.integers(0, 2))
    offset = int(rng.choice([0, 2]))
    rot = N / 2.0 + float(rng.choice([0.0, 0.5, -1.0]))
    pk = dict(N=N, NT=NT, NP=NP, dxy=dxy, dz=dz, zinger=zinger, nhicd=nhicd, offset=offset, rot=rot)
    dk = dict(seed=100 + seed, zfrac=0.01 if zinger else 0.0)
    return pk, dk


def random_case_4d(seed):
    """Frames of interlaced views (the launcher's bit-reversed sub-frames) and
    a phantom with moving ellipsoids."""
    rng = np.random.default_rng(1000 + seed)
    n_time = int(rng.choice([2, 3]))
    K, N_theta = [(4, 16), (2, 8)][int(rng.integers(0, 2))]
    N = int(rng.choice([12, 16]))
    pk = dict(N=N, NT=2, NP=n_time * N_theta, n_time=n_time, nhicd=bool(rng.integers(0, 2)))
    dk = dict(seed=200 + seed, moving=2)
    return pk, dk, (K, N_theta)


def compare(pk, dk, interlaced, seed, tmp_path, monkeypatch):
    p = common.params(**pk)
    monkeypatch.chdir(tmp_path)
    t, a = common.views(p, interlaced)
    xtg.write_view_file("view_info.txt", t, a)
    x, _, y, w = common.data(p, t, a, **dk)
    r = Reference(p)
    o = Oracle(p, t, a)
    try:
        assert np.array_equal(o.derived(), r.derived())
        assert np.array_equal(o.hr(), r.hr())
        for got, want in zip(o.views(), r.views()):
            assert np.array_equal(got, want)
        rng = np.random.default_rng(seed)
        for _ in range(120):
            row, col, view = int(rng.integers(0, r.N_y)), int(rng.integers(0, r.N_x)), int(rng.integers(0, r.N_p))
            vo, io = o.amatrix(row, col, view)
            vr, ir = r.amatrix(row, col, view)
            assert np.array_equal(vo, vr) and np.array_equal(io, ir), (row, col, view)
        for m in (o, r):
            m.set_sino(y, w)
            m.set_object(x)
            m.init_error_sino()
        assert np.array_equal(o.error_sino(), r.error_sino())
        assert np.array_equal(np.float32(o.cost()), np.float32(r.cost()))
        for m in (o, r):
            m.set_object(np.zeros(m.obj_shape, m.real))
            m.init_error_sino()
            m.srandom2(761521)
        for it in range(1, 4):
            o.iterate(it)
            r.iterate(it)
            assert np.array_equal(o.object(), r.object()), f"object after iteration {it}"
            assert np.array_equal(np.float32(o.cost()), np.float32(r.cost())), f"cost after iteration {it}"
            assert np.array_equal(o.offset(), r.offset())
            assert np.float32(o.var()) == np.float32(r.var())
            assert np.array_equal(o.magmap(), r.magmap())
        assert np.array_equal(o.error_sino(), r.error_sino())
    finally:
        o.close()
        r.close()


@pytest.mark.parametrize("seed", range(8))
def test_oracle_matches_reference_live(seed, tmp_path, monkeypatch):
    pk, dk = random_case(seed)
    compare(pk, dk, None, seed, tmp_path, monkeypatch)


@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_reference_live_launcher_geometry(seed, tmp_path, monkeypatch):
    """The launcher's geometry: physical lengths (length_r = 0.65 N_r,
    length_t = 0.65 N_t, so delta_r = delta_t = 0.65 and the voxel update's
    A * delta_t differs from the projector's A, XT_VoxUpdate.c:27,67 against
    XT_ForwardProject.c:17), and positivity off in every other case (the
    launcher's build, 4D_Recon_Launcher_for_Real_Data/XT_Initialize.py:257)."""
    pk, dk = random_case(50 + seed)
    pk.update(pitch=0.65, positivity=seed % 2)
    compare(pk, dk, None, seed, tmp_path, monkeypatch)


@pytest.mark.parametrize("seed", range(4))
def test_oracle_matches_reference_live_4d(seed, tmp_path, monkeypatch):
    pk, dk, views = random_case_4d(seed)
    compare(pk, dk, views, seed, tmp_path, monkeypatch)
