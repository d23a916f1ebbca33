"""The allocation-free NHICD threshold entry point, through the C ABI.

xtg_nhicd_threshold_noalloc serves callers that cannot call cudaMalloc (a
host that owns all device memory through its own pool, for instance a
beamline acquisition loop that must not stall on cudaMalloc's implicit
device-wide synchronisation): the caller passes device buffers, the library's
scratch is a fixed array inside it.  Its thresholds and selections must equal
those of the context-based xtg_nhicd_select -- bit-exact, the tolerance the
other NHICD tests use -- on two calls in a row (the second call reuses the
scratch the first one left behind), and oversized inputs must be refused.

This file is collected last so that a run stopping at the first failure has
run every other test already; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import common
import xtg

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_thresholds_match_context_entry_point_twice():
    import torch

    p = common.params(N=32, NT=8, NP=12, threads=2)
    t, a = common.views(p)
    c = xtg.Context(p, t, a)
    nmaps, ny, nx = c.N_time * c.nzb, c.N_y, c.N_x
    lib = xtg.gpu_lib()
    for call in range(2):
        rng = np.random.default_rng(100 + call)
        m = rng.random((c.N_time, c.nzb, ny, nx)).astype(np.float32)
        m[m < 0.25 + 0.2 * call] = 0.0
        m[:, :, 5, 2:7] = 0.6  # ties
        usn = np.full(nmaps, 300 + 211 * call, np.int32)
        c.set_magmap(m)
        nn, xs, ys, th = c.nhicd_select(usn)

        kth = np.array([ny * nx - u // 10 for u in usn], np.int32)
        d_map = torch.from_numpy(m).cuda()
        d_thr = torch.full((nmaps,), -1.0, dtype=torch.float32, device="cuda")
        d_sel = torch.full((nmaps * ny * nx,), 7, dtype=torch.uint8, device="cuda")
        rc = lib.xtg_nhicd_threshold_noalloc(_ptr(d_map), nmaps, ny, nx, kth.ctypes.data_as(C.c_void_p),
                                             _ptr(d_thr), _ptr(d_sel), None)
        assert rc == 0, lib.xtg_last_error()
        torch.cuda.synchronize()
        thr = d_thr.cpu().numpy()
        sel = d_sel.cpu().numpy().reshape(nmaps, ny, nx)
        assert np.array_equal(thr, th), (call, thr, th)
        for s in range(nmaps):
            want = np.zeros((ny, nx), np.uint8)
            want[ys[s, :nn[s]], xs[s, :nn[s]]] = 1
            assert np.array_equal(sel[s], want), (call, s)
    c.close()


def test_noalloc_selection_matches_reference_fixture():
    """The same entry point against the reference's own NHICD selection
    (tests/golden/nhicd_select.npz, VSC_based_Voxel_Line_Select with ties):
    the columns above the threshold are exactly the reference's lists."""
    import torch

    g = dict(np.load(f"{common.GOLDEN}/nhicd_select.npz"))
    nt, nzb, ny, nx = g["map"].shape
    nmaps = nt * nzb
    kth = np.array([ny * nx - u // 10 for u in g["usn"]], np.int32)
    lib = xtg.gpu_lib()
    d_map = torch.from_numpy(g["map"]).cuda()
    d_thr = torch.zeros((nmaps,), dtype=torch.float32, device="cuda")
    d_sel = torch.zeros((nmaps * ny * nx,), dtype=torch.uint8, device="cuda")
    rc = lib.xtg_nhicd_threshold_noalloc(_ptr(d_map), nmaps, ny, nx, kth.ctypes.data_as(C.c_void_p), _ptr(d_thr),
                                         _ptr(d_sel), None)
    assert rc == 0, lib.xtg_last_error()
    sel = d_sel.cpu().numpy().reshape(nmaps, ny, nx)
    for s in range(nmaps):
        want = np.zeros((ny, nx), np.uint8)
        n = int(g["nn"][s])
        want[g["ys"][s, :n], g["xs"][s, :n]] = 1
        assert np.array_equal(sel[s], want), s


def test_noalloc_rejects_oversized_input():
    import torch

    lib = xtg.gpu_lib()
    ny = nx = 1024
    nmaps = 2  # 2 M values > the 1 M-value scratch
    d_map = torch.zeros((1,), dtype=torch.float32, device="cuda")
    d_thr = torch.zeros((nmaps,), dtype=torch.float32, device="cuda")
    kth = np.ones(nmaps, np.int32)
    rc = lib.xtg_nhicd_threshold_noalloc(_ptr(d_map), nmaps, ny, nx, kth.ctypes.data_as(C.c_void_p), _ptr(d_thr),
                                         None, None)
    assert rc == -1
    assert b"exceed the fixed scratch" in lib.xtg_last_error()
