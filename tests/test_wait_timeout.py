"""Bounded device waits (no GPU is faulted or hung): the mbarrier waits of the
tensor-core kernels give up after a poll limit, set the device error flag,
and the call returns XTG_E_TIMEOUT with the context still usable.  A
one-CTA self-test waits on a barrier that nothing completes (nothing else is
in flight), then on one it has arrived on; a convolution runs afterwards."""
import ctypes as C

import pytest

import xtg

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_stays_usable():
    import torch
    lib = xtg.gpu_lib()
    lib.xtc_wait_selftest.argtypes = [C.c_int32, C.c_int64]
    assert lib.xtc_wait_selftest(1, 1 << 20) == 0
    assert lib.xtc_wait_selftest(0, 1000) == -5  # XTG_E_TIMEOUT
    assert b"timed out" in lib.xtg_last_error()
    # the flag was cleared and the device still works
    assert lib.xtc_wait_selftest(1, 1 << 20) == 0
    # a convolution afterwards: [nb][Y][X][Z][C] input, K-major packed weights
    from test_cnn_conv import case, kpad, pack_w, to_cl
    shape = (1, 8, 8, 8, 8, 16)
    nb, Y, X, Z, cin, cout = shape
    x, w, b = case(shape)
    xd = to_cl(x).to(torch.bfloat16).cuda()
    wd = pack_w(w).cuda()
    bd = b.float().cuda()
    out = torch.empty(nb, Y, X, Z, cout, dtype=torch.float32, device="cuda")
    rc = lib.xtc_conv3d(C.c_void_p(xd.data_ptr()), C.c_void_p(wd.data_ptr()), C.c_void_p(bd.data_ptr()),
                        C.c_void_p(out.data_ptr()), nb, Y, X, Z, cin, cout, kpad(cin), 2, 1)
    assert rc == 0, lib.xtg_last_error()
    assert torch.isfinite(out).all()
    lib.xtc_wait_selftest.argtypes = None
