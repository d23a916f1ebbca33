"""The warm-start network's tcgen05 implicit-GEMM convolutions against a plain
PyTorch fp32 reference on the CPU (same BF16-rounded inputs and weights).

Both kernels are covered: the gather kernel (operands gathered per K stage)
and the tile kernel (the input tile staged once by TMA, each tap a shifted
shared-memory view; X a multiple of 128, Z even, cout <= 64), and both
weight gradients (gather; TMA tiles with the dy taps along M and the dz taps
along N, cout 32).

Tolerance: FP32 accumulation in a different order over K = 27*cin terms,
|got - ref| <= 1e-4 * max|ref| (FP32 output), plus one BF16 rounding of the
result (2^-8 relative) for BF16 outputs.
"""
import ctypes as C

import numpy as np
import pytest
import torch
import torch.nn.functional as F

import xtg

pytestmark = pytest.mark.gpu

SHAPES = [  # nb, Y, X, Z, cin, cout
    (1, 8, 8, 8, 8, 16),
    (2, 6, 10, 4, 32, 48),
    (1, 16, 16, 8, 64, 32),
    (1, 8, 8, 16, 160, 64),
]


TILE_SHAPES = [  # nb, Y, X, Z, cin, cout: 16-channel chunks, a half chunk, batches, tile edges
    (1, 3, 128, 4, 32, 32),
    (2, 2, 128, 6, 48, 64),
    (1, 2, 256, 2, 8, 16),
    (1, 3, 128, 4, 80, 32),
    (1, 2, 128, 2, 24, 48),
]
GATHER, TILE, AUTO = 1, 2, 0


def kpad(cin):
    return (27 * cin + 63) // 64 * 64


def pack_w(w):
    """torch [cout][cin][3][3][3] -> K-major [cout][kpad], k = tap*cin + ci."""
    cout, cin = w.shape[:2]
    m = w.permute(0, 2, 3, 4, 1).reshape(cout, 27 * cin)
    out = torch.zeros(cout, kpad(cin), dtype=torch.bfloat16)
    out[:, :27 * cin] = m.to(torch.bfloat16)
    return out


def to_cl(x):  # [nb][C][Y][X][Z] -> [nb][Y][X][Z][C]
    return x.permute(0, 2, 3, 4, 1).contiguous()


def from_cl(x):
    return x.permute(0, 4, 1, 2, 3).contiguous()


def ptr(t):
    return C.c_void_p(t.data_ptr())


def check(rc):
    assert rc == 0, xtg.gpu_lib().xtg_last_error()


def case(shape, seed=0):
    nb, Y, X, Z, cin, cout = shape
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(nb, cin, Y, X, Z, generator=g).to(torch.bfloat16).float()
    w = (torch.randn(cout, cin, 3, 3, 3, generator=g) / np.sqrt(27 * cin)).to(torch.bfloat16).float()
    b = torch.randn(cout, generator=g) * 0.1
    return x, w, b


@pytest.mark.parametrize("shape", SHAPES)
def test_conv_forward_fp32_and_relu(shape):
    lib = xtg.gpu_lib()
    nb, Y, X, Z, cin, cout = shape
    x, w, b = case(shape)
    ref = F.conv3d(x, w, padding=1)
    xd = to_cl(x).to(torch.bfloat16).cuda()
    wd = pack_w(w).cuda()
    bd = b.float().cuda()
    out = torch.empty(nb, Y, X, Z, cout, dtype=torch.float32, device="cuda")
    check(lib.xtc_conv3d(ptr(xd), ptr(wd), ptr(bd), ptr(out), nb, Y, X, Z, cin, cout, kpad(cin), 2, 1))
    got = from_cl(out.cpu())
    assert torch.max(torch.abs(got - ref)) <= 1e-4 * torch.max(torch.abs(ref))
    outb = torch.empty(nb, Y, X, Z, cout, dtype=torch.bfloat16, device="cuda")
    check(lib.xtc_conv3d(ptr(xd), ptr(wd), ptr(bd), ptr(outb), nb, Y, X, Z, cin, cout, kpad(cin), 0, 1))
    refr = torch.relu(ref + b.view(1, -1, 1, 1, 1))
    gotr = from_cl(outb.float().cpu())
    assert torch.max(torch.abs(gotr - refr)) <= 1e-4 * torch.max(torch.abs(refr)) + 2 ** -8 * torch.max(torch.abs(refr))


@pytest.mark.parametrize("shape", [s for s in SHAPES if s[4] % 16 == 0])
def test_conv_input_gradient(shape):
    lib = xtg.gpu_lib()
    nb, Y, X, Z, cin, cout = shape
    x, w, b = case(shape, 1)
    g = torch.Generator().manual_seed(7)
    dy = torch.randn(nb, cout, Y, X, Z, generator=g).to(torch.bfloat16).float()
    ref = torch.nn.grad.conv3d_input(x.shape, w, dy, padding=1)
    # transposed weights Wt[ci][tap][co]
    wt = w.permute(1, 0, 2, 3, 4).contiguous()  # [cin][cout][3][3][3]
    wtd = pack_w(wt).cuda()
    dyd = to_cl(dy).to(torch.bfloat16).cuda()
    out = torch.empty(nb, Y, X, Z, cin, dtype=torch.float32, device="cuda")
    check(lib.xtc_conv3d(ptr(dyd), ptr(wtd), None, ptr(out), nb, Y, X, Z, cout, cin, kpad(cout), 2, -1))
    got = from_cl(out.cpu())
    assert torch.max(torch.abs(got - ref)) <= 1e-4 * torch.max(torch.abs(ref))


@pytest.mark.parametrize("shape", SHAPES)
def test_conv_weight_gradient(shape):
    lib = xtg.gpu_lib()
    nb, Y, X, Z, cin, cout = shape
    x, w, b = case(shape, 2)
    g = torch.Generator().manual_seed(9)
    dy = torch.randn(nb, cout, Y, X, Z, generator=g).to(torch.bfloat16).float()
    ref = torch.nn.grad.conv3d_weight(x, w.shape, dy, padding=1)  # [cout][cin][3][3][3]
    ref_rows = ref.permute(2, 3, 4, 1, 0).reshape(27 * cin, cout)
    dw = torch.zeros(27 * cin, cout, dtype=torch.float32, device="cuda")
    # keep the device tensors referenced for the duration of the call
    xd = to_cl(x).to(torch.bfloat16).cuda()
    dyd = to_cl(dy).to(torch.bfloat16).cuda()
    check(lib.xtc_conv3d_wgrad(ptr(xd), ptr(dyd), ptr(dw), nb, Y, X, Z, cin, cout))
    got = dw.cpu()
    assert torch.max(torch.abs(got - ref_rows)) <= 1e-4 * torch.max(torch.abs(ref_rows))


WGRAD_TILE_SHAPES = [  # nb, Y, X, Z, cin, cout: 1-5 input chunks (one or two chunk groups), batches, y edges
    (1, 3, 128, 4, 32, 32),
    (2, 2, 128, 6, 48, 32),
    (1, 3, 256, 2, 80, 32),
    (1, 1, 128, 2, 16, 32),
]


@pytest.mark.parametrize("shape", WGRAD_TILE_SHAPES)
def test_tile_weight_gradient(shape):
    """The TMA tile weight gradient (dy taps stacked along M, dz taps along
    N) against PyTorch, and the gather kernel on the same data."""
    lib = xtg.gpu_lib()
    nb, Y, X, Z, cin, cout = shape
    x, w, b = case(shape, 4)
    g = torch.Generator().manual_seed(11)
    dy = torch.randn(nb, cout, Y, X, Z, generator=g).to(torch.bfloat16).float()
    ref = torch.nn.grad.conv3d_weight(x, w.shape, dy, padding=1)
    ref_rows = ref.permute(2, 3, 4, 1, 0).reshape(27 * cin, cout)
    xd = to_cl(x).to(torch.bfloat16).cuda()
    dyd = to_cl(dy).to(torch.bfloat16).cuda()
    got = {}
    for path in (TILE, GATHER, AUTO):
        dw = torch.zeros(27 * cin, cout, dtype=torch.float32, device="cuda")
        check(lib.xtc_conv3d_wgrad_path(ptr(xd), ptr(dyd), ptr(dw), nb, Y, X, Z, cin, cout, path))
        got[path] = dw.cpu()
    tol = 1e-4 * torch.max(torch.abs(ref_rows))
    assert torch.max(torch.abs(got[TILE] - ref_rows)) <= tol
    assert torch.max(torch.abs(got[GATHER] - ref_rows)) <= tol
    assert torch.max(torch.abs(got[AUTO] - got[TILE])) <= tol  # the automatic choice is the tile kernel


def conv_path(lib, xd, wd, bd, out, shape, epi, sign, path):
    nb, Y, X, Z, cin, cout = shape
    return lib.xtc_conv3d_path(ptr(xd), ptr(wd), ptr(bd) if bd is not None else None, ptr(out), nb, Y, X, Z, cin,
                               cout, kpad(cin), epi, sign, path)


@pytest.mark.parametrize("shape", TILE_SHAPES)
def test_tile_conv_forward(shape):
    lib = xtg.gpu_lib()
    nb, Y, X, Z, cin, cout = shape
    x, w, b = case(shape, 3)
    ref = F.conv3d(x, w, padding=1)
    xd = to_cl(x).to(torch.bfloat16).cuda()
    wd = pack_w(w).cuda()
    bd = b.float().cuda()
    out = torch.empty(nb, Y, X, Z, cout, dtype=torch.float32, device="cuda")
    check(conv_path(lib, xd, wd, bd, out, shape, 2, 1, TILE))
    got = from_cl(out.cpu())
    assert torch.max(torch.abs(got - ref)) <= 1e-4 * torch.max(torch.abs(ref))
    # the automatic choice is the tile kernel: the same sums in the same order
    out2 = torch.empty_like(out)
    check(conv_path(lib, xd, wd, bd, out2, shape, 2, 1, AUTO))
    assert torch.equal(out, out2)
    refr = torch.relu(ref + b.view(1, -1, 1, 1, 1))
    tol = 1e-4 * torch.max(torch.abs(refr)) + 2 ** -8 * torch.max(torch.abs(refr))
    for epi, want in ((0, refr), (1, ref)):
        outb = torch.empty(nb, Y, X, Z, cout, dtype=torch.bfloat16, device="cuda")
        check(conv_path(lib, xd, wd, bd, outb, shape, epi, 1, TILE))
        assert torch.max(torch.abs(from_cl(outb.float().cpu()) - want)) <= tol + 2 ** -8 * torch.max(torch.abs(want))
    # and the gather kernel agrees with it
    outg = torch.empty_like(out)
    check(conv_path(lib, xd, wd, bd, outg, shape, 2, 1, GATHER))
    assert torch.max(torch.abs(outg - out)).item() <= 1e-5 * torch.max(torch.abs(ref)).item()


@pytest.mark.parametrize("shape", [s for s in TILE_SHAPES if s[4] % 16 == 0 and s[4] <= 64])
def test_tile_conv_input_gradient(shape):
    lib = xtg.gpu_lib()
    nb, Y, X, Z, cin, cout = shape
    x, w, b = case(shape, 4)
    g = torch.Generator().manual_seed(8)
    dy = torch.randn(nb, cout, Y, X, Z, generator=g).to(torch.bfloat16).float()
    ref = torch.nn.grad.conv3d_input(x.shape, w, dy, padding=1)
    wtd = pack_w(w.permute(1, 0, 2, 3, 4).contiguous()).cuda()
    dyd = to_cl(dy).to(torch.bfloat16).cuda()
    out = torch.empty(nb, Y, X, Z, cin, dtype=torch.float32, device="cuda")
    check(lib.xtc_conv3d_path(ptr(dyd), ptr(wtd), None, ptr(out), nb, Y, X, Z, cout, cin, kpad(cout), 2, -1, TILE))
    got = from_cl(out.cpu())
    assert torch.max(torch.abs(got - ref)) <= 1e-4 * torch.max(torch.abs(ref))


def test_tile_conv_rejects_unsupported_shapes():
    lib = xtg.gpu_lib()
    shape = (1, 2, 96, 4, 32, 32)  # X not a multiple of 128
    x, w, b = case(shape)
    xd = to_cl(x).to(torch.bfloat16).cuda()
    wd = pack_w(w).cuda()
    out = torch.empty(1, 2, 96, 4, 32, dtype=torch.float32, device="cuda")
    assert conv_path(lib, xd, wd, None, out, shape, 2, 1, TILE) == -1  # XTG_E_ARG
    check(conv_path(lib, xd, wd, None, out, shape, 2, 1, AUTO))
    assert torch.max(torch.abs(from_cl(out.cpu()) - F.conv3d(x, w, padding=1))) <= 1e-4 * float(
        torch.max(torch.abs(F.conv3d(x, w, padding=1))))
