"""The warm-start network: forward output and gradients against the PyTorch
fp32 CPU restatement (tests/warmnet_ref.py), and a short training run.

Tolerances: the library keeps BF16 weights, activations and pre-activation
gradients with FP32 accumulation; the reference rounds the same tensors to
BF16 but keeps gradients in fp32.  Forward: |out - ref| <= 2e-2 of the
correction's range.  Gradients: cosine similarity of the whole gradient
>= 0.998, and per parameter tensor a relative L2 error <= 1e-1 (the
coarsest level's gradients are sums over a few voxels after about ten BF16
roundings along the backward chain; measured worst case 5.3 %).
"""
import numpy as np
import pytest
import torch

import warmnet_ref as ref
import xtg

pytestmark = pytest.mark.gpu


def volumes(shape, seed):
    g = torch.Generator().manual_seed(seed)
    nb, Y, X, Z = shape
    fbp = torch.rand(nb, Y, X, Z, generator=g) * 0.01
    icd = fbp * 0.9 + torch.rand(nb, Y, X, Z, generator=g) * 0.001
    tgt = icd + 0.002 * torch.randn(nb, Y, X, Z, generator=g)
    return fbp, icd, tgt


def random_params(net, seed):
    """The network's He-initialised weights with a non-zero head and biases."""
    p = net.params().copy()
    rng = np.random.default_rng(seed)
    nh = ref.HEAD_C + 1
    p[-nh:] = rng.normal(0, 0.3, nh).astype(np.float32)
    off = 0
    for cin, cout in ref.SPEC:
        off += 27 * cin * cout
        p[off:off + cout] = rng.normal(0, 0.05, cout).astype(np.float32)
        off += cout
    return p


@pytest.mark.parametrize("shape", [(2, 16, 16, 16), (1, 32, 16, 8), (1, 16, 128, 8)])
def test_forward_and_gradients_match_reference(shape):
    net = xtg.WarmNet(seed=3)
    p = random_params(net, 5)
    net.set_params(p)
    fbp, icd, tgt = volumes(shape, 11)
    out = torch.empty(shape, device="cuda")
    fd, idd, td = fbp.cuda(), icd.cuda(), tgt.cuda()
    net.forward(fd, idd, out, shape)
    loss = net.backward(fd, idd, td, shape)
    g = torch.from_numpy(net.params(1))
    rloss, ry, rg = ref.loss_and_grads(p, fbp, icd, tgt)
    corr = (ry - icd)
    assert torch.max(torch.abs(out.cpu() - ry)) <= 2e-2 * float(corr.max() - corr.min())
    assert loss == pytest.approx(rloss, rel=2e-2)
    cos = float(torch.dot(g, rg) / (torch.norm(g) * torch.norm(rg)))
    assert cos >= 0.998, cos
    off = 0
    for i, (cin, cout) in enumerate(ref.SPEC):
        for n in (27 * cin * cout, cout):
            a, b = g[off:off + n], rg[off:off + n]
            assert float(torch.norm(a - b) / (torch.norm(b) + 1e-30)) <= 1e-1, (i, n)
            off += n
    net.close()


def test_training_reduces_loss_and_checkpoint_roundtrip(tmp_path):
    """A denoising task (target = ICD image without its noise): 300 Adam steps
    on 32^3 patches lower the loss by at least half; save/load restores the
    parameters bit for bit."""
    torch.manual_seed(0)
    vols = []
    for v in range(4):
        clean = torch.nn.functional.avg_pool3d(torch.rand(1, 1, 64, 64, 32) * 0.01, 5, 1, 2)[0, 0]
        noisy = clean + 0.0005 * torch.randn_like(clean)
        vols.append((noisy.cuda().contiguous(), noisy.cuda().contiguous(), clean.cuda().contiguous()))
    net = xtg.WarmNet(seed=1)
    losses = net.train([v[0] for v in vols], [v[1] for v in vols], [v[2] for v in vols], (64, 64, 32), (32, 32, 32),
                       4, 300, lr=1e-3)
    assert np.all(np.isfinite(losses))
    assert losses[-20:].mean() < 0.5 * losses[:20].mean(), (losses[:20].mean(), losses[-20:].mean())
    f = tmp_path / "w.bin"
    net.save(f)
    p = net.params()
    net2 = xtg.WarmNet(seed=9)
    net2.load(f)
    assert np.array_equal(net2.params(), p)
    net.close()
    net2.close()
