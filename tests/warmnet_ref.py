"""Plain PyTorch fp32 (CPU) restatement of the warm-start network in
include/xtg_cnn.h, the reference for its forward output and gradients (test
infrastructure only).  The library stores weights, activations and the
pre-activation gradients in BF16; this reference rounds weights, packed
inputs and stored activations to BF16 the same way (straight-through for
gradients) and keeps everything else in fp32."""
import torch
import torch.nn.functional as F

SPEC = [(2, 32), (32, 32), (32, 48), (48, 48), (48, 64), (64, 64), (64, 96), (96, 96), (160, 64), (64, 64),
        (112, 48), (48, 48), (80, 32), (32, 32)]
HEAD_C = 32
SCALE = 100.0


def bf(x):
    """BF16 rounding with a straight-through gradient."""
    return x + (x.to(torch.bfloat16).float() - x).detach()


def unpack(p):
    """Flat parameter vector -> list of (weight [cout][cin][3][3][3], bias), head w, head b."""
    p = torch.as_tensor(p, dtype=torch.float32)
    off, layers = 0, []
    for cin, cout in SPEC:
        n = 27 * cin * cout
        w = p[off:off + n].reshape(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2).contiguous()
        off += n
        b = p[off:off + cout].clone()
        off += cout
        layers.append((w, b))
    hw = p[off:off + HEAD_C].clone()
    hb = p[off + HEAD_C:off + HEAD_C + 1].clone()
    return layers, hw, hb


def flat_grads(layers, hw, hb):
    out = []
    for w, b in layers:
        out.append(w.grad.permute(2, 3, 4, 1, 0).reshape(-1))
        out.append(b.grad.reshape(-1))
    out += [hw.grad.reshape(-1), hb.grad.reshape(-1)]
    return torch.cat(out)


def forward(layers, hw, hb, fbp, icd):
    """fbp, icd: [nb][Y][X][Z] -> output [nb][Y][X][Z]."""
    x = torch.stack([bf(fbp * SCALE), bf(icd * SCALE)], 1)  # [nb][2][Y][X][Z]

    def conv(i, t):
        w, b = layers[i]
        return bf(F.relu(F.conv3d(t, bf(w), b, padding=1)))

    def pool(t):
        return bf(F.avg_pool3d(t, 2))

    def up(t):
        return F.interpolate(t, scale_factor=2, mode="nearest")

    s0 = conv(1, conv(0, x))
    s1 = conv(3, conv(2, pool(s0)))
    s2 = conv(5, conv(4, pool(s1)))
    b3 = conv(7, conv(6, pool(s2)))
    f2 = conv(9, conv(8, torch.cat([up(b3), s2], 1)))
    f1 = conv(11, conv(10, torch.cat([up(f2), s1], 1)))
    f0 = conv(13, conv(12, torch.cat([up(f1), s0], 1)))
    corr = torch.einsum("bcyxz,c->byxz", f0, hw) + hb
    return icd + corr / SCALE


def loss_and_grads(p, fbp, icd, target):
    layers, hw, hb = unpack(p)
    for w, b in layers:
        w.requires_grad_(True)
        b.requires_grad_(True)
    hw.requires_grad_(True)
    hb.requires_grad_(True)
    y = forward(layers, hw, hb, fbp, icd)
    loss = torch.mean(((y - target) * SCALE) ** 2)
    loss.backward()
    return loss.item(), y.detach(), flat_grads(layers, hw, hb)
