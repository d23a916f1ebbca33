"""Trains the learned warm start (include/xtg_cnn.h) on phantoms reconstructed
by this engine, and saves its weights.

    python timbir-python_b200/train_warmstart.py --out timbir-python_b200/weights/warmstart_plain3d.bin \
        --n 512 --nt 64 --views 1024 --volumes 24 --target-iters 30 --steps 6000 --patch 32 128 32

(the committed weights; their .json records the run).  Training set: seeded
ellipsoid phantoms of N^2 x NT voxels (default 256^2 x 32 with 512 views;
the committed weights use the plain-3D-at-scale geometry, 512^2 x 64 with
1024 views), views uniform over 180 degrees, 1e4 photons/ray, 0.5 % zingers
with the generalized-Huber correction on, NHICD on; phantom seeds 1000 and
up, distinct from the benchmark's.  For each phantom the GPU
engine forms the network's inputs, the FBP image and the multi-resolution
start (`coarse_iters` ICD iterations on the 2x coarser grid, upsampled), and
the target, the reconstruction after `target_iters` further iterations on
the fine grid.  Training: Adam (lr 1e-3), batches of random patches
(default 64 x 64 x 32; the committed weights: 32 x 128 x 32, whose first
level runs on the TMA tile kernels).  Data generation and training run on the GPU through
the library; the host only draws the Poisson counts and sequences calls.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import xtg  # noqa: E402


def params(N, NT, NP, zinger=True):
    return xtg.Params(
        p=1.2, sigma_s=200000.0, sigma_t=200000.0, c_s=0.01, c_t=0.01, delta_xy=1.0, delta_z=1.0,
        length_r=float(N), length_t=float(NT), rotation_center=N / 2.0, alpha=1.0, Rtime0=0.0,
        Rtime_delta=float(NP), radius_obj=float(N), zingerT=4.0 if zinger else 100000.0,
        zingerDel=0.5 if zinger else 0.0, iter=100, Rtime_num=1, num_projections=NP, N_r=N, N_t=NT,
        num_threads=1, positivity=1, no_NHICD=0)


def make_set(n_vol, N=256, NT=32, NP=512, n_ell=30, I0=1e4, zfrac=0.005, coarse_iters=30, target_iters=40,
             seed=1000, log=print):
    """(fbp, multi-resolution start, target) device tensors [N][N][NT] per
    phantom, and the geometry."""
    import torch
    p = params(N, NT, NP)
    t, a = xtg.round_views(*xtg.views_uniform(NP))
    ctx = xtg.Context(p, t, a)
    ctx.set_options(a_mode=xtg.XTG_A_AUTO)
    shape = (ctx.N_y, ctx.N_x, ctx.N_z)
    out = []
    t0 = time.time()
    for i in range(n_vol):
        x = xtg.phantom((1, NT, N, N), n_ell, 0.01, seed + i)
        ctx.upload_object(x)
        ax = ctx.forward_project()
        y, w = xtg.measure(ax, I0, seed + 100000 + i, zinger_frac=zfrac)
        ctx.upload_sino(y, w)
        ctx.init_fbp()
        f = torch.empty(shape, device="cuda")
        ctx.object_to_device(f)
        ctx.init_multires(coarse_iters, with_z=NT % 2 == 0 and NT >= 16)
        q = torch.empty(shape, device="cuda")
        ctx.object_to_device(q)
        for it in range(1, target_iters + 1):
            ctx.iteration(it)
        g = torch.empty(shape, device="cuda")
        ctx.object_to_device(g)
        out.append((f, q, g))
        if (i + 1) % 16 == 0:
            log(f"  {i + 1}/{n_vol} phantoms, {time.time() - t0:.1f} s")
    ctx.close()
    return out, shape


def train(data, shape, steps=2000, batch=8, patch=(64, 64, 32), lr=1e-3, seed=1, log=print):
    net = xtg.WarmNet(seed=seed)
    t0 = time.time()
    losses = net.train([d[0] for d in data], [d[1] for d in data], [d[2] for d in data], shape, patch, batch, steps,
                       lr=lr, seed=seed + 7)
    log(f"  trained {steps} steps in {time.time() - t0:.1f} s; loss {losses[:50].mean():.4g} -> "
        f"{losses[-50:].mean():.4g}")
    return net, losses


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--volumes", type=int, default=128)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--nt", type=int, default=32)
    ap.add_argument("--views", type=int, default=512)
    ap.add_argument("--coarse-iters", type=int, default=30)
    ap.add_argument("--target-iters", type=int, default=40)
    ap.add_argument("--patch", type=int, nargs=3, default=(64, 64, 32), metavar=("Y", "X", "Z"),
                    help="training patch; X a multiple of 128 runs the level-0 convolutions (forward and input "
                         "gradient) on the TMA tile kernel")
    args = ap.parse_args()
    t0 = time.time()
    data, shape = make_set(args.volumes, args.n, args.nt, args.views, coarse_iters=args.coarse_iters,
                           target_iters=args.target_iters)
    t1 = time.time()
    net, losses = train(data, shape, steps=args.steps, batch=args.batch, patch=tuple(args.patch))
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    net.save(args.out)
    info = {"volumes": args.volumes, "shape": shape, "views": args.views, "coarse_iters": args.coarse_iters,
            "target_iters": args.target_iters, "steps": args.steps, "batch": args.batch, "patch": list(args.patch),
            "data_s": t1 - t0, "train_s": time.time() - t1, "loss_first50": float(losses[:50].mean()),
            "loss_last50": float(losses[-50:].mean()), "params": net.n_params}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps(info))
    net.close()


if __name__ == "__main__":
    main()
