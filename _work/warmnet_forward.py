"""Times the warm-start network's forward pass (the inference inside the
learned start, include/xtg_cnn.h) on one volume of a given size, with the
committed weights, on cuda:0:

    python timbir-python_b200/warmnet_forward.py --n 512 --nz 64 --reps 5

Inputs are seeded random images of the engine's layout [1][N][N][NZ]; the
line printed gives the CUDA-event time per forward pass and its algorithmic
TFLOP/s (2 x 27 x cin x cout per output voxel and layer).
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import xtg  # noqa: E402

# (cin, cout, level) of the 14 convolutions, level l at 1/2^l the resolution
LAYERS = [(2, 32, 0), (32, 32, 0), (32, 48, 1), (48, 48, 1), (48, 64, 2), (64, 64, 2), (64, 96, 3), (96, 96, 3),
          (160, 64, 2), (64, 64, 2), (112, 48, 1), (48, 48, 1), (80, 32, 0), (32, 32, 0)]


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--nz", type=int, default=64)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--weights", default=os.path.join(HERE, "weights", "warmstart_plain3d.bin"))
    args = ap.parse_args()
    net = xtg.WarmNet()
    net.load(args.weights)
    shape = (1, args.n, args.n, args.nz)
    g = torch.Generator(device="cuda").manual_seed(1)
    f = torch.rand(shape, device="cuda", generator=g) * 0.01
    q = f * 0.9
    o = torch.empty(shape, device="cuda")
    net.forward(f, q, o, shape)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.reps):
        net.forward(f, q, o, shape)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.reps, 1)
    vox = args.n * args.n * args.nz
    flops = sum(2.0 * 27 * ci * co * vox / 8 ** lvl for ci, co, lvl in LAYERS)
    print(json.dumps({"shape": shape, "forward_ms": ms, "tflop": flops / 1e12, "tflops": flops / ms / 1e9}))
    net.close()


if __name__ == "__main__":
    main()
