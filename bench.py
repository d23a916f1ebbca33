"""Benchmark: ICD voxel-updates/s of the B200 TIMBIR engine on the plain-3D-at-scale workload.

Workload (the reference's at-scale configuration, seeded synthetic stand-in
for its beamline data): 64 slices of 512x512 voxels, 512 detector bins x 64
rows, 1024 views uniform over 180 degrees, 30 ellipsoids (attenuation
U(0, 0.01) per voxel length), Poisson counts at 1e4 photons/ray, 0.5 % of the
sinogram entries turned into zingers (+U(2, 5)), generalized-Huber zinger
correction on (T = 4, delta = 0.5), NHICD on, FP32.

A step is one reference iteration (updateVoxelsTimeSlices: one random equit in
10 chunks, each followed by NHICD selection and, from iteration 2 on, an NHICD
pass).  value = voxel updates / device time of the K timed steps (CUDA events
around each iteration on the library's stream, max over ranks).  e2e = the
same metric through the C ABI from pinned host buffers: per step the
sinogram/weights go host->device while Ax is projected (xtg_upload_sino_start),
e = y - Ax - d is formed, one iteration runs and the object goes back
device->host (xtg_download_object_start, overlapping the next step's upload
and projection; the timed region ends when the last step's object is on the
host).

--impl reference times the reference engine's own CPU implementation
(oracle/_ref, compiled from the reference sources, OpenMP on every host core)
on a bounded sample of the same workload: the same geometry, views and data
restricted by --radius_obj to a central disk (radius N/8, about 1/20 of the columns).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "timbir-python_b200")]

import xtg  # noqa: E402

WORKLOADS = {
    # plain 3D at scale: 64 slices of 512^2, 512 bins x 64 rows, 1024 views
    # uniform over 180 deg, 30 ellipsoids, 1e4 photons/ray, 0.5 % zingers,
    # zinger correction on (T = 4, delta = 0.5), NHICD on
    "plain3d": dict(N=512, NT=64, NP=1024, n_time=1, n_ell=30, mu=0.01, I0=1e4, zfrac=0.005, seed=2,
                    zinger=True, interlaced=None, moving=0),
    # 4D TIMBIR: 256^2 x 16 volume x 16 time frames, 8 interlaced sub-frames of
    # 32 views per rotation in bit-reversed order (N_theta = 256), 2 sub-frames
    # (64 views) per frame, 1024 views, 256 bins x 16 rows; 8 ellipsoids moving
    # up to 1 voxel/frame plus one growing; temporal prior weight 0.5
    "timbir4d": dict(N=256, NT=16, NP=1024, n_time=16, n_ell=8, mu=0.01, I0=1e4, zfrac=0.0, seed=3,
                     zinger=False, interlaced=(8, 256), moving=8),
    # largest single-GPU 4D: 1024^2 x 64 voxels x 32 frames (8.6 GB FP32),
    # 1536 bins (voxels 1.5 bins wide), 2 interlaced sub-frames of 64 views per
    # frame (4096 views), 1e4 photons/ray, 0.5 % zingers with correction on,
    # NHICD on; its sinogram is formed by the GPU projector (same A, same sums)
    "timbir4d_large": dict(N=1024, NT=64, NP=4096, n_time=32, n_ell=8, mu=0.01, I0=1e4, zfrac=0.005, seed=5,
                           zinger=True, interlaced=(2, 128), moving=8, dxy=1.5, gpu_fp=True),
}
WORKLOAD = WORKLOADS["plain3d"]
METRIC = "voxel-updates/s (ICD)"
# DRAM bytes per voxel update of the ICD column kernel, from the committed ncu
# summary of a random-pass (chunk) launch; scaled by voxel updates per launch
PROFILE = os.path.join(ROOT, "profiles", "icd_columns_plain3d.md")
AMODES = {"fp32": xtg.XTG_A_FP32, "table32": xtg.XTG_A_TABLE32, "fp16": xtg.XTG_A_FP16}
# bytes per A entry streamed from HBM: computed in registers, FP32 table, FP16 table
A_BYTES = {"fp32": 0.0, "table32": 8.0, "fp16": 6.0}
# the reference's HU conversion of --sigma_s / --sigma_t (XT_Init.c:510-511)
SLOPE_HU = 1000.0 / (0.521225397034623 - 0.496372335005353 * 0.001205) / 0.0001
C_HU = -SLOPE_HU * (0.496372335005353 * 0.001205 * 0.0001)


def sigma_t_arg(sigma_s_arg, delta_rtime, weight):
    """--sigma_t giving the temporal prior `weight` times the spatial one:
    (sigma_t delta_Rtime)^2 = (sigma_s mult_xy)^2 / weight (q = 2, mult_xy = 1)."""
    s = (sigma_s_arg - C_HU) / SLOPE_HU
    return C_HU + SLOPE_HU * s / (delta_rtime * weight ** 0.5)


def bins(w):
    """Detector bins: voxels per side x voxel width in bins."""
    return int(round(w["N"] * w.get("dxy", 1.0)))


def params(w, radius=None):
    nt, dxy = w["n_time"], w.get("dxy", 1.0)
    NR = bins(w)
    rdelta = float(w["NP"] // nt)
    sig = 200000.0
    return xtg.Params(
        p=1.2, sigma_s=sig, sigma_t=sigma_t_arg(sig, rdelta, 0.5) if nt > 1 else sig, c_s=0.01, c_t=0.01,
        delta_xy=dxy, delta_z=1.0, length_r=float(NR), length_t=float(w["NT"]), rotation_center=NR / 2.0,
        alpha=1.0, Rtime0=0.0, Rtime_delta=rdelta, radius_obj=float(NR) if radius is None else float(radius),
        zingerT=4.0 if w["zinger"] else 100000.0, zingerDel=0.5 if w["zinger"] else 0.0, iter=100, Rtime_num=nt,
        num_projections=w["NP"], N_r=NR, N_t=w["NT"], num_threads=1, positivity=1, no_NHICD=0)


def make_data(w):
    p = params(w)
    if w["interlaced"]:
        t, a = xtg.round_views(*xtg.views_interlaced(*w["interlaced"], w["NP"]))
    else:
        t, a = xtg.round_views(*xtg.views_uniform(w["NP"]))
    mv = w["moving"]
    x = xtg.phantom((w["n_time"], w["NT"], w["N"], w["N"]), w["n_ell"], w["mu"], w["seed"], n_moving=mv,
                    max_shift=1.0 if mv else 0.0, growing=1 if mv else 0)
    if w.get("gpu_fp"):
        c = xtg.Context(p, t, a)
        c.upload_object(x)
        ax = c.forward_project()
        c.close()
    else:
        ax = xtg.forward_cpu(p, t, a, x)
    y, wt = xtg.measure(ax, w["I0"], w["seed"] + 100, zinger_frac=w["zfrac"])
    return p, t, a, x, y, wt


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        m = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dram_bytes_per_update():
    """DRAM bytes per voxel update of the ICD kernel from the committed ncu summary."""
    if not os.path.exists(PROFILE):
        return None
    for line in open(PROFILE):
        if line.startswith("dram_bytes_per_voxel_update:"):
            return float(line.split(":")[1])
    return None


def workload_name(w):
    if w["n_time"] > 1:
        return f"timbir4d_{w['N']}x{w['N']}x{w['NT']}x{w['n_time']}frames_{w['NP']}views"
    return f"plain3d_{w['N']}x{w['N']}x{w['NT']}_{w['NP']}views"


def workload(args):
    w = dict(WORKLOADS[args.workload])
    if args.nxy:
        w["N"] = args.nxy
    return w


def base_config(w, amode):
    return {"workload": workload_name(w), "N_xy": w["N"], "N_z": w["NT"], "N_time": w["n_time"], "N_r": bins(w),
            "N_t": w["NT"], "N_p": w["NP"], "views": "interlaced K=%d N_theta=%d" % w["interlaced"]
            if w["interlaced"] else "uniform", "zinger": [4.0, 0.5] if w["zinger"] else None,
            "zinger_frac": w["zfrac"], "temporal_weight": 0.5 if w["n_time"] > 1 else None, "nhicd": True,
            "a_mode": amode}


WEIGHTS = os.path.join(ROOT, "timbir-python_b200", "weights", "warmstart_plain3d.bin")


# (cin, cout, level) of the warm-start network's 3x3x3 convolutions
NET_LAYERS = [(2, 32, 0), (32, 32, 0), (32, 48, 1), (48, 48, 1), (48, 64, 2), (64, 64, 2), (64, 96, 3), (96, 96, 3),
              (160, 64, 2), (64, 64, 2), (112, 48, 1), (48, 48, 1), (80, 32, 0), (32, 32, 0)]


def network_roofline(ctx, net, coarse_iters, reps=3):
    """The warm-start network's forward pass over the whole volume (the
    inference inside the learned start), timed with CUDA events: algorithmic
    FLOPs (2 x 27 x cin x cout per output voxel and layer) over time, against
    the measured dense BF16 tensor-core peak."""
    import torch
    shape = (ctx.N_time, ctx.N_y, ctx.N_x, ctx.N_z)
    f, q, o = (torch.empty(shape, device="cuda") for _ in range(3))
    ctx.init_fbp()
    ctx.object_to_device(f)
    ctx.init_multires(coarse_iters)
    ctx.object_to_device(q)
    net.forward(f, q, o, shape)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.forward(f, q, o, shape)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    vox = ctx.N_time * ctx.N_y * ctx.N_x * ctx.N_z
    flops = sum(2.0 * 27 * ci * co * vox / 8 ** lvl for ci, co, lvl in NET_LAYERS)
    try:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
        kind = "measured (MEASURED_PEAKS.json bf16_tflops, burst)"
    except Exception:
        peak, kind = 1590.0, "fallback 1.59 PFLOP/s"
    return {"forward_ms": ms, "tflop": flops / 1e12, "achieved_tflops": flops / ms / 1e9, "peak_tflops": peak,
            "frac": flops / ms / 1e9 / peak, "peak_kind": kind, "bound": "tensor"}


def projector_timing(ctx, reps=3):
    """Forward-projection calls on the resident (zero) object, each through
    the C ABI (which synchronises its stream): e = y - Ax - d in FP32 (the
    reference's order) and the FP64 resync, with the bin-major A table (the
    default where it fits) and with the table-free gather.  Algorithmic HBM
    bytes of one table launch: y read + e written (+ w read for the resync's
    cost) + 8 B per table entry; the object (a z-line per entry) is re-read
    from L2 and L1."""
    import torch
    out = {}
    for kind, key in ((xtg.XTG_PROJ_GATHER, "gather"), (xtg.XTG_PROJ_AUTO, "table")):
        ctx.set_projector(kind)
        ctx.init_error_sino()  # builds the table (outside the timing)
        r = {}
        for name, fn in (("init_error_ms", ctx.init_error_sino), ("resync_fp64_ms", ctx.resync_fp64)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(reps):
                fn()
            r[name] = (time.perf_counter() - t0) * 1e3 / reps
        used, entries = ctx.projector()
        if key == "table":
            out["kind"] = "table" if used == xtg.XTG_PROJ_TABLE else "gather"
            if used == xtg.XTG_PROJ_TABLE:
                ns = int(np.prod(ctx.sino_shape))
                peak, _ = peaks()
                alg = {"init_error_ms": 8.0 * ns + 8.0 * entries, "resync_fp64_ms": 12.0 * ns + 8.0 * entries}
                r["table_entries"] = entries
                r["hbm_gbs_alg"] = {k: alg[k] / (r[k] / 1e3) / 1e9 for k in alg}
                r["frac_of_measured_hbm"] = {k: alg[k] / (r[k] / 1e3) / 1e9 / peak for k in alg}
        out[key] = r
    return out


def kernel_timings(args, reps=5):
    """`--kernels`: the engine's other north-star kernels, each through its C
    ABI call on the workload (after the FBP start and two iterations, so the
    object and the error sinogram are realistic), timed on the host around
    the call (the call synchronises the library's stream; the mean of `reps`
    calls), with the algorithmic HBM bytes of one call and their rate against
    the measured copy bandwidth.  Bytes: sinogram arrays 4 B per entry each
    (e, w, y read; e written), the bin-major A table 8 B per entry, the
    object 4 B per voxel (its neighbours come from L1/L2), the NHICD maps
    4 B per value per pass.  The ncu summaries in profiles/ capture the same
    command."""
    import torch
    w = workload(args)
    p, t, a, x_true, y, wt = make_data(w)
    ctx = xtg.Context(p, t, a)
    ctx.set_options(a_mode=xtg.XTG_A_TABLE32)
    ctx.upload_sino(y, wt)
    ctx.init_fbp()
    for it in (1, 2):
        ctx.iteration(it)
    ns = int(np.prod(ctx.sino_shape))
    nvox = int(np.prod(ctx.obj_shape))
    _, entries = ctx.projector()
    nmag = int(np.prod(ctx.mag_shape))
    usn = np.full(ctx.N_time * ctx.nzb, ctx.n_masked, np.int32)
    peak, kind = peaks()
    calls = {
        # name: (call, algorithmic bytes, kernels)
        "init_error_sino": (ctx.init_error_sino, 8.0 * ns + 8.0 * entries, "k_fp_csr<1>"),
        "resync_fp64": (ctx.resync_fp64, 12.0 * ns + 8.0 * entries + 4.0 * nvox, "k_fp_csr<2>, k_prior_cost64"),
        "map_cost_fp64": (ctx.cost, 8.0 * ns + 8.0 * entries + 4.0 * nvox, "k_fp_csr<3>, k_prior_cost64"),
        "map_cost_running": (ctx.cost_running, 8.0 * ns + 4.0 * nvox, "k_running_cost64, k_prior_cost64"),
        "zinger_refresh": (lambda: ctx.zinger_refresh(want_mask=False), 8.0 * ns, "k_zinger_refresh"),
        "nhicd_select": (lambda: ctx.nhicd_select(usn), 4.0 * nmag * 6, "k_vsc_filter, k_rs_hist, k_rs_pick, "
                                                                         "k_nhicd_compact"),
    }
    out = {"workload": workload_name(w), "sinogram_entries": ns, "voxels": nvox, "table_entries": entries,
           "peak_gbs": peak, "peak_kind": peak_kind_note(kind), "calls": {}}
    for name, (fn, alg, kern) in calls.items():
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        ms = (time.perf_counter() - t0) * 1e3 / reps
        gbs = alg / (ms / 1e3) / 1e9
        out["calls"][name] = {"ms": ms, "alg_bytes": alg, "gbs": gbs, "frac": gbs / peak, "kernels": kern}
    # the A column table of the ICD kernel: an iteration that rebuilds it
    # against one that does not
    its = []
    for rebuild in (False, True):
        if rebuild:
            ctx.set_options(a_mode=xtg.XTG_A_FP16)
            ctx.set_options(a_mode=xtg.XTG_A_TABLE32)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.iteration(3)
        torch.cuda.synchronize()
        its.append((time.perf_counter() - t0) * 1e3)
    out["calls"]["column_table_build"] = {"ms": its[1] - its[0], "kernels": "k_table_count, k_table_fill",
                                          "note": "iteration with the rebuild minus one without"}
    ctx.close()
    print(json.dumps(out), flush=True)


def network_forward(nxy, nz, reps, weights=WEIGHTS):
    """`--network-forward`: the warm-start network's forward pass alone (the
    inference inside the learned start) on one volume [1][nxy][nxy][nz] of
    seeded random images, committed weights, cuda:0; CUDA-event time per pass
    and algorithmic TFLOP/s (2 x 27 x cin x cout per output voxel and layer)."""
    import torch
    net = xtg.WarmNet()
    net.load(weights)
    shape = (1, nxy, nxy, nz)
    g = torch.Generator(device="cuda").manual_seed(1)
    f = torch.rand(shape, device="cuda", generator=g) * 0.01
    q = f * 0.9
    o = torch.empty(shape, device="cuda")
    net.forward(f, q, o, shape)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.forward(f, q, o, shape)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(reps, 1)
    vox = nxy * nxy * nz
    flops = sum(2.0 * 27 * ci * co * vox / 8 ** lvl for ci, co, lvl in NET_LAYERS)
    print(json.dumps({"network_forward": list(shape), "forward_ms": ms, "tflop": flops / 1e12,
                      "tflops": flops / ms / 1e9}), flush=True)
    net.close()


def network_train(nxy, nz, steps, patch, batch=8, volumes=4):
    """`--network-train`: training steps of the warm-start network alone
    (xtc_net_train: batches of random patches, forward, backward, Adam) on
    `volumes` seeded random volumes [nxy][nxy][nz], after 5 untimed steps;
    time per step and algorithmic TFLOP/s (3 x the forward's 2 x 27 x cin x
    cout per voxel and layer)."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(0)
    vols = [torch.rand(nxy, nxy, nz, device="cuda", generator=g) * 0.01 for _ in range(volumes)]
    data = [(v, v * 0.9, v * 0.95) for v in vols]
    net = xtg.WarmNet(seed=1)
    args = ([d[0] for d in data], [d[1] for d in data], [d[2] for d in data], (nxy, nxy, nz), tuple(patch), batch)
    net.train(*args, 5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = net.train(*args, steps)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    vox = batch * patch[0] * patch[1] * patch[2]
    flops = 3 * sum(2.0 * 27 * ci * co * vox / 8 ** lvl for ci, co, lvl in NET_LAYERS)
    net.close()
    return {"network_train": {"patch": list(patch), "batch": batch, "steps": steps, "volumes": [nxy, nxy, nz]},
            "ms_per_step": dt * 1e3 / steps, "tflops": flops * steps / dt / 1e12,
            "loss_last20": float(losses[-20:].mean())}


def converge(ctx, amode, tol=1e-4, max_iters=400, stall=1e-7, resync_every=10, coarse_iters=30, learned=True,
             weights=WEIGHTS, starts=("zero", "fbp", "multires", "learned"), cstar_start="fbp"):
    """Seconds to MAP cost <= (1 + tol) C* from four starts:
      zero     -- the reference's start, plain ICD with the benchmark's A storage;
      fbp      -- the FBP image, same A storage;
      multires -- the launcher's coarse-to-fine scheme in one process:
                  `coarse_iters` iterations on the 2x coarser grid from its FBP
                  image, upsampled (xtg_init_object_multires), same A storage;
      learned  -- the warm-start network (timbir-python_b200/weights) applied
                  to the FBP image and the multi-resolution start, ICD with
                  FP16 A (the FP16-A precision form); the multi-resolution
                  start is kept if the network's image is not lower in cost.

    Pass 1 (untimed) reconstructs from the FBP start until the FP64 MAP cost
    stalls (relative decrease over 10 iterations below `stall`, or
    `max_iters`); its final FP64 cost (full resync e = y - Ax - d) is C*.  Each
    timed pass starts again (the start's own computation is inside the timed
    region) and is timed on the wall clock, cost test included: after every
    iteration the MAP cost of the running error sinogram (FP64 sums), every
    `resync_every` iterations and at the stop the FP64 resync; it stops at the
    first FP64-resynced cost <= (1 + tol) C*.  After each pass (outside its
    timed region) its object is compared with the C* object: `rmse_rel` =
    RMS difference / max |x*|."""
    import torch
    zero = np.zeros(ctx.obj_shape, np.float32)
    torch.cuda.synchronize()
    if cstar_start == "multires":
        ctx.init_multires(coarse_iters)
    else:
        ctx.init_fbp()
    hist = []
    for it in range(1, max_iters + 1):
        ctx.iteration(it)
        c = ctx.resync_fp64()[0] if it % resync_every == 0 else ctx.cost_running()[0]
        hist.append(c)
        if it >= 20 and (hist[-11] - hist[-1]) < stall * abs(hist[-1]):
            break
    c_star = ctx.resync_fp64()[0]
    x_star = ctx.object()
    x_scale = float(np.abs(x_star).max()) or 1.0
    out = {"c_star": c_star, "c_star_iterations": len(hist), "tol": tol, "c_star_start": cstar_start,
           "c_star_source": f"this engine from the {cstar_start} start run until its FP64 cost stalls; the MAP cost of "
                            "that object is re-evaluated on the host in c_star_check (the oracle with the GPU's "
                            "arithmetic, and the reference's FP64 build's arithmetic).  With the same options "
                            "at 128^2 x 16 / 512 views the parallel schedule reaches the reference FP64 engine's "
                            "own converged cost (tests/test_config_c2_pinned.py)",
           "_x_star": x_star}
    net = None
    if learned and "learned" in starts and os.path.exists(weights) and all(d % 8 == 0 for d in (ctx.N_x, ctx.N_y, ctx.N_z)):
        net = xtg.WarmNet()
        net.load(weights)
        # the network's activation buffers and the start images for this
        # volume are allocated once, outside the timed region (like the A table
        # and the coarse context): one learned start with a single coarse
        # iteration
        ctx.init_learned(net, 1)
    # the coarse context of the multi-resolution start is built once, outside
    # the timed region (like the fine context and its A table)
    ctx.init_multires(1)
    runs = [(k, AMODES[amode]) for k in ("zero", "fbp", "multires") if k in starts]
    if net is not None:
        runs.append(("learned", xtg.XTG_A_FP16))
    for kind, am in runs:
        target = c_star * (1.0 + tol)
        ctx.set_options(a_mode=am)
        ctx.upload_object(zero)
        ctx.iteration(1)  # builds the A storage of this mode outside the timed region
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, extra = 0, {}
        if kind == "fbp":
            ctx.init_fbp()
        elif kind == "multires":
            ctx.init_multires(coarse_iters)
            extra = {"coarse_iterations": coarse_iters}
        elif kind == "learned":
            used, cn, ci = ctx.init_learned(net, coarse_iters)
            extra = {"network_used": used, "cost_network_start": cn, "cost_multires_start": ci,
                     "coarse_iterations": coarse_iters}
        else:
            ctx.upload_object(zero)
            ctx.init_error_sino()
        c = float("inf")
        while it < max_iters:
            it += 1
            ctx.iteration(it)
            c = ctx.cost_running()[0]
            if c <= target or it % resync_every == 0:
                c = ctx.resync_fp64()[0]
                if c <= target:
                    break
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        rmse = float(np.sqrt(np.mean((ctx.object() - x_star) ** 2))) / x_scale
        out[kind] = {"s": secs if c <= target else None, "iterations": it, "cost": c, "rmse_rel": rmse,
                     "a_mode": {v: k for k, v in AMODES.items()}[am], **extra}
    if net is not None:
        out["network"] = network_roofline(ctx, net, coarse_iters)
        net.close()
        # training throughput of the same network with the library's own
        # forward / backward / Adam kernels (wall clock around the steps)
        out["network"]["training"] = network_train(256, 32, 100, (32, 128, 32))
    ctx.set_options(a_mode=AMODES[amode])
    z = out.get("zero", {}).get("s")
    for k in ("fbp", "multires", "learned"):
        v = out.get(k, {}).get("s")
        out[f"speedup_{k}_vs_zero"] = z / v if z and v else None
    return out


def nnz_per_column(ctx, p, t, a, n_cols=512, seed=0):
    """Average A-matrix entries of a column over the views of its frame
    (sampled columns, frame 0; every frame has the same number of views)."""
    rng = np.random.default_rng(seed)
    g = ctx.geometry()
    views = np.nonzero(xtg.host_geometry(p, t, a)[3] == 0)[0]
    rows = rng.integers(0, ctx.N_y, n_cols)
    cols = rng.integers(0, ctx.N_x, n_cols)
    keep = [(r, c) for r, c in zip(rows, cols)
            if ((g.x0 + (c + 0.5) * g.delta_xy) ** 2 + (g.y0 + (r + 0.5) * g.delta_xy) ** 2) < g.radius_obj ** 2]
    rr = np.repeat([k[0] for k in keep], len(views))
    cc = np.repeat([k[1] for k in keep], len(views))
    vv = np.tile(views, len(keep))
    _, _, cnt = ctx.amatrix(rr, cc, vv)
    return float(cnt.sum()) / len(keep)


def job_totals(ms, updates, world, device):
    """Whole-job figures of N independent replicas: the slowest rank's device
    time (max over ranks) and the voxel updates of all ranks (sum)."""
    if world <= 1:
        return float(ms), float(updates)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms), float(updates)], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(t[1])


def dist_setup():
    n = int(os.environ.get("WORLD_SIZE", "1"))
    r = int(os.environ.get("RANK", "0"))
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    return n, r, lr


def run_ours(args):
    import torch
    world, rank, lrank = dist_setup()
    torch.cuda.set_device(lrank)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    w = workload(args)
    p, t, a, x_true, y, wt = make_data(w)
    ctx = xtg.Context(p, t, a)
    ctx.set_options(a_mode=AMODES[args.amode], max_columns=args.columns)
    ctx.set_zslab(args.zslab)
    ctx.upload_sino(y, wt)
    ctx.init_error_sino()
    proj = projector_timing(ctx) if world == 1 else None
    fp_ms = proj["table" if proj["kind"] == "table" else "gather"]["init_error_ms"] if proj else None
    nnz = nnz_per_column(ctx, p, t, a)
    it = 0
    for _ in range(args.warmup):
        it += 1
        ctx.iteration(it)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launch_count()
    clk = Clocks(lrank)
    ms_tot, upd, kms, rows, n_icd, zsk = 0.0, 0, 0.0, 0, 0, 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        it += 1
        st = ctx.iteration(it)
        ms_tot += st.ms
        upd += st.voxel_updates
        zsk += st.zero_skipped
        k_ms, _, k_n = ctx.last_kernel_time()
        kms += k_ms
        n_icd += k_n
        rows += st.columns
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = clk.stop()
    launches = ctx.launch_count() - launches0
    cost = ctx.cost()[0]
    ms_job, upd_job = job_totals(ms_tot, upd, world, "cuda")
    value = upd_job / (ms_job / 1e3)

    # e2e: through the C ABI from pinned host buffers, host<->device inside the region
    yp = torch.from_numpy(y).pin_memory()
    wp = torch.from_numpy(wt).pin_memory()
    xo = [torch.empty(ctx.obj_shape, dtype=torch.float32).pin_memory() for _ in range(2)]
    e2e_upd = 0
    n_e2e = max(1, min(args.steps, 3))

    def e2e_step(s):
        # y, w cross to the device while Ax of the resident object is
        # projected (and while the previous step's object leaves for the host)
        ctx.lib.xtg_upload_sino_start(ctx.h, xtg.C.c_void_p(yp.data_ptr()), xtg.C.c_void_p(wp.data_ptr()), None)
        st = ctx.iteration(it + 1 + s)
        ctx.download_object_start(xo[s % 2].data_ptr())
        return st

    e2e_step(0)  # warms this path up, untimed
    ctx.download_wait()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for s in range(1, n_e2e + 1):
        e2e_upd += e2e_step(s).voxel_updates
    ctx.download_wait()  # the last step's object is on the host
    torch.cuda.synchronize()
    e2e_t = time.perf_counter() - t1
    e2e = e2e_upd / e2e_t * world

    # roofline of the ICD column kernel.  Algorithmic bytes per voxel update:
    # nnz x zovl x 12 B (e read, w read, e write per (view, bin, row)) plus the
    # column's A entries shared by its N_z voxels; per average ICD launch
    b_upd = nnz * ctx.zovl * 12.0 + nnz * A_BYTES[args.amode] / ctx.N_z
    alg_per_launch = upd * b_upd / max(n_icd, 1)
    ms_per_launch = kms / max(n_icd, 1)
    peak, kind = peaks()
    achieved = alg_per_launch / (ms_per_launch / 1e3) / 1e9 if kms > 0 else 0.0
    dpu = dram_bytes_per_update()
    traffic = dpu * upd / max(n_icd, 1) if dpu else None
    line = {
        "metric": METRIC, "value": value, "unit": "voxel-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_job / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic (seeded ellipsoid phantom{', moving' if w['moving'] else ''}, reference A, "
                f"Poisson {w['I0']:.0e} photons/ray, {100 * w['zfrac']:g}% zingers)",
        "config": {**base_config(w, args.amode), "masked_columns": ctx.n_masked, "zslab": ctx.zslab(),
                   "iterations_timed": [args.warmup + 1, args.warmup + args.steps],
                   "l2": f"inputs larger than L2 (e + w = {2 * y.nbytes / 1e6:.0f} MB)",
                   "parallelism": f"replicas{world}",
                   "cost_after": cost, "wall_s_timed": wall, "forward_projection_ms": fp_ms, "projector": proj,
                   "zero_skipped_per_step": zsk / args.steps,
                   "counted": "voxel updates exclude zero-skipped voxels (x = 0 with no positive neighbour)"},
        "e2e": {"value": e2e, "unit": "voxel-updates/s", "h2d_bytes_per_step": int(y.nbytes + wt.nbytes),
                "d2h_bytes_per_step": int(xo[0].numel() * 4)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind_note(kind), "kernel": "k_icd_columns",
                     "alg_bytes_per_launch": alg_per_launch, "ms_per_launch": ms_per_launch,
                     "icd_launches_timed": n_icd, "bytes_per_voxel_update": b_upd, "nnz_per_column": nnz,
                     "dram_bytes_per_voxel_update": dpu,
                     "traffic_note": "ncu DRAM bytes per voxel (iteration average of a random-pass and an NHICD "
                                     "launch, 384^2 capture, cold L2) x voxel updates per launch",
                     "kernel_ms_per_step": kms / args.steps, "column_items_per_step": rows / args.steps},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    x_star = None
    if not args.no_converge and world == 1:
        # a single-GPU metric: with N replicas every rank would repeat it.
        # The committed warm-start weights were trained for the plain-3D geometry
        line["time_to_cost"] = converge(ctx, args.amode, learned=args.workload == "plain3d" and not args.nxy,
                                        weights=args.weights, starts=tuple(args.starts.split(",")),
                                        cstar_start=args.cstar_start, max_iters=args.max_iters)
        x_star = line["time_to_cost"].pop("_x_star")
        # the reference's CPU-runnable configuration, to its own FP64 converged cost
        line["time_to_cost_config1"] = config1_gpu(args.amode)
    ctx.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
        if x_star is not None:
            line["time_to_cost"]["c_star_check"] = c_star_check(p, t, a, y, wt, x_star,
                                                                line["time_to_cost"]["c_star"])
    if world == 1 and args.workload == "plain3d" and not args.nxy and not args.no_other:
        line["other_workloads"] = {name: other_workload(name, args) for name in ("timbir4d", "timbir4d_large")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


# the reference's CPU-runnable configuration (4 slices of 128^2, 128 bins,
# 180 views at i degrees, 10 ellipsoids U(0, 0.01), 2e4 photons/ray, no zinger
# correction, no NHICD, positivity on) and its converged cost: the reference's
# -DREAL_IS_DOUBLE build run 150 iterations from zero
# (tests/golden/config_c1.npz, made by tests/golden/make_golden.py)
C1_FIXTURE = os.path.join(ROOT, "tests", "golden", "config_c1.npz")


def config1_case():
    p = xtg.Params(p=1.2, sigma_s=200000.0, sigma_t=200000.0, c_s=0.01, c_t=0.01, delta_xy=1.0, delta_z=1.0,
                   length_r=128.0, length_t=4.0, rotation_center=64.0, alpha=1.0, Rtime0=0.0, Rtime_delta=180.0,
                   radius_obj=128.0, zingerT=100000.0, zingerDel=0.0, iter=20, Rtime_num=1, num_projections=180,
                   N_r=128, N_t=4, num_threads=1, positivity=1, no_NHICD=1)
    t, a = xtg.round_views(*xtg.views_uniform(180))
    x = xtg.phantom((1, 4, 128, 128), 10, 0.01, 1)
    y, w = xtg.measure(xtg.forward_cpu(p, t, a, x), 2e4, 101)
    g = np.load(C1_FIXTURE)
    # the seeded generator reproduces the inputs the reference ran on
    assert abs(y.astype(np.float64).sum() / float(g["y_sum"]) - 1) < 1e-12
    assert abs(w.astype(np.float64).sum() / float(g["w_sum"]) - 1) < 1e-12
    return p, t, a, y, w, float(g["costs64"][-1])


def config1_gpu(amode, tol=1e-4, resync_every=10):
    """Seconds from the zero start to MAP cost <= (1 + tol) C* on configuration
    1 (wall clock, e = y - Ax - d and the cost tests included; the A storage
    is built beforehand, like the reference's tables).  C* is the reference's
    own FP64 converged cost; its own time for the same run is the reference
    arm's time_to_cost_config1."""
    import torch
    p, t, a, y, w, c_star = config1_case()
    c = xtg.Context(p, t, a)
    c.set_options(a_mode=AMODES[amode])
    c.upload_sino(y, w)
    zero = np.zeros(c.obj_shape, np.float32)
    c.upload_object(zero)
    c.iteration(1)
    c.upload_object(zero)
    torch.cuda.synchronize()
    target = c_star * (1 + tol)
    t0 = time.perf_counter()
    c.init_error_sino()
    it, cost = 0, float("inf")
    while it < 200:
        it += 1
        c.iteration(it)
        cost = c.cost_running()[0]
        if cost <= target or it % resync_every == 0:
            cost = c.resync_fp64()[0]
            if cost <= target:
                break
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    c.close()
    return {"workload": "config1_128x128x4_180views", "s": secs if cost <= target else None, "iterations": it,
            "cost": cost, "c_star": c_star, "tol": tol, "a_mode": amode,
            "c_star_source": "the reference's -DREAL_IS_DOUBLE engine, 150 iterations from zero "
                             "(tests/golden/config_c1.npz)"}


def config1_reference(tol=1e-4, threads=None):
    """The reference engine's own routines (oracle/_ref, its default FP32
    build, OpenMP on every host core) on configuration 1 from its zero start:
    seconds until its object's MAP cost is <= (1 + tol) C*.  Timed: e = y - Ax
    and per iteration updateVoxelsTimeSlices plus computeCost (its cost build
    evaluates the cost every iteration).  Not timed: the judge, an FP64
    evaluation of each iteration's object (the reference's own FP32 cost sums
    in float and reads ~3e-5 low here, so it would stop early)."""
    from oracle.oracle import Oracle, Reference
    p, t, a, y, w, c_star = config1_case()
    p.num_threads = threads or os.cpu_count()
    judge = Oracle(p, t, a)
    judge.set_sino(y, w)
    cwd = os.getcwd()
    d = tempfile.mkdtemp()
    os.chdir(d)
    try:
        xtg.write_view_file("view_info.txt", t, a)
        r = Reference(p)
        r.set_sino(y, w)
        r.srandom2(761521)
        target = c_star * (1 + tol)
        t0 = time.perf_counter()
        r.init_error_sino()
        r.cost()
        secs = time.perf_counter() - t0
        cost, it = float("inf"), 0
        while it < 200 and cost > target:
            it += 1
            t0 = time.perf_counter()
            r.iterate(it)
            r.cost()
            secs += time.perf_counter() - t0
            judge.set_object(r.object())
            cost = judge.map_cost_fp64()[0]
        r.close()
    finally:
        os.chdir(cwd)
        judge.close()
    return {"workload": "config1_128x128x4_180views", "s": secs if cost <= target else None, "iterations": it,
            "cost": cost, "c_star": c_star, "tol": tol, "threads": p.num_threads,
            "judge": "MAP cost of each iteration's object with FP64 sums (not timed)",
            "note": "the reference runs N_time x num_z_blocks / 2 = 2 tasks at once on 4 slices "
                    "(XT_Init.c:396-400, XT_ICD_update.c:800-801)"}


def c_star_check(p, t, a, y, w, x_star, c_star):
    """The host re-evaluates the MAP cost of the C* object (part of the CPU
    leg; the oracle is the checker here): with the GPU's arithmetic (FP32 A
    and constants of the reference's default build, FP64 sums) and with the
    reference's -DREAL_IS_DOUBLE arithmetic."""
    from oracle.oracle import Oracle
    out = {}
    for double, key in ((False, "oracle_gpu_arithmetic"), (True, "oracle_reference_fp64_build")):
        t0 = time.perf_counter()
        o = Oracle(p, t, a, double=double)
        o.set_sino(y, w)
        o.set_object(x_star)
        v = o.map_cost_fp64()[0]
        o.close()
        out[key] = {"cost": v, "rel_diff": v / c_star - 1.0, "s": time.perf_counter() - t0}
    return out


def other_workload(name, args, steps=None):
    """Throughput (and for the 4D workload seconds to cost) of the other
    configurations, measured after the headline one."""
    import torch
    w = dict(WORKLOADS[name])
    p, t, a, x_true, y, wt = make_data(w)
    ctx = xtg.Context(p, t, a)
    ctx.set_options(a_mode=xtg.XTG_A_AUTO)
    ctx.upload_sino(y, wt)
    ctx.init_error_sino()
    big = name == "timbir4d_large"
    warm, steps = (1, 2) if big else (3, 10)
    it = 0
    for _ in range(warm):
        it += 1
        ctx.iteration(it)
    torch.cuda.synchronize()
    ms, upd, kms, n_icd = 0.0, 0, 0.0, 0
    for _ in range(steps):
        it += 1
        st = ctx.iteration(it)
        ms += st.ms
        upd += st.voxel_updates
        k_ms, _, k_n = ctx.last_kernel_time()
        kms += k_ms
        n_icd += k_n
    nnz = nnz_per_column(ctx, p, t, a)
    amode = {xtg.XTG_A_FP32: "fp32", xtg.XTG_A_TABLE32: "table32", xtg.XTG_A_FP16: "fp16"}[ctx.a_mode_used()]
    b_upd = nnz * ctx.zovl * 12.0 + nnz * A_BYTES[amode] / ctx.N_z
    peak, kind = peaks()
    achieved = upd * b_upd / (kms / 1e3) / 1e9 if kms > 0 else 0.0
    out = {"config": base_config(w, amode), "value": upd / (ms / 1e3), "unit": "voxel-updates/s",
           "ms_per_step": ms / steps, "steps": steps, "warmup": warm,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "bytes_per_voxel_update": b_upd, "nnz_per_column": nnz, "kernel_ms_per_step": kms / steps,
                        "icd_launches_per_step": n_icd / steps, "peak_kind": peak_kind_note(kind)}}
    if not big and not args.no_converge:
        out["time_to_cost"] = converge(ctx, amode, learned=False)
        out["time_to_cost"].pop("_x_star")
        out["time_to_cost"]["learned"] = "not run: the committed network was trained for the plain-3D geometry"
    elif big:
        out["time_to_cost"] = ("not run by default (about 30 minutes of 4-5 s iterations: a 120-iteration run "
                               "to C* from the multi-resolution start, then each start); time it with "
                               "`python bench.py --workload timbir4d_large --steps 1 --warmup 1 --no-cpu-baseline "
                               "--cstar-start multires --max-iters 120`")
    ctx.close()
    return out


def peak_kind_note(kind):
    return f"{kind} (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else "fallback 6.65 TB/s"


_SAMPLE_DATA = {}


def ref_sample_run(w, iters=1, threads=None):
    """Times the reference engine's own updateVoxelsTimeSlices (oracle/_ref,
    via oracle/ref_harness.c) on the bounded sample; returns
    (voxel updates/s, seconds, voxels per iteration, threads)."""
    from oracle.oracle import Reference, ref_available
    if not ref_available():
        return None
    threads = threads or os.cpu_count()
    radius = w["N"] / 8.0  # central disk: about 1/20 of the columns
    key = json.dumps(w, sort_keys=True)
    if key not in _SAMPLE_DATA:  # the same seeded data for every step
        _SAMPLE_DATA[key] = make_data(w)
    p, t, a, x_true, y, wt = _SAMPLE_DATA[key]
    p = xtg.Params(**{k: getattr(p, k) for k in p.__dataclass_fields__})
    p.radius_obj = radius
    p.num_threads = threads
    cwd = os.getcwd()
    d = tempfile.mkdtemp()
    os.chdir(d)
    try:
        xtg.write_view_file("view_info.txt", t, a)
        r = Reference(p)
        r.set_sino(y, wt)
        # the object starts at zero, so e = y - A 0 - d = y: set it directly
        # instead of running the reference's single-threaded full-volume
        # forward projection, which is not part of the timed iteration
        r.set_error_sino(y)
        r.srandom2(761521)
        c = np.arange(w["N"]) + 0.5 - w["N"] / 2.0
        n_masked = int(((c[None, :] ** 2 + c[:, None] ** 2) < radius * radius).sum())
        g = None
        vox = n_masked * w["NT"] * w["n_time"]
        t0 = time.perf_counter()
        for it in range(1, iters + 1):
            r.iterate(it)
        dt = time.perf_counter() - t0
        r.close()
    finally:
        os.chdir(cwd)
    return vox * iters / dt, dt, vox, threads, g


def cpu_baseline(args):
    res = ref_sample_run(workload(args), 1)
    if res is None:
        return {"value": None, "unit": "voxel-updates/s", "cores": 0, "kind": "reference",
                "sample": "oracle/_ref not built"}
    v, dt, vox, thr, _ = res
    return {"value": v, "unit": "voxel-updates/s", "cores": thr, "kind": "reference",
            "sample": f"reference XT_Engine routines (updateVoxelsTimeSlices, iteration 1) on the same workload "
                      f"restricted to a central disk of radius {workload(args)['N'] // 8} voxels: {vox} voxel updates in {dt:.1f} s, "
                      f"OpenMP {thr} threads"}


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    vals, tot = [], 0.0
    for s in range(args.warmup + args.steps):
        res = ref_sample_run(workload(args), 1)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference build) missing"}))
            return
        v, dt, vox, thr, _ = res
        if s >= args.warmup:
            vals.append(v)
            tot += dt
    value = float(np.mean(vals))
    c1 = config1_reference()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "voxel-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (same seeded workload, central-disk sample)",
            "config": dict(base_config(workload(args), args.amode),
                           sample=f"radius_obj {workload(args)['N'] // 8} (about 1/20 of the columns)",
                           parallelism="cpu"),
            "cpu_baseline": {"value": value, "unit": "voxel-updates/s", "cores": thr, "kind": "reference",
                             "sample": "one reference iteration per step on the central-disk sample"},
            "e2e": {"value": value, "unit": "voxel-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "time_to_cost_config1": c1}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--amode", default="table32", choices=sorted(AMODES),
                    help="A storage: table32 (exact FP32 column table), fp16 (FP16 column table), "
                         "fp32 (computed at every column visit)")
    ap.add_argument("--columns", type=int, default=0)
    ap.add_argument("--workload", default="plain3d", choices=sorted(WORKLOADS))
    ap.add_argument("--nxy", type=int, default=0,
                    help="voxels per side (= detector bins) instead of the workload's; for profiling captures")
    ap.add_argument("--zslab", type=int, default=0,
                    help="z slices per ICD work piece (0: chosen from the L2 size)")
    ap.add_argument("--network-forward", action="store_true",
                    help="time only the warm-start network's forward pass on [1][nxy][nxy][nz] (profiling)")
    ap.add_argument("--network-train", action="store_true",
                    help="time only training steps of the warm-start network on [nxy][nxy][nz] volumes (profiling)")
    ap.add_argument("--patch", type=int, nargs=3, default=(64, 64, 32), help="training patch for --network-train")
    ap.add_argument("--nz", type=int, default=64, help="slices for --network-forward / --network-train")
    ap.add_argument("--reps", type=int, default=5, help="forward passes timed by --network-forward")
    ap.add_argument("--kernels", action="store_true",
                    help="time the non-ICD kernels of the engine on the workload (profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other", action="store_true", help="skip the 4D workloads after the headline one")
    ap.add_argument("--weights", default=WEIGHTS, help="warm-start network weights for the learned start")
    ap.add_argument("--starts", default="zero,fbp,multires,learned",
                    help="starts timed by time_to_cost (comma-separated subset)")
    ap.add_argument("--max-iters", type=int, default=400,
                    help="iteration limit of the run to a stall and of each timed start")
    ap.add_argument("--cstar-start", default="fbp", choices=["fbp", "multires"],
                    help="start of the run to a stall that defines C* (multires: fewer iterations on large volumes)")
    ap.add_argument("--no-converge", action="store_true", help="skip the seconds-to-converged-cost run")
    args = ap.parse_args()
    if args.network_forward:
        network_forward(args.nxy or 512, args.nz, args.reps)
    elif args.network_train:
        print(json.dumps(network_train(args.nxy or 256, args.nz, args.steps, args.patch)), flush=True)
    elif args.kernels:
        kernel_timings(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
