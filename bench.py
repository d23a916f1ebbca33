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
sinogram/weights go host->device, e = y - Ax - d is rebuilt, one iteration
runs and the object comes back device->host.

--impl reference times the reference engine's own CPU implementation
(oracle/_ref, compiled from the reference sources, OpenMP on every host core)
on a bounded sample of the same workload: the same geometry, views and data
restricted by --radius_obj to a central disk of 1/16 of the columns.
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

WORKLOAD = dict(N=512, NT=64, NP=1024, n_ell=30, mu=0.01, I0=1e4, zfrac=0.005, seed=2)
METRIC = "voxel-updates/s (ICD, plain 3D at scale: 512^2 x 64 voxels, 1024 views)"
AMODES = {"fp32": xtg.XTG_A_FP32, "table32": xtg.XTG_A_TABLE32, "fp16": xtg.XTG_A_FP16}


def params(w, radius=None):
    N = w["N"]
    return xtg.Params(
        p=1.2, sigma_s=200000.0, sigma_t=200000.0, c_s=0.01, c_t=0.01, delta_xy=1.0, delta_z=1.0,
        length_r=float(N), length_t=float(w["NT"]), rotation_center=N / 2.0, alpha=1.0, Rtime0=0.0,
        Rtime_delta=float(w["NP"]), radius_obj=float(N) if radius is None else float(radius),
        zingerT=4.0, zingerDel=0.5, iter=100, Rtime_num=1, num_projections=w["NP"], N_r=N, N_t=w["NT"],
        num_threads=1, positivity=1, no_NHICD=0)


def make_data(w):
    p = params(w)
    t, a = xtg.round_views(*xtg.views_uniform(w["NP"]))
    x = xtg.phantom((1, w["NT"], w["N"], w["N"]), w["n_ell"], w["mu"], w["seed"])
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


def traffic_per_launch():
    """DRAM bytes per ICD launch from the committed ncu summary, if present."""
    f = os.path.join(ROOT, "profiles", "icd_columns_plain3d_512.md")
    if not os.path.exists(f):
        return None
    for line in open(f):
        if line.startswith("traffic_bytes_per_chunk_launch:"):
            return float(line.split(":")[1])
    return None


def nnz_per_column(ctx, n_cols=512, seed=0):
    """Average A-matrix entries per column over all views (sampled columns)."""
    rng = np.random.default_rng(seed)
    g = ctx.geometry()
    rows = rng.integers(0, ctx.N_y, n_cols)
    cols = rng.integers(0, ctx.N_x, n_cols)
    keep = [(r, c) for r, c in zip(rows, cols)
            if ((g.x0 + (c + 0.5) * g.delta_xy) ** 2 + (g.y0 + (r + 0.5) * g.delta_xy) ** 2) < g.radius_obj ** 2]
    rr = np.repeat([k[0] for k in keep], ctx.N_p)
    cc = np.repeat([k[1] for k in keep], ctx.N_p)
    vv = np.tile(np.arange(ctx.N_p), len(keep))
    _, _, cnt = ctx.amatrix(rr, cc, vv)
    return float(cnt.sum()) / len(keep)


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
    w = WORKLOAD
    p, t, a, x_true, y, wt = make_data(w)
    ctx = xtg.Context(p, t, a)
    ctx.set_options(a_mode=AMODES[args.amode], max_columns=args.columns)
    ctx.upload_sino(y, wt)
    ctx.init_error_sino()
    torch.cuda.synchronize()
    tf = time.perf_counter()
    ctx.init_error_sino()  # e = y - Ax - d (fast projector), timed once for the log
    fp_ms = (time.perf_counter() - tf) * 1e3
    nnz = nnz_per_column(ctx)
    it = 0
    for _ in range(args.warmup):
        it += 1
        ctx.iteration(it)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launch_count()
    clk = Clocks(lrank)
    ms_tot, upd, kms, rows = 0.0, 0, 0.0, 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        it += 1
        st = ctx.iteration(it)
        ms_tot += st.ms
        upd += st.voxel_updates
        k_ms, _ = ctx.last_kernel_time()
        kms += k_ms
        rows += st.columns
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = clk.stop()
    launches = ctx.launch_count() - launches0
    cost = ctx.cost()[0]
    if world > 1:
        tt = torch.tensor([ms_tot, float(upd)], dtype=torch.float64, device="cuda")
        mx = tt.clone()
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.SUM)
        ms_job, upd_job = float(mx[0]), float(tt[1])
    else:
        ms_job, upd_job = ms_tot, float(upd)
    value = upd_job / (ms_job / 1e3)

    # e2e: through the C ABI from pinned host buffers, host<->device inside the region
    yp = torch.from_numpy(y).pin_memory()
    wp = torch.from_numpy(wt).pin_memory()
    xo = torch.empty(ctx.obj_shape, dtype=torch.float32).pin_memory()
    e2e_upd, e2e_t = 0, 0.0
    for s in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ctx.lib.xtg_upload_sino(ctx.h, xtg.C.c_void_p(yp.data_ptr()), xtg.C.c_void_p(wp.data_ptr()), None)
        ctx.init_error_sino()
        st = ctx.iteration(it + 1 + s)
        ctx.lib.xtg_download_object(ctx.h, xtg.C.c_void_p(xo.data_ptr()))
        torch.cuda.synchronize()
        e2e_t += time.perf_counter() - t1
        e2e_upd += st.voxel_updates
    e2e = e2e_upd / e2e_t * world

    # roofline of the ICD column kernel: algorithmic bytes = rows x nnz x 12 B
    # (e read, w read, e write per (view, bin, row)), per ICD launch time
    n_items = rows
    rows_touched = upd * p.delta_z  # every updated voxel streams its zovl rows
    alg_bytes = rows_touched * nnz * 12.0
    peak, kind = peaks()
    achieved = alg_bytes / (kms / 1e3) / 1e9 if kms > 0 else 0.0
    line = {
        "metric": METRIC, "value": value, "unit": "voxel-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_job / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ellipsoid phantom, reference A, Poisson 1e4, 0.5% zingers)",
        "config": {"workload": "plain3d_512x512x64_1024views", "N_xy": 512, "N_z": 64, "N_r": 512, "N_t": 64,
                   "N_p": 1024, "zinger": [4.0, 0.5], "nhicd": True, "a_mode": args.amode,
                   "iterations_timed": [args.warmup + 1, args.warmup + args.steps],
                   "l2": "inputs larger than L2 (e + w = 268 MB)", "parallelism": f"replicas{world}",
                   "cost_after": cost, "wall_s_timed": wall, "forward_projection_ms": fp_ms},
        "e2e": {"value": e2e, "unit": "voxel-updates/s", "h2d_bytes_per_step": int(y.nbytes + wt.nbytes),
                "d2h_bytes_per_step": int(xo.numel() * 4)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic_per_launch(),
                     "peak_kind": peak_kind_note(kind),
                     "bytes_per_voxel_update": nnz * 12.0, "nnz_per_column": nnz,
                     "kernel_ms_per_step": kms / args.steps, "column_items_per_step": n_items / args.steps},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def peak_kind_note(kind):
    return f"{kind} (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else "fallback 6.65 TB/s"


def ref_sample_run(iters=1, threads=None):
    """Times the reference engine's own updateVoxelsTimeSlices (oracle/_ref,
    via oracle/ref_harness.c) on the bounded sample; returns
    (voxel updates/s, seconds, voxels per iteration, threads)."""
    from oracle.oracle import Reference, ref_available
    if not ref_available():
        return None
    w = WORKLOAD
    threads = threads or os.cpu_count()
    radius = w["N"] / 8.0  # central disk: about 1/16 of the columns
    p, t, a, x_true, y, wt = make_data(w)
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
        vox = n_masked * w["NT"]
        t0 = time.perf_counter()
        for it in range(1, iters + 1):
            r.iterate(it)
        dt = time.perf_counter() - t0
        r.close()
    finally:
        os.chdir(cwd)
    return vox * iters / dt, dt, vox, threads, g


def cpu_baseline(args):
    res = ref_sample_run(1)
    if res is None:
        return {"value": None, "unit": "voxel-updates/s", "cores": 0, "kind": "reference",
                "sample": "oracle/_ref not built"}
    v, dt, vox, thr, _ = res
    return {"value": v, "unit": "voxel-updates/s", "cores": thr, "kind": "reference",
            "sample": f"reference XT_Engine routines (updateVoxelsTimeSlices, iteration 1) on the same workload "
                      f"restricted to a central disk of radius 64 voxels: {vox} voxel updates in {dt:.1f} s, "
                      f"OpenMP {thr} threads"}


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    vals, tot = [], 0.0
    for s in range(args.warmup + args.steps):
        res = ref_sample_run(1)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference build) missing"}))
            return
        v, dt, vox, thr, _ = res
        if s >= args.warmup:
            vals.append(v)
            tot += dt
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "voxel-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (same seeded workload, central-disk sample)",
            "config": {"workload": "plain3d_512x512x64_1024views", "sample": "radius_obj 64 (1/16 of columns)"},
            "cpu_baseline": {"value": value, "unit": "voxel-updates/s", "cores": thr, "kind": "reference",
                             "sample": "one reference iteration per step on the central-disk sample"},
            "e2e": {"value": value, "unit": "voxel-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
