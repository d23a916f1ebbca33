"""One reconstruction split into z slabs over several processes (one GPU each),
the B200 form of the reference's MPI decomposition.

The reference runs one MPI rank per contiguous z slab: rank r of R owns
N_t / R detector rows (Length_T / R, XT_Init.c:290-294), the N_z / R slices
they see (parallel-beam geometry is z-invariant, so a slab's rows depend on
its own slices only), and two halo slices holding its neighbours' adjacent
slices, exchanged after every half-pass (MPI_Send_Recv_Z_Slices /
MPI_Wait_Z_Slices, XT_MPI.c:47-122).  The costs, the variance and the stop
statistic are summed over ranks (XT_ICD_update.c:296-312, 651, 900-902).

Here each slab is an engine context (xtg.Context with the slab's N_t and
length_t); the library calls back at its exchange points (xtg_set_slab) and
the `comm` object moves one x-y plane per frame to each neighbour:

* DistExchange   -- torch.distributed point-to-point (NCCL between GPUs,
                    gloo on the CPU) and all-reduce for the sums;
* ThreadExchange -- the slabs as host threads of one process (testing on one
                    GPU: the host exchanges between launches, no kernel waits
                    on another).

The driver (SlabReconstruction) works with any engine exposing the same few
calls, which is how the CPU tests run the decomposition on the CPU oracle.
Variance and offset re-estimation inside an iteration need sums over every
slab; the library refuses them for slabs.
"""
from __future__ import annotations

import dataclasses
import threading

import numpy as np

import xtg


def slab_params(p: xtg.Params, ranks: int) -> xtg.Params:
    """A rank's command line: N_t / ranks detector rows and Length_T / ranks
    (XT_Init.c:293-294); the slab's slices then follow as N_t / delta_z."""
    if ranks < 1 or p.N_t % ranks:
        raise ValueError(f"N_t = {p.N_t} detector rows do not split into {ranks} slabs")
    rows = p.N_t // ranks
    if rows % int(p.delta_z):
        raise ValueError(f"{rows} rows per slab are not a whole number of {p.delta_z}-row slices")
    return dataclasses.replace(p, N_t=rows, length_t=p.length_t / ranks)


def slab_rows(p: xtg.Params, ranks: int, rank: int) -> tuple[int, int]:
    """Detector rows [t0, t1) of slab `rank` (the whole detector's numbering)."""
    rows = p.N_t // ranks
    return rank * rows, (rank + 1) * rows


def slab_sino(a, p: xtg.Params, ranks: int, rank: int):
    """The slab's rows of a whole-detector array [..][N_t] (sinogram
    [N_p][N_r][N_t] or offset [N_r][N_t])."""
    t0, t1 = slab_rows(p, ranks, rank)
    return np.ascontiguousarray(np.asarray(a)[..., t0:t1])


class DistExchange:
    """Halo planes and sums through torch.distributed: rank r sends its bottom
    slice to r - 1 and its top slice to r + 1 and receives theirs."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.ranks = dist.get_world_size(group)

    def exchange(self, send_below, send_above, recv_below, recv_above):
        dist = self.dist
        ops = []
        if send_below is not None:
            ops += [dist.P2POp(dist.isend, send_below, self.rank - 1, self.group),
                    dist.P2POp(dist.irecv, recv_below, self.rank - 1, self.group)]
        if send_above is not None:
            ops += [dist.P2POp(dist.isend, send_above, self.rank + 1, self.group),
                    dist.P2POp(dist.irecv, recv_above, self.rank + 1, self.group)]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        t = next((x for x in (recv_below, recv_above) if x is not None), None)
        if t is not None and t.is_cuda:
            import torch
            torch.cuda.synchronize(t.device)  # the engine's next launch reads the planes

    def reduce(self, values, op="sum"):
        import torch
        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM if op == "sum" else self.dist.ReduceOp.MAX,
                             group=self.group)
        return t.cpu().numpy()

    def gather(self, a):
        """Every rank's array (equal shapes), in rank order."""
        import torch
        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        out = [torch.empty_like(t) for _ in range(self.ranks)]
        self.dist.all_gather(out, t, group=self.group)
        return [o.cpu().numpy() for o in out]


class ThreadExchange:
    """The slabs as host threads of one process: a rendezvous per exchange.
    Make one object for all ranks and call `view(rank)` in each thread."""

    def __init__(self, ranks: int, timeout: float = 120.0):
        self.ranks = ranks
        self.timeout = timeout
        self.barrier = threading.Barrier(ranks)
        self.slots = [None] * ranks

    def view(self, rank):
        return _ThreadRank(self, rank)


class _ThreadRank:
    def __init__(self, hub, rank):
        self.hub, self.rank, self.ranks = hub, rank, hub.ranks

    def _sync(self):
        self.hub.barrier.wait(self.hub.timeout)

    def exchange(self, send_below, send_above, recv_below, recv_above):
        h, r = self.hub, self.rank
        h.slots[r] = (send_below, send_above)
        self._sync()
        if recv_below is not None:
            recv_below.copy_(h.slots[r - 1][1])
        if recv_above is not None:
            recv_above.copy_(h.slots[r + 1][0])
        t = next((x for x in (recv_below, recv_above) if x is not None), None)
        if t is not None and t.is_cuda:
            import torch
            torch.cuda.synchronize(t.device)
        self._sync()  # nobody refills its planes before every copy is done

    def reduce(self, values, op="sum"):
        h, r = self.hub, self.rank
        h.slots[r] = np.array([float(v) for v in values], np.float64)
        self._sync()
        stack = np.stack(h.slots)
        out = stack.sum(0) if op == "sum" else stack.max(0)
        self._sync()
        return out

    def gather(self, a):
        h, r = self.hub, self.rank
        h.slots[r] = np.asarray(a)
        self._sync()
        out = list(h.slots)
        self._sync()
        return out


class XtgSlabEngine:
    """A slab as an engine context on this process's GPU; the halo planes are
    CUDA tensors owned here and handed to the library."""

    def __init__(self, p_slab: xtg.Params, times, angles, below: bool, above: bool):
        import torch
        self.ctx = xtg.Context(p_slab, times, angles)
        shape = (self.ctx.N_time, self.ctx.N_y, self.ctx.N_x)

        def plane(on):
            return torch.zeros(shape, dtype=torch.float32, device="cuda") if on else None

        self.planes = (plane(below), plane(above), plane(below), plane(above))
        self._fn = None

    def set_exchange(self, fn):
        self._fn = fn
        self.ctx.set_slab(*self.planes, exchange=lambda phase: fn(*self.planes))

    def exchange(self):
        self.ctx.slab_exchange()

    def __getattr__(self, name):  # upload_sino, init_fbp, iteration, cost, object, ...
        return getattr(self.ctx, name)


class SlabReconstruction:
    """Slab `rank` of `ranks` of one reconstruction.  Every rank makes the same
    calls in the same order (each call may exchange planes or sum over ranks).

    engine: None for the GPU engine, or a factory engine(p_slab, times,
    angles, below, above) returning an object with the XtgSlabEngine calls."""

    def __init__(self, p: xtg.Params, times, angles, ranks: int, rank: int, comm, engine=None):
        self.p, self.ranks, self.rank, self.comm = p, ranks, rank, comm
        self.p_slab = slab_params(p, ranks)
        make = engine or XtgSlabEngine
        self.eng = make(self.p_slab, times, angles, rank > 0, rank < ranks - 1)
        self.eng.set_exchange(comm.exchange)

    def upload_sino(self, y, w, d=None, whole_detector=True):
        """y, w [N_p][N_r][N_t] (d [N_r][N_t]) of the whole detector, or of this
        slab's rows with whole_detector=False."""
        if whole_detector:
            y, w = (slab_sino(a, self.p, self.ranks, self.rank) for a in (y, w))
            d = None if d is None else slab_sino(d, self.p, self.ranks, self.rank)
        self.eng.upload_sino(y, w, d)

    def start(self, kind="zero", **kw):
        """The start of every slab (zero, fbp, multires), then one exchange so
        the halos hold the neighbours' starting slices."""
        if kind == "fbp":
            self.eng.init_fbp()
        elif kind == "multires":
            self.eng.init_multires(**kw)
        else:
            self.eng.upload_object(np.zeros(self.eng.obj_shape, np.float32))
            self.eng.init_error_sino()
        self.eng.exchange()

    def iteration(self, it):
        """One reference iteration on every slab; the whole volume's stop
        statistic (XT_ICD_update.c:900-925) from the slabs' sums."""
        st = self.eng.iteration(it)
        s = self.comm.reduce([st.voxel_updates, st.zero_skipped, st.columns, st.mag_sum, st.vox_mag, st.total_pix])
        ms = self.comm.reduce([st.ms], op="max")[0]
        out = {"voxel_updates": int(s[0]), "zero_skipped": int(s[1]), "columns": int(s[2]), "mag_sum": s[3],
               "vox_mag": s[4], "total_pix": s[5], "ms_max": ms}
        out["avg_update_pct"] = 100.0 * s[3] / s[4] if s[4] > 0 else float("inf")
        return out

    def cost(self):
        """The whole volume's MAP cost (cost, forward, prior): the slabs' sums."""
        c = self.eng.cost()
        return tuple(float(v) for v in self.comm.reduce(list(c)))

    def object(self):
        """This slab's slices [N_time][N_z / ranks][N_y][N_x]."""
        return self.eng.object()

    def gather_object(self):
        """The whole volume [N_time][N_z][N_y][N_x] on every rank."""
        return np.concatenate(self.comm.gather(self.object()), axis=1)
