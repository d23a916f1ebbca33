"""The z-slab decomposition over processes (timbir-python_b200/xtg_slab.py),
the reference's MPI rank split (XT_Init.c:290-294, XT_MPI.c:47-122), on the
CPU: two gloo ranks (127.0.0.1), each slab run by the FP64 oracle made
rank-aware as the reference's ranks are (halo slices in the voxel update,
XT_VoxUpdate.c:94-99; the prior's pairs into the slab above,
XT_ICD_update.c:203-205).

  * the partition gives each rank N_t / ranks detector rows and
    Length_T / ranks, and the whole detector's rows in order;
  * after an exchange each rank's halo planes hold its neighbours' boundary
    slices;
  * the sum of the slabs' MAP costs equals the whole-volume cost of the
    gathered object (1e-9 relative: the decomposition of the data term, the
    log term and the prior pairs across the slab boundary is exact);
  * run to convergence, the decomposed reconstruction reaches the converged
    cost of the undivided one (within 1e-6 relative; no zinger correction,
    so the objective is convex and both reach the same minimum).

The GPU form (the library's exchange hook, slabs as threads on one GPU) is in
tests/test_slab_gpu.py.
"""
import os
import socket
import types

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import common
import xtg
import xtg_slab
from oracle.oracle import Oracle

N, NT, NP, ITERS = 16, 8, 24, 80


def case():
    p = common.params(N=N, NT=NT, NP=NP, nhicd=True)
    t, a = common.views(p)
    x, ax, y, w = common.data(p, t, a, seed=31)
    return p, t, a, y, w


class OracleSlabEngine:
    """A slab run by the FP64 oracle, with the engine calls the driver makes."""

    def __init__(self, p_slab, times, angles, below, above):
        self.o = Oracle(p_slab, times, angles, double=True)
        self.o.set_slab(below, above)
        self.o.srandom2(761521)
        shape = (self.o.N_time, self.o.N_y, self.o.N_x)
        self.planes = tuple(torch.zeros(shape, dtype=torch.float64) if on else None
                            for on in (below, above, below, above))

    @property
    def obj_shape(self):
        return self.o.obj_shape

    def set_exchange(self, fn):
        self.fn = fn

    def exchange(self):
        lo, hi = self.o.boundary()
        if self.planes[0] is not None:
            self.planes[0].copy_(torch.from_numpy(lo))
        if self.planes[1] is not None:
            self.planes[1].copy_(torch.from_numpy(hi))
        self.fn(*self.planes)
        self.o.set_halo(None if self.planes[2] is None else self.planes[2].numpy(),
                        None if self.planes[3] is None else self.planes[3].numpy())

    def upload_sino(self, y, w, d=None):
        self.o.set_sino(y, w, d)

    def upload_object(self, x):
        self.o.set_object(x)

    def init_error_sino(self):
        self.o.init_error_sino()

    def iteration(self, it):
        self.exchange()
        self.o.iterate(it)
        self.exchange()
        return types.SimpleNamespace(voxel_updates=0, zero_skipped=0, columns=0, mag_sum=0.0, vox_mag=1.0,
                                     total_pix=0.0, ms=0.0)

    def cost(self):
        return self.o.map_cost_fp64()

    def object(self):
        return self.o.object().astype(np.float32)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        p, t, a, y, w = case()
        comm = xtg_slab.DistExchange()
        r = xtg_slab.SlabReconstruction(p, t, a, world, rank, comm, engine=OracleSlabEngine)
        r.upload_sino(y, w)
        r.start("zero")
        # halo routing: each halo plane is the neighbour's boundary slice
        lo, hi = r.eng.o.boundary()
        bounds = comm.gather(np.stack([lo, hi]))
        if rank > 0:
            assert np.array_equal(r.eng.planes[2].numpy(), bounds[rank - 1][1])
        if rank < world - 1:
            assert np.array_equal(r.eng.planes[3].numpy(), bounds[rank + 1][0])
        costs = []
        for it in range(1, ITERS + 1):
            r.iteration(it)
            costs.append(r.cost()[0])
        x = r.gather_object()
        q.put((rank, r.p_slab.N_t, r.p_slab.length_t, costs, x))
    finally:
        dist.destroy_process_group()


def test_slab_partition_matches_reference_split():
    p, t, a, y, w = case()
    for ranks in (1, 2, 4):
        ps = xtg_slab.slab_params(p, ranks)
        assert ps.N_t == p.N_t // ranks and ps.length_t == pytest.approx(p.length_t / ranks)
        rows = [xtg_slab.slab_rows(p, ranks, r) for r in range(ranks)]
        assert rows[0][0] == 0 and rows[-1][1] == p.N_t
        assert all(rows[i][1] == rows[i + 1][0] for i in range(ranks - 1))
        parts = [xtg_slab.slab_sino(y, p, ranks, r) for r in range(ranks)]
        assert np.array_equal(np.concatenate(parts, axis=-1), y)
    with pytest.raises(ValueError):
        xtg_slab.slab_params(p, 3)


def test_two_gloo_ranks_reach_the_undivided_reconstruction():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = {}
    for _ in range(world):
        rank, nt, lt, costs, x = q.get(timeout=600)
        res[rank] = (nt, lt, costs, x)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    p, t, a, y, w = case()
    assert res[0][0] == NT // 2 and res[0][1] == pytest.approx(p.length_t / 2)
    costs, x = res[0][2], res[0][3]
    assert res[1][2] == costs and np.array_equal(res[1][3], x)  # every rank holds the same sums
    # the slabs' summed cost is the whole volume's cost of the gathered object
    o = Oracle(p, t, a, double=True)
    o.set_sino(y, w)
    o.set_object(x)
    whole = o.map_cost_fp64()[0]
    assert costs[-1] == pytest.approx(whole, rel=1e-9)
    # the undivided reconstruction's converged cost
    o.set_object(np.zeros(o.obj_shape))
    o.init_error_sino()
    o.srandom2(761521)
    for it in range(1, ITERS + 1):
        o.iterate(it)
    c_star = o.map_cost_fp64()[0]
    print("slab cost", costs[-1], "undivided", c_star, "rel", costs[-1] / c_star - 1)
    assert abs(costs[-1] / c_star - 1) < 1e-6
