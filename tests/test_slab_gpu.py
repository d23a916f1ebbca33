"""The z-slab decomposition on the GPU through the library's exchange hook
(xtg_set_slab): two slabs of one reconstruction as two host threads of one
process on one GPU (timbir-python_b200/xtg_slab.py ThreadExchange).  The
host moves the halo planes between launches; no kernel waits on another.

  * after the start's exchange each slab's halo planes hold its neighbour's
    boundary slices;
  * the sum of the slabs' FP64 MAP costs equals the whole-volume cost of the
    gathered object evaluated by one undivided context (1e-9 relative);
  * the decomposed reconstruction reaches the undivided one's converged cost
    (within 1e-5 relative: both run the parallel schedule to convergence on
    a convex objective);
  * variance re-estimation is refused for a slab.
"""
import dataclasses
import threading

import numpy as np
import pytest

import common
import xtg
import xtg_slab

pytestmark = pytest.mark.gpu

N, NT, NP, ITERS = 64, 16, 128, 60


def case():
    p = common.params(N=N, NT=NT, NP=NP, nhicd=True)
    t, a = common.views(p)
    x, ax, y, w = common.data(p, t, a, seed=41, I0=1e4)
    return p, t, a, y, w


def run_slabs(ranks=2):
    p, t, a, y, w = case()
    hub = xtg_slab.ThreadExchange(ranks)
    out, errs = [None] * ranks, []

    def work(r):
        try:
            s = xtg_slab.SlabReconstruction(p, t, a, ranks, r, hub.view(r))
            s.eng.set_options(a_mode=xtg.XTG_A_TABLE32)
            s.upload_sino(y, w)
            s.start("fbp")
            planes = [None if q is None else q.cpu().numpy() for q in s.eng.planes]
            first = s.object()
            costs = []
            for it in range(1, ITERS + 1):
                s.iteration(it)
                costs.append(s.cost()[0])
            out[r] = (planes, first, costs, s.gather_object())
            s.eng.ctx.close()
        except Exception as e:  # reported by the main thread
            errs.append(e)
            hub.barrier.abort()

    th = [threading.Thread(target=work, args=(r,)) for r in range(ranks)]
    for x in th:
        x.start()
    for x in th:
        x.join(600)
    assert not errs, errs
    return p, t, a, y, w, out


def test_slabs_on_one_gpu_match_the_undivided_reconstruction():
    p, t, a, y, w, out = run_slabs(2)
    (pl0, first0, costs0, x0), (pl1, first1, costs1, x1) = out
    assert costs0 == costs1 and np.array_equal(x0, x1)
    # halo routing after the start: slab 0's plane above is slab 1's bottom
    # slice and vice versa (send planes: own boundary slices)
    assert np.array_equal(pl0[3], first1[:, 0]) and np.array_equal(pl1[2], first0[:, -1])
    assert np.array_equal(pl0[1], first0[:, -1]) and np.array_equal(pl1[0], first1[:, 0])
    # the slabs' summed cost is the whole volume's cost of the gathered object
    c = xtg.Context(p, t, a)
    c.upload_sino(y, w)
    c.upload_object(x0)
    whole = c.cost()[0]
    assert costs0[-1] == pytest.approx(whole, rel=1e-9)
    # the undivided reconstruction
    c.init_fbp()
    for it in range(1, ITERS + 1):
        c.iteration(it)
    c_star = c.resync_fp64()[0]
    print("slabs", costs0[-1], "undivided", c_star, "rel", costs0[-1] / c_star - 1)
    assert abs(costs0[-1] / c_star - 1) < 1e-5
    c.close()


def test_slab_refuses_variance_reestimation():
    import torch
    p, t, a, y, w = case()
    ps = dataclasses.replace(xtg_slab.slab_params(p, 2), do_VarEst=1)
    c = xtg.Context(ps, t, a)
    pl = torch.zeros((c.N_time, c.N_y, c.N_x), device="cuda")
    with pytest.raises(RuntimeError):
        c.set_slab(pl, None, pl, None, lambda phase: None)
    c.close()
