"""The learned warm start end to end on the engine (small geometry: 64^2 x 16
voxels, 128 views, 1e4 photons/ray, 0.5 % zingers):

  * an untrained network (zero head) returns its ICD input, which is not
    lower in cost, so the fallback keeps the ICD image;
  * a network trained on 16 phantoms reconstructed by the engine lowers the
    MAP cost of a held-out phantom's start below the ICD image it was given,
    and the reconstruction from it reaches (1 + 1e-3) of the converged cost in
    fewer iterations than the FBP start.
"""
import os
import sys

import numpy as np
import pytest
import torch

import common
import xtg

sys.path.insert(0, os.path.join(common.ROOT, "timbir-python_b200"))
import train_warmstart as tw  # noqa: E402

pytestmark = pytest.mark.gpu

N, NT, NP = 64, 16, 128


def held_out_ctx(seed=77):
    p = tw.params(N, NT, NP)
    t, a = xtg.round_views(*xtg.views_uniform(NP))
    c = xtg.Context(p, t, a)
    c.set_options(a_mode=xtg.XTG_A_AUTO)
    x = xtg.phantom((1, NT, N, N), 30, 0.01, seed)
    c.upload_object(x)
    y, w = xtg.measure(c.forward_project(), 1e4, seed + 5, zinger_frac=0.005)
    c.upload_sino(y, w)
    return c


def iters_to(c, start_iter, target, limit=200):
    for it in range(start_iter, start_iter + limit):
        c.iteration(it)
        if c.resync_fp64()[0] <= target:
            return it - start_iter + 1
    return None


def test_untrained_network_falls_back_to_icd_image():
    c = held_out_ctx()
    net = xtg.WarmNet(seed=2)
    used, cn, ci = c.init_learned(net, 2)
    # the zero head returns the ICD image itself: equal cost, so it is not used
    assert not used and cn == ci
    # the context holds the ICD image with a fresh e: its cost is the one reported
    assert c.cost_running()[0] == pytest.approx(ci, rel=1e-12)
    net.close()


def test_trained_network_lowers_start_cost_and_iterations():
    data, shape = tw.make_set(16, N, NT, NP, equits=2, target_iters=40, seed=500, log=lambda *a: None)
    net, losses = tw.train(data, shape, steps=400, batch=8, patch=(32, 32, 16), log=lambda *a: None)
    assert losses[-50:].mean() < losses[:50].mean()
    # converged cost of the held-out phantom
    c = held_out_ctx()
    c.init_fbp()
    for it in range(1, 121):
        c.iteration(it)
    c_star = c.resync_fp64()[0]
    target = c_star * (1 + 1e-3)
    c = held_out_ctx()
    used, cn, ci = c.init_learned(net, 2)
    assert used and cn < ci, (cn, ci)
    n_learned = iters_to(c, 3, target)
    c = held_out_ctx()
    c.init_fbp()
    n_fbp = iters_to(c, 1, target)
    print("iterations to 1e-3:", "learned", n_learned, "+2", "fbp", n_fbp)
    assert n_learned is not None and n_fbp is not None
    assert n_learned + 2 <= n_fbp
    net.close()
