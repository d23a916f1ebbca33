"""The multi-resolution and learned warm starts end to end on the engine
(small geometry: 64^2 x 16 voxels, 128 views, 1e4 photons/ray, 0.5 %
zingers):

  * the GPU upsampling reproduces the reference's upsample_object_bilinear_2D
    and _3D bit for bit (tests/golden/upsample.npz);
  * the multi-resolution start reaches (1 + 1e-3) of the converged cost in
    fewer fine iterations than the FBP start;
  * its binned variant reconstructs the coarse grid from the detector binned
    2 x 2 (weights summed, projections weight-averaged), as a context created
    on that binned sinogram does; a counts-ingested context (sinobin 3) bins
    its coarse stage the same way;
  * an untrained network (zero head) returns its start image, which is not
    lower in cost, so the fallback keeps the multi-resolution start;
  * a network trained on 16 phantoms reconstructed by the engine lowers the
    MAP cost of a held-out phantom's start below the multi-resolution start
    it was given, and needs strictly fewer iterations than it to reach
    (1 + 1e-4) of the converged cost.
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


def held_out_ctx(seed=77, sino=False):
    p = tw.params(N, NT, NP)
    t, a = xtg.round_views(*xtg.views_uniform(NP))
    c = xtg.Context(p, t, a)
    c.set_options(a_mode=xtg.XTG_A_AUTO)
    x = xtg.phantom((1, NT, N, N), 30, 0.01, seed)
    c.upload_object(x)
    y, w = xtg.measure(c.forward_project(), 1e4, seed + 5, zinger_frac=0.005)
    c.upload_sino(y, w)
    return (c, y, w) if sino else c


def close_images(a, b):
    """Equal up to the order in which concurrent column updates meet in the
    error sinogram (timing-dependent; both sides run to near convergence)."""
    d = np.abs(a - b)
    return d.mean() < 1e-3 * np.abs(b).mean() and d.max() < 2e-2 * np.abs(b).max(), (d.mean(), d.max())


def iters_to(c, start_iter, target, limit=200):
    for it in range(start_iter, start_iter + limit):
        c.iteration(it)
        if c.resync_fp64()[0] <= target:
            return it - start_iter + 1
    return None


def converged(seed=77):
    c = held_out_ctx(seed)
    c.init_fbp()
    for it in range(1, 121):
        c.iteration(it)
    return c.resync_fp64()[0]


def test_upsampling_bit_exact():
    g = dict(np.load(os.path.join(common.GOLDEN, "upsample.npz")))
    c = held_out_ctx()
    assert np.array_equal(c.upsample(g["inp"][None], with_z=False)[0], g["xy"])
    assert np.array_equal(c.upsample(g["inp"][None], with_z=True)[0], g["xyz"])


def test_multires_start_beats_fbp_start():
    target = converged() * (1 + 1e-3)
    c = held_out_ctx()
    c.init_multires(20)
    n_multi = iters_to(c, 1, target)
    c = held_out_ctx()
    c.init_fbp()
    n_fbp = iters_to(c, 1, target)
    print("iterations to 1e-3: multires", n_multi, "fbp", n_fbp)
    assert n_multi is not None and n_fbp is not None and n_multi < n_fbp


def test_binned_multires_matches_binned_context():
    import dataclasses
    c, y, w = held_out_ctx(sino=True)
    c.init_multires(40, binned=True)
    got = c.object()
    # the coarse problem built by hand: detector bins and rows binned 2 x 2
    wb = w.reshape(NP, N // 2, 2, NT // 2, 2).sum(axis=(2, 4))
    yb = (w * y).reshape(NP, N // 2, 2, NT // 2, 2).sum(axis=(2, 4)) / wb
    p = dataclasses.replace(tw.params(N, NT, NP), delta_xy=2.0, delta_z=2.0, sinobin=3)
    t, a = xtg.round_views(*xtg.views_uniform(NP))
    cb = xtg.Context(p, t, a)
    cb.set_options(a_mode=xtg.XTG_A_AUTO)
    assert cb.obj_shape == (1, NT // 2, N // 2, N // 2)
    cb.upload_sino(yb, wb)
    cb.init_fbp()
    for it in range(1, 41):
        cb.iteration(it)
    ok, err = close_images(got, c.upsample(cb.object()))
    assert ok, err
    # the binned start is a reconstruction: below the FBP start's cost
    c.init_error_sino()
    cost_bin = c.cost()[0]
    c.init_fbp()
    assert cost_bin < c.cost()[0]
    cb.close()
    c.close()


def test_counts_ingest_multires_bins_its_coarse_stage():
    import dataclasses
    c, y, w = held_out_ctx(sino=True)
    counts = np.maximum(w, 1.0).astype(np.float32)
    bright = np.full((N, NT), 1e4, np.float32)
    # the same measurement as projections and weights
    c.upload_sino(np.log(1e4 / counts.astype(np.float64)).astype(np.float32), counts)
    c.init_multires(40, binned=True)
    want = c.object()
    p = dataclasses.replace(tw.params(N, NT, NP), sinobin=3)
    t, a = xtg.round_views(*xtg.views_uniform(NP))
    c3 = xtg.Context(p, t, a)
    c3.set_options(a_mode=xtg.XTG_A_AUTO)
    c3.upload_counts(bright, counts)
    c3.init_multires(40)
    ok, err = close_images(c3.object(), want)
    assert ok, err
    c3.close()
    c.close()


def test_untrained_network_falls_back_to_multires_start():
    c = held_out_ctx()
    net = xtg.WarmNet(seed=2)
    used, cn, ci = c.init_learned(net, 20)
    # the zero head returns the start image itself: equal cost, so it is not used
    assert not used and cn == pytest.approx(ci, rel=1e-12)
    # the context holds the multi-resolution start with a fresh e
    assert c.cost_running()[0] == pytest.approx(ci, rel=1e-12)
    net.close()


def test_trained_network_lowers_start_cost():
    """What the network gains over the method without it: on a held-out
    phantom its start needs strictly fewer fine iterations than the
    multi-resolution start it refines to reach MAP cost <= (1 + 1e-4) of the
    converged cost (the benchmark's tolerance)."""
    data, shape = tw.make_set(16, N, NT, NP, coarse_iters=20, target_iters=40, seed=500, log=lambda *a: None)
    net, losses = tw.train(data, shape, steps=400, batch=8, patch=(32, 32, 16), log=lambda *a: None)
    assert losses[-50:].mean() < losses[:50].mean()
    target = converged() * (1 + 1e-4)
    c = held_out_ctx()
    used, cn, ci = c.init_learned(net, 20)
    assert used and cn < ci, (cn, ci)
    n_learned = iters_to(c, 1, target)
    c = held_out_ctx()
    c.init_multires(20)
    n_multi = iters_to(c, 1, target)
    print("iterations to 1e-4: learned", n_learned, "multires", n_multi, "start costs", cn, ci)
    assert n_learned is not None and n_multi is not None and n_learned < n_multi
    net.close()
