"""The reference's CPU-runnable configuration end to end on the GPU: 4 slices
of 128^2, 128 bins, 180 views at i degrees, 10 ellipsoids, 2e4 photons/ray,
no zinger correction, no NHICD, 20 ICD equits (tests/golden/config_c1.npz
holds the reference's FP64 cost per iteration for 150 iterations, the last
being its converged cost C*, its FP32 costs for the 20 equits, and its
converged object).

Criteria (the reconstruction is measured by the reference's MAP cost):
  * after the configuration's 20 iterations the GPU's FP64 cost is within
    1e-4 of C* -- what the reference reaches at iteration 19;
  * the parallel schedule needs at most twice the reference's iterations to
    reach (1 + 1e-4) C*;
  * RMSE against the reference's converged object below 1 % of its maximum.
"""
import os

import numpy as np
import pytest

import common
import xtg

pytestmark = pytest.mark.gpu


def c1_case():
    g = dict(np.load(os.path.join(common.GOLDEN, "config_c1.npz")))
    p = common.params(N=128, NT=4, NP=180, nhicd=False)
    t, a = g["times"], g["angles"]
    x, ax, y, w = common.data(p, t, a, seed=1, n_ell=10, I0=2e4)
    # the seeded generator reproduces the reference's inputs
    assert y.astype(np.float64).sum() == pytest.approx(float(g["y_sum"]), rel=1e-12)
    assert w.astype(np.float64).sum() == pytest.approx(float(g["w_sum"]), rel=1e-12)
    return g, p, t, a, y, w


@pytest.mark.parametrize("amode", [xtg.XTG_A_TABLE32, xtg.XTG_A_FP16])
def test_config_c1_reaches_reference_converged_cost(amode):
    g, p, t, a, y, w = c1_case()
    c_star = float(g["costs64"][-1])
    ref_iters = int(np.argmax(g["costs64"] <= c_star * (1 + 1e-4)))
    c = xtg.Context(p, t, a)
    c.set_options(a_mode=amode)
    c.upload_sino(y, w)
    c.init_error_sino()
    costs = []
    for it in range(1, 2 * ref_iters + 1):
        c.iteration(it)
        costs.append(c.resync_fp64()[0])
    costs = np.array(costs)
    print("C*", c_star, "reference iterations", ref_iters, "GPU costs", costs[[0, 9, 19, -1]])
    assert costs[19] <= c_star * (1 + 1e-4)
    assert costs.min() <= c_star * (1 + 1e-4)
    x = c.object()
    xs = g["x_star"]
    rmse = float(np.sqrt(np.mean((x - xs) ** 2)))
    assert rmse / float(np.abs(xs).max()) < 1e-2
    c.close()
