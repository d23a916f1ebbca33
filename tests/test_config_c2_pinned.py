"""The at-scale configuration's options, pinned to the reference's own FP64
converged cost.

Reduced size (tests/golden/config_c2_small.npz, made by the reference's
-DREAL_IS_DOUBLE build from its zero start until its cost stalled: 16 slices
of 128^2, 128 bins x 16 rows, 512 views, 30 ellipsoids, 1e4 photons/ray,
0.5 % zingers, generalized-Huber zinger correction T = 4, delta = 0.5, NHICD
on).  The reference's cost per iteration is stored; the last is its
converged cost C*, reached within 1e-4 at iteration 19.  For each start
(zero, FBP, multi-resolution, learned + FP16-A) and A storage the parallel
schedule runs until its own FP64 cost is within 1e-4 of C*; then the MAP
cost of its object is evaluated on the host

  * by the oracle with the GPU's arithmetic (the float build's A and
    constants, FP64 sums): equal to xtg_map_cost_fp64 to 1e-9 relative;
  * by the oracle's double build, i.e. the reference's REAL_IS_DOUBLE cost of
    that object: at most (1 + 1e-4) C*.

Iterations: from zero at most twice the reference's, from a warm start no
more than the reference's.  RMSE against the reference's converged object is
stated (zinger correction makes the data term non-convex; 5 % of its maximum
bounds it).

Full size (512^2 x 64, 1024 views, the benchmark's workload): after the FBP
start and 8 iterations the host oracle re-evaluates the MAP cost of the
GPU's object (1e-9 with the GPU's arithmetic, 2e-4 against the double build,
whose detector response differs in the FP32 build's rounding).
"""
import os

import numpy as np
import pytest

import common
import xtg
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(common.ROOT, "timbir-python_b200", "weights", "warmstart_plain3d.bin")
TOL = 1e-4


def c2s_case():
    g = dict(np.load(os.path.join(common.GOLDEN, "config_c2_small.npz")))
    p = common.params(N=128, NT=16, NP=512, zinger=True, nhicd=True, threads=8)
    t, a = g["times"], g["angles"]
    x, ax, y, w = common.data(p, t, a, seed=7, n_ell=30, mu=0.01, I0=1e4, zfrac=0.005)
    # the seeded generator reproduces the reference's inputs
    assert y.astype(np.float64).sum() == pytest.approx(float(g["y_sum"]), rel=1e-12)
    assert w.astype(np.float64).sum() == pytest.approx(float(g["w_sum"]), rel=1e-12)
    return g, p, t, a, y, w


def host_costs(p, t, a, y, w, x):
    """(GPU arithmetic, reference FP64 build) MAP costs of x on the host."""
    out = []
    for double in (False, True):
        o = Oracle(p, t, a, double=double)
        o.set_sino(y, w)
        o.set_object(x)
        out.append(o.map_cost_fp64()[0])
        o.close()
    return out


@pytest.mark.parametrize("start,amode", [("zero", xtg.XTG_A_TABLE32), ("zero", xtg.XTG_A_FP16),
                                         ("fbp", xtg.XTG_A_TABLE32), ("multires", xtg.XTG_A_TABLE32),
                                         ("learned", xtg.XTG_A_FP16)])
def test_reaches_reference_converged_cost(start, amode):
    g, p, t, a, y, w = c2s_case()
    c_star = float(g["costs64"][-1])
    ref_iters = int(np.argmax(g["costs64"] <= c_star * (1 + TOL)))
    c = xtg.Context(p, t, a)
    c.set_options(a_mode=amode)
    c.upload_sino(y, w)
    net = None
    if start == "zero":
        c.init_error_sino()
    elif start == "fbp":
        c.init_fbp()
    elif start == "multires":
        c.init_multires(20)
    else:
        net = xtg.WarmNet()
        net.load(WEIGHTS)
        c.init_learned(net, 20)
    limit = 2 * ref_iters if start == "zero" else ref_iters
    costs = []
    for it in range(1, limit + 1):
        c.iteration(it)
        costs.append(c.resync_fp64()[0])
        if costs[-1] <= c_star * (1 + TOL):
            break
    x = c.object()
    gpu_cost = c.cost()[0]
    mine, ref64 = host_costs(p, t, a, y, w, x)
    rmse = float(np.sqrt(np.mean((x - g["x_star"]) ** 2))) / float(np.abs(g["x_star"]).max())
    print(f"{start}: {len(costs)} iterations (reference {ref_iters}), GPU cost {gpu_cost!r}, reference FP64 "
          f"cost of the GPU object {ref64!r} = C* (1 + {ref64 / c_star - 1:.2e}), RMSE {rmse:.2e} of max")
    assert gpu_cost == pytest.approx(mine, rel=1e-9)
    assert ref64 <= c_star * (1 + TOL)
    assert rmse < 5e-2
    c.close()
    if net is not None:
        net.close()


def test_full_size_cost_matches_host_oracle():
    """The benchmark's workload: the GPU's FP64 MAP cost of its object equals
    the host oracle's evaluation of the same object."""
    N, NT, NP = 512, 64, 1024
    p = common.params(N=N, NT=NT, NP=NP, zinger=True, nhicd=True)
    t, a = common.views(p)
    x_true = xtg.phantom((1, NT, N, N), 30, 0.01, 2)
    c = xtg.Context(p, t, a)
    c.set_options(a_mode=xtg.XTG_A_TABLE32)
    c.upload_object(x_true)
    y, w = xtg.measure(c.forward_project(), 1e4, 102, zinger_frac=0.005)
    c.upload_sino(y, w)
    c.init_fbp()
    for it in range(1, 9):
        c.iteration(it)
    x = c.object()
    gpu = c.cost()[0]
    mine, ref64 = host_costs(p, t, a, y, w, x)
    print(f"GPU {gpu!r}, oracle (GPU arithmetic) {mine!r}, reference FP64 build {ref64!r}")
    assert gpu == pytest.approx(mine, rel=1e-9)
    assert gpu == pytest.approx(ref64, rel=2e-4)
    c.close()
