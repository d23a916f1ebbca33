"""The oracle's FP64 MAP-cost evaluator (xo_map_cost_fp64), the checker the
GPU tests use for MAP costs of large objects, against the oracle's own
restatement of computeCost (XT_ICD_update.c:181-314).

  * double build: equal to computeCost on e = y - delta_t A x - d to 1e-12
    relative (the same terms, summed in another order);
  * float build (FP32 A entries and constants, FP64 sums -- the GPU's
    arithmetic): within 2e-5 of the float build's own computeCost (FP32
    sums), and within 2e-4 of the double build.  The two builds are slightly
    different problems: the float build sums the detector response H_r
    (XT_Profile.c:128-171) in FP32, so its A entries differ from the double
    build's by up to ~3e-4 relative in the response's tails, and a residual
    at noise level turns that into ~1e-5 to 1e-4 of the data term.
"""
import numpy as np
import pytest

import common
import xtg
from oracle.oracle import Oracle


@pytest.mark.parametrize("pk,interlaced", [
    (dict(N=32, NT=4, NP=36, zinger=True, nhicd=True), None),
    (dict(N=24, NT=4, NP=30, pitch=0.65, positivity=0, zinger=True), None),
    (dict(N=16, NT=2, NP=48, n_time=3), (4, 16)),
    (dict(N=32, NT=4, NP=30, dxy=2.0, dz=2.0), None),
])
def test_map_cost_fp64_matches_compute_cost(pk, interlaced):
    p = common.params(**pk)
    t, a = common.views(p, interlaced)
    x, _, y, w = common.data(p, t, a, seed=21, zfrac=0.01 if pk.get("zinger") else 0.0,
                             moving=2 if interlaced else 0)
    xr = np.maximum(x + 0.002 * np.random.default_rng(2).standard_normal(x.shape), 0).astype(np.float32)
    o64 = Oracle(p, t, a, double=True)
    o64.set_sino(y, w)
    o64.set_object(xr)
    o64.init_error_sino_model()
    want = o64.cost()
    got = o64.map_cost_fp64()
    for g_, w_ in zip(got, want):
        assert g_ == pytest.approx(w_, rel=1e-12, abs=1e-9)
    o32 = Oracle(p, t, a)
    o32.set_sino(y, w)
    o32.set_object(xr)
    got32 = o32.map_cost_fp64()
    o32.init_error_sino_model()
    assert got32[0] == pytest.approx(o32.cost()[0], rel=2e-5)
    assert got32[0] == pytest.approx(want[0], rel=2e-4)
    o64.close()
    o32.close()
