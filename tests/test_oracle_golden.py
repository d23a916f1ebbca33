"""The CPU oracle restatement (oracle/xt_oracle.c) against the golden fixtures
made by running the reference engine itself (tests/golden/make_golden.py).

Float32 results are compared bit for bit: the restatement keeps the
reference's evaluation order and float/double promotions.
"""
import os

import numpy as np
import pytest

import common
from oracle.oracle import Oracle

CASES = {
    "plain3d": (dict(N=32, NT=4, NP=36), None),
    "zinger_nhicd": (dict(N=24, NT=4, NP=30, zinger=True, nhicd=True, offset=2, var=1), None),
    "offset_zero_mean": (dict(N=20, NT=2, NP=24, offset=2, zero_mean=1, zinger=True), None),
    "timbir4d": (dict(N=16, NT=2, NP=48, n_time=3), (4, 16)),
    "blocks_z": (dict(N=16, NT=8, NP=20, threads=4, nhicd=True), None),
    "coarse_xy2": (dict(N=32, NT=4, NP=30, dxy=2.0, dz=2.0), None),
    "launcher_geom": (dict(N=32, NT=4, NP=36, pitch=0.65, positivity=0, zinger=True, nhicd=True, offset=2), None),
}


def same_cost(got, want, threads):
    """Bit-exact for one thread; the reference's OpenMP reduction
    (XT_ICD_update.c:188, :206) sums in thread order otherwise."""
    got, want = np.array(got, np.float32), np.asarray(want).astype(np.float32)
    if threads == 1:
        return np.array_equal(got, want)
    return np.allclose(got, want, rtol=1e-5, atol=1e-3)


def load(name):
    return dict(np.load(os.path.join(common.GOLDEN, name + ".npz")))


def oracle_for(name, double=False):
    pk, _ = CASES[name]
    g = load(name + ("_fp64" if double else ""))
    p = common.params(**pk)
    return Oracle(p, g["times"], g["angles"], double=double), g


@pytest.mark.parametrize("name", sorted(CASES))
def test_setup_tables(name):
    o, g = oracle_for(name)
    assert np.array_equal(o.derived(), g["derived"])
    assert np.array_equal(o.hr(), g["hr"])
    v, cs, sn, pn, pi = o.views()
    for a, b in ((v, "view_rad"), (cs, "cosv"), (sn, "sinv"), (pn, "proj_num"), (pi, "proj_idx")):
        assert np.array_equal(a, g[b]), b


@pytest.mark.parametrize("name", sorted(CASES))
def test_amatrix(name):
    o, g = oracle_for(name)
    for q, (row, col, view) in enumerate(g["a_trip"]):
        vals, idx = o.amatrix(int(row), int(col), int(view))
        n = int((g["a_idx"][q] >= 0).sum())
        assert len(vals) == n
        assert np.array_equal(vals, g["a_vals"][q, :n]) and np.array_equal(idx, g["a_idx"][q, :n])


@pytest.mark.parametrize("name", sorted(CASES))
def test_forward_and_cost(name):
    o, g = oracle_for(name)
    o.set_sino(g["y"], g["w"])
    o.set_object(g["x_true"])
    assert np.array_equal(o.forward_project(), g["ax"])
    o.init_error_sino()
    assert np.array_equal(o.error_sino(), g["e_true"])
    assert same_cost(o.cost(), g["cost_true"], CASES[name][0].get("threads", 1))


@pytest.mark.parametrize("name", sorted(CASES))
def test_iterations(name):
    o, g = oracle_for(name)
    o.set_sino(g["y"], g["w"])
    o.init_error_sino()
    th = CASES[name][0].get("threads", 1)
    assert same_cost(o.cost(), g["cost_0"], th)
    o.srandom2(761521)
    for it in range(len(g["objs"])):
        o.iterate(it + 1)
        assert np.array_equal(o.object(), g["objs"][it]), f"object after iteration {it + 1}"
        assert same_cost(o.cost(), g["costs"][it], th)
        assert np.array_equal(o.offset(), g["offsets"][it])
        assert np.float32(o.var()) == np.float32(g["vars"][it])
        assert np.array_equal(o.magmap(), g["magmaps"][it])
    assert np.array_equal(o.error_sino(), g["e_final"])


def test_iterations_fp64():
    o, g = oracle_for("plain3d", double=True)
    o.set_sino(g["y"], g["w"])
    o.init_error_sino()
    o.srandom2(761521)
    for it in range(len(g["objs"])):
        o.iterate(it + 1)
        assert np.array_equal(o.object(), g["objs"][it])
        assert np.array_equal(np.array(o.cost()), g["costs"][it])


def test_rng_known_answers():
    """Park-Miller KAT printed in the reference source (randlib.c:69-91)."""
    o, _ = oracle_for("plain3d")
    o.srandom2(1)
    got = [round(o.random2() * 2147483647) for _ in range(20)]
    assert got == load("rng_kat")["table"].tolist()


def test_nhicd_selection():
    g = load("nhicd_select")
    p = common.params(N=32, NT=8, NP=12, threads=2)
    t, a = common.views(p)
    o = Oracle(p, t, a)
    o.set_magmap(g["map"])
    o.srandom2(99)
    nn, xs, ys = o.nhicd_select(g["usn"])
    assert np.array_equal(nn, g["nn"])
    for s in range(len(nn)):
        assert np.array_equal(xs[s, :nn[s]], g["xs"][s, :nn[s]])
        assert np.array_equal(ys[s, :nn[s]], g["ys"][s, :nn[s]])


def test_upsampling():
    g = load("upsample")
    o, _ = oracle_for("plain3d")
    assert np.array_equal(o.upsample_xy(g["inp"]), g["xy"])
    assert np.array_equal(o.upsample_xyz(g["inp"]), g["xyz"])
