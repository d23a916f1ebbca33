"""Generates the golden fixtures in tests/golden from the reference itself.

Runs the reference engine's own routines (gromitsun/timbir-python
Source_Code_4D_Fast, compiled by `make -C oracle` into oracle/_ref) on small
seeded cases and stores inputs and outputs as .npz files.  The CPU tests pin
the oracle restatement (oracle/xt_oracle.c) against these files, so the pin
holds on machines without the reference tree.

    python tests/golden/make_golden.py      # needs oracle/_ref (this container)
    python tests/golden/make_golden.py NAME # one case of CASES
    python tests/golden/make_golden.py config_c1 | config_c2_small
                                            # the long converged runs

The RNG known-answer table is read from the reference source's own comment
(Source_Code_4D_Fast/randlib.c:69-91) and checked against the compiled
generator before it is stored.
"""
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "timbir-python_b200"), os.path.join(ROOT, "tests")]

import common  # noqa: E402
import xtg  # noqa: E402
from oracle.oracle import Reference, ref_available  # noqa: E402

# the reference tree (read-only); TIMBIR_REFERENCE overrides its location
REF_TREE = os.environ.get("TIMBIR_REFERENCE", "/root/reference")
REF_SRC = os.path.join(REF_TREE, "Source_Code_4D_Fast", "randlib.c")

CASES = {
    # name: (params kwargs, view kind, data kwargs, iterations)
    "plain3d": (dict(N=32, NT=4, NP=36), None, dict(seed=1), 3),
    "zinger_nhicd": (dict(N=24, NT=4, NP=30, zinger=True, nhicd=True, offset=2, var=1), None,
                     dict(seed=2, zfrac=0.01), 4),
    "offset_zero_mean": (dict(N=20, NT=2, NP=24, offset=2, zero_mean=1, zinger=True), None,
                         dict(seed=6, zfrac=0.02), 2),
    "timbir4d": (dict(N=16, NT=2, NP=48, n_time=3), (4, 16), dict(seed=3, moving=2), 3),
    "blocks_z": (dict(N=16, NT=8, NP=20, threads=4, nhicd=True), None, dict(seed=4), 3),
    "coarse_xy2": (dict(N=32, NT=4, NP=30, dxy=2.0, dz=2.0), None, dict(seed=5), 2),
    # the launcher's geometry: physical lengths (delta_r = delta_t = 0.65),
    # positivity off, zinger correction, NHICD and offset re-estimation
    "launcher_geom": (dict(N=32, NT=4, NP=36, pitch=0.65, positivity=0, zinger=True, nhicd=True, offset=2), None,
                      dict(seed=8, zfrac=0.01), 3),
}


def run_case(name, pk, vk, dk, iters, double=False):
    p = common.params(**pk)
    with tempfile.TemporaryDirectory() as d:
        cwd = os.getcwd()
        os.chdir(d)
        try:
            t, a = common.views(p, vk)
            xtg.write_view_file("view_info.txt", t, a)
            x, ax, y, w = common.data(p, t, a, **dk)
            r = Reference(p, double=double)
            out = dict(times=t, angles=a, y=y, w=w, x_true=x, ax=ax)
            out["derived"] = r.derived()
            out["hr"] = r.hr()
            v, cs, sn, pn, pi = r.views()
            out.update(view_rad=v, cosv=cs, sinv=sn, proj_num=pn, proj_idx=pi)
            rng = np.random.default_rng(11)
            trip = np.stack([rng.integers(0, r.N_y, 400), rng.integers(0, r.N_x, 400),
                             rng.integers(0, r.N_p, 400)], 1).astype(np.int32)
            av = np.zeros((400, 16), r.real)
            ai = np.full((400, 16), -1, np.int32)
            for q, (row, col, view) in enumerate(trip):
                vals, idx = r.amatrix(int(row), int(col), int(view))
                av[q, :len(vals)] = vals
                ai[q, :len(idx)] = idx
            out.update(a_trip=trip, a_vals=av, a_idx=ai)
            r.set_sino(y, w)
            r.set_object(x)
            r.init_error_sino()
            out["e_true"] = r.error_sino()
            out["cost_true"] = np.array(r.cost())
            r.set_object(np.zeros(r.obj_shape, r.real))
            r.init_error_sino()
            out["cost_0"] = np.array(r.cost())
            r.srandom2(761521)
            objs, costs, offs, vars_, mags = [], [], [], [], []
            for it in range(1, iters + 1):
                r.iterate(it)
                objs.append(r.object())
                costs.append(r.cost())
                offs.append(r.offset())
                vars_.append(r.var())
                mags.append(r.magmap())
            out.update(objs=np.array(objs), costs=np.array(costs), offsets=np.array(offs), vars=np.array(vars_),
                       magmaps=np.array(mags), e_final=r.error_sino())
            r.close()
        finally:
            os.chdir(cwd)
    return out


def rng_kat():
    txt = open(REF_SRC).read()
    blk = txt[txt.index("TABLE:"):txt.index("Test for verifying")]
    table = np.array([int(s) for s in re.findall(r"^\s*(\d+)\s*$", blk, re.M)], np.int64)
    assert len(table) == 20, table
    p = common.params()
    with tempfile.TemporaryDirectory() as d:
        cwd = os.getcwd()
        os.chdir(d)
        try:
            xtg.write_view_file("view_info.txt", *common.views(p))
            r = Reference(p)
            r.srandom2(1)
            got = np.array([round(r.random2() * 2147483647) for _ in range(20)], np.int64)
            r.close()
        finally:
            os.chdir(cwd)
    assert np.array_equal(got, table), (got, table)
    return table


def nhicd_case():
    p = common.params(N=32, NT=8, NP=12, threads=2)
    with tempfile.TemporaryDirectory() as d:
        cwd = os.getcwd()
        os.chdir(d)
        try:
            xtg.write_view_file("view_info.txt", *common.views(p))
            r = Reference(p)
            rng = np.random.default_rng(5)
            m = rng.random((r.N_time, r.nzb, r.N_y, r.N_x)).astype(np.float32)
            m[m < 0.3] = 0.0
            m[:, :, 3, 4:9] = 0.75  # ties
            r.set_magmap(m)
            usn = np.full(r.N_time * r.nzb, 700, np.int32)
            r.srandom2(99)
            nn, xs, ys = r.nhicd_select(usn)
            r.close()
        finally:
            os.chdir(cwd)
    return dict(map=m, usn=usn, nn=nn, xs=xs, ys=ys)


def upsample_case():
    p = common.params()
    with tempfile.TemporaryDirectory() as d:
        cwd = os.getcwd()
        os.chdir(d)
        try:
            xtg.write_view_file("view_info.txt", *common.views(p))
            r = Reference(p)
            a = np.random.default_rng(3).random((3, 5, 6)).astype(np.float32)
            out = dict(inp=a, xy=r.upsample_xy(a), xyz=r.upsample_xyz(a))
            r.close()
        finally:
            os.chdir(cwd)
    return out


def config_c1():
    """The reference's CPU-runnable configuration: 4 slices of 128^2, 128 bins,
    180 views at i degrees, 10 ellipsoids, 2e4 photons/ray, no zinger
    correction, no NHICD.  The FP64 reference runs 150 iterations (its cost
    per iteration; the last is the converged cost C*), the FP32 reference the
    20 iterations the configuration names."""
    p = common.params(N=128, NT=4, NP=180, nhicd=False)
    with tempfile.TemporaryDirectory() as d:
        cwd = os.getcwd()
        os.chdir(d)
        try:
            t, a = common.views(p)
            xtg.write_view_file("view_info.txt", t, a)
            x, ax, y, w = common.data(p, t, a, seed=1, n_ell=10, I0=2e4)
            out = dict(times=t, angles=a, y_sum=np.float64(y.astype(np.float64).sum()),
                       w_sum=np.float64(w.astype(np.float64).sum()))
            for double, iters, key in ((True, 150, "costs64"), (False, 20, "costs32")):
                r = Reference(p, double=double)
                r.set_sino(y, w)
                r.init_error_sino()
                r.srandom2(761521)
                cs = [r.cost()[0]]
                for it in range(1, iters + 1):
                    r.iterate(it)
                    cs.append(r.cost()[0])
                out[key] = np.array(cs)
                if double:
                    out["x_star"] = r.object().astype(np.float32)
                r.close()
        finally:
            os.chdir(cwd)
    return out


def config_c2_small(max_iters=500, stall=1e-9):
    """The at-scale configuration's options at a size the CPU finishes: 16
    slices of 128^2, 128 bins x 16 rows, 512 views uniform over 180 degrees,
    30 ellipsoids, 1e4 photons/ray, 0.5 % of the sinogram entries turned into
    zingers (+U(2, 5)), generalized-Huber zinger correction on (T = 4,
    delta = 0.5), NHICD on, positivity on.  The FP64 reference runs from its
    own zero start until its cost stalls (decrease over 10 iterations below
    `stall` relative) or `max_iters`; its cost per iteration (the last is the
    converged cost C*) and its converged object are stored."""
    p = common.params(N=128, NT=16, NP=512, zinger=True, nhicd=True, threads=8)
    with tempfile.TemporaryDirectory() as d:
        cwd = os.getcwd()
        os.chdir(d)
        try:
            t, a = common.views(p)
            xtg.write_view_file("view_info.txt", t, a)
            x, ax, y, w = common.data(p, t, a, seed=7, n_ell=30, mu=0.01, I0=1e4, zfrac=0.005)
            out = dict(times=t, angles=a, y_sum=np.float64(y.astype(np.float64).sum()),
                       w_sum=np.float64(w.astype(np.float64).sum()))
            r = Reference(p, double=True)
            r.set_sino(y, w)
            r.init_error_sino()
            r.srandom2(761521)
            cs = [r.cost()[0]]
            for it in range(1, max_iters + 1):
                r.iterate(it)
                cs.append(r.cost()[0])
                print(f"config_c2_small iteration {it}: cost {cs[-1]!r}", flush=True)
                if it >= 30 and cs[-11] - cs[-1] < stall * abs(cs[-1]):
                    break
            out["costs64"] = np.array(cs)
            out["x_star"] = r.object().astype(np.float32)
            r.close()
        finally:
            os.chdir(cwd)
    return out


def main():
    if not ref_available():
        sys.exit("oracle/_ref is not built (make -C oracle needs the reference tree)")
    for name, (pk, vk, dk, iters) in CASES.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **run_case(name, pk, vk, dk, iters))
        print("wrote", name)
    o64 = run_case("plain3d", *CASES["plain3d"], double=True)
    np.savez_compressed(os.path.join(HERE, "plain3d_fp64.npz"), **o64)
    np.savez_compressed(os.path.join(HERE, "rng_kat.npz"), table=rng_kat())
    np.savez_compressed(os.path.join(HERE, "nhicd_select.npz"), **nhicd_case())
    np.savez_compressed(os.path.join(HERE, "upsample.npz"), **upsample_case())
    np.savez_compressed(os.path.join(HERE, "config_c1.npz"), **config_c1())
    print("done")


if __name__ == "__main__":
    if sys.argv[1:] == ["config_c1"]:
        np.savez_compressed(os.path.join(HERE, "config_c1.npz"), **config_c1())
    elif sys.argv[1:] == ["config_c2_small"]:
        np.savez_compressed(os.path.join(HERE, "config_c2_small.npz"), **config_c2_small())
    elif len(sys.argv) == 2 and sys.argv[1] in CASES:
        np.savez_compressed(os.path.join(HERE, f"{sys.argv[1]}.npz"), **run_case(sys.argv[1], *CASES[sys.argv[1]]))
    else:
        main()
