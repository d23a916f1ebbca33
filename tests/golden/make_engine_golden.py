"""Generates the XT_Engine command-line fixtures in tests/golden from the
reference engine binary itself.

Each case writes the launcher's input files (view_info.txt, projection /
weight or bright / counts, and for the multi-resolution stage the coarser
object, magnitude-update map, offset and variance), runs the reference
XT_Engine (gromitsun/timbir-python Source_Code_4D_Fast, built by
`make -C oracle` as oracle/_ref/XT_Engine_ref32, or XT_Engine_ref32_nopos for a
case with positivity off) with the launcher's options
in a scratch directory, and stores every input and output file byte for byte
together with the argument list:

    python tests/golden/make_engine_golden.py [NAME ...]   # needs oracle/_ref (this container)

tests/test_engine_cli.py replays the same command against this engine's
bin/XT_Engine and compares the output files.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "timbir-python_b200"), os.path.join(ROOT, "tests")]

import common  # noqa: E402
import xtg  # noqa: E402

REF_ENGINE = os.path.join(ROOT, "oracle", "_ref", "XT_Engine_ref32")


def plain_case():
    """sinobin 1, zinger correction, NHICD, offset and variance estimation, 3 iterations."""
    p = common.params(N=32, NT=4, NP=36, zinger=True, nhicd=True, offset=2, var=1)
    t, a = common.views(p)
    x, ax, y, w = common.data(p, t, a, seed=7, zfrac=0.01)
    files = {"projection_n0.bin": y.tobytes(), "weight_n0.bin": w.tobytes()}
    return p, t, a, files


def counts_multires_case():
    """sinobin 3 (bright + counts summed over 2x1 detector blocks), initICD 2
    (bilinear 2x in x-y from the coarser stage), --initMagUpMap, offset read
    from the coarser stage and re-estimated (updateProjOffset 3), 2 iterations."""
    p = common.params(N=32, NT=4, NP=30, dxy=2.0, nhicd=True, offset=3, var=1)
    p.sinobin, p.initICD, p.initMagUpMap, p.iter = 3, 2, 1, 2
    t, a = common.views(p)
    fine = common.params(N=32, NT=4, NP=30, dxy=2.0)
    x, ax, _, counts = common.data(fine, t, a, seed=9, I0=3e4)
    rng = np.random.default_rng(9)
    bright = (3e4 * (1.0 + 0.02 * rng.standard_normal((32, 4)))).astype(np.float32)
    # coarse stage (voxels 4 detector bins wide): 8 x 8 x 4 object, one frame
    coarse = np.maximum(x[0, :, ::2, ::2] + 0.001 * rng.standard_normal((4, 8, 8)), 0).astype(np.float32)
    magmap = rng.random((1, 2, 8, 8)).astype(np.float32)
    offset = (0.01 * rng.standard_normal((8, 4))).astype(np.float32)
    files = {"bright_n0.bin": bright.tobytes(), "weight_n0.bin": counts.tobytes(),
             "object_n0_time_0.bin": coarse.tobytes(), "mag_update_map_n0.bin": magmap.tobytes(),
             "proj_offset_n0.bin": offset.tobytes(), "variance_estimate_n0.bin": np.float32(1.3).tobytes()}
    return p, t, a, files


def launcher_case():
    """The launcher's geometry: physical lengths (length_r = 0.65 N_r,
    length_t = 0.65 N_t, so delta_t != 1: quirk of XT_VoxUpdate.c:27,67 against
    XT_ForwardProject.c:17), positivity off (the launcher's compile line,
    4D_Recon_Launcher_for_Real_Data/XT_Initialize.py:257: the reference
    binary built without POSITIVITY_CONSTRAINT), zinger correction, NHICD,
    offset and variance estimation, 3 iterations."""
    p = common.params(N=32, NT=4, NP=36, pitch=0.65, positivity=0, zinger=True, nhicd=True, offset=2, var=1)
    t, a = common.views(p)
    x, ax, y, w = common.data(p, t, a, seed=12, zfrac=0.01)
    files = {"projection_n0.bin": y.tobytes(), "weight_n0.bin": w.tobytes()}
    return p, t, a, files


CASES = {"engine_plain": plain_case, "engine_counts_multires": counts_multires_case, "engine_launcher": launcher_case}


def run(name):
    p, t, a, files = CASES[name]()
    args = p.cli()
    with tempfile.TemporaryDirectory() as d:
        xtg.write_view_file(os.path.join(d, "view_info.txt"), t, a)
        for f, b in files.items():
            with open(os.path.join(d, f), "wb") as fh:
                fh.write(b)
        before = set(os.listdir(d))
        ins = {f: open(os.path.join(d, f), "rb").read() for f in sorted(before)}
        engine = REF_ENGINE if p.positivity else REF_ENGINE + "_nopos"
        r = subprocess.run([engine] + args, cwd=d, capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        outs = {f: open(os.path.join(d, f), "rb").read() for f in sorted(os.listdir(d))
                if f.endswith(".bin") and (f not in before or open(os.path.join(d, f), "rb").read() != ins.get(f))}
    rec = {"args": np.array(args), "positivity": np.int32(p.positivity)}
    for f, b in ins.items():
        rec["in:" + f] = np.frombuffer(b, np.uint8)
    for f, b in outs.items():
        rec["out:" + f] = np.frombuffer(b, np.uint8)
    return rec


def main():
    if not os.path.exists(REF_ENGINE):
        sys.exit("oracle/_ref is not built (make -C oracle needs the reference tree)")
    for name in sys.argv[1:] or CASES:
        rec = run(name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
        print("wrote", name, sorted(k for k in rec if k.startswith("out:")))


if __name__ == "__main__":
    main()
