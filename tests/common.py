"""Shared test cases: small geometries in the XT_Engine parameterisation."""
import os

import numpy as np

import xtg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def params(N=32, NT=4, NP=36, n_time=1, dxy=1.0, dz=1.0, zinger=False, nhicd=False, threads=1, rot=None,
           positivity=1, sigma=200000.0, c=0.01, alpha=1.0, offset=0, var=0, zero_mean=0, rtime_delta=None, pitch=1.0):
    """pitch: detector pitch in length units (length_r = pitch N_r, length_t =
    pitch N_t); the launcher passes physical lengths, so its delta_r and
    delta_t differ from 1."""
    return xtg.Params(
        p=1.2, sigma_s=sigma, sigma_t=sigma, c_s=c, c_t=c, delta_xy=dxy, delta_z=dz, length_r=pitch * float(N),
        length_t=pitch * float(NT), rotation_center=float(N) / 2 if rot is None else rot, alpha=alpha, Rtime0=0.0,
        Rtime_delta=float(NP // n_time) if rtime_delta is None else rtime_delta, radius_obj=float(N),
        zingerT=4.0 if zinger else 100000.0, zingerDel=0.5 if zinger else 0.0, iter=3,
        Rtime_num=n_time, num_projections=NP, N_r=N, N_t=NT, num_threads=threads, positivity=positivity,
        no_NHICD=0 if nhicd else 1, updateProjOffset=offset, do_VarEst=var, EnforceZeroMeanOffset=zero_mean)


def views(p, interlaced=None):
    if interlaced:
        K, N_theta = interlaced
        t, a = xtg.views_interlaced(K, N_theta, p.num_projections)
    else:
        t, a = xtg.views_uniform(p.num_projections)
    return xtg.round_views(t, a)


def data(p, t, a, seed=1, n_ell=6, mu=0.01, I0=2e4, zfrac=0.0, moving=0):
    """Phantom at the finest grid of p, its sinogram with Poisson noise."""
    N_x = int(p.N_r / p.delta_xy)
    N_z = int(p.N_t / p.delta_z)
    x = xtg.phantom((p.Rtime_num, N_z, N_x, N_x), n_ell, mu, seed, n_moving=moving, max_shift=1.0 if moving else 0.0,
                    growing=1 if moving else 0)
    ax = xtg.forward_cpu(p, t, a, x)
    y, w = xtg.measure(ax, I0, seed + 100, zinger_frac=zfrac)
    return x, ax, y, w
