"""FP64 numpy restatement of the engine's FBP warm start, the checker for
xtg_init_object_fbp (test infrastructure only).

Parallel-beam FBP (Kak & Slaney, Principles of Computerized Tomographic
Imaging, ch. 3, eqs. 61-63) on the engine's geometry: ramp filter
h(0) = 1/(4 dr^2), h(odd m) = -1/(m^2 pi^2 dr^2) applied along the detector
bins of y - d (times dr), backprojection r = x cos(th) - y sin(th) with linear
interpolation between bin centres R0 + (i + 0.5) dr, weight pi / (views of the
frame), zovl detector rows averaged per slice, 0 outside the reconstruction
disk, clamped at 0 with positivity.  Returns [N_time][N_z][N_y][N_x].
"""
import numpy as np

import xtg


def fbp(p, times, angles, y, d=None):
    g, cs, sn, fov, _ = xtg.host_geometry(p, times, angles)
    N_r, N_t, N_x, N_y, N_z = g.N_r, g.N_t, g.N_x, g.N_y, g.N_z
    dr = float(g.delta_r)
    yd = y.astype(np.float64) - (0.0 if d is None else d.astype(np.float64)[None])
    m = np.arange(-(N_r - 1), N_r)
    h = np.zeros(m.size)
    h[m == 0] = 1.0 / (4 * dr * dr)
    odd = m % 2 != 0
    h[odd] = -1.0 / (m[odd].astype(np.float64) ** 2 * np.pi ** 2 * dr * dr)
    # q[p][r][t] = dr * sum_n h[r - n] yd[p][n][t]
    H = h[(np.arange(N_r)[:, None] - np.arange(N_r)[None, :]) + (N_r - 1)]
    q = dr * np.einsum("rn,pnt->prt", H, yd)
    xs = g.x0 + (np.arange(N_x) + 0.5) * g.delta_xy
    ys = g.y0 + (np.arange(N_y) + 0.5) * g.delta_xy
    X, Y = np.meshgrid(xs, ys)  # [N_y][N_x]
    mask = (X.astype(np.float32) ** 2 + Y.astype(np.float32) ** 2) < np.float32(g.radius_obj) ** 2
    out = np.zeros((g.N_time, N_z, N_y, N_x))
    for f in range(g.N_time):
        views = np.nonzero(fov == f)[0]
        acc = np.zeros((N_y, N_x, N_t))
        for pv in views:
            r = X * float(cs[pv]) - Y * float(sn[pv])
            u = (r - g.R0) / dr - 0.5
            i = np.floor(u).astype(int)
            fr = u - i
            for ii, wt in ((i, 1.0 - fr), (i + 1, fr)):
                ok = (ii >= 0) & (ii < N_r)
                acc[ok] += wt[ok, None] * q[pv, ii[ok], :]
        acc *= np.pi / len(views)
        sl = acc.reshape(N_y, N_x, N_z, g.zovl).mean(axis=3)  # [N_y][N_x][N_z]
        sl[~mask] = 0.0
        if p.positivity:
            sl = np.maximum(sl, 0.0)
        out[f] = np.transpose(sl, (2, 0, 1))
    return out
