"""ctypes front end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Two implementations with one Python API:

* ``Oracle``    -- the CPU restatement in xt_oracle.c (libxtoracle{32,64}.so);
* ``Reference`` -- the reference engine's own routines, compiled from
  gromitsun/timbir-python Source_Code_4D_Fast by oracle/Makefile into
  oracle/_ref/libxtref{32,64}.so and driven by ref_harness.c.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
``--impl reference`` legs may use this module, and only as the checker.

``params`` is any object with the XT_Engine option names as attributes
(the tests pass the product's ``xtg.Params``).  ``double=True`` selects the
FP64 build (the reference's -DREAL_IS_DOUBLE).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, n)) for n in
               ("libxtref32.so", "libxtref64.so", "XT_Engine_ref32", "XT_Engine_ref64"))


class XoParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "p", "sigma_s", "sigma_t", "c_s", "c_t", "mult_xy", "mult_z", "length_r", "length_t",
        "rot_center", "alpha", "Rtime0", "Rtime_delta", "zingerT", "zingerDel", "var_est",
        "voxel_thresh", "radius_obj")] + [(n, C.c_int32) for n in (
        "N_r", "N_t", "N_p", "N_time", "num_threads", "positivity", "no_nhicd",
        "update_proj_offset", "zero_mean_offset", "update_var")]


def xo_params(p):
    c = XoParams()
    c.p, c.sigma_s, c.sigma_t, c.c_s, c.c_t = p.p, p.sigma_s, p.sigma_t, p.c_s, p.c_t
    c.mult_xy, c.mult_z, c.length_r, c.length_t = p.delta_xy, p.delta_z, p.length_r, p.length_t
    c.rot_center, c.alpha, c.Rtime0, c.Rtime_delta = p.rotation_center, p.alpha, p.Rtime0, p.Rtime_delta
    c.zingerT, c.zingerDel, c.var_est = p.zingerT, p.zingerDel, p.Est_of_Var
    c.voxel_thresh, c.radius_obj = p.voxel_thresh, p.radius_obj
    c.N_r, c.N_t, c.N_p, c.N_time = p.N_r, p.N_t, p.num_projections, p.Rtime_num
    c.num_threads, c.positivity, c.no_nhicd = p.num_threads, p.positivity, p.no_NHICD
    c.update_proj_offset, c.zero_mean_offset, c.update_var = p.updateProjOffset, p.EnforceZeroMeanOffset, p.do_VarEst
    return c


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class _Base:
    prefix = ""

    def _setup(self, lib, double):
        self.lib = lib
        self.real = np.float64 if double else np.float32
        self.creal = C.c_double if double else C.c_float
        pre = self.prefix
        for name in ("cost", "functional_substitution", "randomized_select", "get_var"):
            getattr(lib, pre + name).restype = self.creal
        getattr(lib, pre + "functional_substitution").argtypes = [C.c_void_p, self.creal, self.creal, self.creal,
                                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        getattr(lib, pre + "randomized_select").argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32]
        getattr(lib, pre + "random2").restype = C.c_double
        getattr(lib, pre + "amatrix").argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
        for name in ("destroy", "dims", "derived", "get_hr", "set_sino", "set_object", "get_object",
                     "get_error_sino", "set_error_sino", "get_weight", "get_offset", "get_magmap", "set_magmap",
                     "init_error_sino", "cost", "iterate", "get_var", "update_offset", "update_variance",
                     "views", "random_lists", "nhicd_select"):
            getattr(lib, pre + name).argtypes = None
        d = np.zeros(9, np.int32)
        self._call("dims", C.c_void_p(self.h), d)
        (self.N_x, self.N_y, self.N_z, self.N_time, self.N_r, self.N_t, self.N_p,
         self.nzb, self.zovl) = (int(v) for v in d)

    def _call(self, name, *a):
        fn = getattr(self.lib, self.prefix + name)
        return fn(*[x if not isinstance(x, np.ndarray) else _ptr(x) for x in a])

    def close(self):
        if getattr(self, "h", None):
            self._call("destroy", C.c_void_p(self.h))
            self.h = None

    @property
    def sino_shape(self):
        return (self.N_p, self.N_r, self.N_t)

    @property
    def obj_shape(self):
        return (self.N_time, self.N_z, self.N_y, self.N_x)

    def _arr(self, shape):
        return np.zeros(shape, self.real)

    def derived(self):
        o = np.zeros(40, np.float64)
        self._call("derived", C.c_void_p(self.h), o)
        return o

    def views(self):
        v, cs, sn = self._arr(self.N_p), self._arr(self.N_p), self._arr(self.N_p)
        pn, pi = np.zeros(self.N_time, np.int32), np.zeros(self.N_p, np.int32)
        self._call("views", C.c_void_p(self.h), v, cs, sn, pn, pi)
        return v, cs, sn, pn, pi

    def hr(self):
        o = self._arr((self.N_p, 65))
        self._call("get_hr", C.c_void_p(self.h), o)
        return o

    def amatrix(self, row, col, view):
        v, i = self._arr(64), np.zeros(64, np.int32)
        n = getattr(self.lib, self.prefix + "amatrix")(C.c_void_p(self.h), row, col, view, _ptr(v), _ptr(i))
        return v[:n].copy(), i[:n].copy()

    def set_sino(self, y, w, d=None):
        y = np.ascontiguousarray(y, self.real)
        w = np.ascontiguousarray(w, self.real)
        d = None if d is None else np.ascontiguousarray(d, self.real)
        self._call("set_sino", C.c_void_p(self.h), y, w, d)

    def set_object(self, x):
        self._call("set_object", C.c_void_p(self.h), np.ascontiguousarray(x, self.real))

    def object(self):
        o = self._arr(self.obj_shape)
        self._call("get_object", C.c_void_p(self.h), o)
        return o

    def error_sino(self):
        o = self._arr(self.sino_shape)
        self._call("get_error_sino", C.c_void_p(self.h), o)
        return o

    def set_error_sino(self, e):
        self._call("set_error_sino", C.c_void_p(self.h), np.ascontiguousarray(e, self.real))

    def weight(self):
        o = self._arr(self.sino_shape)
        self._call("get_weight", C.c_void_p(self.h), o)
        return o

    def offset(self):
        o = self._arr((self.N_r, self.N_t))
        self._call("get_offset", C.c_void_p(self.h), o)
        return o

    def magmap(self):
        o = self._arr((self.N_time, self.nzb, self.N_y, self.N_x))
        self._call("get_magmap", C.c_void_p(self.h), o)
        return o

    def set_magmap(self, m):
        self._call("set_magmap", C.c_void_p(self.h), np.ascontiguousarray(m, self.real))

    def var(self):
        return float(getattr(self.lib, self.prefix + "get_var")(C.c_void_p(self.h)))

    def init_error_sino(self):
        self._call("init_error_sino", C.c_void_p(self.h))

    def cost(self):
        f, p = self.creal(), self.creal()
        c = getattr(self.lib, self.prefix + "cost")(C.c_void_p(self.h), C.byref(f), C.byref(p))
        return float(c), float(f.value), float(p.value)

    def update_offset(self):
        self._call("update_offset", C.c_void_p(self.h))

    def update_variance(self):
        self._call("update_variance", C.c_void_p(self.h))

    def functional_substitution(self, V, th1, th2, nh, tnh, fl, tfl):
        nh = np.ascontiguousarray(nh, self.real)
        tnh = np.ascontiguousarray(tnh, self.real)
        fl = np.ascontiguousarray(fl, np.uint8)
        tfl = np.ascontiguousarray(tfl, np.uint8)
        return float(getattr(self.lib, self.prefix + "functional_substitution")(
            C.c_void_p(self.h), V, th1, th2, _ptr(nh), _ptr(tnh), _ptr(fl), _ptr(tfl)))

    def random_lists(self):
        nseg, nxy = self.N_time * self.nzb, self.N_x * self.N_y
        usn = np.zeros(nseg, np.int32)
        xs, ys = np.zeros((nseg, nxy), np.int32), np.zeros((nseg, nxy), np.int32)
        self._call("random_lists", C.c_void_p(self.h), usn, xs, ys)
        return usn, xs, ys

    def nhicd_select(self, usn):
        nseg, nxy = self.N_time * self.nzb, self.N_x * self.N_y
        usn = np.ascontiguousarray(usn, np.int32)
        nn = np.zeros(nseg, np.int32)
        xs, ys = np.zeros((nseg, nxy), np.int32), np.zeros((nseg, nxy), np.int32)
        self._call("nhicd_select", C.c_void_p(self.h), usn, nn, xs, ys)
        return nn, xs, ys

    def srandom2(self, s):
        getattr(self.lib, self.prefix + "srandom2")(C.c_uint32(s))

    def random2(self):
        return float(getattr(self.lib, self.prefix + "random2")())

    def randomized_select(self, a, i):
        a = np.ascontiguousarray(a, self.real).copy()
        return float(getattr(self.lib, self.prefix + "randomized_select")(_ptr(a), 0, len(a) - 1, i))


_libs = {}


def _lib(path):
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        _libs[path] = C.CDLL(path)
    return _libs[path]


class Oracle(_Base):
    """CPU restatement (xt_oracle.c)."""

    prefix = "xo_"

    def __init__(self, params, times, angles_deg, double=False):
        lib = _lib(os.path.join(HERE, "libxtoracle64.so" if double else "libxtoracle32.so"))
        lib.xo_create.restype = C.c_void_p
        lib.xo_create.argtypes = [C.POINTER(XoParams), C.c_void_p, C.c_void_p]
        self._p = xo_params(params)
        t = np.ascontiguousarray(times, np.float64)
        a = np.ascontiguousarray(angles_deg, np.float64)
        self.h = lib.xo_create(C.byref(self._p), _ptr(t), _ptr(a))
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        self._setup(lib, double)

    def forward_project(self):
        o = self._arr(self.sino_shape)
        self._call("forward_project", C.c_void_p(self.h), o)
        return o

    def map_cost_fp64(self):
        """MAP cost of the object, every sum in FP64 (this build's A and
        constants): (cost, forward, prior)."""
        fn = self.lib.xo_map_cost_fp64
        fn.restype = C.c_double
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        f, p = C.c_double(), C.c_double()
        c = fn(C.c_void_p(self.h), C.byref(f), C.byref(p))
        return float(c), float(f.value), float(p.value)

    def set_slab(self, below, above):
        """This oracle is one z slab of a volume split over ranks."""
        self.lib.xo_set_slab.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
        self.lib.xo_set_slab(C.c_void_p(self.h), int(below), int(above))

    def boundary(self):
        """(bottom slice, top slice), each [N_time][N_y][N_x]."""
        lo, hi = self._arr((self.N_time, self.N_y, self.N_x)), self._arr((self.N_time, self.N_y, self.N_x))
        self.lib.xo_get_boundary.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.xo_get_boundary(C.c_void_p(self.h), _ptr(lo), _ptr(hi))
        return lo, hi

    def set_halo(self, lo, hi):
        lo = None if lo is None else np.ascontiguousarray(lo, self.real)
        hi = None if hi is None else np.ascontiguousarray(hi, self.real)
        self.lib.xo_set_halo.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.xo_set_halo(C.c_void_p(self.h), _ptr(lo), _ptr(hi))

    def init_error_sino_model(self):
        """e = y - delta_t A x - d (the voxel update's matrix)."""
        self.lib.xo_init_error_sino_model.argtypes = None
        self._call("init_error_sino_model", C.c_void_p(self.h))

    def iterate(self, it):
        pct = self.creal()
        f = self.lib.xo_iterate(C.c_void_p(self.h), it, C.byref(pct))
        return int(f), float(pct.value)

    def vsc_filter(self, m):
        m = np.ascontiguousarray(m, self.real)
        o = np.zeros_like(m)
        self.lib.xo_vsc_filter(C.c_void_p(self.h), _ptr(m), _ptr(o))
        return o

    def upsample_xy(self, a):
        a = np.ascontiguousarray(a, self.real)
        nz, ny, nx = a.shape
        o = np.zeros((nz, 2 * ny, 2 * nx), self.real)
        self.lib.xo_upsample_xy(_ptr(a), _ptr(o), nz, ny, nx)
        return o

    def upsample_xyz(self, a):
        a = np.ascontiguousarray(a, self.real)
        nz, ny, nx = a.shape
        o = np.zeros((2 * nz, 2 * ny, 2 * nx), self.real)
        self.lib.xo_upsample_xyz(_ptr(a), _ptr(o), nz, ny, nx)
        return o


class Reference(_Base):
    """The reference engine's own routines (oracle/_ref).  Needs view_info.txt
    in the working directory, like the reference program."""

    prefix = "xr_"

    def __init__(self, params, double=False):
        if getattr(params, "positivity", 1):
            name = "libxtref64.so" if double else "libxtref32.so"
        elif not double:
            name = "libxtref32_nopos.so"  # the reference built without POSITIVITY_CONSTRAINT
        else:
            raise ValueError("no FP64 reference build without positivity")
        lib = _lib(os.path.join(REF_DIR, name))
        lib.xr_create.restype = C.c_void_p
        argv = ["XT_Engine"] + params.cli()
        self._argv = (C.c_char_p * len(argv))(*[s.encode() for s in argv])
        self.h = lib.xr_create(len(argv), self._argv)
        if not self.h:
            raise ValueError("reference set-up failed")
        self._setup(lib, double)

    def iterate(self, it):
        return int(self.lib.xr_iterate(C.c_void_p(self.h), it)), float("nan")

    def upsample_xy(self, a):
        a = np.ascontiguousarray(a, self.real)
        nz, ny, nx = a.shape
        o = np.zeros((nz, 2 * ny, 2 * nx), self.real)
        self.lib.xr_upsample_xy(_ptr(a), _ptr(o), nz, ny, nx)
        return o

    def upsample_xyz(self, a):
        a = np.ascontiguousarray(a, self.real)
        nz, ny, nx = a.shape
        o = np.zeros((2 * nz, 2 * ny, 2 * nx), self.real)
        self.lib.xr_upsample_xyz(_ptr(a), _ptr(o), nz, ny, nx)
        return o
