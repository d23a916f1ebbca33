"""ctypes bindings of libxtgpu.so (include/xtg.h) and libxtgen.so (include/xt_gen.h).

The C ABI is the product boundary; this module only marshals numpy arrays
across it.  It never computes anything itself and it has no CPU fallback:
loading fails loudly when the shared libraries are missing, and
``Context`` raises when no sm_100 GPU is present.

Array layouts are the reference engine's (Source_Code_4D_Fast):
sinogram ``[N_p][N_r][N_t]``, offset ``[N_r][N_t]``, object
``[N_time][N_z][N_y][N_x]``, magnitude-update map ``[N_time][nzb][N_y][N_x]``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field, fields

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")

XTG_A_FP32, XTG_A_FP16, XTG_A_TABLE32, XTG_A_AUTO = 0, 1, 2, 3
XTG_ORDER_PARALLEL, XTG_ORDER_SEQUENTIAL = 0, 1
XTG_MULTIRES_Z, XTG_MULTIRES_BIN = 1, 2
XTG_PROJ_AUTO, XTG_PROJ_GATHER, XTG_PROJ_TABLE = 0, 1, 2

# symbols declared in include/xtg.h and include/xt_gen.h
XTG_SYMBOLS = [
    "xtg_create", "xtg_destroy", "xtg_set_zslab", "xtg_set_slab", "xtg_slab_exchange", "xtg_init_object_fbp", "xtg_object_to_device",
    "xtg_object_from_device", "xtg_upsample", "xtg_init_object_multires", "xtg_get_zslab", "xtg_last_error", "xtg_abi_version", "xtg_dims", "xtg_geometry",
    "xtg_get_hr", "xtg_set_options", "xtg_get_options", "xtg_set_projector", "xtg_get_projector", "xtg_upload_sino", "xtg_upload_sino_start", "xtg_upload_counts", "xtg_upload_object",
    "xtg_download_object", "xtg_get_error_sino", "xtg_set_error_sino", "xtg_get_weight",
    "xtg_get_offset", "xtg_set_offset", "xtg_get_magmap", "xtg_set_magmap", "xtg_get_variance",
    "xtg_set_variance", "xtg_amatrix", "xtg_forward_project", "xtg_init_error_sino",
    "xtg_resync_fp64", "xtg_map_cost_fp64", "xtg_map_cost_running", "xtg_zinger_refresh",
    "xtg_icd_iteration", "xtg_update_columns", "xtg_nhicd_select", "xtg_update_offset",
    "xtg_update_variance", "xtg_device_bytes", "xtg_launch_count", "xtg_last_kernel_time",
    "xtg_nhicd_threshold_noalloc", "xtg_download_object_start", "xtg_download_wait",
]
# warm-start network entry points (include/xtg_cnn.h), also in libxtgpu.so
XTC_SYMBOLS = ["xtc_wait_selftest", "xtc_conv3d", "xtc_conv3d_path", "xtc_conv3d_wgrad", "xtc_conv3d_wgrad_path",
               "xtc_net_create", "xtc_net_destroy", "xtc_net_param_count", "xtc_net_get_params", "xtc_net_set_params", "xtc_net_save", "xtc_net_load", "xtc_net_forward",
               "xtc_net_backward", "xtc_net_adam_step", "xtc_net_train", "xtg_init_object_learned"]
XTGEN_SYMBOLS = [
    "xtgen_views_uniform", "xtgen_views_interlaced", "xtgen_write_view_file", "xtgen_phantom",
    "xtgen_forward", "xtgen_measure", "xtgen_write_bin", "xtgen_geometry", "xtgen_amatrix",
]


class XtParams(C.Structure):
    """xt_params of xt_geom.h: the XT_Engine command line after atof/atoi."""

    _fields_ = [(n, C.c_double) for n in (
        "p", "sigma_s", "sigma_t", "c_s", "c_t", "delta_xy", "delta_z", "length_r", "length_t",
        "voxel_thresh", "cost_thresh", "rotation_center", "alpha", "Rtime0", "Rtime_delta",
        "radius_obj", "zingerT", "zingerDel", "Est_of_Var")] + [(n, C.c_int32) for n in (
        "iter", "sinobin", "initICD", "writeTiff", "Rtime_num", "num_projections", "N_r", "N_t",
        "detector_slice_begin", "detector_slice_num", "num_threads", "phantom_N_xy", "phantom_N_z",
        "updateProjOffset", "x_start", "x_width", "EnforceZeroMeanOffset", "time_reg",
        "RMSE_converged", "WritePerIter", "no_NHICD", "only_Edge_Updates", "initMagUpMap",
        "do_VarEst", "dont_reconstruct", "readSino4mHDF", "NoNoise", "positivity", "real_is_double")]


class XtGeom(C.Structure):
    _fields_ = ([(n, C.c_int32) for n in (
        "N_r", "N_t", "N_p", "N_x", "N_y", "N_z", "N_time", "zovl", "nzb", "zstep", "amax")]
        + [(n, C.c_float) for n in (
            "delta_r", "delta_t", "R0", "RMax", "T0", "x0", "y0", "delta_xy", "delta_z", "OffsetR",
            "mult_xy", "mult_z", "MRF_P", "C_S", "C_T", "alpha", "Sigma_S_Q", "Sigma_S_Q_P",
            "Sigma_T_Q", "Sigma_T_Q_P")]
        + [("SF", C.c_float * 27)]
        + [(n, C.c_float) for n in (
            "TF", "T", "delta", "var_est", "StopThreshold", "radius_obj", "Rtime0", "delta_Rtime")])


class XtgStats(C.Structure):
    _fields_ = [("avg_update_pct", C.c_double), ("mag_sum", C.c_double), ("vox_mag", C.c_double),
                ("total_pix", C.c_double), ("voxel_updates", C.c_int64), ("zero_skipped", C.c_int64),
                ("columns", C.c_int64), ("converged", C.c_int32), ("ms", C.c_float)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class PhantomSpec(C.Structure):
    _fields_ = [("n_ellipsoids", C.c_int32), ("mu_max", C.c_double), ("n_moving", C.c_int32),
                ("max_shift", C.c_double), ("growing", C.c_int32), ("seed", C.c_uint64)]


def _load(name):
    path = os.path.join(LIBDIR, name)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `make -C timbir-python_b200` "
                           "(there is no CPU fallback)")
    return C.CDLL(path, mode=C.RTLD_GLOBAL)


_gpu = None
_gen = None


def gpu_lib():
    global _gpu
    if _gpu is None:
        lib = _load("libxtgpu.so")
        lib.xtg_last_error.restype = C.c_char_p
        lib.xtg_create.argtypes = [C.POINTER(XtParams), C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]
        for n in ("xtg_destroy",):
            getattr(lib, n).argtypes = [C.c_void_p]
            getattr(lib, n).restype = None
        lib.xtg_device_bytes.restype = C.c_int64
        lib.xtg_device_bytes.argtypes = [C.c_void_p]
        lib.xtg_launch_count.restype = C.c_int64
        lib.xtg_launch_count.argtypes = [C.c_void_p]
        lib.xtg_set_options.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_uint64]
        lib.xtg_set_variance.argtypes = [C.c_void_p, C.c_double]
        lib.xtg_upload_counts.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        lib.xtg_nhicd_threshold_noalloc.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p]
        _gpu = lib
    return _gpu


def gen_lib():
    global _gen
    if _gen is None:
        lib = _load("libxtgen.so")
        lib.xtgen_phantom.argtypes = [C.POINTER(PhantomSpec), C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
        lib.xtgen_forward.argtypes = [C.POINTER(XtParams), C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        lib.xtgen_measure.argtypes = [C.c_size_t, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_uint64, C.c_void_p, C.c_void_p]
        lib.xtgen_views_uniform.argtypes = [C.c_int32, C.c_void_p, C.c_void_p]
        lib.xtgen_views_interlaced.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
        lib.xtgen_write_view_file.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p]
        lib.xtgen_write_bin.argtypes = [C.c_char_p, C.c_void_p, C.c_size_t, C.c_int]
        _gen = lib
    return _gen


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


@dataclass
class Params:
    """Python mirror of the XT_Engine command line (same names as the long options)."""

    p: float = 1.2
    sigma_s: float = 0.0
    sigma_t: float = 0.0
    c_s: float = 0.01
    c_t: float = 0.01
    delta_xy: float = 1.0
    delta_z: float = 1.0
    length_r: float = 0.0
    length_t: float = 0.0
    voxel_thresh: float = 0.0
    cost_thresh: float = 100.0
    rotation_center: float = 0.0
    alpha: float = 1.0
    Rtime0: float = 0.0
    Rtime_delta: float = 0.0
    radius_obj: float = 0.0
    zingerT: float = 100000.0
    zingerDel: float = 0.0
    Est_of_Var: float = 1.0
    iter: int = 20
    sinobin: int = 1
    initICD: int = 0
    writeTiff: int = 0
    Rtime_num: int = 1
    num_projections: int = 0
    N_r: int = 0
    N_t: int = 0
    detector_slice_begin: int = 0
    detector_slice_num: int = 0
    num_threads: int = 1
    phantom_N_xy: int = 0
    phantom_N_z: int = 0
    updateProjOffset: int = 0
    x_start: int = 0
    x_width: int = 0
    EnforceZeroMeanOffset: int = 0
    time_reg: int = 0
    RMSE_converged: int = 0
    WritePerIter: int = 0
    no_NHICD: int = 0
    only_Edge_Updates: int = 0
    initMagUpMap: int = 0
    do_VarEst: int = 0
    dont_reconstruct: int = 0
    readSino4mHDF: int = 0
    NoNoise: int = 0
    positivity: int = 1
    real_is_double: int = 0

    def to_c(self):
        c = XtParams()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c

    def cli(self, extra=()):
        """The XT_Engine argument list (reference option names)."""
        a = ["--p", repr(self.p), "--sigma_s", repr(self.sigma_s), "--sigma_t", repr(self.sigma_t),
             "--c_s", repr(self.c_s), "--c_t", repr(self.c_t), "--delta_xy", repr(self.delta_xy),
             "--delta_z", repr(self.delta_z), "--length_r", repr(self.length_r),
             "--length_t", repr(self.length_t), "--voxel_thresh", repr(self.voxel_thresh),
             "--cost_thresh", repr(self.cost_thresh), "--iter", str(self.iter),
             "--rotation_center", repr(self.rotation_center), "--alpha", repr(self.alpha),
             "--sinobin", str(self.sinobin), "--initICD", str(self.initICD), "--Rtime0", repr(self.Rtime0),
             "--Rtime_delta", repr(self.Rtime_delta), "--Rtime_num", str(self.Rtime_num),
             "--num_projections", str(self.num_projections), "--N_r", str(self.N_r), "--N_t", str(self.N_t),
             "--num_threads", str(self.num_threads), "--radius_obj", repr(self.radius_obj),
             "--updateProjOffset", str(self.updateProjOffset), "--writeTiff", str(self.writeTiff),
             "--zingerT", repr(self.zingerT), "--zingerDel", repr(self.zingerDel),
             "--Est_of_Var", repr(self.Est_of_Var)]
        if self.no_NHICD:
            a.append("--no_NHICD")
        if self.EnforceZeroMeanOffset:
            a.append("--EnforceZeroMeanOffset")
        if self.do_VarEst:
            a.append("--do_VarEst")
        if self.initMagUpMap:
            a.append("--initMagUpMap")
        if self.WritePerIter:
            a.append("--WritePerIter")
        return a + list(extra)


def _check(rc, what):
    if rc != 0:
        msg = gpu_lib().xtg_last_error()
        raise RuntimeError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")


class Context:
    """One device-resident reconstruction (xtg_ctx)."""

    def __init__(self, params: Params, times, angles_deg):
        lib = gpu_lib()
        self.lib = lib
        self.params = params
        self._cp = params.to_c()
        t = np.ascontiguousarray(times, dtype=np.float64)
        a = np.ascontiguousarray(angles_deg, dtype=np.float64)
        h = C.c_void_p()
        _check(lib.xtg_create(C.byref(self._cp), _p(t), _p(a), len(t), C.byref(h)), "xtg_create")
        self.h = h
        d = np.zeros(11, np.int32)
        lib.xtg_dims(h, _p(d))
        (self.N_x, self.N_y, self.N_z, self.N_time, self.N_r, self.N_t, self.N_p,
         self.nzb, self.zovl, self.amax, self.n_masked) = (int(v) for v in d)

    def close(self):
        if getattr(self, "h", None):
            self.lib.xtg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # shapes
    @property
    def sino_shape(self):
        return (self.N_p, self.N_r, self.N_t)

    @property
    def obj_shape(self):
        return (self.N_time, self.N_z, self.N_y, self.N_x)

    @property
    def mag_shape(self):
        return (self.N_time, self.nzb, self.N_y, self.N_x)

    def geometry(self):
        g = XtGeom()
        _check(self.lib.xtg_geometry(self.h, C.byref(g)), "xtg_geometry")
        return g

    def hr(self):
        out = np.zeros((self.N_p, 65), np.float32)
        _check(self.lib.xtg_get_hr(self.h, _p(out)), "xtg_get_hr")
        return out

    def init_fbp(self):
        _check(self.lib.xtg_init_object_fbp(self.h), "xtg_init_object_fbp")

    def upsample(self, a, with_z=True):
        a = _f32(a)
        nt, nz, ny, nx = a.shape
        out = np.zeros((nt, 2 * nz if with_z else nz, 2 * ny, 2 * nx), np.float32)
        _check(self.lib.xtg_upsample(self.h, _p(a), _p(out), nt, nz, ny, nx, int(with_z)), "xtg_upsample")
        return out

    def init_multires(self, coarse_iters=40, with_z=True, binned=False):
        """Multi-resolution start: coarse_iters ICD iterations on the grid with
        voxels twice as large (x-y, and z when with_z), upsampled; binned runs
        them against the detector binned to the coarse voxel size."""
        flags = (XTG_MULTIRES_Z if with_z else 0) | (XTG_MULTIRES_BIN if binned else 0)
        _check(self.lib.xtg_init_object_multires(self.h, int(coarse_iters), flags), "xtg_init_object_multires")

    def object_to_device(self, dst):
        _check(self.lib.xtg_object_to_device(self.h, WarmNet._dev(dst)), "xtg_object_to_device")

    def object_from_device(self, src):
        _check(self.lib.xtg_object_from_device(self.h, WarmNet._dev(src)), "xtg_object_from_device")

    def init_learned(self, net, coarse_iters=30):
        """Learned warm start over the multi-resolution start; returns
        (used, cost_net, cost_base).  ICD continues at iteration 1."""
        used, cn, ci = C.c_int32(), C.c_double(), C.c_double()
        _check(self.lib.xtg_init_object_learned(self.h, net.h, int(coarse_iters), C.byref(used), C.byref(cn),
                                                C.byref(ci)), "xtg_init_object_learned")
        return bool(used.value), cn.value, ci.value

    # the exchange hook's C type: int (*)(void *user, int32_t phase)
    EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32)

    def set_slab(self, send_below, send_above, recv_below, recv_above, exchange):
        """This context is one z slab of a larger volume (xtg_set_slab): device
        planes [N_time][N_y][N_x] (torch CUDA tensors or None per side) and
        exchange(phase) -> None, called whenever the neighbours' slices are
        due; it must fill recv_* from the neighbours' send_* before it
        returns."""
        def hook(user, phase):
            try:
                exchange(int(phase))
                return 0
            except Exception as err:  # reported through the library's error path
                self._hook_error = err
                return 1
        self._hook = self.EXCHANGE_FN(hook)  # kept alive as long as the context uses it
        self._slab_planes = (send_below, send_above, recv_below, recv_above)
        ptr = [None if t is None else C.c_void_p(t.data_ptr()) for t in self._slab_planes]
        _check(self.lib.xtg_set_slab(self.h, ptr[0], ptr[1], ptr[2], ptr[3], self._hook, None), "xtg_set_slab")

    def slab_exchange(self):
        _check(self.lib.xtg_slab_exchange(self.h), "xtg_slab_exchange")

    def set_zslab(self, slices):
        _check(self.lib.xtg_set_zslab(self.h, int(slices)), "xtg_set_zslab")

    def zslab(self):
        v = C.c_int32()
        _check(self.lib.xtg_get_zslab(self.h, C.byref(v)), "xtg_get_zslab")
        return v.value

    def set_options(self, a_mode=XTG_A_FP32, order=XTG_ORDER_PARALLEL, max_columns=0, seed=0x5EED5EED):
        _check(self.lib.xtg_set_options(self.h, a_mode, order, max_columns, seed), "xtg_set_options")

    def set_projector(self, kind):
        _check(self.lib.xtg_set_projector(self.h, int(kind)), "xtg_set_projector")

    def projector(self):
        """(projector in use, entries of its bin-major table)."""
        k, n = C.c_int32(), C.c_int64()
        _check(self.lib.xtg_get_projector(self.h, C.byref(k), C.byref(n)), "xtg_get_projector")
        return k.value, n.value

    def a_mode_used(self):
        """The A storage in force (XTG_A_AUTO resolved)."""
        m = C.c_int32()
        _check(self.lib.xtg_get_options(self.h, C.byref(m), None, None, None), "xtg_get_options")
        return m.value

    def upload_sino(self, y, w, d=None):
        y, w = _f32(y), _f32(w)
        d = None if d is None else _f32(d)
        _check(self.lib.xtg_upload_sino(self.h, _p(y), _p(w), _p(d)), "xtg_upload_sino")

    def upload_sino_start(self, y, w, d=None):
        """upload_sino + init_error_sino for the resident object, the copies
        overlapping the projection (pinned torch CPU tensors overlap best)."""
        if hasattr(y, "data_ptr"):
            ptrs = [C.c_void_p(t.data_ptr()) if t is not None else None for t in (y, w, d)]
        else:
            y, w = _f32(y), _f32(w)
            d = None if d is None else _f32(d)
            ptrs = [_p(y), _p(w), _p(d)]
        _check(self.lib.xtg_upload_sino_start(self.h, *ptrs), "xtg_upload_sino_start")

    def upload_counts(self, bright, counts, bh=0.0, d=None):
        b, c = _f32(bright), _f32(counts)
        d = None if d is None else _f32(d)
        _check(self.lib.xtg_upload_counts(self.h, _p(b), _p(c), bh, _p(d)), "xtg_upload_counts")

    def upload_object(self, x):
        x = _f32(x)
        assert x.size == int(np.prod(self.obj_shape))
        _check(self.lib.xtg_upload_object(self.h, _p(x)), "xtg_upload_object")

    def object(self):
        out = np.zeros(self.obj_shape, np.float32)
        _check(self.lib.xtg_download_object(self.h, _p(out)), "xtg_download_object")
        return out

    def download_object_start(self, ptr):
        """Start copying the object to host memory at `ptr` (an address, e.g.
        a pinned torch tensor's data_ptr(), of obj_shape float32 values);
        complete after download_wait()."""
        _check(self.lib.xtg_download_object_start(self.h, C.c_void_p(ptr)), "xtg_download_object_start")

    def download_wait(self):
        _check(self.lib.xtg_download_wait(self.h), "xtg_download_wait")

    def _get(self, fn, shape):
        out = np.zeros(shape, np.float32)
        _check(getattr(self.lib, fn)(self.h, _p(out)), fn)
        return out

    def error_sino(self):
        return self._get("xtg_get_error_sino", self.sino_shape)

    def set_error_sino(self, e):
        e = _f32(e)
        _check(self.lib.xtg_set_error_sino(self.h, _p(e)), "xtg_set_error_sino")

    def weight(self):
        return self._get("xtg_get_weight", self.sino_shape)

    def offset(self):
        return self._get("xtg_get_offset", (self.N_r, self.N_t))

    def set_offset(self, d):
        d = _f32(d)
        _check(self.lib.xtg_set_offset(self.h, _p(d)), "xtg_set_offset")

    def magmap(self):
        return self._get("xtg_get_magmap", self.mag_shape)

    def set_magmap(self, m):
        m = _f32(m)
        _check(self.lib.xtg_set_magmap(self.h, _p(m)), "xtg_set_magmap")

    def variance(self):
        v = C.c_double()
        _check(self.lib.xtg_get_variance(self.h, C.byref(v)), "xtg_get_variance")
        return v.value

    def amatrix(self, rows, cols, views):
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        views = np.ascontiguousarray(views, np.int32)
        n = len(rows)
        vals = np.zeros((n, self.amax), np.float32)
        idx = np.zeros((n, self.amax), np.int32)
        cnt = np.zeros(n, np.int32)
        _check(self.lib.xtg_amatrix(self.h, n, _p(rows), _p(cols), _p(views), _p(vals), _p(idx), _p(cnt)),
               "xtg_amatrix")
        return vals, idx, cnt

    def forward_project(self):
        out = np.zeros(self.sino_shape, np.float32)
        _check(self.lib.xtg_forward_project(self.h, _p(out)), "xtg_forward_project")
        return out

    def init_error_sino(self):
        _check(self.lib.xtg_init_error_sino(self.h), "xtg_init_error_sino")

    def _cost3(self, fn):
        c, f, p = C.c_double(), C.c_double(), C.c_double()
        _check(getattr(self.lib, fn)(self.h, C.byref(c), C.byref(f), C.byref(p)), fn)
        return c.value, f.value, p.value

    def resync_fp64(self):
        return self._cost3("xtg_resync_fp64")

    def cost(self):
        return self._cost3("xtg_map_cost_fp64")

    def cost_running(self):
        return self._cost3("xtg_map_cost_running")

    def zinger_refresh(self, want_mask=True):
        sel = np.zeros(self.sino_shape, np.uint8) if want_mask else None
        n = C.c_int64()
        _check(self.lib.xtg_zinger_refresh(self.h, _p(sel), C.byref(n)), "xtg_zinger_refresh")
        return sel, n.value

    def iteration(self, it):
        st = XtgStats()
        _check(self.lib.xtg_icd_iteration(self.h, it, C.byref(st)), "xtg_icd_iteration")
        return st

    def update_columns(self, it, items):
        items = np.ascontiguousarray(items, np.int32).reshape(-1, 4)
        st = XtgStats()
        _check(self.lib.xtg_update_columns(self.h, it, len(items), _p(items), C.byref(st)), "xtg_update_columns")
        return st

    def nhicd_select(self, update_select_num):
        usn = np.ascontiguousarray(update_select_num, np.int32)
        nseg = self.N_time * self.nzb
        nn = np.zeros(nseg, np.int32)
        xs = np.zeros((nseg, self.N_x * self.N_y), np.int32)
        ys = np.zeros((nseg, self.N_x * self.N_y), np.int32)
        th = np.zeros(nseg, np.float32)
        _check(self.lib.xtg_nhicd_select(self.h, _p(usn), _p(nn), _p(xs), _p(ys), _p(th)), "xtg_nhicd_select")
        return nn, xs, ys, th

    def update_offset(self):
        _check(self.lib.xtg_update_offset(self.h), "xtg_update_offset")

    def update_variance(self):
        _check(self.lib.xtg_update_variance(self.h), "xtg_update_variance")

    def device_bytes(self):
        return int(self.lib.xtg_device_bytes(self.h))

    def launch_count(self):
        return int(self.lib.xtg_launch_count(self.h))

    def last_kernel_time(self):
        ms, items, launches = C.c_float(), C.c_int64(), C.c_int64()
        _check(self.lib.xtg_last_kernel_time(self.h, C.byref(ms), C.byref(items), C.byref(launches)),
               "xtg_last_kernel_time")
        return ms.value, items.value, launches.value


# ------------------------------------------------------ warm-start network --
class WarmNet:
    """The learned warm start (include/xtg_cnn.h) over device buffers.  Volume
    arguments are CUDA tensors (torch) or raw device addresses (int)."""

    def __init__(self, seed=1):
        lib = gpu_lib()
        self.lib = lib
        lib.xtc_net_create.argtypes = [C.c_uint64, C.POINTER(C.c_void_p)]
        lib.xtc_net_destroy.argtypes = [C.c_void_p]
        lib.xtc_net_destroy.restype = None
        lib.xtc_net_param_count.argtypes = [C.c_void_p]
        lib.xtc_net_param_count.restype = C.c_int64
        lib.xtc_net_adam_step.argtypes = [C.c_void_p, C.c_float]
        lib.xtc_net_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                      C.c_uint64, C.c_void_p]
        h = C.c_void_p()
        _check(lib.xtc_net_create(C.c_uint64(seed), C.byref(h)), "xtc_net_create")
        self.h = h
        self.n_params = int(lib.xtc_net_param_count(h))

    @staticmethod
    def _dev(t):
        return C.c_void_p(t if isinstance(t, int) else t.data_ptr())

    def params(self, which=0):
        out = np.zeros(self.n_params, np.float32)
        _check(self.lib.xtc_net_get_params(self.h, _p(out), int(which)), "xtc_net_get_params")
        return out

    def set_params(self, p):
        p = _f32(p)
        assert p.size == self.n_params
        _check(self.lib.xtc_net_set_params(self.h, _p(p)), "xtc_net_set_params")

    def forward(self, fbp, icd, out, shape):
        nb, Y, X, Z = shape
        _check(self.lib.xtc_net_forward(self.h, self._dev(fbp), self._dev(icd), self._dev(out), nb, Y, X, Z),
               "xtc_net_forward")

    def backward(self, fbp, icd, target, shape):
        nb, Y, X, Z = shape
        loss = C.c_double()
        _check(self.lib.xtc_net_backward(self.h, self._dev(fbp), self._dev(icd), self._dev(target), nb, Y, X, Z,
                                         C.byref(loss)), "xtc_net_backward")
        return loss.value

    def adam_step(self, lr):
        _check(self.lib.xtc_net_adam_step(self.h, C.c_float(lr)), "xtc_net_adam_step")

    def train(self, fbp, icd, target, vol_shape, patch, batch, steps, lr=1e-3, seed=7):
        """fbp / icd / target: lists of device volumes [Y][X][Z]; returns the losses."""
        n = len(fbp)
        arr = C.c_void_p * n
        pf, pi, pt = (arr(*[self._dev(t) for t in lst]) for lst in (fbp, icd, target))
        losses = np.zeros(steps, np.float32)
        Y, X, Z = vol_shape
        py, px, pz = patch
        _check(self.lib.xtc_net_train(self.h, pf, pi, pt, n, Y, X, Z, py, px, pz, batch, steps, C.c_float(lr),
                                      C.c_uint64(seed), _p(losses)), "xtc_net_train")
        return losses

    def save(self, path):
        _check(self.lib.xtc_net_save(self.h, str(path).encode()), "xtc_net_save")

    def load(self, path):
        _check(self.lib.xtc_net_load(self.h, str(path).encode()), "xtc_net_load")

    def close(self):
        if getattr(self, "h", None):
            self.lib.xtc_net_destroy(self.h)
            self.h = None


# ------------------------------------------------------------ generator ----
def views_uniform(n_p):
    t, a = np.zeros(n_p), np.zeros(n_p)
    assert gen_lib().xtgen_views_uniform(n_p, _p(t), _p(a)) == 0
    return t, a


def views_interlaced(K, N_theta, n_p):
    t, a = np.zeros(n_p), np.zeros(n_p)
    assert gen_lib().xtgen_views_interlaced(K, N_theta, n_p, _p(t), _p(a)) == 0
    return t, a


def write_view_file(path, times, angles):
    """Writes view_info.txt; returns the (times, angles) a reader parses back."""
    t = np.array(times, np.float64)
    a = np.array(angles, np.float64)
    assert gen_lib().xtgen_write_view_file(path.encode(), len(t), _p(t), _p(a)) == 0
    return t, a


def round_views(times, angles):
    """The values a view_info.txt reader gets back for these views."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        return write_view_file(os.path.join(d, "view_info.txt"), times, angles)


def phantom(shape, n_ellipsoids=10, mu_max=0.01, seed=1, n_moving=0, max_shift=0.0, growing=0):
    nt, nz, ny, nx = shape
    s = PhantomSpec(n_ellipsoids, mu_max, n_moving, max_shift, growing, seed)
    x = np.zeros(shape, np.float32)
    assert gen_lib().xtgen_phantom(C.byref(s), nt, nz, ny, nx, _p(x)) == 0
    return x


def forward_cpu(params: Params, times, angles, x):
    """A x on the host with the reference A and summation order (libxtgen)."""
    t = np.ascontiguousarray(times, np.float64)
    a = np.ascontiguousarray(angles, np.float64)
    x = _f32(x)
    cp = params.to_c()
    n_t = int(params.N_t)
    out = np.zeros((len(t), int(params.N_r), n_t), np.float32)
    rc = gen_lib().xtgen_forward(C.byref(cp), _p(t), _p(a), len(t), _p(x), _p(out))
    if rc != 0:
        raise RuntimeError("xtgen_forward failed")
    return out


def host_geometry(params: Params, times, angles):
    """The engine's host-side set-up (no GPU): geometry, cos/sin, frame of each view, H_r."""
    lib = gen_lib()
    t = np.ascontiguousarray(times, np.float64)
    a = np.ascontiguousarray(angles, np.float64)
    n = len(t)
    g = XtGeom()
    cs, sn = np.zeros(n, np.float32), np.zeros(n, np.float32)
    fov = np.zeros(n, np.int32)
    hr = np.zeros((n, 65), np.float32)
    err = C.create_string_buffer(512)
    cp = params.to_c()
    lib.xtgen_geometry.argtypes = [C.POINTER(XtParams), C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(XtGeom),
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    if lib.xtgen_geometry(C.byref(cp), _p(t), _p(a), n, C.byref(g), _p(cs), _p(sn), _p(fov), _p(hr), err, 512):
        raise ValueError(err.value.decode())
    return g, cs, sn, fov, hr


def host_amatrix(params: Params, times, angles, row, col, view):
    lib = gen_lib()
    t = np.ascontiguousarray(times, np.float64)
    a = np.ascontiguousarray(angles, np.float64)
    v, i = np.zeros(16, np.float32), np.zeros(16, np.int32)
    cp = params.to_c()
    lib.xtgen_amatrix.argtypes = [C.POINTER(XtParams), C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                  C.c_int32, C.c_void_p, C.c_void_p]
    n = lib.xtgen_amatrix(C.byref(cp), _p(t), _p(a), len(t), row, col, view, _p(v), _p(i))
    return v[:n].copy(), i[:n].copy()


def measure(ax, I0, seed, zinger_frac=0.0, zinger_lo=2.0, zinger_hi=5.0):
    ax = _f32(ax)
    y = np.zeros_like(ax)
    w = np.zeros_like(ax)
    gen_lib().xtgen_measure(ax.size, _p(ax), float(I0), float(zinger_frac), float(zinger_lo),
                            float(zinger_hi), int(seed), _p(y), _p(w))
    return y, w
