"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only to compare the product's results with, or (the CPU baseline) to
time the reference's kernels on the host.  It wraps:

* ``libxpr_oracle.so`` -- the C restatement of the reference path (xpr_oracle.c);
* ``libxpr_ref.so``    -- the reference's own OpenCL kernels compiled for the CPU
  (oracle/build.py), used to pin the restatement.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

STRICT, FAST = 0, 1
FIXED_ONE = 1 << 22

_oracle = None
_ref = None
_ref_relaxed = None

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


class Launch(C.Structure):
    _fields_ = [
        ("vmin", C.c_int32 * 3), ("vmax", C.c_int32 * 3),
        ("origin", C.c_float * 3), ("voxel", C.c_float * 3),
        ("det_w", C.c_uint32), ("rows", C.c_uint32), ("row_offset", C.c_int32),
        ("n_angles", C.c_uint32), ("modules", C.c_uint32),
        ("list_mvp", C.c_void_p), ("list_img", C.c_void_p), ("n_list", C.c_uint32),
        ("arith", C.c_int32), ("compat_pad", C.c_int32), ("nan_skip", C.c_int32),
    ]


class GeomParams(C.Structure):
    _fields_ = [
        ("so", C.c_float), ("sd", C.c_float), ("angle", C.c_float), ("heli_offset", C.c_float),
        ("px", C.c_float), ("rx_px", C.c_float), ("sx", C.c_float), ("sy", C.c_float),
        ("module_number", C.c_int64), ("module_angle_offset_set", C.c_int32),
        ("module_angle_offset", C.c_float), ("module_center_offset_z", C.c_float),
        ("dwidth", C.c_int64), ("dheight", C.c_int64), ("projections", C.c_int64), ("sit", C.c_int64),
        ("angle_list", C.c_void_p), ("mod_offset", C.c_void_p), ("mod_rpy", C.c_void_p),
    ]


class GeomOut(C.Structure):
    _fields_ = [("vx", C.c_float), ("vwidth", C.c_int64), ("vheight", C.c_int64),
                ("orig", C.c_float * 3), ("concurrent", C.c_int64)]


class ReconParams(C.Structure):
    _fields_ = [("it", C.c_int64), ("sit", C.c_int64), ("weight", C.c_float), ("weight_factor", C.c_float),
                ("seed", C.c_uint32), ("arith", C.c_int32), ("compat_pad", C.c_int32)]


class MT(C.Structure):
    _fields_ = [("mt", C.c_uint32 * 624), ("idx", C.c_int)]


def lib():
    global _oracle
    if _oracle is None:
        path = _build.ORACLE_SO
        if not os.path.exists(path):
            path = _build.build_oracle()
        L = C.CDLL(path)
        L.orc_expf.restype = C.c_float
        L.orc_expf.argtypes = [C.c_float]
        L.orc_logf.restype = C.c_float
        L.orc_logf.argtypes = [C.c_float]
        L.orc_mt_seed.argtypes = [C.POINTER(MT), C.c_uint32]
        L.orc_mt_next.restype = C.c_uint32
        L.orc_mt_next.argtypes = [C.POINTER(MT)]
        L.orc_uniform_float.restype = C.c_float
        L.orc_uniform_float.argtypes = [C.POINTER(MT), C.c_float, C.c_float]
        L.orc_float_to_fixed.restype = C.c_uint32
        L.orc_float_to_fixed.argtypes = [C.c_float]
        L.orc_ndrange.restype = C.c_uint64
        L.orc_ndrange.argtypes = [C.c_uint64]
        L.orc_forward.argtypes = [f32p, u32p, f32p, C.POINTER(Launch)]
        L.orc_backward.argtypes = [f32p, f32p, f32p, C.POINTER(Launch)]
        L.orc_error.argtypes = [f32p, u32p, C.c_uint64, C.c_float]
        L.orc_error_first_1c.argtypes = [f32p, f32p, C.c_uint64]
        L.orc_error_1c.argtypes = [f32p, u32p, C.c_uint64, C.c_float]
        L.orc_minmax_normal.argtypes = [f32p, C.c_uint64, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_preprocess.argtypes = [f32p, C.c_uint64, C.c_int, C.c_float, C.c_float, C.c_int]
        L.orc_geometry.argtypes = [C.POINTER(GeomParams), C.c_int, f32p, C.POINTER(GeomOut)]
        L.orc_cull_layer.restype = C.c_int
        L.orc_cull_layer.argtypes = [C.POINTER(GeomParams), C.POINTER(GeomOut), f32p, C.c_int64, C.c_int64,
                                     C.c_int, u16p, u16p]
        L.orc_plan_chunks.restype = C.c_int
        L.orc_plan_chunks.argtypes = [C.POINTER(GeomParams), C.POINTER(GeomOut), f32p, C.c_uint64, C.c_uint64,
                                      C.c_float, i64p, C.c_int]
        for fn in ("orc_recon_naive", "orc_recon_1c"):
            getattr(L, fn).restype = C.c_int
            getattr(L, fn).argtypes = [C.POINTER(GeomParams), C.POINTER(ReconParams), f32p, f32p]
        L.orc_recon_chunks.restype = C.c_int
        L.orc_recon_chunks.argtypes = [C.POINTER(GeomParams), C.POINTER(ReconParams), f32p, i64p, C.c_int, f32p]
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.orc_geometry_f64.argtypes = [C.POINTER(GeomParams), f64p, f64p, C.POINTER(GeomOut)]
        L.orc64_forward.argtypes = [f64p, f64p, f64p, f64p, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                    C.POINTER(C.c_double), C.c_double, C.c_int64, C.c_int64]
        L.orc64_preprocess.argtypes = [f32p, f64p, C.c_uint64, C.c_int]
        L.orc64_recon_naive.restype = C.c_int
        L.orc64_recon_naive.argtypes = [C.POINTER(GeomParams), C.POINTER(ReconParams), f64p, f64p]
        _oracle = L
    return _oracle


def ref_lib(relaxed: bool = False):
    """The reference's own kernels compiled for the CPU (IEEE single precision), or with
    relaxed=True the same sources under relaxed floating point; None if unavailable."""
    global _ref, _ref_relaxed
    cached = _ref_relaxed if relaxed else _ref
    if cached is None:
        target = _build.REF_RELAXED_SO if relaxed else _build.REF_SO
        if not os.path.exists(target):
            _build.build_ref()
        if not os.path.exists(target):
            return None
        R = C.CDLL(target)
        u32x = C.POINTER(C.c_uint32)
        f4 = C.POINTER(C.c_float)
        i32x = C.POINTER(C.c_int32)
        R.refk_forward.argtypes = [f32p, u32p, f32p, u32x, f4, C.c_uint32, C.c_uint32, i32x, i32x, i32x, f4, C.c_uint64]
        R.refk_backward.argtypes = [f32p, f32p, f32p, u32x, f4, C.c_uint32, C.c_uint32, i32x, i32x, i32x, f4, C.c_uint64]
        R.refk_error.argtypes = [f32p, u32p, u32x, C.c_uint32, C.c_float, C.c_uint64]
        R.refk_forwardh.argtypes = [f32p, u32p, f32p, u16p, u16p, C.c_uint32, C.c_uint32, f4, C.c_float,
                                    C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
        R.refk_backwardh.argtypes = [f32p, f32p, f32p, u16p, u16p, C.c_uint32, C.c_uint32, f4, C.c_float,
                                     C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
        if relaxed:
            _ref_relaxed = R
        else:
            _ref = R
        cached = R
    return cached


# --------------------------------------------------------------------------- helpers
def ndrange(n: int) -> int:
    """Work-items of the reference NDRange for n items (kernel.hpp:73-81)."""
    return n + (32 - n % 32)


def make_launch(vmin, vmax, origin, voxel, det_w, rows, row_offset, n_angles, modules,
                arith=STRICT, compat_pad=0, nan_skip=0, list_mvp=None, list_img=None) -> tuple:
    L = Launch()
    L.vmin[:] = [int(v) for v in vmin]
    L.vmax[:] = [int(v) for v in vmax]
    L.origin[:] = [float(v) for v in origin]
    L.voxel[:] = [float(v) for v in voxel]
    L.det_w, L.rows, L.row_offset = int(det_w), int(rows), int(row_offset)
    L.n_angles, L.modules = int(n_angles), int(modules)
    L.arith, L.compat_pad, L.nan_skip = int(arith), int(compat_pad), int(nan_skip)
    keep = []
    if list_mvp is not None:
        lm = np.ascontiguousarray(list_mvp, dtype=np.uint16)
        li = np.ascontiguousarray(list_img, dtype=np.uint16)
        keep = [lm, li]
        L.list_mvp = lm.ctypes.data
        L.list_img = li.ctypes.data
        L.n_list = len(lm)
    return L, keep


def geom_params(so=100.0, sd=1000.0, angle=360.0, heli_offset=0.0, px=0.1, rx=0.0, sx=0.0, sy=0.0,
                module_number=1, module_angle_offset=None, module_center_offset_z=0.0,
                dwidth=64, dheight=64, projections=36, sit=4, angle_list=None,
                mod_offset=None, mod_rpy=None):
    g = GeomParams()
    g.so, g.sd, g.angle, g.heli_offset = so, sd, angle, heli_offset
    g.px, g.rx_px, g.sx, g.sy = px, rx, sx, sy
    g.module_number = module_number
    g.module_angle_offset_set = 0 if module_angle_offset is None else 1
    g.module_angle_offset = 0.0 if module_angle_offset is None else module_angle_offset
    g.module_center_offset_z = module_center_offset_z
    g.dwidth, g.dheight, g.projections, g.sit = dwidth, dheight, projections, sit
    keep = []
    for name, arr in (("angle_list", angle_list), ("mod_offset", mod_offset), ("mod_rpy", mod_rpy)):
        if arr is not None:
            a = np.ascontiguousarray(arr, dtype=np.float32)
            keep.append(a)
            setattr(g, name, a.ctypes.data)
    g._keep = keep
    return g


def geometry(g: GeomParams, fp64: bool = False):
    """(ProjData float32[P*M, 20], GeomOut)"""
    out = np.zeros((g.projections * g.module_number, 20), np.float32)
    go = GeomOut()
    lib().orc_geometry(C.byref(g), int(fp64), out, C.byref(go))
    return out, go


def subset_projdata(all_pd: np.ndarray, P: int, S: int, M: int, sit: int, Pc: int) -> np.ndarray:
    """ProjData of the first Pc angles of sub-iteration `sit` (geometry.hpp:306-327)."""
    idx = [(sit + k * S) * M + m for k in range(Pc) for m in range(M)]
    return np.ascontiguousarray(all_pd[idx])


def forward(vol, sums, pd, L):
    lib().orc_forward(vol, sums, pd, C.byref(L))


def backward(vol, ratio, pd, L):
    lib().orc_backward(vol, ratio, pd, C.byref(L))


def error(images, sums, weight):
    lib().orc_error(images, sums, sums.size, weight)


def jitter_sequence(seed: int, n: int, vx: float) -> np.ndarray:
    g = MT()
    lib().orc_mt_seed(C.byref(g), seed)
    return np.array([lib().orc_uniform_float(C.byref(g), 0.0, vx) for _ in range(n)], np.float32)


def mt_outputs(seed: int, n: int) -> np.ndarray:
    g = MT()
    lib().orc_mt_seed(C.byref(g), seed)
    return np.array([lib().orc_mt_next(C.byref(g)) for _ in range(n)], np.uint64)


# --------------------------------------------------------------------------- reference kernels
def _c_arr(ctype, vals):
    return (ctype * len(vals))(*vals)


def ref_forward(vol, sums, pd, det_w, det_h, origin, n_angles, modules, vmin, vmax, line_offset, voxel, pad=True, relaxed=False):
    R = ref_lib(relaxed)
    n = int(np.prod(np.subtract(vmax, vmin)))
    R.refk_forward(vol, sums, pd, _c_arr(C.c_uint32, [det_w, det_h, det_w, 1]),
                   _c_arr(C.c_float, [*origin, 0.0]), n_angles, modules,
                   _c_arr(C.c_int32, list(vmin)), _c_arr(C.c_int32, list(vmax)),
                   _c_arr(C.c_int32, list(line_offset)), _c_arr(C.c_float, [*voxel, 1.0]),
                   ndrange(n) if pad else n)


def ref_backward(vol, ratio, pd, det_w, det_h, origin, n_angles, modules, vmin, vmax, line_offset, voxel, pad=True, relaxed=False):
    R = ref_lib(relaxed)
    n = int(np.prod(np.subtract(vmax, vmin)))
    R.refk_backward(vol, ratio, pd, _c_arr(C.c_uint32, [det_w, det_h, det_w, 1]),
                    _c_arr(C.c_float, [*origin, 0.0]), n_angles, modules,
                    _c_arr(C.c_int32, list(vmin)), _c_arr(C.c_int32, list(vmax)),
                    _c_arr(C.c_int32, list(line_offset)), _c_arr(C.c_float, [*voxel, 1.0]),
                    ndrange(n) if pad else n)


def ref_error(images, sums, det_w, det_h, weight, relaxed=False):
    R = ref_lib(relaxed)
    R.refk_error(images, sums, _c_arr(C.c_uint32, [det_w, det_h, det_w, 1]), sums.size, weight, ndrange(sums.size))


# ----------------------------------------------------------------------------- FP64 oracle
def geometry_f64(g: GeomParams):
    """(mvp float64[P*M, 16], vp float64[P*M, 4], GeomOut): the geometry in double."""
    n = g.projections * g.module_number
    mvp = np.zeros((n, 16), np.float64)
    vp = np.zeros((n, 4), np.float64)
    go = GeomOut()
    lib().orc_geometry_f64(C.byref(g), mvp, vp, C.byref(go))
    return mvp, vp, go


def forward_f64(vol, mvp, vp, modules, W, Hv, origin, voxel, det_w, rows):
    """Double-precision forward of a W x Hv x W volume against len(mvp) (angle, module)
    entries; returns the detector sums, float64[len(mvp) // modules, rows, det_w]."""
    n_img = mvp.shape[0] // modules
    out = np.zeros(n_img * rows * det_w, np.float64)
    o = (C.c_double * 3)(*origin)
    lib().orc64_forward(np.ascontiguousarray(vol, np.float64).ravel(), out, np.ascontiguousarray(mvp),
                        np.ascontiguousarray(vp), mvp.shape[0], modules, W, Hv, o, voxel, det_w, rows)
    return out.reshape(n_img, rows, det_w)


def recon_naive_f64(gp: GeomParams, rp: ReconParams, raw: np.ndarray, mlog: bool = True) -> np.ndarray:
    """The naive reconstruction in double from raw (un-preprocessed) float32 images."""
    raw = np.ascontiguousarray(raw, np.float32).ravel()
    imgs = np.zeros(raw.size, np.float64)
    lib().orc64_preprocess(raw, imgs, raw.size, int(mlog))
    go = GeomOut()
    tmp = np.zeros((gp.projections * gp.module_number, 20), np.float32)
    lib().orc_geometry(C.byref(gp), 1, tmp, C.byref(go))
    vol = np.zeros(int(go.vwidth) * int(go.vheight) * int(go.vwidth), np.float64)
    assert lib().orc64_recon_naive(C.byref(gp), C.byref(rp), imgs, vol) == 0
    return vol


# ----------------------------------------------------------------------------- naive loop over a kernel set
def recon_loop(kernels, pd_all, go, P, S, M, imgs, Wd, Hd, it, weight, weight_factor, seed, box=None,
               arith=STRICT, pad=False):
    """The naive reconstruction of reconstruction_n.hpp:27-88 as a host loop over one
    kernel set: kernels = "ref" runs the reference's own Forward / Error / Backward
    (oracle/_ref, its OpenCL sources compiled for the CPU; IEEE single precision, the
    STRICT contract by construction), "ref_relaxed" the same sources under relaxed
    floating point (the reference's -cl-fast-relaxed-math, emulated), "oracle" the C
    restatement in contract `arith`.

    Volume 1.0 (:59), sums FIXED_ONE before the first sub-iteration (:60), which skips
    the forward (:70); per sub-iteration the origin is jittered by three
    uniform_real_distribution<float>(0, vx) draws of std::mt19937(seed)
    (reconstruction.hpp:268-272), the error is written over the sums (KernelError.cl)
    and the sums are zeroed after the backward; weight *= weight_factor after each main
    iteration (:80).  imgs: preprocessed float32[P, Hd, Wd] in acquisition order;
    sub-iteration s uses acquisitions s, s + S, ... (geometry.hpp:306-327).  box =
    (vmin, vmax) reconstructs that part of the grid only (the kernels' volume box);
    pad launches the reference's NDRange padding work-items (kernel.hpp:73-81).
    Returns the box's volume, float32[n]."""
    W, Hv = int(go.vwidth), int(go.vheight)
    vmin, vmax = ((0, 0, 0), (W, Hv, W)) if box is None else box
    n = int(np.prod(np.subtract(vmax, vmin)))
    Pc = P // S
    vol = np.ones(ndrange(n) if pad else n, np.float32)
    sums = np.full(Pc * Wd * Hd, FIXED_ONE, np.uint32)
    g = MT()
    lib().orc_mt_seed(C.byref(g), int(seed))
    w = np.float32(weight)
    imgs = np.asarray(imgs, np.float32).reshape(P, Hd, Wd)
    for mit in range(it):
        for s in range(S):
            origin = [float(np.float32(go.orig[i]) + np.float32(lib().orc_uniform_float(C.byref(g), 0.0, go.vx)))
                      for i in range(3)]
            pd = np.ascontiguousarray(subset_projdata(pd_all, P, S, M, s, Pc), np.float32)
            sub = np.ascontiguousarray(imgs[[s + k * S for k in range(Pc)]]).ravel()
            if kernels in ("ref", "ref_relaxed"):
                rx = kernels == "ref_relaxed"
                if mit > 0 or s > 0:
                    ref_forward(vol, sums, pd, Wd, Hd, origin, Pc, M, vmin, vmax, (0, Hd), [go.vx] * 3, pad=pad,
                                relaxed=rx)
                ref_error(sub, sums, Wd, Hd, float(w), relaxed=rx)
                ref_backward(vol, sums.view(np.float32), pd, Wd, Hd, origin, Pc, M, vmin, vmax, (0, Hd),
                             [go.vx] * 3, pad=pad, relaxed=rx)
            else:
                L, keep = make_launch(vmin, vmax, origin, [go.vx] * 3, Wd, Hd, 0, Pc, M, arith=arith,
                                      compat_pad=int(pad))
                if mit > 0 or s > 0:
                    forward(vol, sums, pd, L)
                error(sub, sums, float(w))
                backward(vol, sums.view(np.float32), pd, L)
            sums[:] = 0
        w = np.float32(w * np.float32(weight_factor))
    return vol[:n].copy()
