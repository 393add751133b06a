"""ctypes binding of ``lib/libxpr.so`` (the C ABI declared in include/xpr.h).

Loading fails loudly when the library has not been built: there is no CPU or
pure-Python fallback for any operator.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# XPR_LIB names another build of the same C ABI (a deployment's own copy of the library)
LIB_PATH = os.environ.get("XPR_LIB") or os.path.join(HERE, "lib", "libxpr.so")

XPR_OK = 0
# status codes (enum xpr_status)
ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_CAP, ERR_IO, ERR_PARAM, ERR_UNSUPPORTED = 1, 2, 3, 4, 5, 6, 7
STRICT, FAST = 0, 1
F32, BF16, F16 = 0, 1, 2
ERROR_STD, ERROR_FIRST_1C, ERROR_1C = 0, 1, 2


class XprError(RuntimeError):
    pass


class ProjData(C.Structure):
    _fields_ = [("mvp", C.c_float * 16), ("vp", C.c_float * 4)]


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


class BatchProblem(C.Structure):
    _fields_ = [
        ("vol", C.c_void_p), ("images", C.c_void_p), ("projdata", C.c_void_p),
        ("det_w", C.c_uint32), ("det_h", C.c_uint32), ("per_subset", C.c_uint32), ("modules", C.c_uint32),
        ("sit", C.c_uint32), ("it", C.c_uint32), ("vwidth", C.c_uint32), ("vheight", C.c_uint32),
        ("voxel", C.c_float), ("orig", C.c_float * 3), ("seed", C.c_uint32),
        ("weight", C.c_float), ("weight_factor", C.c_float), ("residual", C.c_void_p),
    ]


class BatchOpts(C.Structure):
    _fields_ = [("arith", C.c_int32), ("storage", C.c_int32), ("init_volume", C.c_int32),
                ("use_graph", C.c_int32), ("autotune", C.c_int32), ("fwd_splits", C.c_int32),
                ("bwd_column", C.c_int32), ("ctas_per_sm", C.c_int32), ("image_storage_set", C.c_int32),
                ("image_storage", C.c_int32), ("fwd_layers", C.c_int32)]


_lib = None
vp = C.c_void_p
u64 = C.c_uint64
i32 = C.c_int


def _sig(L, name, res, args):
    fn = getattr(L, name)
    fn.restype = res
    fn.argtypes = args


def lib():
    """Load libxpr.so (raises ImportError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libxpr.so is not built (%s); run `python -m xpulse_recon_b200.build`" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    _sig(L, "xpr_last_error", C.c_char_p, [])
    _sig(L, "xpr_abi_version", i32, [])
    _sig(L, "xpr_ndrange", u64, [u64])
    _sig(L, "xpr_create", i32, [i32, u64, C.POINTER(vp)])
    _sig(L, "xpr_destroy", i32, [vp])
    _sig(L, "xpr_mem_available", i32, [vp, C.POINTER(u64)])
    _sig(L, "xpr_alloc", i32, [vp, u64, C.POINTER(vp)])
    _sig(L, "xpr_free", i32, [vp, vp])
    _sig(L, "xpr_alloc_pinned", i32, [vp, u64, C.POINTER(vp)])
    _sig(L, "xpr_free_pinned", i32, [vp, vp])
    _sig(L, "xpr_upload", i32, [vp, vp, vp, u64, vp])
    _sig(L, "xpr_download", i32, [vp, vp, vp, u64, vp])
    _sig(L, "xpr_fill_u32", i32, [vp, vp, C.c_uint32, u64, vp])
    _sig(L, "xpr_synchronize", i32, [vp, vp])
    _sig(L, "xpr_forward", i32, [vp, vp, vp, vp, C.c_uint32, C.POINTER(Launch), vp])
    _sig(L, "xpr_backward", i32, [vp, vp, vp, i32, vp, C.c_uint32, C.POINTER(Launch), vp])
    _sig(L, "xpr_error", i32, [vp, vp, i32, vp, vp, i32, u64, C.c_float, i32, i32, vp, vp])
    _sig(L, "xpr_preprocess_minmax", i32, [vp, vp, u64, vp, vp])
    _sig(L, "xpr_preprocess_apply", i32, [vp, vp, vp, i32, u64, i32, vp, i32, vp])
    _sig(L, "xpr_subiteration", i32, [vp, vp, vp, vp, i32, vp, i32, vp, C.c_uint32, C.POINTER(Launch),
                                      C.c_float, i32, vp, vp])
    _sig(L, "xpr_geometry", i32, [C.POINTER(GeomParams), i32, vp, C.POINTER(GeomOut)])
    _sig(L, "xpr_jitter", i32, [C.c_uint32, u64, C.c_float, vp])
    _sig(L, "xpr_batch_create", i32, [vp, C.POINTER(BatchProblem), C.c_uint32, C.POINTER(BatchOpts), vp,
                                      C.POINTER(vp)])
    _sig(L, "xpr_batch_run", i32, [vp, vp])
    _sig(L, "xpr_batch_step", i32, [vp, C.c_uint32, vp])
    _sig(L, "xpr_batch_steps", C.c_uint32, [vp])
    _sig(L, "xpr_batch_schedule", i32, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_int32), C.POINTER(C.c_double)])
    _sig(L, "xpr_batch_destroy", i32, [vp])
    _lib = L
    return L


def check(status: int, what: str = "") -> None:
    if status != XPR_OK:
        msg = lib().xpr_last_error().decode(errors="replace")
        raise XprError("%s failed (status %d): %s" % (what or "xpr call", status, msg))


def exported_symbols(header: str) -> list[str]:
    """Names of the functions declared in a C header (`int xpr_x(` style)."""
    import re
    with open(header) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(xpr_[a-z0-9_]+)\s*\(", text)))
