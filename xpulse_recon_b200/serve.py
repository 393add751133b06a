"""Continuous-batching request loop (``xpr_serve_*`` of include/xpr.h).

Each request is a naive reconstruction of raw projections with parameters in the
XPRecon JSON schema; requests of any size are admitted by device memory and advance
together, one sub-iteration per tick.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import _lib
from ._lib import check, lib

QUEUED, ACTIVE, DONE, FAILED = 0, 1, 2, 3


class ServeOpts(C.Structure):
    _fields_ = [("arith", C.c_int32), ("storage", C.c_int32), ("mem_budget", C.c_uint64),
                ("max_active", C.c_uint32), ("image_storage_set", C.c_int32), ("image_storage", C.c_int32)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("error", C.c_int32), ("submit_s", C.c_double), ("admit_s", C.c_double),
                ("done_s", C.c_double), ("pairs", C.c_uint64), ("device_bytes", C.c_uint64)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("ticks", C.c_uint64), ("pairs", C.c_uint64), ("active", C.c_uint32), ("queued", C.c_uint32),
                ("bytes_in_use", C.c_uint64), ("peak_bytes", C.c_uint64)]


def _signatures(L):
    vp, i32 = C.c_void_p, C.c_int
    if getattr(L, "_serve_sigs", False):
        return
    L.xpr_serve_create.restype = i32
    L.xpr_serve_create.argtypes = [vp, C.POINTER(ServeOpts), C.POINTER(vp)]
    L.xpr_serve_submit.restype = i32
    L.xpr_serve_submit.argtypes = [vp, C.c_char_p, vp, C.c_int64, C.c_uint32, C.c_uint32, vp, C.c_uint64,
                                   C.POINTER(C.c_uint64)]
    L.xpr_serve_poll.restype = i32
    L.xpr_serve_poll.argtypes = [vp, C.c_uint64, C.POINTER(RequestInfo)]
    L.xpr_serve_wait.restype = i32
    L.xpr_serve_wait.argtypes = [vp, C.c_uint64, C.c_double, C.POINTER(RequestInfo)]
    L.xpr_serve_stats_get.restype = i32
    L.xpr_serve_stats_get.argtypes = [vp, C.POINTER(ServeStats)]
    L.xpr_serve_destroy.restype = i32
    L.xpr_serve_destroy.argtypes = [vp]
    L._serve_sigs = True


def grid_of(params: dict, width: int, height: int) -> tuple:
    """(vwidth, vheight) of the reconstruction grid the reference derives (geometry.hpp:55-60)."""
    from .projector import geometry
    d = params.get("detector", {})
    g = params.get("geometry", {})
    _, out = geometry(so=g.get("so", 100.0), sd=g.get("sd", 1000.0), heli_offset=g.get("heli_offset", 0.0),
                      px=d.get("px", 0.1), dwidth=width, dheight=height, projections=1, sit=1)
    return int(out["vwidth"]), int(out["vheight"])


class Server:
    """xpr_server handle; keeps every submitted request's raw images and output alive."""

    def __init__(self, ctx, arith: int = _lib.STRICT, storage: int = _lib.F32, mem_budget: int = 0,
                 max_active: int = 0, image_storage: int = None):
        """storage: the ratios' dtype, and the images' unless image_storage is given."""
        L = lib()
        _signatures(L)
        self.ctx = ctx
        h = C.c_void_p()
        o = ServeOpts(arith, storage, mem_budget, max_active, int(image_storage is not None),
                      storage if image_storage is None else image_storage)
        check(L.xpr_serve_create(ctx.handle, C.byref(o), C.byref(h)), "xpr_serve_create")
        self.handle = h
        self._keep = {}

    def submit(self, params: dict, raw: np.ndarray, out: np.ndarray = None) -> int:
        """raw: (projections, height, width) float32 intensities; out: optional float32
        array of the grid's size for the result (page-locked buffers -- e.g. numpy views
        of pinned torch tensors -- are copied without staging).  Returns the ticket."""
        raw = np.ascontiguousarray(raw, np.float32)
        P, H, W = raw.shape
        vw, vh = grid_of(params, W, H)
        if out is None:
            out = np.full(vw * vh * vw, np.nan, np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.size >= vw * vh * vw
        t = C.c_uint64()
        check(lib().xpr_serve_submit(self.handle, json.dumps(params).encode(), raw.ctypes.data, P, W, H,
                                     out.ctypes.data, out.size, C.byref(t)), "xpr_serve_submit")
        self._keep[t.value] = (raw, out)
        return t.value

    def result(self, ticket: int) -> np.ndarray:
        return self._keep[ticket][1]

    def poll(self, ticket: int) -> RequestInfo:
        info = RequestInfo()
        check(lib().xpr_serve_poll(self.handle, ticket, C.byref(info)), "xpr_serve_poll")
        return info

    def wait(self, ticket: int, timeout: float = -1.0) -> RequestInfo:
        info = RequestInfo()
        check(lib().xpr_serve_wait(self.handle, ticket, timeout, C.byref(info)), "xpr_serve_wait")
        return info

    def stats(self) -> ServeStats:
        st = ServeStats()
        check(lib().xpr_serve_stats_get(self.handle, C.byref(st)), "xpr_serve_stats_get")
        return st

    def close(self) -> None:
        if self.handle:
            lib().xpr_serve_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
