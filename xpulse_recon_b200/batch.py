"""Batched reconstructions: many independent naive reconstructions in lock-step
(``xpr_batch_*`` of include/xpr.h), with PyTorch tensors for device memory.

``Problem.from_raw`` prepares one reconstruction the way the reference's naive method
sees it (geometry.hpp:35-76 + computeMVPs; preprocessing of data_loader.hpp:48-101;
subset-major image order of dataset.hpp:133-140), all on the device through the C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, lib
from .projector import Context, _stream, geometry

_TORCH_DTYPE = None


def torch_dtype(storage: int):
    import torch
    return {_lib.F32: torch.float32, _lib.BF16: torch.bfloat16, _lib.F16: torch.float16}[storage]


@dataclass
class Problem:
    """One naive reconstruction resident on the device."""
    vol: object                    # torch float32 [vheight * vwidth * vwidth]
    images: object                 # torch [sit * per_subset * det_h * det_w], image storage dtype, subset-major
    projdata: object               # torch float32 [sit * per_subset * modules, 20], subset-major
    det_w: int
    det_h: int
    per_subset: int
    modules: int
    sit: int
    it: int
    vwidth: int
    vheight: int
    voxel: float
    orig: tuple
    seed: int = 5489
    weight: float = 1.0
    weight_factor: float = 0.9
    residual: object = None        # optional torch float64 [it * sit]
    extra: dict = field(default_factory=dict)

    @staticmethod
    def from_raw(ctx: Context, raw: np.ndarray, geom: dict, it: int, sit: int, seed: int = 5489,
                 weight: float = 1.0, weight_factor: float = 0.9, storage: int = _lib.F32, mlog: bool = True,
                 fp64_geometry: bool = False, residual: bool = False) -> "Problem":
        """raw: (projections, det_h, det_w) float32 intensities in acquisition order;
        storage: the dtype the preprocessed images are kept in."""
        import torch
        P, H, W = raw.shape
        M = int(geom.get("module_number", 1))
        pd_all, g = geometry(dwidth=W, dheight=H, projections=P, sit=sit, fp64=fp64_geometry, **geom)
        Pc = int(g["concurrent"])
        order = [s + k * sit for s in range(sit) for k in range(Pc)]
        sub_raw = np.ascontiguousarray(raw[order], np.float32)
        pd = np.ascontiguousarray(pd_all.reshape(P, M, 20)[order].reshape(-1, 20))
        d_raw = torch.from_numpy(sub_raw.ravel()).cuda()
        images = torch.empty(d_raw.numel(), dtype=torch_dtype(storage), device="cuda")
        check(lib().xpr_preprocess_apply(ctx.handle, d_raw.data_ptr(), images.data_ptr(), storage, d_raw.numel(),
                                         0, None, int(mlog), _stream()), "xpr_preprocess_apply")
        vw, vh = int(g["vwidth"]), int(g["vheight"])
        vol = torch.ones(vw * vh * vw, dtype=torch.float32, device="cuda")
        res = torch.zeros(it * sit, dtype=torch.float64, device="cuda") if residual else None
        return Problem(vol=vol, images=images, projdata=torch.from_numpy(pd).cuda(), det_w=W, det_h=H,
                       per_subset=Pc, modules=M, sit=sit, it=it, vwidth=vw, vheight=vh, voxel=float(g["vx"]),
                       orig=tuple(float(v) for v in g["orig"]), seed=seed, weight=weight,
                       weight_factor=weight_factor, residual=res, extra={"storage": storage})

    def c_struct(self) -> _lib.BatchProblem:
        p = _lib.BatchProblem()
        p.vol, p.images, p.projdata = self.vol.data_ptr(), self.images.data_ptr(), self.projdata.data_ptr()
        p.det_w, p.det_h, p.per_subset, p.modules = self.det_w, self.det_h, self.per_subset, self.modules
        p.sit, p.it, p.vwidth, p.vheight = self.sit, self.it, self.vwidth, self.vheight
        p.voxel = self.voxel
        p.orig[:] = list(self.orig)
        p.seed, p.weight, p.weight_factor = self.seed, self.weight, self.weight_factor
        p.residual = None if self.residual is None else self.residual.data_ptr()
        return p

    def run_alone(self, ctx: Context, arith: int = _lib.STRICT, storage: int = _lib.F32) -> None:
        """The same reconstruction without the batch: one xpr_subiteration per
        sub-iteration (reconstruction_n.hpp:65-76), from a fresh volume of 1.0;
        storage is the ratio's dtype (the images keep theirs)."""
        import torch
        L = lib()
        self.vol.fill_(1.0)
        E = self.per_subset * self.modules
        npix = self.per_subset * self.det_w * self.det_h
        sums = torch.full((npix,), 1 << 22, dtype=torch.int32, device="cuda")  # FIXED_ONE
        ratio = torch.empty(npix, dtype=torch_dtype(storage), device="cuda")
        steps = self.it * self.sit
        jit = np.zeros(3 * steps, np.float32)
        check(L.xpr_jitter(self.seed, jit.size, self.voxel, jit.ctypes.data), "xpr_jitter")
        w = np.float32(self.weight)
        isz = self.images.element_size()
        idt = {torch.float32: _lib.F32, torch.bfloat16: _lib.BF16, torch.float16: _lib.F16}[self.images.dtype]
        for k in range(steps):
            s = k % self.sit
            d = _lib.Launch()
            d.vmax[:] = [self.vwidth, self.vheight, self.vwidth]
            d.origin[:] = [float(np.float32(self.orig[c]) + jit[3 * k + c]) for c in range(3)]
            d.voxel[:] = [self.voxel] * 3
            d.det_w, d.rows, d.n_angles, d.modules, d.arith = self.det_w, self.det_h, self.per_subset, \
                self.modules, arith
            res = None if self.residual is None else self.residual.data_ptr() + 8 * k
            check(L.xpr_subiteration(ctx.handle, self.vol.data_ptr(), sums.data_ptr(),
                                     self.images.data_ptr() + s * npix * isz, idt, ratio.data_ptr(), storage,
                                     self.projdata.data_ptr() + s * E * 80, E, C.byref(d), float(w), int(k == 0),
                                     res, _stream()), "xpr_subiteration")
            if s == self.sit - 1:
                w = np.float32(w * np.float32(self.weight_factor))


class Batch:
    """xpr_batch handle over a list of Problems (kept alive with it)."""

    def __init__(self, ctx: Context, problems: list, arith: int = _lib.STRICT, storage: int = _lib.F32,
                 init_volume: bool = True, use_graph: bool = True, autotune: bool = True, fwd_splits: int = 0,
                 bwd_column: int = 0, ctas_per_sm: int = 0, image_storage: int = None, fwd_layers: int = 0):
        """storage: the ratio's dtype, and the images' unless image_storage is given;
        fwd_layers: the forward brick's layers (0: automatic or tuned; 8, or 16 in STRICT)."""
        self.ctx, self.problems = ctx, list(problems)
        arr = (_lib.BatchProblem * len(self.problems))(*[p.c_struct() for p in self.problems])
        o = _lib.BatchOpts(arith, storage, int(init_volume), int(use_graph), int(autotune), fwd_splits, bwd_column,
                           ctas_per_sm, int(image_storage is not None),
                           storage if image_storage is None else image_storage, fwd_layers)
        h = C.c_void_p()
        check(lib().xpr_batch_create(ctx.handle, arr, len(self.problems), C.byref(o), _stream(), C.byref(h)),
              "xpr_batch_create")
        self.handle = h

    @property
    def steps(self) -> int:
        return int(lib().xpr_batch_steps(self.handle))

    def run(self, stream=None) -> None:
        check(lib().xpr_batch_run(self.handle, _stream() if stream is None else stream), "xpr_batch_run")

    def step(self, k: int, stream=None) -> None:
        check(lib().xpr_batch_step(self.handle, k, _stream() if stream is None else stream), "xpr_batch_step")

    def schedule(self) -> dict:
        s, ly, c, n, t = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        check(lib().xpr_batch_schedule(self.handle, C.byref(s), C.byref(ly), C.byref(c), C.byref(n), C.byref(t)),
              "xpr_batch_schedule")
        return {"fwd_splits": s.value, "fwd_layers": ly.value, "bwd_column": c.value, "ctas_per_sm": n.value,
                "tuned_ms": t.value}

    def close(self) -> None:
        if self.handle:
            lib().xpr_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
