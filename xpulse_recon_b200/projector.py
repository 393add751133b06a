"""Host-side mirror of the reference's operator seam.

``Reconstruction`` reproduces the protected API of the reference's
``class Reconstruction`` (src/reconstruction.hpp:30-316): buffers and kernel
scalars are bound with ``set_*`` calls named as in the reference, then
``forward()``, ``error()`` and ``backward()`` enqueue the three operators.  Here
they call the sm_100a kernels through the C ABI (include/xpr.h); device memory
and streams come from PyTorch (plumbing only -- no torch op runs on the path).

Differences from the reference, all deliberate:
  * the origin jitter uses a seeded std::mt19937 (the reference seeds it from
    std::random_device, reconstruction.hpp:31-36, so two of its runs differ);
  * ``arith`` selects the arithmetic contract (STRICT = the reference kernels
    under IEEE single precision; FAST = fused contract), see xpr_math.cuh;
  * the ratio may be stored in a separate BF16 / FP16 buffer
    (``set_ratio_buffer``); by default it is written over the sums in FP32 as the
    reference does (KernelError.cl:20-23).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib

_TORCH_DT = None


def _dtype_code(t) -> int:
    import torch
    return {torch.float32: _lib.F32, torch.bfloat16: _lib.BF16, torch.float16: _lib.F16}[t.dtype]


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Context:
    """A device context (replaces gpu::Context, context.hpp:32-113)."""

    def __init__(self, device: int = 0, mem_cap: int = 0):
        self.handle = C.c_void_p()
        check(lib().xpr_create(device, mem_cap, C.byref(self.handle)), "xpr_create")
        self.device = device

    def close(self):
        if self.handle:
            lib().xpr_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().xpr_synchronize(self.handle, None), "xpr_synchronize")


class JitterSource:
    """std::mt19937(seed) feeding std::uniform_real_distribution<float>(0, b)."""

    def __init__(self, seed: int):
        self.seed = int(seed) & 0xFFFFFFFF
        self._canon = np.zeros(0, np.float32)
        self._pos = 0

    def draw(self, b: float) -> float:
        if self._pos >= len(self._canon):
            n = max(64, 2 * len(self._canon))
            buf = np.zeros(n, np.float32)
            check(lib().xpr_jitter(self.seed, n, 1.0, buf.ctypes.data), "xpr_jitter")
            self._canon = buf
        c = self._canon[self._pos]
        self._pos += 1
        return float(np.float32(c) * np.float32(b))


class Reconstruction:
    """Operator seam of reconstruction.hpp:160-316 over the C ABI."""

    def __init__(self, ctx: Context, seed: int = 5489, arith: int = _lib.STRICT):
        self.ctx = ctx
        self.arith = arith
        self.compat_pad = 0
        self.jitter = JitterSource(seed)
        self._images = None
        self._sums = None
        self._ratio = None
        self._volume = None
        self._projdata = None
        self._n_pd = 0
        self._lists = None
        self._nan_skip = 0
        self._size = (0, 0, 0)
        self._vmin = (0, 0, 0)
        self._vmax = (0, 0, 0)
        self._voxel = (0.0, 0.0, 0.0)
        self._origin = (0.0, 0.0, 0.0)
        self._angles = (0, 1)
        self._offset = (0, 0)
        self._weight = 1.0
        self._elements = 0

    # -- buffers (reconstruction.hpp:166-199)
    def set_images_buffer(self, t):
        self._images = t

    def set_sum_images_buffer(self, t):
        self._sums = t

    def set_ratio_buffer(self, t):
        """Separate ratio storage (FP32/BF16/FP16); None = in place over the sums."""
        self._ratio = t

    def set_volume_buffer(self, t):
        self._volume = t

    def set_projdata_buffer(self, t):
        """t: device tensor of n x 20 float32 (ProjData, constants.cl:25-28)."""
        self._projdata = t
        self._n_pd = t.numel() // 20

    def set_angle_list(self, mvp_idx, img_idx, nan_skip: bool = False):
        """ForwardH / BackwardH index lists (device uint16 tensors) or None."""
        self._lists = None if mvp_idx is None else (mvp_idx, img_idx)
        self._nan_skip = int(nan_skip)

    # -- scalars (reconstruction.hpp:208-288)
    def set_image_parameters(self, width: int, height: int, number: int):
        self._size = (int(width), int(height), int(number))
        self._elements = int(width) * int(height) * int(number)

    def set_volume_parameters(self, vmin, vmax, voxel):
        self._vmin, self._vmax, self._voxel = tuple(vmin), tuple(vmax), tuple(voxel)

    def set_angle_number(self, number: int, module_per_angle: int):
        self._angles = (int(number), int(module_per_angle))

    def set_weight(self, weight: float):
        self._weight = float(weight)

    def set_origin(self, origin, randomized_offset=(0.0, 0.0, 0.0)):
        o = [np.float32(origin[i]) for i in range(3)]
        for i in range(3):
            o[i] = np.float32(o[i] + np.float32(self.jitter.draw(randomized_offset[i])))
        self._origin = tuple(float(v) for v in o)

    def set_image_offset(self, offset_rows):
        self._offset = (int(offset_rows[0]), int(offset_rows[1]))

    def set_image_elements(self, elements: int):
        self._elements = int(elements)

    # -- operators (reconstruction.hpp:294-312)
    def launch(self) -> _lib.Launch:
        L = _lib.Launch()
        L.vmin[:] = list(self._vmin)
        L.vmax[:] = list(self._vmax)
        L.origin[:] = list(self._origin)
        L.voxel[:] = list(self._voxel)
        L.det_w = self._size[0]
        L.rows = self._offset[1] if self._offset[1] else self._size[1]
        L.row_offset = self._offset[0]
        L.n_angles, L.modules = self._angles
        if self._lists is not None:
            L.list_mvp = self._lists[0].data_ptr()
            L.list_img = self._lists[1].data_ptr()
            L.n_list = self._lists[0].numel()
        L.arith = self.arith
        L.compat_pad = self.compat_pad
        L.nan_skip = self._nan_skip
        return L

    def forward(self):
        L = self.launch()
        check(lib().xpr_forward(self.ctx.handle, self._volume.data_ptr(), self._sums.data_ptr(),
                                self._projdata.data_ptr(), self._n_pd, C.byref(L), _stream()), "forward")

    def error(self, mode: int = _lib.ERROR_STD, residual=None):
        ratio = self._ratio if self._ratio is not None else self._sums
        rdt = _dtype_code(self._ratio) if self._ratio is not None else _lib.F32
        check(lib().xpr_error(self.ctx.handle, self._images.data_ptr(), _dtype_code(self._images),
                              self._sums.data_ptr(), ratio.data_ptr(), rdt, self._elements, self._weight, mode,
                              0, None if residual is None else residual.data_ptr(), _stream()), "error")

    def backward(self):
        L = self.launch()
        ratio = self._ratio if self._ratio is not None else self._sums
        rdt = _dtype_code(self._ratio) if self._ratio is not None else _lib.F32
        check(lib().xpr_backward(self.ctx.handle, self._volume.data_ptr(), ratio.data_ptr(), rdt,
                                 self._projdata.data_ptr(), self._n_pd, C.byref(L), _stream()), "backward")


def geometry(so=100.0, sd=1000.0, angle=360.0, heli_offset=0.0, px=0.1, rx=0.0, sx=0.0, sy=0.0,
             module_number=1, module_angle_offset=None, module_center_offset_z=0.0,
             dwidth=64, dheight=64, projections=36, sit=4, angle_list=None, mod_offset=None, mod_rpy=None,
             fp64=False):
    """ProjData (float32 [P*M, 20]) and the derived grid (geometry.hpp:35-76, 298-328)."""
    g = _lib.GeomParams()
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
    out = np.zeros((projections * module_number, 20), np.float32)
    go = _lib.GeomOut()
    check(lib().xpr_geometry(C.byref(g), int(fp64), out.ctypes.data, C.byref(go)), "xpr_geometry")
    return out, {"vx": go.vx, "vwidth": go.vwidth, "vheight": go.vheight, "orig": tuple(go.orig),
                 "concurrent": go.concurrent}
