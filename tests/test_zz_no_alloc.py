"""xpr_subiteration_static: one sub-iteration for callers that cannot allocate device
memory while they run (a host application that owns the device budget and hands the
library only inputs and outputs, or a frame loop that must not stall on or fail in an
allocation).  Its detector scratch is a fixed device array inside the library, so its
results must equal those of xpr_subiteration, whose scratch the caller allocates.

Collected last (file name) so that a run stopping at the first failure has already run
every other test; self-contained, so it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tests.cases import assert_same_bits  # noqa: E402
from xpulse_recon_b200 import _lib  # noqa: E402
from xpulse_recon_b200.projector import Context, geometry  # noqa: E402

pytestmark = pytest.mark.gpu


def _signatures(L):
    vp, i32 = C.c_void_p, C.c_int
    L.xpr_subiteration_static.restype = i32
    L.xpr_subiteration_static.argtypes = [vp, vp, vp, i32, vp, C.c_uint32, C.POINTER(_lib.Launch), C.c_float, i32, vp]
    L.xpr_subiteration_static_capacity.restype = C.c_uint64
    L.xpr_subiteration_static_capacity.argtypes = []


TORCH_DT = {_lib.F32: torch.float32, _lib.BF16: torch.bfloat16, _lib.F16: torch.float16}


@pytest.mark.parametrize("image_dtype,arith,lists", [
    (_lib.F32, _lib.FAST, False),
    (_lib.F32, _lib.STRICT, False),
    (_lib.BF16, _lib.FAST, False),
    (_lib.F16, _lib.STRICT, False),
    (_lib.F32, _lib.STRICT, True),   # ForwardH / BackwardH index lists
])
def test_static_scratch_subiteration_matches_allocating_entry(image_dtype, arith, lists):
    L = _lib.lib()
    _signatures(L)
    ctx = Context(0)
    try:
        kw = dict(dwidth=48, dheight=40, projections=24, sit=3, rx=1.0, sy=0.5)
        pd_all, g = geometry(**kw)
        W, Hv, Pc, Wd, Hd, S = g["vwidth"], g["vheight"], g["concurrent"], kw["dwidth"], kw["dheight"], kw["sit"]
        n = Pc * Wd * Hd
        assert n <= L.xpr_subiteration_static_capacity()
        rng = np.random.default_rng(0)
        raw = rng.uniform(0.05, 0.95, (kw["projections"], Hd, Wd)).astype(np.float32)
        meas = (-np.log(raw)).astype(np.float32)
        imgs = [torch.from_numpy(np.ascontiguousarray(meas[[s + k * S for k in range(Pc)]]).ravel()).cuda()
                .to(TORCH_DT[image_dtype]) for s in range(S)]
        pds = [torch.from_numpy(np.ascontiguousarray(pd_all[[s + k * S for k in range(Pc)]])).cuda() for s in range(S)]
        keep = []
        if lists:  # every entry but one, in reverse order: entry i -> ProjData and image slot Pc - 1 - i
            order = np.arange(Pc - 1, 0, -1, dtype=np.uint16)
            keep = [torch.from_numpy(order.copy()).cuda(), torch.from_numpy(order.copy()).cuda()]
        vol_alloc = torch.ones(W * Hv * W, dtype=torch.float32, device="cuda")
        vol_static = torch.ones_like(vol_alloc)
        sums = torch.full((n,), 1 << 22, dtype=torch.int32, device="cuda")  # the caller's scratch
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        for call, sit in enumerate((0, 1)):  # two calls in a row: the first (no forward), then a full one
            Ld = _lib.Launch()
            Ld.vmin[:] = [0, 0, 0]
            Ld.vmax[:] = [W, Hv, W]
            Ld.origin[:] = [g["orig"][i] + 0.3 * g["vx"] * (call + 1) for i in range(3)]
            Ld.voxel[:] = [g["vx"]] * 3
            Ld.det_w, Ld.rows, Ld.row_offset, Ld.n_angles, Ld.modules = Wd, Hd, 0, Pc, 1
            Ld.arith = arith
            if lists:
                Ld.list_mvp, Ld.list_img, Ld.n_list = keep[0].data_ptr(), keep[1].data_ptr(), keep[0].numel()
            first = 1 if call == 0 else 0
            if first:
                sums.fill_(1 << 22)
            _lib.check(L.xpr_subiteration(ctx.handle, vol_alloc.data_ptr(), sums.data_ptr(), imgs[sit].data_ptr(),
                                          image_dtype, sums.data_ptr(), _lib.F32, pds[sit].data_ptr(), Pc,
                                          C.byref(Ld), 1.0, first, None, stream), "xpr_subiteration")
            _lib.check(L.xpr_subiteration_static(ctx.handle, vol_static.data_ptr(), imgs[sit].data_ptr(),
                                                 image_dtype, pds[sit].data_ptr(), Pc, C.byref(Ld), 1.0, first,
                                                 stream), "xpr_subiteration_static")
            torch.cuda.synchronize()
            # the tolerance of this suite's FP32 path: identical bits (NaN positions identical)
            assert_same_bits(vol_static.cpu().numpy(), vol_alloc.cpu().numpy())
        assert np.isfinite(vol_static.cpu().numpy()).mean() > 0.5

        # a sub-iteration larger than the static scratch is refused, before any GPU work
        Lbig = _lib.Launch()
        Lbig.vmin[:] = [0, 0, 0]
        Lbig.vmax[:] = [W, Hv, W]
        Lbig.voxel[:] = [g["vx"]] * 3
        Lbig.det_w, Lbig.rows, Lbig.n_angles, Lbig.modules = 4096, 4096, 1, 1
        rc = L.xpr_subiteration_static(ctx.handle, vol_static.data_ptr(), imgs[0].data_ptr(), image_dtype,
                                       pds[0].data_ptr(), Pc, C.byref(Lbig), 1.0, 1, stream)
        assert rc == _lib.ERR_CAP
        assert b"static scratch" in L.xpr_last_error()
    finally:
        ctx.close()
