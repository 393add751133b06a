"""Edge cases of the operators on the GPU against the CPU oracle (tolerance 0 ulp):
one-voxel boxes, a box at the far corner of the grid, no projections (every voxel's
count is 0, so the update is 0/0 = NaN as in the reference), empty error calls, and
arguments the C ABI must refuse before any GPU work."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from tests.cases import assert_same_bits, make_case, oracle_backward, oracle_forward, ratio_from  # noqa: E402
from tests.test_gpu_parity import gpu_backward, gpu_forward  # noqa: E402
from xpulse_recon_b200 import _lib  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("arith", [O.STRICT, O.FAST])
@pytest.mark.parametrize("box", [((10, 10, 10), (11, 11, 11)), ((47, 0, 0), (48, 1, 48)), ((30, 40, 30), (48, 48, 48))])
def test_small_and_corner_boxes(ctx, arith, box):
    c = make_case("plain48", sit=1, seed=21, box=box)
    sums = gpu_forward(ctx, c, arith)
    np.testing.assert_array_equal(sums, oracle_forward(c, arith))
    ratio = ratio_from(c, oracle_forward(c, arith))
    assert_same_bits(gpu_backward(ctx, c, ratio, arith), oracle_backward(c, ratio, arith))


def test_no_projections(ctx):
    c = make_case("offsets64", sit=1, seed=22)
    c1 = dict(c)
    c1["Pc"] = 0  # n_angles = 0: no (voxel, projection) pair, so every update is 0 / 0
    ratio = np.zeros(64 * 40, np.float32)
    got = gpu_backward(ctx, c1, ratio, O.FAST)
    assert np.isnan(got[:c["n"]]).all()  # the buffer's padding past n is not part of the box
    assert_same_bits(got, oracle_backward(c1, ratio, O.FAST))


def test_empty_error_and_fill(ctx):
    L = _lib.lib()
    buf = torch.zeros(4, dtype=torch.int32, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.xpr_error(ctx.handle, buf.data_ptr(), _lib.F32, buf.data_ptr(), buf.data_ptr(), _lib.F32, 0, 1.0,
                           _lib.ERROR_STD, 0, None, s), "error")
    _lib.check(L.xpr_fill_u32(ctx.handle, buf.data_ptr(), 7, 0, s), "fill")
    torch.cuda.synchronize()
    assert (buf.cpu().numpy() == 0).all()


def _launch(**kw):
    d = _lib.Launch()
    d.vmin[:] = kw.get("vmin", [0, 0, 0])
    d.vmax[:] = kw.get("vmax", [8, 8, 8])
    d.voxel[:] = [0.01] * 3
    d.det_w, d.rows, d.n_angles, d.modules = kw.get("det_w", 16), kw.get("rows", 16), kw.get("n_angles", 1), 1
    d.arith = kw.get("arith", _lib.FAST)
    if "n_list" in kw:
        d.list_mvp, d.list_img, d.n_list = kw["lists"][0], kw["lists"][1], kw["n_list"]
    return d


@pytest.mark.parametrize("bad,match", [
    (dict(det_w=(1 << 22) + 1), "2^22"),
    (dict(vmin=[4, 0, 0], vmax=[4, 8, 8]), "vmin < vmax"),
    (dict(n_angles=3), "exceeds the ProjData count"),
    (dict(arith=7), "arith"),
])
def test_invalid_launches_are_refused(ctx, bad, match):
    L = _lib.lib()
    vol = torch.zeros(512, dtype=torch.float32, device="cuda")
    sums = torch.zeros(16 * 16, dtype=torch.int32, device="cuda")
    pd = torch.zeros(2 * 20, dtype=torch.float32, device="cuda")
    d = _launch(**bad)
    rc = L.xpr_forward(ctx.handle, vol.data_ptr(), sums.data_ptr(), pd.data_ptr(), 2, C.byref(d), None)
    assert rc == 1  # XPR_ERR_INVALID
    assert match.encode() in L.xpr_last_error()


def test_too_many_list_entries_are_refused(ctx):
    L = _lib.lib()
    vol = torch.zeros(512, dtype=torch.float32, device="cuda")
    sums = torch.zeros(16 * 16, dtype=torch.int32, device="cuda")
    pd = torch.zeros(20, dtype=torch.float32, device="cuda")
    lm = torch.zeros(70000, dtype=torch.int16, device="cuda")
    d = _launch(n_list=70000, lists=(lm.data_ptr(), lm.data_ptr()))
    rc = L.xpr_forward(ctx.handle, vol.data_ptr(), sums.data_ptr(), pd.data_ptr(), 1, C.byref(d), None)
    assert rc == 1
    assert b"65535" in L.xpr_last_error()


def test_null_buffers_are_refused(ctx):
    L = _lib.lib()
    d = _launch()
    assert L.xpr_forward(ctx.handle, None, None, None, 1, C.byref(d), None) == 1


@pytest.mark.parametrize("nbytes", [4096, 48 << 20])
def test_pinned_host_memory_round_trip(ctx, nbytes):
    """xpr_alloc_pinned below and above the size at which large buffers are mapped with
    huge pages and registered (32 MB): device copies on a stream run from and to it, it
    holds what is written, and xpr_free_pinned releases it."""
    L = _lib.lib()
    hp, hq = C.c_void_p(), C.c_void_p()
    _lib.check(L.xpr_alloc_pinned(ctx.handle, nbytes, C.byref(hp)), "alloc_pinned")
    _lib.check(L.xpr_alloc_pinned(ctx.handle, nbytes, C.byref(hq)), "alloc_pinned")
    try:
        a = np.frombuffer((C.c_uint8 * nbytes).from_address(hp.value), np.uint8)
        b = np.frombuffer((C.c_uint8 * nbytes).from_address(hq.value), np.uint8)
        a[:] = np.random.default_rng(5).integers(0, 256, nbytes, dtype=np.uint8)
        b[:] = 0
        dev = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(L.xpr_upload(ctx.handle, dev.data_ptr(), hp, nbytes, s), "upload")
        _lib.check(L.xpr_download(ctx.handle, hq, dev.data_ptr(), nbytes, s), "download")
        _lib.check(L.xpr_synchronize(ctx.handle, s), "synchronize")
        np.testing.assert_array_equal(a, b)
    finally:
        _lib.check(L.xpr_free_pinned(ctx.handle, hp), "free_pinned")
        _lib.check(L.xpr_free_pinned(ctx.handle, hq), "free_pinned")
