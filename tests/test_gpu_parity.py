"""GPU parity: the sm_100a kernels through the C ABI against the CPU oracle.

Integer work (forward sums, pixel indices) must be bit-exact; the floating-point
steps (error ratio, backward update) are also bit-exact because both sides
implement the same operation-by-operation contracts (xpr_math.cuh /
xpr_oracle.h) -- the tolerance for the FP32 path is therefore 0 ulp.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from tests.cases import (CASES, assert_same_bits, make_case, oracle_backward, oracle_forward,  # noqa: E402
                         ratio_from)
from xpulse_recon_b200 import _lib  # noqa: E402
from xpulse_recon_b200.projector import Reconstruction  # noqa: E402

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host_u32(t):
    return t.cpu().numpy().view(np.uint32)


def operator_for(ctx, c, arith, compat_pad=0, lists=None, nan_skip=False):
    r = Reconstruction(ctx, arith=arith)
    r.compat_pad = compat_pad
    n_img = c["Pc"] if lists is None else max(int(np.max(lists[1])) + 1, c["Pc"])
    r.set_image_parameters(c["Wd"], c["Hd"], n_img)
    r.set_volume_parameters(c["vmin"], c["vmax"], [c["go"].vx] * 3)
    r.set_angle_number(n_img, c["M"])
    r.set_image_offset((c["row_offset"], c["rows"]))
    r._origin = tuple(c["origin"])
    pd = c["pd"] if lists is None else c["pd_all"]
    r.set_projdata_buffer(dev(pd))
    if lists is not None:
        r.set_angle_list(dev(lists[0].astype(np.int16)), dev(lists[1].astype(np.int16)), nan_skip)
    return r, n_img


def gpu_forward(ctx, c, arith, compat_pad=0, lists=None):
    r, n_img = operator_for(ctx, c, arith, compat_pad, lists)
    vol = dev(c["vol"])
    sums = torch.zeros(n_img * c["Wd"] * c["rows"], dtype=torch.int32, device="cuda")
    r.set_volume_buffer(vol)
    r.set_sum_images_buffer(sums)
    r.forward()
    torch.cuda.synchronize()
    return host_u32(sums)


def gpu_backward(ctx, c, ratio, arith, compat_pad=0, lists=None, nan_skip=False, ratio_dtype=torch.float32):
    r, n_img = operator_for(ctx, c, arith, compat_pad, lists, nan_skip)
    vol = dev(c["vol"])
    rt = dev(ratio.astype(np.float32)).to(ratio_dtype)
    r.set_volume_buffer(vol)
    r.set_sum_images_buffer(rt)
    r.set_ratio_buffer(rt)
    r.backward()
    torch.cuda.synchronize()
    return vol.cpu().numpy()


@pytest.mark.parametrize("arith", [O.STRICT, O.FAST])
@pytest.mark.parametrize("name", sorted(CASES))
def test_forward_bit_exact(ctx, name, arith):
    c = make_case(name, sit=1, seed=11)
    np.testing.assert_array_equal(gpu_forward(ctx, c, arith), oracle_forward(c, arith))


@pytest.mark.parametrize("arith", [O.STRICT, O.FAST])
def test_forward_compat_padding(ctx, ref, arith):
    """The reference NDRange's padding work-items (kernel.hpp:73-81) reproduced on demand."""
    c = make_case("plain48", sit=3, seed=12)
    got = gpu_forward(ctx, c, arith, compat_pad=1)
    np.testing.assert_array_equal(got, oracle_forward(c, arith, compat_pad=1))
    if arith == O.STRICT:  # and against the reference's own kernel
        sums_ref = np.zeros_like(got)
        O.ref_forward(c["vol"], sums_ref, c["pd"], c["Wd"], c["Hd"], c["origin"], c["Pc"], c["M"], c["vmin"],
                      c["vmax"], (0, c["rows"]), [c["go"].vx] * 3)
        np.testing.assert_array_equal(got, sums_ref)


@pytest.mark.parametrize("arith", [O.STRICT, O.FAST])
@pytest.mark.parametrize("name", ["offsets64", "modules2", "ragged"])
def test_forward_row_window_and_box(ctx, name, arith):
    base = make_case(name)
    H = base["Hd"]
    c = make_case(name, sit=0, seed=13, row_window=(H // 4, H // 2),
                  box=((3, 5, 1), (base["W"] - 2, base["go"].vheight - 4, base["W"] - 5)))
    np.testing.assert_array_equal(gpu_forward(ctx, c, arith), oracle_forward(c, arith))


@pytest.mark.parametrize("arith", [O.STRICT, O.FAST])
def test_forward_backward_with_angle_lists(ctx, arith):
    c = make_case("offsets64", sit=1, seed=14)
    gp, go, W = c["gp"], c["go"], c["W"]
    layer = 21
    lm = np.zeros(64, np.uint16)
    li = np.zeros(64, np.uint16)
    n = O.lib().orc_cull_layer(O.C.byref(gp), O.C.byref(go), c["pd_all"], 1, layer, 0, lm, li)
    lists = (lm[:n].copy(), li[:n].copy())
    c["vmin"], c["vmax"] = (0, layer, 0), (W, layer + 3, W)
    c["vol"] = c["vol"][: 3 * W * W].copy()
    np.testing.assert_array_equal(gpu_forward(ctx, c, arith, lists=lists),
                                  oracle_forward(c, arith, lists=lists, pd=c["pd_all"]))
    ratio = c["images"][: (c["Pc"] + 1) * c["Wd"] * c["Hd"]].copy()
    ratio[::5] = np.nan
    got = gpu_backward(ctx, c, ratio, arith, lists=lists, nan_skip=True)
    exp = oracle_backward(c, ratio, arith, nan_skip=1, lists=lists, pd=c["pd_all"])
    assert_same_bits(got, exp[: got.size])


@pytest.mark.parametrize("arith", [O.STRICT, O.FAST])
@pytest.mark.parametrize("name", ["plain48", "offsets64", "modules3_rpy", "helical", "widecone"])
def test_backward_bit_exact(ctx, name, arith):
    c = make_case(name, sit=2, seed=15)
    ratio = ratio_from(c, oracle_forward(c, arith))
    got = gpu_backward(ctx, c, ratio, arith)
    exp = oracle_backward(c, ratio, arith)
    assert_same_bits(got[: c["n"]], exp[: c["n"]])


@pytest.mark.parametrize("dt", [torch.bfloat16, torch.float16])
def test_backward_reduced_precision_ratio(ctx, dt):
    """BF16 / FP16 ratio storage: exact against the oracle fed the same rounded ratios."""
    c = make_case("offsets64", sit=2, seed=16)
    ratio = ratio_from(c, oracle_forward(c, O.FAST))
    rounded = torch.from_numpy(ratio).to(dt).to(torch.float32).numpy()
    got = gpu_backward(ctx, c, ratio, O.FAST, ratio_dtype=dt)
    exp = oracle_backward(c, rounded, O.FAST)
    assert_same_bits(got[: c["n"]], exp[: c["n"]])


@pytest.mark.parametrize("mode", [_lib.ERROR_STD, _lib.ERROR_FIRST_1C, _lib.ERROR_1C])
@pytest.mark.parametrize("idt,rdt", [(torch.float32, torch.float32), (torch.bfloat16, torch.bfloat16),
                                     (torch.float32, torch.float16)])
def test_error_bit_exact(ctx, mode, idt, rdt):
    rng = np.random.default_rng(17)
    n = 100_003
    img = rng.uniform(-0.1, 6.0, n).astype(np.float32)
    img[:50] = [0.0, -0.0, 1e-30, np.inf, np.nan] * 10
    sums = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    sums[:64] = [0, 1, 2, 0xFFFFFFFF] * 16
    img_r = torch.from_numpy(img).to(idt).to(torch.float32).numpy()
    exp = sums.copy()
    if mode == _lib.ERROR_STD:
        O.lib().orc_error(img_r, exp, n, 0.729)
    elif mode == _lib.ERROR_FIRST_1C:
        tmp = np.zeros(n, np.float32)
        O.lib().orc_error_first_1c(img_r, tmp, n)
        exp = tmp.view(np.uint32)
    else:
        O.lib().orc_error_1c(img_r, exp, n, 0.729)
    exp_f = torch.from_numpy(exp.view(np.float32).copy()).to(rdt).to(torch.float32).numpy()
    import ctypes as C
    d_img = dev(img).to(idt)
    d_sum = dev(sums.view(np.int32))
    d_ratio = torch.zeros(n, dtype=rdt, device="cuda")
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().xpr_error(ctx.handle, d_img.data_ptr(), {torch.float32: 0, torch.bfloat16: 1}[idt],
                                    d_sum.data_ptr(), d_ratio.data_ptr(),
                                    {torch.float32: 0, torch.bfloat16: 1, torch.float16: 2}[rdt], n, 0.729, mode,
                                    1, res.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    got = d_ratio.to(torch.float32).cpu().numpy()
    assert_same_bits(got, exp_f)
    assert (d_sum.cpu().numpy() == 0).all()  # zero_sum
    finite = np.isfinite(exp.view(np.float32))
    r64 = exp.view(np.float32)[finite].astype(np.float64)
    if rdt == torch.float32:
        assert abs(res.item() - float((r64 ** 2).sum())) <= 1e-9 * float((r64 ** 2).sum()) or not finite.all()


def gpu_naive(ctx, gp_kwargs, images, it, sit, weight, wf, seed, arith, compat_pad):
    """reconstruction_n.hpp:27-88 driven through the operator mirror."""
    from xpulse_recon_b200.projector import geometry
    pd_all, g = geometry(**gp_kwargs)
    P, M = gp_kwargs["projections"], gp_kwargs.get("module_number", 1)
    Pc, W, Hv = g["concurrent"], g["vwidth"], g["vheight"]
    Wd, Hd = gp_kwargs["dwidth"], gp_kwargs["dheight"]
    r = Reconstruction(ctx, seed=seed, arith=arith)
    r.compat_pad = compat_pad
    n = W * Hv * W
    vol = torch.ones(O.ndrange(n) if compat_pad else n, dtype=torch.float32, device="cuda")
    sums = torch.full((Pc * Wd * Hd,), 1 << 22, dtype=torch.int32, device="cuda")
    subsets = []
    for s in range(sit):
        idx = [s + k * sit for k in range(Pc)]
        subsets.append((dev(images.reshape(P, -1)[idx].ravel()),
                        dev(np.concatenate([pd_all[i * M:(i + 1) * M] for i in idx]))))
    r.set_sum_images_buffer(sums)
    r.set_volume_buffer(vol)
    r.set_image_parameters(Wd, Hd, Pc)
    r.set_volume_parameters((0, 0, 0), (W, Hv, W), [g["vx"]] * 3)
    r.set_image_offset((0, Hd))
    r.set_angle_number(Pc, M)
    w = np.float32(weight)
    for mit in range(it):
        r.set_weight(float(w))
        for s in range(sit):
            r.set_origin(g["orig"], [g["vx"]] * 3)
            r.set_images_buffer(subsets[s][0])
            r.set_projdata_buffer(subsets[s][1])
            if s > 0 or mit > 0:
                r.forward()
            r.error()
            r.backward()
            sums.zero_()
        w = np.float32(w * np.float32(wf))
    torch.cuda.synchronize()
    return vol.cpu().numpy()


@pytest.mark.parametrize("arith,compat_pad", [(O.STRICT, 0), (O.STRICT, 1), (O.FAST, 0)])
def test_naive_reconstruction_bit_exact(ctx, arith, compat_pad):
    """A whole seeded naive reconstruction (it=2, sit=4): identical volume, bit for bit."""
    kw = dict(dwidth=40, dheight=32, projections=36, sit=4, rx=1.0, sx=-0.5, sy=0.8)
    rng = np.random.default_rng(18)
    images = rng.uniform(0.05, 1.5, 36 * 40 * 32).astype(np.float32)
    got = gpu_naive(ctx, kw, images, 2, 4, 1.0, 0.9, 77, arith, compat_pad)
    gp = O.geom_params(**kw)
    rp = O.ReconParams(2, 4, 1.0, 0.9, 77, arith, compat_pad)
    exp = np.zeros(got.size, np.float32)
    assert O.lib().orc_recon_naive(O.C.byref(gp), O.C.byref(rp), images, exp) == 0
    assert_same_bits(got, exp)
    assert np.isfinite(got).mean() > 0.5


@pytest.mark.parametrize("arith", [O.STRICT, O.FAST])
def test_forward_medium_size_and_slab_split(ctx, arith):
    """160^3 grid, 40 projections: bit-exact against the oracle, and a forward split into
    y-slabs (the layer / chunk streaming of methods 1a/1b/2) equals one launch."""
    c = make_case("plain48", seed=19)
    gp = O.geom_params(dwidth=160, dheight=160, projections=80, sit=2, rx=2.5, sy=-1.0)
    pd_all, go = O.geometry(gp)
    c.update(gp=gp, go=go, pd_all=pd_all, Pc=40, M=1, W=160, Wd=160, Hd=160, rows=160, row_offset=0,
             pd=O.subset_projdata(pd_all, 80, 2, 1, 1, 40), vmin=(0, 0, 0), vmax=(160, 160, 160))
    rng = np.random.default_rng(20)
    c["vol"] = rng.uniform(0, 1, 160 ** 3).astype(np.float32)
    c["origin"] = [float(np.float32(go.orig[i]) + np.float32(0.3 * go.vx)) for i in range(3)]
    whole = gpu_forward(ctx, c, arith)
    np.testing.assert_array_equal(whole, oracle_forward(c, arith))
    acc = np.zeros_like(whole)
    for y0, y1 in ((0, 37), (37, 100), (100, 160)):
        cc = dict(c, vmin=(0, y0, 0), vmax=(160, y1, 160), vol=c["vol"][y0 * 160 * 160: y1 * 160 * 160])
        acc += gpu_forward(ctx, cc, arith)
    np.testing.assert_array_equal(acc, whole)


def test_forward_linearity_at_full_detector(ctx):
    """768 x 768 detector, 72 projections over a 256^3 box of the 768^3 grid:
    forward(a) + forward(b) == forward(a + b) exactly when a, b are multiples of 2^-22."""
    gp = O.geom_params(dwidth=768, dheight=768, projections=720, sit=10, rx=1.5, sx=-2.0, sy=3.0)
    pd_all, go = O.geometry(gp)
    pd = O.subset_projdata(pd_all, 720, 10, 1, 3, 72)
    rng = np.random.default_rng(21)
    q = np.float32(2.0 ** -22)
    a = (rng.integers(0, 1 << 20, 256 ** 3).astype(np.float32) * q).astype(np.float32)
    b = (rng.integers(0, 1 << 20, 256 ** 3).astype(np.float32) * q).astype(np.float32)
    base = dict(gp=gp, go=go, pd_all=pd_all, pd=pd, Pc=72, M=1, W=768, Wd=768, Hd=768, rows=768, row_offset=0,
                vmin=(256, 256, 256), vmax=(512, 512, 512),
                origin=[float(np.float32(go.orig[i]) + np.float32(0.41 * go.vx)) for i in range(3)])
    fa = gpu_forward(ctx, dict(base, vol=a), O.FAST)
    fb = gpu_forward(ctx, dict(base, vol=b), O.FAST)
    fab = gpu_forward(ctx, dict(base, vol=(a + b).astype(np.float32)), O.FAST)
    np.testing.assert_array_equal(fa + fb, fab)
    assert fab.astype(np.uint64).sum() > 0
