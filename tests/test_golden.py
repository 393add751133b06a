"""Golden vectors of the reference's own kernels (tests/golden/ref_kernels.npz, made by
tests/golden/make_golden.py from KernelForward/Error/Backward(.H).cl compiled for the CPU).

CPU tests replay every record through the oracle (STRICT contract, the reference's
padded NDRange); GPU tests replay them through the C ABI.  Tolerance: none -- the
forward sums are integers and the STRICT contract reproduces the reference's IEEE
single-precision arithmetic, so every output must be bit-identical (any NaN matches
any NaN at the same position)."""
import ctypes as C
import json

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as G
from tests.cases import assert_same_bits, launch


def _oracle_kernels(c):
    L, keep = launch(c, O.STRICT, compat_pad=1)
    sums = np.zeros(c["sums"].size, np.uint32)
    O.forward(c["vol"], sums, c["pd"], L)
    ratio = sums.copy()
    O.error(c["images"], ratio, float(c["weight"]))
    vol = c["vol"].copy()
    O.backward(vol, ratio.view(np.float32), c["pd"], L)
    return sums, ratio, vol


# ----------------------------------------------------------------------------- CPU: the oracle
@pytest.mark.parametrize("name", G.KERNEL_CASES)
def test_oracle_reproduces_golden_kernels(name):
    c = G.case(name)
    sums, ratio, vol = _oracle_kernels(c)
    assert c["sums"].sum(dtype=np.uint64) > 0
    np.testing.assert_array_equal(sums, c["sums"])
    np.testing.assert_array_equal(ratio, c["ratio"])
    assert_same_bits(vol, c["vol_out"])


def test_oracle_reproduces_golden_culled_layer():
    c = G.case("lists")
    L, keep = O.make_launch(c["vmin"], c["vmax"], c["origin"], [c["go"].vx] * 3, c["Wd"], c["Hd"], 0, c["Pc"], 1,
                            compat_pad=1, list_mvp=c["list_mvp"], list_img=c["list_img"])
    sums = np.zeros_like(c["sums"])
    O.forward(c["vol"], sums, c["pd_all"], L)
    np.testing.assert_array_equal(sums, c["sums"])
    L.nan_skip = 1
    vol = c["vol"].copy()
    O.backward(vol, c["ratio_in"], c["pd_all"], L)
    assert_same_bits(vol, c["vol_out"])


def _recon_inputs():
    z = G.load()
    dw, dh, P = (int(v) for v in z["recon.geom"])
    rx, sx, sy = (float(v) for v in z["recon.offsets"])
    it, sit, seed = (int(v) for v in z["recon.params"])
    w, wf = (float(v) for v in z["recon.weights"])
    return dict(dwidth=dw, dheight=dh, projections=P, rx=rx, sx=sx, sy=sy), dict(it=it, sit=sit, seed=seed,
                                                                                 weight=w, weight_factor=wf)


def test_oracle_reproduces_golden_reconstruction():
    geom, rc = _recon_inputs()
    z = G.load()
    raw = z["recon.raw"]
    imgs = np.ascontiguousarray(raw, np.float32).ravel().copy()
    O.lib().orc_preprocess(imgs, imgs.size, 0, 0.0, 0.0, 1)
    gp = O.geom_params(sit=rc["sit"], **geom)
    rp = O.ReconParams(rc["it"], rc["sit"], rc["weight"], rc["weight_factor"], rc["seed"], O.STRICT, 1)
    n = z["recon.vol_out"].size
    out = np.zeros(O.ndrange(n), np.float32)
    assert O.lib().orc_recon_naive(C.byref(gp), C.byref(rp), imgs, out) == 0
    assert_same_bits(out[:n], z["recon.vol_out"])


def test_golden_file_is_what_the_script_makes(ref):
    """Regenerating the fixture from the reference kernels gives the committed bytes."""
    from tests.golden import make_golden as M
    rng = np.random.default_rng(2024)
    z = G.load()

    def same(v, key):
        a, b = np.asarray(v), z[key]
        assert a.dtype == b.dtype and a.shape == b.shape, key
        assert a.tobytes() == b.tobytes(), key

    for name, spec in M.KERNEL_CASES.items():
        for k, v in M._kernel_case(name, spec, rng).items():
            same(v, f"{name}.{k}")
    for k, v in M._lists_case(rng).items():
        same(v, f"lists.{k}")
    for k, v in M._recon_case(rng).items():
        same(v, f"recon.{k}")


# ----------------------------------------------------------------------------- GPU: the product
@pytest.mark.gpu
@pytest.mark.parametrize("name", G.KERNEL_CASES)
def test_gpu_reproduces_golden_kernels(ctx, name):
    import torch
    from xpulse_recon_b200.projector import Reconstruction
    c = G.case(name)
    r = Reconstruction(ctx, arith=O.STRICT)
    r.compat_pad = 1
    r.set_image_parameters(c["Wd"], c["Hd"], c["Pc"])
    r.set_volume_parameters(c["vmin"], c["vmax"], [c["go"].vx] * 3)
    r.set_angle_number(c["Pc"], c["M"])
    r.set_image_offset((c["row_offset"], c["rows"]))
    r._origin = tuple(c["origin"])
    r.set_weight(float(c["weight"]))
    r.set_image_elements(c["sums"].size)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    vol, sums, imgs = dev(c["vol"]), torch.zeros(c["sums"].size, dtype=torch.int32, device="cuda"), dev(c["images"])
    r.set_projdata_buffer(dev(c["pd"]))
    r.set_volume_buffer(vol)
    r.set_sum_images_buffer(sums)
    r.set_images_buffer(imgs)
    r.forward()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sums.cpu().numpy().view(np.uint32), c["sums"])
    r.error()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sums.cpu().numpy().view(np.uint32), c["ratio"])
    r.backward()
    torch.cuda.synchronize()
    assert_same_bits(vol.cpu().numpy(), c["vol_out"])


@pytest.mark.gpu
def test_gpu_reproduces_golden_culled_layer(ctx):
    import torch
    from xpulse_recon_b200.projector import Reconstruction
    c = G.case("lists")
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    r = Reconstruction(ctx, arith=O.STRICT)
    r.compat_pad = 1
    r.set_image_parameters(c["Wd"], c["Hd"], c["Pc"])
    r.set_volume_parameters(c["vmin"], c["vmax"], [c["go"].vx] * 3)
    r.set_angle_number(c["Pc"], 1)
    r.set_image_offset((0, c["Hd"]))
    r._origin = tuple(c["origin"])
    r.set_projdata_buffer(dev(c["pd_all"]))
    r.set_angle_list(dev(c["list_mvp"].astype(np.int16)), dev(c["list_img"].astype(np.int16)), nan_skip=True)
    vol = dev(c["vol"])
    sums = torch.zeros(c["sums"].size, dtype=torch.int32, device="cuda")
    r.set_volume_buffer(vol)
    r.set_sum_images_buffer(sums)
    r.forward()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sums.cpu().numpy().view(np.uint32), c["sums"])
    ratio = dev(c["ratio_in"])
    r.set_sum_images_buffer(ratio)
    r.set_ratio_buffer(ratio)
    r.backward()
    torch.cuda.synchronize()
    assert_same_bits(vol.cpu().numpy(), c["vol_out"])


@pytest.mark.gpu
def test_gpu_reproduces_golden_reconstruction():
    """A whole naive reconstruction through the drop-in host entry point (the JSON schema
    of the command line), STRICT contract with the reference's NDRange padding."""
    from xpulse_recon_b200 import _lib
    geom, rc = _recon_inputs()
    z = G.load()
    raw = z["recon.raw"]
    cfg = {"recon": {"method": "naive", "it": rc["it"], "sit": rc["sit"], "seed": rc["seed"], "arith": "strict",
                     "geometry": "fp32", "compat_pad": True, "mlog": True, "weight": rc["weight"],
                     "weight_factor": rc["weight_factor"]},
           "geometry": {"so": 100.0, "sd": 1000.0, "angle": 360.0},
           "detector": {"px": 0.1, "rx": geom["rx"], "sx": geom["sx"], "sy": geom["sy"]}}
    L = _lib.lib()
    L.xpr_reconstruct_host.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.c_uint64, C.POINTER(C.c_double)]
    P, H, W = raw.shape
    out = np.full(z["recon.vol_out"].size, np.nan, np.float32)
    secs = C.c_double()
    rc_ = L.xpr_reconstruct_host(json.dumps(cfg).encode(), np.ascontiguousarray(raw).ctypes.data, P, W, H,
                                 out.ctypes.data, out.size, C.byref(secs))
    assert rc_ == 0, L.xpr_last_error()
    assert_same_bits(out, z["recon.vol_out"])
