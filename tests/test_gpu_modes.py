"""Whole reconstructions on the GPU through the C ABI / the xprecon command line, one
per memory mode, against the CPU oracle (bit-exact, same seed and contract)."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.cases import assert_same_bits
from xpulse_recon_b200 import _lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "xpulse_recon_b200", "lib", "xprecon")

GEOM = dict(dwidth=40, dheight=32, projections=36, sit=4, rx=1.0, sx=-0.5, sy=0.8)
FLT_MIN, FLT_MAX = np.finfo(np.float32).tiny, np.finfo(np.float32).max


def raw_images(seed=0, P=36, H=32, W=40):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.05, 0.98, (P, H, W)).astype(np.float32)


def config(method, arith="strict", it=2, seed=77, geometry="fp32", **recon):
    cfg = {"recon": {"method": method, "it": it, "sit": GEOM["sit"], "seed": seed, "arith": arith,
                     "geometry": geometry, "mlog": True, "weight": 1.0, "weight_factor": 0.9, **recon},
           "geometry": {"so": 100.0, "sd": 1000.0, "angle": 360.0},
           "detector": {"px": 0.1, "rx": GEOM["rx"], "sx": GEOM["sx"], "sy": GEOM["sy"]}}
    return cfg


def run_host(cfg, raw):
    L = _lib.lib()
    L.xpr_reconstruct_host.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.c_uint64, C.POINTER(C.c_double)]
    P, H, W = raw.shape
    out = np.full(W * H * W, np.nan, np.float32)
    secs = C.c_double()
    rc = L.xpr_reconstruct_host(json.dumps(cfg).encode(), np.ascontiguousarray(raw).ctypes.data, P, W, H,
                                out.ctypes.data, out.size, C.byref(secs))
    assert rc == 0
    return out


def oracle_preprocessed(raw, normalize=False, mlog=True):
    imgs = np.ascontiguousarray(raw, np.float32).ravel().copy()
    mn, mx = C.c_float(FLT_MAX), C.c_float(FLT_MIN)
    if normalize:
        O.lib().orc_minmax_normal(imgs, imgs.size, C.byref(mn), C.byref(mx))
    O.lib().orc_preprocess(imgs, imgs.size, int(normalize), mn.value, mx.value, int(mlog))
    return imgs, mn.value, mx.value


def oracle_params(cfg):
    r = cfg["recon"]
    gp = O.geom_params(**GEOM)
    rp = O.ReconParams(r["it"], r["sit"], r["weight"], r["weight_factor"], r["seed"],
                       O.STRICT if r["arith"] == "strict" else O.FAST, int(r.get("compat_pad", False)))
    return gp, rp


@pytest.mark.parametrize("arith", ["strict", "fast"])
def test_naive_matches_oracle(arith):
    raw = raw_images(1)
    cfg = config("naive", arith)
    got = run_host(cfg, raw)
    imgs, _, _ = oracle_preprocessed(raw)
    gp, rp = oracle_params(cfg)
    exp = np.zeros(got.size, np.float32)
    assert O.lib().orc_recon_naive(C.byref(gp), C.byref(rp), imgs, exp) == 0
    assert_same_bits(got, exp)


@pytest.mark.parametrize("method", ["method_1a", "method_1b"])
@pytest.mark.parametrize("arith", ["strict", "fast"])
def test_layer_streaming_equals_naive(method, arith):
    """methods 1a / 1b stream the volume through the device in y-slabs; integer forward
    sums and per-voxel updates make them bit-identical to the resident naive method."""
    raw = raw_images(2)
    naive = run_host(config("naive", arith), raw)
    streamed = run_host(config(method, arith, slab=5), raw)
    assert_same_bits(streamed, naive)


@pytest.mark.parametrize("cache", [1, 3])
@pytest.mark.parametrize("method", ["method_1b", "method_1c"])
def test_slab_cache_evictions_change_nothing(method, cache):
    """method_1b / 1c keep slabs in a device cache and write a slab back only when its
    buffer is needed: with 1 or 3 buffers for 7 slabs every pass evicts and reloads,
    and the volume must equal the run whose slabs all stay resident."""
    raw = raw_images(4)
    resident = run_host(config(method, "fast", slab=5), raw)
    evicting = run_host(config(method, "fast", slab=5, slab_cache=cache), raw)
    assert np.isfinite(resident).mean() > 0.5
    assert_same_bits(evicting, resident)


@pytest.mark.parametrize("arith", ["strict", "fast"])
def test_method_1c_matches_oracle(arith):
    """method_1c semantics (reconstruction_lplh.hpp): 1/W start, unweighted first error,
    NaN-skipping back projection, every angle of a sub-iteration; the oracle culls per
    layer, the product streams slabs with the full angle list."""
    raw = raw_images(3, P=38)  # 38 projections, sit 4: sub-iterations of 10 and 9 angles
    cfg = config("method_1c", arith, slab=6)
    got = run_host(cfg, raw)
    imgs, _, _ = oracle_preprocessed(raw)
    gp, rp = oracle_params(cfg)
    gp.projections = 38
    exp = np.zeros(got.size, np.float32)
    assert O.lib().orc_recon_1c(C.byref(gp), C.byref(rp), imgs, exp) == 0
    assert_same_bits(got, exp)


@pytest.mark.parametrize("arith", ["strict", "fast"])
def test_method_2_chunks_match_oracle(arith):
    raw = raw_images(4)
    cap = 200_000
    cfg = config("method_2", arith, mem_cap=cap)
    got = run_host(cfg, raw)
    imgs, _, _ = oracle_preprocessed(raw)
    gp, rp = oracle_params(cfg)
    pd_all, go = O.geometry(gp)
    budget = int(cap * 0.98)
    chunks = np.zeros((64, 6), np.int64)
    n = O.lib().orc_plan_chunks(C.byref(gp), C.byref(go), pd_all, budget, budget, 1.0, chunks, 64)
    assert n >= 2
    exp = np.full(got.size, np.nan, np.float32)
    assert O.lib().orc_recon_chunks(C.byref(gp), C.byref(rp), imgs, chunks, n, exp) == 0
    assert_same_bits(got, exp)
    assert np.isfinite(got).any()


def test_bf16_storage_close_to_fp32():
    raw = raw_images(5)
    a = run_host(config("naive", "fast", it=3), raw)
    b = run_host(config("naive", "fast", it=3, storage="bf16"), raw)
    m = np.isfinite(a) & np.isfinite(b)
    assert m.mean() > 0.5 and (np.isnan(a) == np.isnan(b)).all()
    rel = np.linalg.norm(a[m] - b[m]) / np.linalg.norm(a[m])
    assert rel < 2e-2, rel


def phantom_images(P=36, H=32, W=40, seed=11):
    """Consistent data: noise-free transmission images exp(-p) of a seeded ellipsoid
    phantom, p the fixed-point forward projection of the oracle (FAST contract)."""
    rng = np.random.default_rng(seed)
    y, z, x = np.meshgrid(np.arange(H), np.arange(W), np.arange(W), indexing="ij")
    vol = np.zeros((H, W, W), np.float32)
    for _ in range(6):
        c = rng.uniform([H * 0.3, W * 0.3, W * 0.3], [H * 0.7, W * 0.7, W * 0.7])
        a = rng.uniform(3, 10, 3)
        inside = ((y - c[0]) / a[0]) ** 2 + ((z - c[1]) / a[1]) ** 2 + ((x - c[2]) / a[2]) ** 2 <= 1
        vol[inside] += rng.uniform(0.002, 0.01)
    gp = O.geom_params(**dict(GEOM, projections=P))
    pd_all, go = O.geometry(gp)
    v = np.ascontiguousarray(vol.ravel())
    imgs = np.zeros((P, H, W), np.float32)
    L, keep = O.make_launch((0, 0, 0), (W, H, W), list(go.orig), [go.vx] * 3, W, H, 0, P, 1, arith=O.FAST)
    sums = np.zeros(P * W * H, np.uint32)
    O.forward(v, sums, pd_all, L)
    p = sums.astype(np.float64) / 4194304.0
    return np.exp(-p).astype(np.float32).reshape(P, H, W)


def rel_l2(a, b):
    assert (np.isnan(a) == np.isnan(b)).all()
    m = np.isfinite(a)
    return float(np.linalg.norm(a[m] - b[m]) / np.linalg.norm(b[m]))


def test_default_contract_is_close_to_reference_semantics():
    """On consistent projections of a phantom, the default FAST contract stays within
    1e-4 relative L2 of the reference semantics (STRICT contract) after it = 2.  The
    FP64 matrix construction moves pixel assignments by up to ~7e-4 px against the
    reference's FP32 glm construction; its deviation is measured and bounded loosely."""
    raw = phantom_images()
    ref = run_host(config("naive", "strict", it=2, geometry="fp32"), raw)
    fast = run_host(config("naive", "fast", it=2, geometry="fp32"), raw)
    geo = run_host(config("naive", "strict", it=2, geometry="fp64"), raw)
    r_fast, r_geo = rel_l2(fast, ref), rel_l2(geo, ref)
    print("rel L2 vs reference semantics: fast contract %.3g, fp64 geometry %.3g" % (r_fast, r_geo))
    assert r_fast < 1e-4, r_fast
    assert r_geo < 1e-2, r_geo


def write_stack(dirpath, raw):
    L = _lib.lib()
    L.xpr_tiff_write.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32]
    os.makedirs(dirpath, exist_ok=True)
    P, H, W = raw.shape
    for i in range(P):
        img = np.ascontiguousarray(raw[i])
        assert L.xpr_tiff_write(os.path.join(dirpath, "p_%05d.tif" % i).encode(), img.ctypes.data, W, H) == 0


def read_tiff(path):
    L = _lib.lib()
    L.xpr_tiff_read.argtypes = [C.c_char_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    w, h = C.c_uint32(), C.c_uint32()
    assert L.xpr_tiff_read(path.encode(), None, 0, C.byref(w), C.byref(h)) == 0
    out = np.zeros(w.value * h.value, np.float32)
    assert L.xpr_tiff_read(path.encode(), out.ctypes.data, out.size, C.byref(w), C.byref(h)) == 0
    return out.reshape(h.value, w.value)


@pytest.mark.parametrize("method,normalize", [("naive", False), ("method_1b", True)])
def test_cli_end_to_end(tmp_path, method, normalize):
    raw = raw_images(7) * 3.0  # not in (0, 1): exercises normalisation
    write_stack(str(tmp_path / "in"), raw)
    cfg = config(method, "strict", slab=7, normalize=normalize)
    cfg["recon"].update(input=str(tmp_path / "in"), output=str(tmp_path / "out"))
    cf = tmp_path / "cfg.json"
    cf.write_text(json.dumps(cfg))
    r = subprocess.run([CLI, str(cf)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    H, W = raw.shape[1:]
    vol = np.stack([read_tiff(str(tmp_path / "out" / ("layer_%05d.tif" % l))) for l in range(H)])
    imgs, mn, mx = oracle_preprocessed(raw, normalize=normalize)
    gp, rp = oracle_params(cfg)
    exp = np.zeros(W * H * W, np.float32)
    assert O.lib().orc_recon_naive(C.byref(gp), C.byref(rp), imgs, exp) == 0
    if normalize:  # saved layers are scaled back by (max - min) (data_loader.hpp:135-139)
        exp = (exp * np.float32(np.float32(mx) - np.float32(mn))).astype(np.float32)
    assert_same_bits(vol.ravel(), exp)


def test_simulation_matches_oracle(tmp_path):
    """forward_exec (reconstruction.hpp:66-158): 32 jittered samples of the saved layers
    (divided by 32, cylinder mask) per sub-iteration, written as p_%010d.tif."""
    P, H, W, S = 24, 32, 40, 4
    raw = raw_images(8, P=P)
    write_stack(str(tmp_path / "in"), raw)
    rng = np.random.default_rng(9)
    vol = rng.uniform(0.0, 0.01, (H, W, W)).astype(np.float32)
    out = tmp_path / "out"
    os.makedirs(out)
    L = _lib.lib()
    for l in range(H):
        layer = np.ascontiguousarray(vol[l])
        assert L.xpr_tiff_write(str(out / ("layer_%05d.tif" % l)).encode(), layer.ctypes.data, W, W) == 0
    cfg = config("naive", "fast", seed=5)
    cfg["recon"].update(input=str(tmp_path / "in"), output=str(out), proj_output=str(tmp_path / "sim"),
                        simulation=True)
    r = subprocess.run([CLI, json.dumps(cfg)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    # oracle
    gp = O.geom_params(**dict(GEOM, projections=P))
    pd_all, go = O.geometry(gp)
    Pc = P // S
    j = np.arange(W)
    mask = ((2 * j[None, :] - W) ** 2 + (2 * j[:, None] - W) ** 2) >= (W - 2) ** 2  # [z, x]
    v = (vol / np.float32(32)).astype(np.float32)
    v[:, mask] = 0.0
    v = np.ascontiguousarray(v.ravel())
    jit = O.jitter_sequence(5, 3 * 32 * S, go.vx)
    n = 0
    for sit in range(S):
        sums = np.zeros(Pc * W * H, np.uint32)
        pd = O.subset_projdata(pd_all, P, S, 1, sit, Pc)
        for _ in range(32):
            origin = [float(np.float32(go.orig[i]) + jit[n + i]) for i in range(3)]
            n += 3
            Lx, keep = O.make_launch((0, 0, 0), (W, H, W), origin, [go.vx] * 3, W, H, 0, Pc, 1, arith=O.FAST)
            O.forward(v, sums, pd, Lx)
        for k in range(Pc):
            got = read_tiff(str(tmp_path / "sim" / ("p_%010d.tif" % (sit + k * S))))
            exp = (sums[k * W * H:(k + 1) * W * H].astype(np.float32) / np.float32(4194304.0)).reshape(H, W)
            np.testing.assert_array_equal(got.view(np.uint32), exp.view(np.uint32))


def write_layers(dirpath, vol, H, W):
    """A volume (H layers of W x W, y outermost) as the layer_%05d.tif stack a run saves."""
    L = _lib.lib()
    L.xpr_tiff_write.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32]
    os.makedirs(dirpath, exist_ok=True)
    v = vol.reshape(H, W, W)
    for l in range(H):
        layer = np.ascontiguousarray(v[l])
        assert L.xpr_tiff_write(os.path.join(dirpath, "layer_%05d.tif" % l).encode(), layer.ctypes.data, W, W) == 0


@pytest.mark.parametrize("method", ["naive", "method_1a", "method_1b", "method_1c"])
def test_resume_continues_the_run(tmp_path, method):
    """Iterations 0 .. 1 of a run, then iteration 2 resumed from their saved layers
    (recon.resume, recon.first_iteration 2), equal the uninterrupted 3-iteration run bit for
    bit: the resumed run takes iteration 2's weight and origin-jitter draws and projects in
    its first sub-iteration."""
    raw = raw_images(11)
    H, W = raw.shape[1:]
    whole = run_host(config(method, it=3, slab=5), raw)
    part = run_host(config(method, it=2, slab=5), raw)
    write_layers(str(tmp_path / "ckpt"), part, H, W)
    resumed = run_host(config(method, it=3, slab=5, resume=str(tmp_path / "ckpt"), first_iteration=2), raw)
    assert np.isfinite(whole).mean() > 0.5
    assert_same_bits(resumed, whole)
    assert not np.array_equal(part.view(np.uint32), whole.view(np.uint32))  # the last iteration did change it


def test_resume_rejects_a_stack_of_another_size(tmp_path):
    raw = raw_images(12)
    H, W = raw.shape[1:]
    write_layers(str(tmp_path / "ckpt"), np.ones((H + 2) * (W + 2) * (W + 2), np.float32), H + 2, W + 2)
    L = _lib.lib()
    L.xpr_reconstruct_host.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.c_uint64, C.POINTER(C.c_double)]
    out = np.zeros(W * H * W, np.float32)
    cfg = config("naive", it=2, resume=str(tmp_path / "ckpt"), first_iteration=1)
    rc = L.xpr_reconstruct_host(json.dumps(cfg).encode(), np.ascontiguousarray(raw).ctypes.data, raw.shape[0], W, H,
                                out.ctypes.data, out.size, C.byref(C.c_double()))
    assert rc != 0
    assert b"layer size mismatch" in L.xpr_last_error()
