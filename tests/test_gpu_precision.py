"""Precision of the reduced-storage forms against the FP64 oracle.

Whole naive reconstructions through the drop-in host entry point (STRICT contract,
geometry matrices built in double, detector images and ratios stored in FP32, BF16 or
FP16 with FP32 accumulation and an FP32 volume) are compared with the same algorithm
run in double precision on the CPU (oracle/xpr_oracle.c, orc64_recon_naive), on
projections of a seeded ellipsoid phantom with Poisson noise (simulated with the FAST
forward projector).

Measure: relative RMSE = ||v - v64||_2 / ||v64||_2 over the measurement region: the
voxels finite in both inside the grid's inscribed cylinder, without the two layers at
each end of the grid.  The end layers are seen by few detector rows; on noisy data the
multiplicative update drives a few hundred of their voxels to 1e12 in either precision
(the ratio is only clamped at 2^-22), so over all voxels the measure says nothing about
storage precision (it is reported as rel_rmse_all).  The voxels no projection reaches
are NaN in both, by the algorithm's 0/0.

Storage forms (ratio / measured images): fp32, fp16, bf16 = BF16 ratio with FP16
images, bf16_fp32img = BF16 ratio with FP32 images, bf16_all = BF16 ratio and BF16
images.  Tolerance (written here): 1e-3 relative RMSE, the precision target, which
FP32 and FP16 storage meet (measured 5.5e-4 - 7.6e-4 on B200).  Every BF16 form is a
known miss, kept as a strict xfail so that the miss stays visible: a BF16 ratio alone
gives 1.1e-3 - 1.4e-3 (its 2^-9 relative rounding of the log-ratio, largest in the
first sub-iterations, survives the averaging over a sub-iteration's projections), BF16
measured images 1.6e-3 - 2.2e-3 (a 2^-9 relative error of the measured value is an
absolute error of the same size in the log-ratio).  Setting XPR_PRECISION_REPORT=<path>
appends one JSON line per (workload, storage) with the measured values (region and all
voxels; over all voxels the few hundred end-layer voxels that run to 1e12 in either
precision dominate, so that figure is 1.0 for every form)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from xpulse_recon_b200 import _lib  # noqa: E402
from xpulse_recon_b200.projector import Context, Reconstruction, geometry  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-3
# form: (ratio storage, image storage)
FORMS = {"fp32": ("fp32", "fp32"), "fp16": ("fp16", "fp16"), "bf16": ("bf16", "fp16"),
         "bf16_fp32img": ("bf16", "fp32"), "bf16_all": ("bf16", "bf16")}

# name: (geometry, it, sit, ellipsoids, phantom fraction of the grid, seed)
WORKLOADS = {
    # the small plain workload: 192^2 detector, 180 projections, it 1, sit 10
    "plain192": (dict(dwidth=192, dheight=192, projections=180), 1, 10, 10, 2.0 / 3.0, 1),
    # the 768^2 / 720-projection offset geometry at quarter scale, it 3, sit 10
    "offsets192_it3": (dict(dwidth=192, dheight=192, projections=180, rx=1.5, sx=-2.0, sy=3.0), 3, 10, 40,
                       2.0 / 3.0, 2),
    # three modules of 64 px tilted by roll / pitch / yaw (the batched workload's detector), it 2
    "modules3_rpy": (dict(dwidth=192, dheight=128, projections=180, module_number=3,
                          mod_rpy=[1.5, -1.0, 0.5, -0.5, 1.2, -1.8, 0.9, 0.4, -1.1]), 2, 10, 20, 0.6, 3),
}


def _phantom(W, Hv, n_ell, frac, rng):
    """Ellipsoids (attenuation per voxel uniform in [0, 0.02)) inside the central
    frac-sized cube of the grid."""
    e = int(round(W * frac))
    lo, lov = (W - e) // 2, (Hv - e) // 2
    zz, yy, xx = np.meshgrid(np.arange(e), np.arange(e), np.arange(e), indexing="ij")
    sub = np.zeros((e, e, e), np.float32)  # [y, z, x]
    r_in = e / 2.0
    for _ in range(n_ell):
        while True:
            c = rng.uniform(-r_in, r_in, 3)
            if c[0] ** 2 + c[2] ** 2 < (0.8 * r_in) ** 2:
                break
        c += r_in
        a = rng.uniform(0.03, 0.25, 3) * e
        m = ((xx - c[0]) / a[0]) ** 2 + ((zz - c[1]) / a[1]) ** 2 + ((yy - c[2]) / a[2]) ** 2 < 1.0
        sub[m] += np.float32(rng.uniform(0.0, 0.02))
    vol = np.zeros((Hv, W, W), np.float32)
    vol[lov:lov + e, lo:lo + e, lo:lo + e] = sub
    return vol


def _projections(ctx, vol, pd_all, g, det, rng, i0=1e5, jitters=4, modules=1):
    """Raw intensities I / I0 of the phantom: the average of `jitters` jittered GPU
    forward projections (all P angles), then Poisson noise at i0 photons per pixel."""
    W, Hv, P = int(g["vwidth"]), int(g["vheight"]), pd_all.shape[0]
    Wd, Hd = det
    P_img = P // modules
    dvol = torch.from_numpy(vol.ravel()).cuda()
    dpd = torch.from_numpy(pd_all).cuda()
    acc = np.zeros(P_img * Wd * Hd, np.float64)
    r = Reconstruction(ctx, arith=_lib.FAST)
    r.set_image_parameters(Wd, Hd, P_img)
    r.set_volume_parameters((0, 0, 0), (W, Hv, W), [g["vx"]] * 3)
    r.set_angle_number(P // modules, modules)
    r.set_image_offset((0, Hd))
    r.set_projdata_buffer(dpd)
    r.set_volume_buffer(dvol)
    for _ in range(jitters):
        sums = torch.zeros(P_img * Wd * Hd, dtype=torch.int32, device="cuda")
        r._origin = tuple(float(np.float32(g["orig"][i]) + np.float32(rng.uniform(0, g["vx"]))) for i in range(3))
        r.set_sum_images_buffer(sums)
        r.forward()
        torch.cuda.synchronize()
        acc += sums.cpu().numpy().view(np.uint32).astype(np.float64) / 4194304.0
    p = acc / jitters
    counts = rng.poisson(i0 * np.exp(-p))
    return (np.maximum(counts, 1) / i0).astype(np.float32).reshape(P_img, Hd, Wd)


def _product(raw, geom, it, sit, form):
    storage, image_storage = FORMS[form]
    cfg = {"recon": {"method": "naive", "it": it, "sit": sit, "seed": 5, "arith": "strict", "geometry": "fp64",
                     "storage": storage, "image_storage": image_storage, "mlog": True, "weight": 1.0,
                     "weight_factor": 0.9},
           "geometry": {"so": 100.0, "sd": 1000.0, "angle": 360.0},
           "detector": {"px": 0.1, "rx": geom.get("rx", 0.0), "sx": geom.get("sx", 0.0), "sy": geom.get("sy", 0.0)}}
    if "mod_rpy" in geom:
        a = geom["mod_rpy"]
        cfg["detector"]["module_number"] = geom["module_number"]
        cfg["detector"]["modules"] = [{"roll": a[3 * m], "pitch": a[3 * m + 1], "yaw": a[3 * m + 2]}
                                      for m in range(geom["module_number"])]
    L = _lib.lib()
    L.xpr_reconstruct_host.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.c_uint64, C.POINTER(C.c_double)]
    P, H, W = raw.shape
    out = np.full(W * H * W, np.nan, np.float32)
    secs = C.c_double()
    rc = L.xpr_reconstruct_host(json.dumps(cfg).encode(), np.ascontiguousarray(raw).ctypes.data, P, W, H,
                                out.ctypes.data, out.size, C.byref(secs))
    assert rc == 0, L.xpr_last_error()
    return out


def _region(W, Hv, margin=2):
    """inscribed cylinder of the grid (x, z), layers [margin, Hv - margin); layout (y, z, x)"""
    c = np.arange(W) + 0.5 - W / 2.0
    disk = (c[None, :] ** 2 + c[:, None] ** 2) < (W / 2.0) ** 2
    m = np.zeros((Hv, W, W), bool)
    m[margin:Hv - margin] = disk[None]
    return m.ravel()


def _rel_rmse(v, ref, region=None):
    m = np.isfinite(v) & np.isfinite(ref)
    if region is not None:
        m &= region
    d = v[m].astype(np.float64) - ref[m]
    return float(np.sqrt(np.mean(d * d)) / np.sqrt(np.mean(ref[m] * ref[m])))


_cache = {}


def _workload(name):
    if name not in _cache:
        geom, it, sit, n_ell, frac, seed = WORKLOADS[name]
        rng = np.random.default_rng(seed)
        pd_all, g = geometry(sit=sit, fp64=True, **geom)
        W, Hv = int(g["vwidth"]), int(g["vheight"])
        vol = _phantom(W, Hv, n_ell, frac, rng)
        ctx = Context(0)
        try:
            raw = _projections(ctx, vol, pd_all, g, (geom["dwidth"], geom["dheight"]), rng,
                               modules=geom.get("module_number", 1))
        finally:
            ctx.close()
        gp = O.geom_params(sit=sit, **geom)
        rp = O.ReconParams(it, sit, 1.0, 0.9, 5, O.FAST, 0)
        v64 = O.recon_naive_f64(gp, rp, raw)
        _cache[name] = (raw, v64)
    return _cache[name]


BF16_MISS = {"bf16": "BF16 ratio: 1.1e-3 - 1.4e-3 relative RMSE, above the 1e-3 bound",
             "bf16_fp32img": "BF16 ratio: 1.1e-3 - 1.4e-3 relative RMSE, above the 1e-3 bound",
             "bf16_all": "BF16 ratio and images: 1.6e-3 - 2.2e-3 relative RMSE, above the 1e-3 bound"}


@pytest.mark.parametrize("storage", ["fp32", "fp16"] + [pytest.param(f, marks=pytest.mark.xfail(strict=True, reason=r))
                                                         for f, r in BF16_MISS.items()])
@pytest.mark.parametrize("name", sorted(WORKLOADS))
def test_relative_rmse_against_fp64_oracle(name, storage):
    geom, it, sit = WORKLOADS[name][:3]
    raw, v64 = _workload(name)
    v = _product(raw, geom, it, sit, storage)
    # the voxels no projection reaches are NaN in both; a voxel on the edge of the field
    # of view may be reached in one precision and not in the other
    nan_mismatch = float(np.mean(np.isnan(v) != np.isnan(v64)))
    W = geom["dwidth"]
    Hv = v.size // (W * W)  # the grid is dwidth x (dheight + helical extent) x dwidth
    err = _rel_rmse(v, v64, _region(W, Hv))
    err_all = _rel_rmse(v, v64)
    report = os.environ.get("XPR_PRECISION_REPORT")
    if report:
        with open(report, "a") as f:
            f.write(json.dumps({"workload": name, "storage": storage, "ratio": FORMS[storage][0],
                                "images": FORMS[storage][1], "geometry": "fp64", "arith": "strict",
                                "it": it, "sit": sit, "rel_rmse_vs_fp64": err, "rel_rmse_all": err_all,
                                "voxels": int(np.isfinite(v64).sum()), "nan_mismatch": nan_mismatch}) + "\n")
    assert nan_mismatch <= 1e-5, nan_mismatch
    assert err <= TOL, (name, storage, err)
