"""Generate tests/golden/ref_kernels.npz: golden vectors of the reference's own kernels.

The reference (ebarjou/xpulse_recon) ships no tests, fixtures or golden vectors, so
they are made here from its OpenCL kernel sources compiled for the CPU
(oracle/_ref/libxpr_ref.so, built by oracle/build.py from the reference tree):

  KernelForward.cl   -> forward sums (u32)
  KernelError.cl     -> ratio (f32 bits in the u32 buffer)
  KernelBackward.cl  -> updated volume (f32)
  KernelForwardH.cl / KernelBackwardH.cl -> one layer with culled angle lists

Inputs are stored whole (ProjData, origin, box, volume, images), so the fixture needs
neither the reference nor the oracle's geometry to be replayed.  Every kernel runs over
the reference's padded NDRange (n + 32 - n % 32 work-items) on a padded volume buffer,
as the reference launches them (kernel.hpp:73-81).

One further record, `recon`, is a whole naive reconstruction (reconstruction_n.hpp:27-88:
volume 1.0, sums FIXED_ONE on the first sub-iteration, mt19937 jitter of the origin,
weight *= weight_factor per main iteration) whose three kernels are the reference's; its
host loop and the -log preprocessing (data_loader.hpp:48-101) are the oracle's
restatement.

Run from the repository root, in a tree where the reference is present:

    python -m tests.golden.make_golden
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "ref_kernels.npz")
FIXED_ONE = 1 << 22

# name: geometry, sub-iteration, box (vmin, vmax) or None for the full grid, row window or None
KERNEL_CASES = {
    "plain": dict(geom=dict(dwidth=32, dheight=24, projections=16, sit=4), sit=1,
                  box=((8, 4, 8), (24, 20, 24)), window=None, weight=0.9),
    "offsets_m2": dict(geom=dict(dwidth=40, dheight=24, projections=12, sit=3, module_number=2, rx=1.5, sx=-2.0,
                                 sy=3.0), sit=2, box=((12, 4, 12), (28, 20, 28)), window=None, weight=0.81),
    "rpy_m3": dict(geom=dict(dwidth=30, dheight=20, projections=8, sit=2, module_number=3,
                             mod_rpy=[1.0, -0.5, 0.8, 0.0, 0.3, -1.2, -1.5, 0.9, 0.2]),
                   sit=1, box=((6, 2, 6), (24, 18, 24)), window=None, weight=1.0),
    "ragged": dict(geom=dict(dwidth=37, dheight=29, projections=23, sit=3, rx=-0.7, sy=0.4), sit=0,
                   box=((10, 5, 9), (27, 24, 28)), window=None, weight=0.9),
    # method_2's cropped detector row window; the box stops short of the last layer so the
    # reference's unclipped lower bound never indexes past the window
    "window": dict(geom=dict(dwidth=32, dheight=24, projections=16, sit=4), sit=3,
                   box=((8, 2, 8), (24, 23, 24)), window=(6, 18), weight=0.9),
}


def _kernel_case(name, spec, rng):
    gp = O.geom_params(**{k: v for k, v in spec["geom"].items() if k != "mod_rpy"},
                       mod_rpy=None if "mod_rpy" not in spec["geom"] else
                       np.asarray(spec["geom"]["mod_rpy"], np.float32))
    pd_all, go = O.geometry(gp)
    P, S, M = gp.projections, gp.sit, gp.module_number
    Pc = int(go.concurrent)
    pd = np.ascontiguousarray(O.subset_projdata(pd_all, P, S, M, spec["sit"], Pc), np.float32)
    Wd, Hd = gp.dwidth, gp.dheight
    vmin, vmax = spec["box"]
    row_offset, rows = (0, Hd) if spec["window"] is None else spec["window"]
    n = int(np.prod(np.subtract(vmax, vmin)))
    vol = rng.uniform(0.0, 2.0, O.ndrange(n)).astype(np.float32)
    origin = np.array([np.float32(go.orig[i]) + np.float32(rng.uniform(0, go.vx)) for i in range(3)], np.float32)
    images = rng.uniform(0.2, 4.0, Pc * Wd * rows).astype(np.float32)
    vx = float(go.vx)
    sums = np.zeros(Pc * Wd * rows, np.uint32)
    O.ref_forward(vol, sums, pd, Wd, Hd, [float(o) for o in origin], Pc, M, vmin, vmax, (row_offset, rows),
                  [vx] * 3)
    ratio = sums.copy()
    O.ref_error(images, ratio, Wd, rows, spec["weight"])
    vol_out = vol.copy()
    O.ref_backward(vol_out, ratio.view(np.float32), pd, Wd, Hd, [float(o) for o in origin], Pc, M, vmin, vmax,
                   (row_offset, rows), [vx] * 3)
    assert sums.sum(dtype=np.uint64) > 0, name
    return {"pd": pd, "det": np.array([Wd, Hd, rows, row_offset, Pc, M], np.int64),
            "box": np.array([*vmin, *vmax], np.int64), "origin": origin, "voxel": np.float32(vx),
            "weight": np.float32(spec["weight"]), "vol": vol, "images": images, "sums": sums, "ratio": ratio,
            "vol_out": vol_out}


def _lists_case(rng):
    """KernelForwardH / KernelBackwardH: one y-layer, the angle list culled for it, and a
    ratio with NaN entries that the NaN-skipping backward must pass over."""
    gp = O.geom_params(dwidth=40, dheight=24, projections=20, sit=4, rx=1.5, sx=-2.0, sy=3.0)
    pd_all, go = O.geometry(gp)
    Pc, W, Wd, Hd = int(go.concurrent), int(go.vwidth), gp.dwidth, gp.dheight
    layer = 9
    lm = np.zeros(64, np.uint16)
    li = np.zeros(64, np.uint16)
    n = O.lib().orc_cull_layer(C.byref(gp), C.byref(go), pd_all, 1, layer, 0, lm, li)
    lm, li = lm[:n].copy(), li[:n].copy()
    assert 0 < n <= Pc + 1
    origin = np.array([np.float32(go.orig[i]) + np.float32(rng.uniform(0, go.vx)) for i in range(3)], np.float32)
    vol = rng.uniform(0.0, 2.0, O.ndrange(W * W)).astype(np.float32)
    o4 = (C.c_float * 4)(*[float(v) for v in origin], 1.0)
    sums = np.zeros((Pc + 1) * Wd * Hd, np.uint32)
    R = O.ref_lib()
    pd_all = np.ascontiguousarray(pd_all, np.float32)
    R.refk_forwardh(vol, sums, pd_all, lm, li, n, layer, o4, go.vx, Wd, Hd, W, O.ndrange(W * W))
    ratio = rng.uniform(0.2, 4.0, sums.size).astype(np.float32)
    ratio[::7] = np.nan
    vol_out = vol.copy()
    R.refk_backwardh(vol_out, ratio, pd_all, lm, li, n, layer, o4, go.vx, Wd, Hd, W, O.ndrange(W * W))
    return {"pd_all": pd_all, "det": np.array([Wd, Hd, Hd, 0, Pc + 1, 1], np.int64),
            "box": np.array([0, layer, 0, W, layer + 1, W], np.int64), "origin": origin,
            "voxel": np.float32(go.vx), "list_mvp": lm, "list_img": li, "vol": vol, "sums": sums,
            "ratio_in": ratio, "vol_out": vol_out}


RECON_GEOM = dict(dwidth=24, dheight=20, projections=16, sit=4, rx=1.0, sx=-0.5, sy=0.8)
RECON = dict(it=2, sit=4, weight=1.0, weight_factor=0.9, seed=77)


def _recon_case(rng):
    gp = O.geom_params(**RECON_GEOM)
    pd_all, go = O.geometry(gp)
    P, S, M = gp.projections, gp.sit, gp.module_number
    Pc, W, Hv, Wd, Hd = int(go.concurrent), int(go.vwidth), int(go.vheight), gp.dwidth, gp.dheight
    raw = rng.uniform(0.05, 0.98, (P, Hd, Wd)).astype(np.float32)
    imgs = raw.ravel().copy()
    O.lib().orc_preprocess(imgs, imgs.size, 0, 0.0, 0.0, 1)  # -log, no normalisation
    imgs = imgs.reshape(P, Hd, Wd)
    n = W * Hv * W
    vol = np.ones(O.ndrange(n), np.float32)
    sums = np.full(Pc * Wd * Hd, FIXED_ONE, np.uint32)
    g = O.MT()
    O.lib().orc_mt_seed(C.byref(g), RECON["seed"])
    weight = np.float32(RECON["weight"])
    for mit in range(RECON["it"]):
        for s in range(S):
            origin = [float(np.float32(go.orig[i]) + np.float32(O.lib().orc_uniform_float(C.byref(g), 0.0, go.vx)))
                      for i in range(3)]
            pd = np.ascontiguousarray(O.subset_projdata(pd_all, P, S, M, s, Pc), np.float32)
            sub = np.ascontiguousarray(imgs[[s + k * S for k in range(Pc)]]).ravel()
            if mit > 0 or s > 0:
                O.ref_forward(vol, sums, pd, Wd, Hd, origin, Pc, M, (0, 0, 0), (W, Hv, W), (0, Hd), [go.vx] * 3)
            O.ref_error(sub, sums, Wd, Hd, float(weight))
            O.ref_backward(vol, sums.view(np.float32), pd, Wd, Hd, origin, Pc, M, (0, 0, 0), (W, Hv, W), (0, Hd),
                           [go.vx] * 3)
            sums[:] = 0
        weight = np.float32(weight * np.float32(RECON["weight_factor"]))
    return {"raw": raw, "vol_out": vol[:n].copy(),
            "params": np.array([RECON["it"], RECON["sit"], RECON["seed"]], np.int64),
            "weights": np.array([RECON["weight"], RECON["weight_factor"]], np.float32),
            "geom": np.array([RECON_GEOM["dwidth"], RECON_GEOM["dheight"], RECON_GEOM["projections"]], np.int64),
            "offsets": np.array([RECON_GEOM["rx"], RECON_GEOM["sx"], RECON_GEOM["sy"]], np.float32)}


def main():
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref/libxpr_ref.so is not built (python -m oracle.build needs the reference tree)")
    rng = np.random.default_rng(2024)
    out = {}
    for name, spec in KERNEL_CASES.items():
        for k, v in _kernel_case(name, spec, rng).items():
            out[f"{name}.{k}"] = v
    for k, v in _lists_case(rng).items():
        out[f"lists.{k}"] = v
    for k, v in _recon_case(rng).items():
        out[f"recon.{k}"] = v
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
