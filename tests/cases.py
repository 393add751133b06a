"""Seeded parity cases shared by the CPU and GPU tests.

A case is a geometry (XPRecon JSON parameters), one sub-iteration's ProjData,
a jittered origin, a volume box and seeded data.  Sizes are small enough for
the CPU oracle to finish in well under a second.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

# name: geometry overrides (detector, offsets, modules) + launch variations
CASES = {
    "plain48": dict(dwidth=48, dheight=48, projections=36, sit=4),
    "offsets64": dict(dwidth=64, dheight=40, projections=40, sit=5, rx=1.5, sx=-2.0, sy=3.0),
    "ragged": dict(dwidth=37, dheight=29, projections=23, sit=3, rx=-0.7, sy=0.4),
    "modules2": dict(dwidth=64, dheight=32, projections=24, sit=3, module_number=2),
    "modules3_rpy": dict(dwidth=60, dheight=30, projections=18, sit=2, module_number=3,
                         mod_rpy=[[1.0, -0.5, 0.8], [0.0, 0.3, -1.2], [-1.5, 0.9, 0.2]]),
    "helical": dict(dwidth=40, dheight=24, projections=30, sit=3, heli_offset=0.05),
    "shortscan": dict(dwidth=48, dheight=48, projections=30, sit=3, angle=200.0),
    # wide cone (source close to the object): near-source bricks project large enough that
    # the forward splats them with global atomics instead of a shared-memory tile
    "widecone": dict(dwidth=96, dheight=40, projections=24, sit=3, so=2.0, sd=4.0, rx=0.5, sy=1.0),
    "anglelist": dict(dwidth=32, dheight=32, projections=12, sit=2,
                      angle_list=[0.0, 7.5, 31.0, 44.0, 90.0, 95.5, 180.0, 181.0, 250.0, 271.0, 300.0, 359.0]),
}


def make_case(name: str, sit: int = 1, seed: int = 0, box=None, row_window=None, fp64=False):
    """Returns dict(pd_all, pd, go, gp, Pc, M, W, H, origin, vmin, vmax, rows, row_offset, vol, images)."""
    kw = dict(CASES[name])
    mod_rpy = kw.pop("mod_rpy", None)
    angle_list = kw.pop("angle_list", None)
    gp = O.geom_params(mod_rpy=None if mod_rpy is None else np.asarray(mod_rpy, np.float32).ravel(),
                       angle_list=angle_list, **kw)
    pd_all, go = O.geometry(gp, fp64=fp64)
    P, S, M = gp.projections, gp.sit, gp.module_number
    Pc = int(go.concurrent)
    pd = O.subset_projdata(pd_all, P, S, M, sit % S, Pc)
    W, Hv = int(go.vwidth), int(go.vheight)
    Wd, Hd = gp.dwidth, gp.dheight
    rng = np.random.default_rng(seed)
    origin = [float(np.float32(go.orig[i]) + np.float32(rng.uniform(0, go.vx))) for i in range(3)]
    vmin, vmax = (0, 0, 0), (W, Hv, W)
    if box is not None:
        vmin, vmax = box
    n = int(np.prod(np.subtract(vmax, vmin)))
    vol = np.ascontiguousarray(rng.uniform(0.0, 2.0, O.ndrange(n)).astype(np.float32))
    row_offset, rows = 0, Hd
    if row_window is not None:
        row_offset, rows = row_window
    images = np.ascontiguousarray(rng.uniform(0.2, 4.0, (Pc + 1) * Wd * rows).astype(np.float32))
    return dict(pd_all=pd_all, pd=pd, go=go, gp=gp, Pc=Pc, M=M, W=W, Wd=Wd, Hd=Hd, origin=origin, vmin=vmin,
                vmax=vmax, rows=rows, row_offset=row_offset, vol=vol, images=images, n=n)


def launch(c, arith=O.STRICT, compat_pad=0, nan_skip=0, lists=None):
    lm, li = (None, None) if lists is None else lists
    return O.make_launch(c["vmin"], c["vmax"], c["origin"], [c["go"].vx] * 3, c["Wd"], c["rows"], c["row_offset"],
                         c["Pc"] if lists is None else max(int(np.max(li)) + 1, c["Pc"]), c["M"], arith=arith,
                         compat_pad=compat_pad, nan_skip=nan_skip, list_mvp=lm, list_img=li)


def oracle_forward(c, arith=O.STRICT, compat_pad=0, lists=None, pd=None):
    L, keep = launch(c, arith, compat_pad, lists=lists)
    n_img = c["Pc"] if lists is None else max(int(np.max(lists[1])) + 1, c["Pc"])
    sums = np.zeros(n_img * c["Wd"] * c["rows"], np.uint32)
    O.forward(c["vol"], sums, c["pd"] if pd is None else pd, L)
    return sums


def oracle_backward(c, ratio, arith=O.STRICT, compat_pad=0, nan_skip=0, lists=None, pd=None):
    L, keep = launch(c, arith, compat_pad, nan_skip, lists=lists)
    vol = c["vol"].copy()
    O.backward(vol, np.ascontiguousarray(ratio, np.float32), c["pd"] if pd is None else pd, L)
    return vol


def ratio_from(c, sums, weight=0.9):
    r = sums.copy()
    O.error(c["images"][: r.size], r, weight)
    return r.view(np.float32)


def assert_same_bits(got, exp):
    """Bit-identical float32 arrays, except that any NaN matches any NaN (CPU and GPU
    produce different NaN payloads; the NaN positions must agree)."""
    got = np.asarray(got, np.float32)
    exp = np.asarray(exp, np.float32)
    assert got.shape == exp.shape
    gn, en = np.isnan(got), np.isnan(exp)
    np.testing.assert_array_equal(gn, en)
    np.testing.assert_array_equal(got[~gn].view(np.uint32), exp[~en].view(np.uint32))
