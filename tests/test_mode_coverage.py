"""Coverage of the forward kernel's per-(brick, projection) modes by the parity cases.

The forward (`compute_meta` in xpulse_recon_b200/csrc/xpr_kernels.cu) projects each
brick's 8 corners, bounds the footprint with a 2-pixel margin, clips it to the viewport
and the buffer rows, and picks: skip (no overlap), a shared-memory tile (footprint within
TILE_CAP pixels) or a direct splat with global atomics; it also marks footprints that the
clipping left unchanged ("inside": no bounds tests).  This test restates that choice on
the CPU (in double precision: only the counts matter here) so that the GPU parity cases
are known to reach every mode: if a change to the brick shape, the tile capacity or the
cases stopped exercising one, the GPU tests would pass without testing it.
"""
import re
from pathlib import Path

import numpy as np
import pytest

from tests.cases import make_case

KERNELS = Path(__file__).resolve().parents[1] / "xpulse_recon_b200" / "csrc" / "xpr_kernels.cu"


def kernel_constant(name):
    m = re.search(r"constexpr int %s = (\d+);" % name, KERNELS.read_text())
    assert m, name
    return int(m.group(1))


def modes(c):
    bx, by, bz, cap = (kernel_constant(n) for n in ("BX", "BY", "BZ", "TILE_CAP"))
    pd = np.asarray(c["pd"], np.float64).reshape(-1, 20)
    vx, org = float(c["go"].vx), np.asarray(c["origin"], np.float64)
    vmin, vmax, off = c["vmin"], c["vmax"], c["row_offset"]
    out = dict(skip=0, tile=0, direct=0, inside=0)
    for x0 in range(vmin[0], vmax[0], bx):
        for y0 in range(vmin[1], vmax[1], by):
            for z0 in range(vmin[2], vmax[2], bz):
                corners = np.array([[x, y, z] for x in (x0, x0 + bx - 1) for y in (y0, y0 + by - 1)
                                    for z in (z0, z0 + bz - 1)], np.float64) * vx + org
                for e in range(pd.shape[0]):
                    cu, cv, cw = pd[e, 0:4], pd[e, 4:8], pd[e, 12:16]
                    nu, nv, nw = (corners @ r[:3] + r[3] for r in (cu, cv, cw))
                    l, r, b, t = pd[e, 16:20]
                    l, r = max(int(np.ceil(l)), 0), min(int(np.ceil(r)), c["Wd"])
                    b, t = max(int(np.ceil(b)), 0), min(int(np.ceil(t)), c["rows"])
                    ok = bool((nw > 0).all())
                    if ok:
                        u, v = nu / nw, nv / nw - off
                        fl, fr = int(np.floor(u.min())) - 2, int(np.ceil(u.max())) + 3
                        fb, ft = int(np.floor(v.min())) - 2, int(np.ceil(v.max())) + 3
                        out["inside"] += fl >= l and fr <= r and fb >= b and ft <= t
                        l, r, b, t = max(l, fl), min(r, fr), max(b, fb), min(t, ft)
                    if r <= l or t <= b:
                        out["skip"] += 1
                    elif ok and (r - l) * (t - b) <= cap:
                        out["tile"] += 1
                    else:
                        out["direct"] += 1
    return out


@pytest.mark.parametrize("name,need", [("widecone", ("tile", "direct", "inside")),
                                       ("offsets64", ("tile", "inside")),
                                       ("modules2", ("tile", "skip"))])
def test_parity_cases_reach_every_forward_mode(name, need):
    m = modes(make_case(name, sit=1, seed=11))  # the forward parity test's case
    for k in need:
        assert m[k] > 0, (name, m)
