"""Loader of tests/golden/ref_kernels.npz (golden vectors of the reference's own kernels,
made by tests/golden/make_golden.py) into the case dictionaries of tests/cases.py."""
from __future__ import annotations

import os
from types import SimpleNamespace

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_kernels.npz")
KERNEL_CASES = ["plain", "offsets_m2", "rpy_m3", "ragged", "window"]

_cache = {}


def load():
    if "z" not in _cache:
        with np.load(PATH) as z:
            _cache["z"] = {k: z[k] for k in z.files}
    return _cache["z"]


def case(name: str) -> dict:
    """Inputs and outputs of one golden record, in the keys tests/cases.py uses."""
    z = load()
    g = {k.split(".", 1)[1]: v for k, v in z.items() if k.startswith(name + ".")}
    Wd, Hd, rows, row_offset, Pc, M = (int(v) for v in g["det"])
    box = [int(v) for v in g["box"]]
    c = dict(Wd=Wd, Hd=Hd, rows=rows, row_offset=row_offset, Pc=Pc, M=M, vmin=tuple(box[:3]),
             vmax=tuple(box[3:]), origin=[float(v) for v in g["origin"]],
             go=SimpleNamespace(vx=float(g["voxel"])), n=int(np.prod(np.subtract(box[3:], box[:3]))))
    c.update(g)
    if "pd" not in c:
        c["pd"] = c["pd_all"]
    return c
