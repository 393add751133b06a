"""Slab sharding of one reconstruction over ranks (xpulse_recon_b200/shard.py) on the CPU:
world_size 2 and 3 gloo process groups on 127.0.0.1, with the oracle as the arithmetic,
both with detector-row windows (point-to-point exchange of the shared rows, the default)
and with the whole detector all-reduced.  The gathered volume must equal the
single-process oracle reconstruction bit for bit (the exchanged sums are integers)."""
import ctypes as C
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from tests.cases import assert_same_bits  # noqa: E402
from xpulse_recon_b200 import _lib  # noqa: E402
from xpulse_recon_b200.shard import (SlabReconstruction, exchange_plan, exchange_rows, row_window,  # noqa: E402
                                     slab_bounds)

GEOM = dict(dwidth=40, dheight=32, projections=24, sit=4, rx=1.0, sx=-0.5, sy=0.8)


class OracleOps:
    """The slab operators on the CPU oracle (FAST contract, FP32 storage)."""
    arith = O.FAST

    def tensor(self, a):
        return np.array(a, copy=True)

    def zeros_u32(self, n):
        return np.zeros(n, np.uint32)

    def full_u32(self, n, v):
        return np.full(n, v, np.uint32)

    def ones_f32(self, n):
        return np.ones(n, np.float32)

    def ratio_buffer(self, n):
        return np.zeros(n, np.float32)

    def preprocess(self, raw):
        x = np.ascontiguousarray(raw, np.float32).copy()
        O.lib().orc_preprocess(x, x.size, 0, 0.0, 0.0, 1)
        return x

    def _launch(self, L):
        box = (tuple(L.vmin), tuple(L.vmax))
        return O.make_launch(box[0], box[1], list(L.origin), list(L.voxel), L.det_w, L.rows, L.row_offset,
                             L.n_angles, L.modules, arith=O.FAST)

    def forward(self, vol, sums, pd, n_pd, L):
        d, keep = self._launch(L)
        O.forward(vol, sums, np.ascontiguousarray(pd, np.float32), d)

    def error(self, images, sums, ratio, n, weight):
        O.error(np.ascontiguousarray(images[:n]), sums, weight)
        ratio[:] = sums.view(np.float32)
        sums[:] = 0

    def backward(self, vol, ratio, pd, n_pd, L):
        d, keep = self._launch(L)
        O.backward(vol, ratio, np.ascontiguousarray(pd, np.float32), d)

    def all_reduce_sum(self, sums, group=None):
        import torch.distributed as dist
        t = torch.from_numpy(sums.view(np.int32))  # u32 addition modulo 2^32 == wrapping int32 addition
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)

    def exchange(self, sums, plan, r0, n_img, rows, width, group=None):
        return exchange_rows(torch.from_numpy(sums.view(np.int32)), plan, r0, n_img, rows, width, group)

    def synchronize(self):
        pass

    def to_host(self, t):
        return t


def _inputs():
    gp = O.geom_params(**GEOM)
    pd_all, go = O.geometry(gp)
    g = {"vwidth": go.vwidth, "vheight": go.vheight, "vx": go.vx, "orig": tuple(go.orig), "concurrent": go.concurrent}
    raw = np.random.default_rng(5).uniform(0.05, 0.98, (GEOM["projections"], GEOM["dheight"],
                                                        GEOM["dwidth"])).astype(np.float32)
    return raw, pd_all, g


def _rank_main(rank, world, port, out_dir, windowed):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        raw, pd_all, g = _inputs()
        r = SlabReconstruction(OracleOps(), raw, pd_all, g, it=2, sit=GEOM["sit"], seed=77, rank=rank, world=world,
                               windowed=windowed)
        r.run()
        vol = r.gather()
        sent = [None] * world
        dist.all_gather_object(sent, r.exchanged_bytes)
        if rank == 0:
            np.save(os.path.join(out_dir, "vol_%d.npy" % world), vol)
            np.save(os.path.join(out_dir, "bytes_%d.npy" % world), np.array(sent))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slab_bounds_partition():
    for H in (1, 7, 32, 33, 768):
        for world in (1, 2, 3, 8):
            b = [slab_bounds(H, world, r) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == H
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            assert max(y1 - y0 for y0, y1 in b) - min(y1 - y0 for y0, y1 in b) <= 1


@pytest.mark.parametrize("windowed", [True, False])
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_equals_single_process(tmp_path, world, windowed):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path), windowed), nprocs=world, join=True)
    got = np.load(tmp_path / ("vol_%d.npy" % world))
    raw, pd_all, g = _inputs()
    imgs = raw.ravel().copy()
    O.lib().orc_preprocess(imgs, imgs.size, 0, 0.0, 0.0, 1)
    gp = O.geom_params(**GEOM)
    rp = O.ReconParams(2, GEOM["sit"], 1.0, 0.9, 77, O.FAST, 0)
    exp = np.zeros(got.size, np.float32)
    assert O.lib().orc_recon_naive(C.byref(gp), C.byref(rp), imgs, exp) == 0
    assert np.isfinite(got).mean() > 0.5
    assert_same_bits(got, exp)
    # one exchange per sub-iteration with a forward: the whole detector, or the shared rows
    npix = g["concurrent"] * GEOM["dwidth"] * GEOM["dheight"]
    sent = np.load(tmp_path / ("bytes_%d.npy" % world))
    forwards = 2 * GEOM["sit"] - 1
    if not windowed:
        assert all(int(b) == 4 * npix * forwards for b in sent)
    else:
        windows = [row_window(pd_all, g, *slab_bounds(int(g["vheight"]), world, q), GEOM["dheight"])
                   for q in range(world)]
        for q in range(world):
            shared = sum(b - a for _, a, b in exchange_plan(windows, q))
            assert int(sent[q]) == 4 * g["concurrent"] * GEOM["dwidth"] * shared * forwards
            assert shared < GEOM["dheight"]


def test_row_windows_cover_every_voxel_pixel():
    """Every in-bounds pixel a slab's voxels reach (oracle forward of the slab, all
    projections, jittered origins) lies in the slab's row window."""
    raw, pd_all, g = _inputs()
    gp = O.geom_params(**GEOM)
    W, Hv, Wd, Hd = int(g["vwidth"]), int(g["vheight"]), GEOM["dwidth"], GEOM["dheight"]
    P = GEOM["projections"]
    rng = np.random.default_rng(3)
    for world in (2, 3, 5):
        for q in range(world):
            y0, y1 = slab_bounds(Hv, world, q)
            r0, r1 = row_window(pd_all, g, y0, y1, Hd)
            vol = np.ones(W * (y1 - y0) * W, np.float32)
            for _ in range(3):
                origin = [float(np.float32(g["orig"][i]) + np.float32(rng.uniform(0, g["vx"]))) for i in range(3)]
                L, keep = O.make_launch((0, y0, 0), (W, y1, W), origin, [g["vx"]] * 3, Wd, Hd, 0, P, 1, arith=O.FAST)
                sums = np.zeros(P * Wd * Hd, np.uint32)
                O.forward(vol, sums, np.ascontiguousarray(pd_all), L)
                hit = sums.reshape(P, Hd, Wd).any(axis=(0, 2))
                rows = np.nonzero(hit)[0]
                assert rows.min() >= r0 and rows.max() < r1, (world, q, rows.min(), rows.max(), r0, r1)
