"""Slab sharding on the GPU: two ranks (processes) share the one GPU of the test machine,
each running this library's kernels (STRICT contract) on its y-slab, the detector
partial sums of the rows the two slabs' windows share exchanged through a gloo process
group (host staging; the ranks' kernels never wait on each other).  The gathered volume
must equal the single-rank GPU run and the CPU oracle bit for bit."""
import ctypes as C
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from tests.cases import assert_same_bits  # noqa: E402

pytestmark = pytest.mark.gpu

GEOM = dict(dwidth=48, dheight=40, projections=36, sit=4, rx=1.0, sx=-0.5, sy=0.8)


def _run(rank, world, port, out_dir):
    import torch.distributed as dist
    from xpulse_recon_b200.projector import Context, geometry
    from xpulse_recon_b200.shard import GpuOps, SlabReconstruction
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
    ctx = Context(0)
    try:
        pd_all, g = geometry(**GEOM)
        raw = np.random.default_rng(9).uniform(0.05, 0.98, (GEOM["projections"], GEOM["dheight"],
                                                            GEOM["dwidth"])).astype(np.float32)
        r = SlabReconstruction(GpuOps(ctx), raw, pd_all, g, it=2, sit=GEOM["sit"], seed=31, rank=rank, world=world)
        r.run()
        vol = r.gather()
        if rank == 0:
            np.save(os.path.join(out_dir, "vol_%d.npy" % world), vol)
    finally:
        ctx.close()
        if world > 1:
            dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_slab_ranks_equal_one_gpu_and_the_oracle(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_run, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    mp.spawn(_run, args=(1, 0, str(tmp_path)), nprocs=1, join=True)
    two, one = np.load(tmp_path / "vol_2.npy"), np.load(tmp_path / "vol_1.npy")
    assert np.isfinite(one).mean() > 0.5
    assert_same_bits(two, one)
    raw = np.random.default_rng(9).uniform(0.05, 0.98, (GEOM["projections"], GEOM["dheight"],
                                                        GEOM["dwidth"])).astype(np.float32)
    imgs = raw.ravel().copy()
    O.lib().orc_preprocess(imgs, imgs.size, 0, 0.0, 0.0, 1)
    gp = O.geom_params(**GEOM)
    rp = O.ReconParams(2, GEOM["sit"], 1.0, 0.9, 31, O.STRICT, 0)
    exp = np.zeros(one.size, np.float32)
    assert O.lib().orc_recon_naive(C.byref(gp), C.byref(rp), imgs, exp) == 0
    assert_same_bits(one, exp)
