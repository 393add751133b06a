"""One reconstruction sharded over ranks by y-slabs (one process per GPU).

Rank r owns layers [y0_r, y1_r) of the volume (the slab split of method_2's chunks,
geometry_chunk.hpp:92-197, without their padding: slabs here are exact partitions).
Its voxels reach only a window of detector rows [r0_r, r1_r) (method_2's cropped
image window, the iOffset / iSize of geometry_chunk.hpp:120-168, here computed from the
slab's corners over every projection with a margin), and the windows of neighbouring
slabs overlap by the rows that rays through both slabs reach.  A sub-iteration
(reconstruction_n.hpp:65-76) becomes

    forward of the rank's slab into a window buffer of u32 partial sums
    -> exchange: each rank sends its partial sums over the rows it shares with another
       rank's window and adds what it receives (point-to-point, NCCL over NVLink); the
       u32 sums are integers, so every window then holds the single-GPU forward's sums
       bit for bit (addition modulo 2^32)
    -> error on the rank's window
    -> backward of the rank's slab (it reads only its window of the ratio)

so the sharded volume equals the single-GPU volume bit for bit.  The exchange is the one
real data dependency of the path; it moves only the overlap rows (about 3 % of the
detector per neighbour pair at the 768^2 x 72 configuration on 8 ranks, against the
170 MB of a whole-detector all-reduce, which `windowed=False` keeps).  The forward of
the next sub-iteration reads the volume this one's backward writes, so the exchange
cannot overlap it; it is kept small instead.

The arithmetic is supplied by an `ops` object (forward / error / backward on one slab):
`GpuOps` runs this library's kernels through the C ABI; tests may supply any other.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

FIXED_ONE = 1 << 22


def slab_bounds(height: int, world: int, rank: int) -> tuple:
    """Layers [y0, y1) of rank `rank` when `height` layers are split over `world` ranks."""
    base, extra = divmod(height, world)
    y0 = rank * base + min(rank, extra)
    return y0, y0 + base + (1 if rank < extra else 0)


def row_window(pd_all, g, y0: int, y1: int, rows: int, margin: int = 3) -> tuple:
    """Detector rows [r0, r1) that voxels of layers [y0, y1) can reach in any of the
    ProjData entries pd_all (n x 20: glm columns, then the viewport), origin jitter of up
    to one voxel included.  The slab is a box, so in front of the source its image is the
    convex hull of its corners' images; the corners are projected in double precision and
    the window widened by `margin` rows (far above any single-precision rounding of a
    pixel coordinate).  The whole detector when some corner is not in front of the source."""
    if y1 <= y0:
        return 0, 0
    m = np.asarray(pd_all, np.float64).reshape(-1, 20)
    W, vx = int(g["vwidth"]), float(g["vx"])
    o = np.asarray(g["orig"], np.float64)
    xs = o[0] + vx * np.array([-1.0, W + 1.0])
    ys = o[1] + vx * np.array([y0 - 1.0, y1 + 1.0])
    zs = o[2] + vx * np.array([-1.0, W + 1.0])
    P = np.array([[x, y, z, 1.0] for x in xs for y in ys for z in zs])  # 8 corners
    nv = P @ m[:, 4:8].T   # (corner, entry)
    nw = P @ m[:, 12:16].T
    if not (nw > 0).all():
        return 0, rows
    v = nv / nw
    r0 = max(0, int(np.floor(v.min())) - margin)
    r1 = min(rows, int(np.ceil(v.max())) + margin + 1)
    return (r0, r1) if r1 > r0 else (0, 0)


def exchange_plan(windows, rank: int) -> list:
    """(peer, a, b) for every other rank whose window shares rows [a, b) with this rank's
    (absolute detector rows), in peer order."""
    r0, r1 = windows[rank]
    plan = []
    for q, (q0, q1) in enumerate(windows):
        a, b = max(r0, q0), min(r1, q1)
        if q != rank and a < b:
            plan.append((q, a, b))
    return plan


def exchange_rows(sums, plan, r0: int, n_img: int, rows: int, width: int, group=None):
    """Adds to `sums` (torch int32 tensor of the window's u32 sums, [n_img, rows, width]
    from detector row r0) every peer's partial sums over the rows they share: both sides
    send their own partials and add the peer's (wrapping int32 addition is u32 addition
    modulo 2^32).  Device tensors go through host memory when the backend is not NCCL.
    Returns the bytes sent."""
    import torch
    import torch.distributed as dist
    if not plan:
        return 0
    v = sums.view(n_img, rows, width)
    host = dist.get_backend(group) != "nccl" and v.is_cuda
    ops, pending, sent = [], [], 0
    for q, a, b in plan:
        send = v[:, a - r0:b - r0, :].contiguous()
        if host:
            send = send.cpu()
        recv = torch.empty_like(send)
        peer = q if group is None else dist.get_global_rank(group, q)
        ops += [dist.P2POp(dist.isend, send, peer, group), dist.P2POp(dist.irecv, recv, peer, group)]
        pending.append((a, b, send, recv))
        sent += send.numel() * 4
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    for a, b, _, recv in pending:
        v[:, a - r0:b - r0, :] += recv.to(v.device) if host else recv
    return sent


class GpuOps:
    """The slab operators on this library's kernels (torch tensors on the context's GPU)."""

    def __init__(self, ctx, arith: int = _lib.STRICT, storage: int = _lib.F32):
        import torch
        self.torch, self.ctx, self.arith, self.storage = torch, ctx, arith, storage
        self.L = _lib.lib()

    def tensor(self, a, dtype=None):
        t = self.torch.from_numpy(np.ascontiguousarray(a)).cuda()
        return t if dtype is None else t.to(dtype)

    def zeros_u32(self, n):
        return self.torch.zeros(n, dtype=self.torch.int32, device="cuda")

    def full_u32(self, n, v):
        return self.torch.full((n,), v, dtype=self.torch.int32, device="cuda")

    def ones_f32(self, n):
        return self.torch.ones(n, dtype=self.torch.float32, device="cuda")

    def ratio_buffer(self, n):
        dt = {_lib.F32: self.torch.float32, _lib.BF16: self.torch.bfloat16, _lib.F16: self.torch.float16}
        return self.torch.empty(n, dtype=dt[self.storage], device="cuda")

    def preprocess(self, raw_f32):
        """-log (data_loader.hpp:84-86) into the storage type."""
        out = self.ratio_buffer(raw_f32.numel())
        _lib.check(self.L.xpr_preprocess_apply(self.ctx.handle, raw_f32.data_ptr(), out.data_ptr(), self.storage,
                                               raw_f32.numel(), 0, None, 1, self._s()), "preprocess")
        return out

    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def forward(self, vol, sums, pd, n_pd, L):
        _lib.check(self.L.xpr_forward(self.ctx.handle, vol.data_ptr(), sums.data_ptr(), pd.data_ptr(), n_pd,
                                      C.byref(L), self._s()), "forward")

    def error(self, images, sums, ratio, n, weight):
        _lib.check(self.L.xpr_error(self.ctx.handle, images.data_ptr(), self.storage, sums.data_ptr(),
                                    ratio.data_ptr(), self.storage, n, weight, _lib.ERROR_STD, 1, None, self._s()),
                   "error")

    def backward(self, vol, ratio, pd, n_pd, L):
        _lib.check(self.L.xpr_backward(self.ctx.handle, vol.data_ptr(), ratio.data_ptr(), self.storage,
                                       pd.data_ptr(), n_pd, C.byref(L), self._s()), "backward")

    def exchange(self, sums, plan, r0, n_img, rows, width, group=None):
        return exchange_rows(sums, plan, r0, n_img, rows, width, group)

    def all_reduce_sum(self, sums, group=None):
        import torch.distributed as dist
        if dist.get_backend(group) == "nccl":
            dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
        else:  # host staging for backends without device buffers
            h = sums.cpu()
            dist.all_reduce(h, op=dist.ReduceOp.SUM, group=group)
            sums.copy_(h)

    def synchronize(self):
        self.torch.cuda.synchronize()

    def to_host(self, t):
        return t.cpu().numpy()


def _rows_of(images, n_img, H, W, r0, r1):
    """Rows [r0, r1) of each of n_img images of H x W (flat numpy array or torch tensor)."""
    v = images.reshape(n_img, H, W)[:, r0:r1, :]
    if isinstance(v, np.ndarray):
        return np.ascontiguousarray(v).reshape(-1)
    return v.contiguous().reshape(-1)


class SlabReconstruction:
    """The naive method on one y-slab per rank.

    raw: (projections, det_h, det_w) float32 intensities (acquisition order), on every rank.
    pd_all: ProjData (projections * modules, 20) in angle-major order and `g` the grid
    description (`projector.geometry`)."""

    def __init__(self, ops, raw, pd_all, g, modules=1, it=1, sit=10, seed=5489, weight=1.0,
                 weight_factor=0.9, rank=0, world=1, group=None, images=None, shape=None, windowed=True):
        """images / shape: already preprocessed subset-major images in the storage type and
        the (projections, det_h, det_w) they come from, instead of `raw`.  windowed: each
        rank keeps the detector rows its slab reaches and exchanges the shared rows with
        the ranks whose windows overlap (else the whole detector and an all-reduce)."""
        self.ops, self.rank, self.world, self.group = ops, rank, world, group
        P, H, W = raw.shape if raw is not None else shape
        self.P, self.Hd, self.Wd, self.M, self.S, self.it = P, H, W, modules, sit, it
        self.Pc = int(g["concurrent"])
        self.Wv, self.Hv, self.vx = int(g["vwidth"]), int(g["vheight"]), float(g["vx"])
        self.orig = [float(v) for v in g["orig"]]
        self.y0, self.y1 = slab_bounds(self.Hv, world, rank)
        self.seed, self.weight, self.weight_factor = seed, weight, weight_factor
        self.windowed = bool(windowed) and world > 1
        if self.windowed:
            self.windows = [row_window(pd_all, g, *slab_bounds(self.Hv, world, q), H) for q in range(world)]
        else:
            self.windows = [(0, H)] * world
        self.r0, self.r1 = self.windows[rank]
        self.rows = self.r1 - self.r0
        self.plan = exchange_plan(self.windows, rank) if self.windowed else []
        self.npix = self.Pc * W * self.rows
        order = [s + k * sit for s in range(sit) for k in range(self.Pc)]
        images = images if images is not None else ops.preprocess(ops.tensor(raw[order].reshape(-1)))
        self.images = images if self.rows == H else _rows_of(images, sit * self.Pc, H, W, self.r0, self.r1)
        pd = np.ascontiguousarray(pd_all.reshape(P, modules, 20)[order].reshape(-1, 20))
        self.pd = [ops.tensor(pd[s * self.Pc * modules:(s + 1) * self.Pc * modules]) for s in range(sit)]
        self.vol = ops.ones_f32(self.Wv * max(self.y1 - self.y0, 0) * self.Wv)
        self.sums = ops.full_u32(self.npix, FIXED_ONE)
        self.ratio = ops.ratio_buffer(self.npix)
        self.exchanged_bytes = 0

    def launch(self, origin):
        d = _lib.Launch()
        d.vmin[:] = [0, self.y0, 0]
        d.vmax[:] = [self.Wv, self.y1, self.Wv]
        d.origin[:] = origin
        d.voxel[:] = [self.vx] * 3
        d.det_w, d.rows, d.row_offset, d.n_angles, d.modules = self.Wd, self.rows, self.r0, self.Pc, self.M
        d.arith = getattr(self.ops, "arith", _lib.STRICT)
        return d

    def _schedule(self):
        steps = self.it * self.S
        jit = np.zeros(3 * steps, np.float32)
        _lib.check(_lib.lib().xpr_jitter(self.seed, jit.size, self.vx, jit.ctypes.data), "xpr_jitter")
        self._origins = [[float(np.float32(self.orig[c]) + jit[3 * k + c]) for c in range(3)] for k in range(steps)]
        w, self._weights = np.float32(self.weight), []
        for k in range(steps):
            self._weights.append(float(w))
            if k % self.S == self.S - 1:
                w = np.float32(w * np.float32(self.weight_factor))

    def step(self, k):
        """Sub-iteration k (< it * sit); the jitter draws are the same on every rank."""
        if not hasattr(self, "_origins"):
            self._schedule()
        s = k % self.S
        L = self.launch(self._origins[k])
        has_slab = self.y1 > self.y0 and self.rows > 0
        n_pd = self.Pc * self.M
        if k > 0:  # the first sub-iteration has no forward (reconstruction_n.hpp:70)
            if has_slab:
                self.ops.forward(self.vol, self.sums, self.pd[s], n_pd, L)
            if self.windowed:
                self.exchanged_bytes += self.ops.exchange(self.sums, self.plan, self.r0, self.Pc, self.rows, self.Wd,
                                                          self.group)
            elif self.world > 1:
                self.ops.all_reduce_sum(self.sums, self.group)
                self.exchanged_bytes += 4 * self.npix
        img = self.images[s * self.npix:(s + 1) * self.npix]
        self.ops.error(img, self.sums, self.ratio, self.npix, self._weights[k])  # zeroes the sums
        if has_slab:
            self.ops.backward(self.vol, self.ratio, self.pd[s], n_pd, L)

    def run(self):
        """All it * sit sub-iterations."""
        for k in range(self.it * self.S):
            self.step(k)
        self.ops.synchronize()

    def gather(self):
        """The whole volume (rank order = slab order), on every rank."""
        v = np.asarray(self.ops.to_host(self.vol), np.float32)
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist
        parts = [None] * self.world
        dist.all_gather_object(parts, v, group=self.group)
        return np.concatenate([np.asarray(p, np.float32) for p in parts])
