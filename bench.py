#!/usr/bin/env python3
"""Throughput of one sub-iteration of XPRecon's iterative cone-beam path on B200.

Metric (the reference's headline): GUPS = voxels x projections-per-sub-iteration
/ sub-iteration time / 1e9, a sub-iteration being forward projection + error +
multiplicative back-projection (reconstruction_n.hpp:65-76) over one angular
subset.  Workload: the 512^3-phantom configuration -- the reference derives a
768^3 reconstruction grid from the 768 x 768 detector (geometry.hpp:50-56);
720 projections over 360 degrees, sit = 10, so 72 projections per sub-iteration;
px 0.1 mm, so 100, sd 1000, rx 1.5 px, sx -2, sy 3 (mm).  Data are synthetic
(seeded ellipsoid phantom + textured background, projected with this library's
forward projector, Poisson noise at 1e5 photons, -log preprocessing on the GPU).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--arith fast|strict] [--storage fp32|bf16|fp16] [--shard]
                  [--config c2|c1|c2slab|c3h|c4|c4s|c4one|c5]

Under torchrun each rank reconstructs its own volume (weak scaling, no
collective on the data path), or with --shard one volume split into y-slabs over
the ranks (strong scaling, one all-reduce of the detector sums per sub-iteration);
the time is the max over ranks.  c3h runs whole reconstructions in every memory
mode under a device-memory cap; c4 / c4s many reconstructions as one batched run;
c5 a request loop with Poisson arrivals (latency percentiles and served GUPS).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c2": dict(desc="768^3 recon grid (512^3 phantom: 40 ellipsoids + 5% textured background), "
                    "720 projections of 768x768, sit=10 -> 72 per sub-iteration",
               dwidth=768, dheight=768, projections=720, sit=10, px=0.1, so=100.0, sd=1000.0, rx=1.5, sx=-2.0,
               sy=3.0, phantom=512, ellipsoids=40, background=0.05, i0=1e5, seed=2),
    # the c2 geometry restricted to the central 256 layers (profiling-sized: ~3 GB on the device)
    "c2slab": dict(desc="c2 geometry, central 256-layer y-slab of the 768^3 grid, 72 projections per sub-iteration",
                   dwidth=768, dheight=768, projections=720, sit=10, px=0.1, so=100.0, sd=1000.0, rx=1.5, sx=-2.0,
                   sy=3.0, phantom=512, ellipsoids=40, background=0.05, i0=1e5, seed=2, slab=(256, 512)),
    "c1": dict(desc="192^3 recon grid (128^3 phantom: 10 ellipsoids), 180 projections of 192x192, sit=10 -> 18",
               dwidth=192, dheight=192, projections=180, sit=10, px=0.1, so=100.0, sd=1000.0, rx=0.0, sx=0.0,
               sy=0.0, phantom=128, ellipsoids=10, background=0.0, i0=1e5, seed=1),
    # many small reconstructions as one batched, graph-captured, autotuned run (BF16 storage)
    "c4": dict(desc="64 independent 384^3 recon grids (256^3 ellipsoid phantoms, so U[80,120], sd U[800,1200]), "
                    "360 projections of 384x384 on 3 modules of 128 px (roll/pitch/yaw U[-2,2] deg), sit=10 -> 36, "
                    "it=2, BF16 image/ratio storage, one batched persistent launch per phase in a CUDA graph",
               batch=64, dwidth=384, dheight=384, projections=360, sit=10, it=2, modules=3, px=0.1, rpy=2.0,
               phantom=256, ellipsoids=12, background=0.0, i0=1e5, seed=4, plain_sample=4),
    # a request loop: Poisson arrivals of mixed-size scans, continuous batching
    "c5": dict(desc="Poisson arrivals (4/s) of 500 scans: phantom edge in {128, 256, 384, 512, 768} (recon "
                    "grid and detector 1.5x: 192 .. 1152), {180, 360, 720, 1080} projections, it 1, sit 10, "
                    "1e5 photons; servers with FP32 storage and with the BF16 form (BF16 ratio, FP16 images)",
               serve=True, requests=500, rate=4.0, edges=[128, 256, 384, 512, 768],
               projections_set=[180, 360, 720, 1080], sit=10, it=1, px=0.1, i0=1e5, seed=5, ellipsoids=10,
               background=0.0, plain_requests=100),
    # out-of-core at half linear scale: the volume does not fit the device-memory cap
    "c3h": dict(desc="c3 at half linear scale: 1536x1024x1536 recon grid (9.7 GB), 1000 projections of "
                     "1536x1024 (6.3 GB), sit 20 -> 50, it 1, under an 8 GB device-memory cap: naive without "
                     "the cap, then method_1b, method_1c and method_2 with it",
                outofcore=True, dwidth=1536, dheight=1024, projections=1000, sit=20, it=1, px=0.1, so=100.0,
                sd=1000.0, phantom=1024, ellipsoids=60, background=0.0, i0=5e4, seed=3, mem_cap=8 << 30,
                methods=["naive", "method_1b", "method_1c", "method_2"]),
    # the batched form where it matters: reconstructions too small to fill the GPU alone
    "c4s": dict(desc="256 small independent reconstructions: 96x64 detector on 3 modules of 32 px (roll/pitch/yaw "
                     "U[-2,2] deg) -> 96x64x96 grid, 180 projections, sit=10 -> 18, it=2, so U[80,120], "
                     "sd U[800,1200], BF16 image/ratio storage, batched persistent launches in a CUDA graph",
                batch=256, dwidth=96, dheight=64, projections=180, sit=10, it=2, modules=3, px=0.1, rpy=2.0,
                phantom=56, ellipsoids=6, background=0.0, i0=1e5, seed=6, plain_sample=16),
    # one problem of the c4 family (profiling-sized)
    "c4one": dict(desc="one 384^3 recon grid of the c4 family (3 tilted modules, 36 projections per sub-iteration)",
                  batch=1, dwidth=384, dheight=384, projections=360, sit=10, it=2, modules=3, px=0.1, rpy=2.0,
                  phantom=256, ellipsoids=12, background=0.0, i0=1e5, seed=4, plain_sample=0),
}

FLOPS_PER_PAIR = 44          # algorithmic FP32 operations per (voxel, projection) pair, forward + backward
NOMINAL_FP32_LANES = 148 * 128
# DRAM bytes (read + write) per voxel per launch, from one ncu capture of each kernel on the
# c2 geometry's central 256-layer slab (150,994,944 voxels, FP32 storage); scaled to a
# launch by its voxel count for the same geometry
MEASURED_TRAFFIC_PER_VOXEL = {
    "strict": {"forward": 716.4e6 / 150994944, "backward": 1211.8e6 / 150994944},
    "fast": {"forward": 716.1e6 / 150994944, "backward": 1219.0e6 / 150994944},
}
# executed-work figures of the same captures (profiles/k_*_c2slab.md): issue-active share,
# l1tex (shared-memory pipe) throughput and thread instructions per (voxel, projection) pair
MEASURED_PROFILE = {
    "strict": {"forward": {"issue_active_pct": 67.7, "l1tex_pct": 74.5, "fma_pipe_pct": 56.2,
                           "thread_inst_per_pair": 14.5, "shared_atomic_replay_pct": 48.6},
               "backward": {"issue_active_pct": 70.7, "l1tex_pct": 46.7, "fma_pipe_pct": 65.8,
                            "thread_inst_per_pair": 15.7},
               "source": "ncu --set full, c2 geometry 256-layer slab: profiles/k_forward_tiled_strict_c2slab.md, "
                         "profiles/k_backward_tiled_strict_c2slab.md"},
    "fast": {"forward": {"issue_active_pct": 76.0, "l1tex_pct": 84.9, "thread_inst_per_pair": 13.0},
             "backward": {"issue_active_pct": 68.7, "thread_inst_per_pair": 11.5},
             "source": "ncu --set full, c2 geometry 256-layer slab: profiles/k_forward_tiled_fast_c2slab.md, "
                       "profiles/k_backward_tiled_fast_c2slab.md"},
}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--arith", choices=["fast", "strict"], default=None,
                   help="projector contract: strict = the reference kernels' IEEE results bit for bit (the "
                        "default), fast = the relaxed-math form (the default of the tilted-module batched "
                        "configurations c4 / c4s / c4one, which have no reference counterpart)")
    p.add_argument("--storage", choices=["fp32", "bf16", "fp16"], default=None,
                   help="image / ratio storage (default: fp32; bf16 for the batched configurations)")
    p.add_argument("--config", choices=sorted(CONFIGS), default="c2")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--shard", action="store_true",
                   help="one reconstruction split into y-slabs over the ranks (the default for N > 1): the "
                        "u32 detector sums of the rows where neighbouring slabs' footprints overlap are "
                        "exchanged each sub-iteration (strong scaling)")
    p.add_argument("--replicas", action="store_true",
                   help="N > 1: an independent reconstruction per rank instead (weak scaling, no exchange)")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def emit(obj):
    print(json.dumps(obj), flush=True)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        import tempfile
        self.path = os.path.join(tempfile.gettempdir(), "xpr_clocks_%d.csv" % os.getpid())

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for i, n in enumerate(names):
                if r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ----------------------------------------------------------------------------- synthetic data
def make_phantom(cfg, vx, W, Hv, device, seed, y0=0, y1=None):
    """Seeded ellipsoid phantom (+ smooth Gaussian-textured background) in the central
    phantom^3 region of the (y, z, x) grid; values are attenuation per voxel (mu * vx).
    Only layers [y0, y1) are materialised."""
    import torch
    rng = np.random.default_rng(seed)
    y1 = Hv if y1 is None else y1
    full = torch.zeros((Hv, W, W), dtype=torch.float32, device=device) if (y0, y1) == (0, Hv) else None
    vol = full if full is not None else torch.zeros((y1 - y0, W, W), dtype=torch.float32, device=device)
    ph = cfg["phantom"]
    c0 = np.array([W / 2.0, Hv / 2.0, W / 2.0])  # x, y, z centre in voxels
    mus = []
    for _ in range(cfg["ellipsoids"]):
        while True:
            cx, cz = rng.uniform(-ph / 2, ph / 2, 2)
            if cx * cx + cz * cz <= (ph / 2) ** 2:
                break
        cy = rng.uniform(-ph / 2, ph / 2)
        axes = rng.uniform(0.03, 0.25, 3) * ph
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        mu = rng.uniform(0.0, 0.02)
        mus.append(mu)
        cen = c0 + np.array([cx, cy, cz])
        r = axes.max()
        lo = np.maximum(np.floor(cen - r).astype(int), 0)
        hi = np.minimum(np.ceil(cen + r).astype(int) + 1, [W, Hv, W])
        if (hi <= lo).any():
            continue
        xs = torch.arange(lo[0], hi[0], device=device, dtype=torch.float32) - float(cen[0])
        ys = torch.arange(lo[1], hi[1], device=device, dtype=torch.float32) - float(cen[1])
        zs = torch.arange(lo[2], hi[2], device=device, dtype=torch.float32) - float(cen[2])
        Y, Z, X = torch.meshgrid(ys, zs, xs, indexing="ij")
        P = torch.stack([X, Y, Z], dim=-1) @ torch.from_numpy(q.astype(np.float32)).to(device)
        inside = ((P / torch.from_numpy(axes.astype(np.float32)).to(device)) ** 2).sum(-1) <= 1.0
        a, b = max(lo[1], y0), min(hi[1], y1)
        if a < b:
            vol[a - y0:b - y0, lo[2]:hi[2], lo[0]:hi[0]] += inside[a - lo[1]:b - lo[1]].float() * float(mu * vx)
        del Y, Z, X, P, inside
    if cfg["background"] > 0:
        g = torch.Generator(device=device).manual_seed(seed)
        noise = torch.randn((1, 1, ph, ph, ph), device=device, generator=g)
        k = torch.exp(-0.5 * (torch.arange(-12, 13, device=device, dtype=torch.float32) / 4.0) ** 2)
        k = k / k.sum()
        import torch.nn.functional as F
        noise = F.conv3d(noise, k.view(1, 1, -1, 1, 1), padding=(12, 0, 0))
        noise = F.conv3d(noise, k.view(1, 1, 1, -1, 1), padding=(0, 12, 0))
        noise = F.conv3d(noise, k.view(1, 1, 1, 1, -1), padding=(0, 0, 12))[0, 0]
        noise = noise / noise.std()
        level = cfg["background"] * float(np.mean(mus)) * vx
        bg = torch.clamp(level * (1.0 + noise), min=0.0)
        py0, x0 = (Hv - ph) // 2, (W - ph) // 2
        a, b = max(py0, y0), min(py0 + ph, y1)
        if a < b:
            vol[a - y0:b - y0, x0:x0 + ph, x0:x0 + ph] += bg[a - py0:b - py0]
        del noise, bg
    return vol.reshape(-1).contiguous()


class Problem:
    """Device-resident state of one reconstruction of the benchmark configuration."""

    def __init__(self, cfg, arith, storage, device_index, seed):
        import torch
        from xpulse_recon_b200 import _lib
        from xpulse_recon_b200.projector import Context, JitterSource, geometry
        self.torch, self.L = torch, _lib.lib()
        self.cfg = cfg
        self.arith = _lib.FAST if arith == "fast" else _lib.STRICT
        self.storage = {"fp32": _lib.F32, "bf16": _lib.BF16, "fp16": _lib.F16}[storage]
        self.tdt = {"fp32": torch.float32, "bf16": torch.bfloat16, "fp16": torch.float16}[storage]
        self.ctx = Context(device_index)
        self.device = torch.device("cuda", device_index)
        kw = {k: cfg[k] for k in ("dwidth", "dheight", "projections", "sit", "px", "so", "sd", "rx", "sx", "sy")}
        self.pd_all, self.g = geometry(**kw)
        self.P, self.S = cfg["projections"], cfg["sit"]
        self.Pc, self.W, self.Hv = self.g["concurrent"], self.g["vwidth"], self.g["vheight"]
        self.Wd, self.Hd = cfg["dwidth"], cfg["dheight"]
        self.y0, self.y1 = cfg.get("slab", (0, self.Hv))
        self.nvox = self.W * (self.y1 - self.y0) * self.W
        self.npix = self.Pc * self.Wd * self.Hd
        self.jitter = JitterSource(seed)
        self.stream = torch.cuda.Stream(device=self.device)
        self.sp = C.c_void_p(self.stream.cuda_stream)
        d = self.device
        self.pd_sub = []
        for s in range(self.S):
            idx = [s + k * self.S for k in range(self.Pc)]
            self.pd_sub.append(torch.from_numpy(np.ascontiguousarray(self.pd_all[idx])).to(d))
        # measured projections: simulate with the forward projector, Poisson noise, -log on the GPU
        with torch.cuda.stream(self.stream):
            phantom = make_phantom(cfg, self.g["vx"], self.W, self.Hv, d, seed, self.y0, self.y1)
            self.images = []
            self.raw_host = []  # the raw intensities I / I0 of each subset (for the raw end-to-end leg)
            sums = torch.zeros(self.npix, dtype=torch.int32, device=d)
            gen = torch.Generator(device=d).manual_seed(seed + 1)
            for s in range(self.S):
                sums.zero_()
                self._forward(phantom, sums, s, list(self.g["orig"]))
                p = sums.view(torch.int32).to(torch.int64).bitwise_and(0xFFFFFFFF).to(torch.float32) / float(1 << 22)
                inten = torch.poisson(cfg["i0"] * torch.exp(-p), generator=gen) / cfg["i0"]
                out = torch.empty(self.npix, dtype=self.tdt, device=d)
                _lib.check(self.L.xpr_preprocess_apply(self.ctx.handle, inten.data_ptr(), out.data_ptr(), self.storage,
                                                       self.npix, 0, None, 1, self.sp), "preprocess")
                self.images.append(out)
                self.raw_host.append(inten.cpu())
                del p, inten
            self.phantom_host = None
            self.phantom = phantom
            self.vol = torch.ones(self.nvox, dtype=torch.float32, device=d)
            self.sums = torch.full((self.npix,), 1 << 22, dtype=torch.int32, device=d)
            self.ratio = self.sums if self.storage == _lib.F32 else torch.empty(self.npix, dtype=self.tdt, device=d)
            self.residual = torch.zeros(1, dtype=torch.float64, device=d)
        self.stream.synchronize()
        self.sit_next = 0
        self.weight = 1.0
        # the first sub-iteration has no forward (reconstruction_n.hpp:70): run it untimed
        self.subiteration(first=True)
        self.stream.synchronize()

    def launch_desc(self, origin):
        from xpulse_recon_b200 import _lib
        L = _lib.Launch()
        L.vmin[:] = [0, self.y0, 0]
        L.vmax[:] = [self.W, self.y1, self.W]
        L.origin[:] = origin
        L.voxel[:] = [self.g["vx"]] * 3
        L.det_w, L.rows, L.row_offset = self.Wd, self.Hd, 0
        L.n_angles, L.modules = self.Pc, 1
        L.arith = self.arith
        return L

    def _forward(self, vol, sums, s, origin):
        from xpulse_recon_b200 import _lib
        L = self.launch_desc(origin)
        _lib.check(self.L.xpr_forward(self.ctx.handle, vol.data_ptr(), sums.data_ptr(), self.pd_sub[s].data_ptr(),
                                      self.Pc, C.byref(L), self.sp), "forward")

    def next_origin(self):
        o = []
        for i in range(3):
            o.append(float(np.float32(np.float32(self.g["orig"][i]) + np.float32(self.jitter.draw(self.g["vx"])))))
        return o

    def subiteration(self, first=False, events=None, images=None):
        """forward -> error -> backward -> reset sums, with optional per-kernel events."""
        from xpulse_recon_b200 import _lib
        s = self.sit_next
        self.sit_next = (s + 1) % self.S
        L = self.launch_desc(self.next_origin())
        h, sp = self.ctx.handle, self.sp
        img = self.images[s] if images is None else images
        if events:
            events[0].record(self.stream)
        if not first:
            _lib.check(self.L.xpr_forward(h, self.vol.data_ptr(), self.sums.data_ptr(), self.pd_sub[s].data_ptr(),
                                          self.Pc, C.byref(L), sp), "forward")
        if events:
            events[1].record(self.stream)
        _lib.check(self.L.xpr_error(h, img.data_ptr(), self.storage, self.sums.data_ptr(), self.ratio.data_ptr(),
                                    self.storage, self.npix, self.weight, _lib.ERROR_STD, 1,
                                    self.residual.data_ptr(), sp), "error")
        if events:
            events[2].record(self.stream)
        _lib.check(self.L.xpr_backward(h, self.vol.data_ptr(), self.ratio.data_ptr(), self.storage,
                                       self.pd_sub[s].data_ptr(), self.Pc, C.byref(L), sp), "backward")
        if events:
            events[3].record(self.stream)
        if self.ratio is self.sums:  # in-place FP32 ratio: reset the sums for the next forward
            _lib.check(self.L.xpr_fill_u32(h, self.sums.data_ptr(), 0, self.npix, sp), "fill")
        return s


# ----------------------------------------------------------------------------- CPU (reference kernels)
REF_SAMPLE_LAYERS = 128  # the central y-slab both CPU legs time when the whole grid is too large


def cpu_reference_step_factory(cfg, seconds_target, max_layers=REF_SAMPLE_LAYERS):
    """The reference's own OpenCL kernels (oracle/_ref, built from its sources) on the host
    cores: forward + error + backward of a y-slab of the grid against one sub-iteration's
    projections -- the whole grid when it is small (c1), else the central max_layers layers
    (the same sample for cpu_baseline and the reference arm, so that their fixed costs --
    the error step over the whole detector -- weigh the same).  seconds_target only sets
    how often a whole small grid is repeated.  Returns (step_fn, info)."""
    from oracle import oracle as O
    R = O.ref_lib()
    kind = "reference"
    if R is None:
        kind = "port"
    gp = O.geom_params(**{k: cfg[k] for k in ("dwidth", "dheight", "projections", "sit", "px", "so", "sd", "rx",
                                               "sx", "sy")})
    pd_all, go = O.geometry(gp)
    Pc, W, Hv, Wd, Hd = int(go.concurrent), int(go.vwidth), int(go.vheight), cfg["dwidth"], cfg["dheight"]
    pd = O.subset_projdata(pd_all, cfg["projections"], cfg["sit"], 1, 1, Pc)
    rng = np.random.default_rng(9)
    images = rng.uniform(0.02, 0.3, Pc * Wd * Hd).astype(np.float32)
    origin = [float(np.float32(go.orig[i]) + np.float32(0.37 * go.vx)) for i in range(3)]
    y_mid = Hv // 2

    def run(layers, reps=1):
        y0 = y_mid - layers // 2
        n = W * layers * W
        vol = rng.uniform(1e-4, 3e-4, O.ndrange(n)).astype(np.float32)
        t = time.perf_counter()
        for _ in range(reps):
            sums = np.zeros(Pc * Wd * Hd, np.uint32)
            if kind == "reference":
                O.ref_forward(vol, sums, pd, Wd, Hd, origin, Pc, 1, (0, y0, 0), (W, y0 + layers, W), (0, Hd),
                              [go.vx] * 3)
                O.ref_error(images, sums, Wd, Hd, 1.0)
                O.ref_backward(vol, sums.view(np.float32), pd, Wd, Hd, origin, Pc, 1, (0, y0, 0),
                               (W, y0 + layers, W), (0, Hd), [go.vx] * 3)
            else:
                L, keep = O.make_launch((0, y0, 0), (W, y0 + layers, W), origin, [go.vx] * 3, Wd, Hd, 0, Pc, 1)
                O.forward(vol, sums, pd, L)
                O.error(images, sums, 1.0)
                O.backward(vol, sums.view(np.float32), pd, L)
        return time.perf_counter() - t, n * Pc * reps

    whole = W * Hv * W * Pc <= 2e9
    layers = Hv if whole else min(Hv, max_layers)
    reps = 1
    if whole:
        dt_full, _ = run(Hv)
        reps = int(max(1, round(seconds_target / max(dt_full, 1e-3))))
    info = {"kind": kind, "cores": os.cpu_count(), "layers": layers, "W": W, "Hv": Hv, "Pc": Pc, "reps": reps}
    if not whole and max_layers <= 16:
        info["probe_s"], _ = run(layers)  # a timing probe of the thin slab
    return (lambda: run(layers, reps)), info


def cpu_baseline(cfg, seconds):
    step, info = cpu_reference_step_factory(cfg, seconds)
    dt, pairs = step()
    return {"value": pairs / dt / 1e9, "unit": "GUPS", "cores": info["cores"], "kind": info["kind"],
            "sample": "forward + error + backward of a %d-layer y-slab (%dx%dx%d voxels) against one "
                      "sub-iteration's %d projections, %d time(s), OpenMP on %d host threads, %.1f s"
                      % (info["layers"], info["W"], info["layers"], info["W"], info["Pc"], info["reps"],
                         info["cores"], dt)}


# ----------------------------------------------------------------------------- main arms
def run_reference(args, cfg, rank, world):
    if rank != 0:
        return 0
    if any(k not in cfg for k in ("so", "sd", "rx", "sx", "sy")):
        emit({"impl": "reference", "unavailable": "the reference runs one reconstruction per process; %s is a "
              "batched / served / out-of-core workload of this library (time its single-problem kernels with "
              "--config c2)" % args.config})
        return 0
    # the cpu_baseline sample (whole small grids once per step; else the central 128-layer slab,
    # thinned to no fewer than 64 layers only if the whole run would take over about five
    # minutes).  A step costs a fixed part (the error step over the whole detector, thread
    # start-up) plus a part per layer; probes of 8 and 16 layers separate the two.
    n = max(1, args.steps + args.warmup)
    _, probe_info = cpu_reference_step_factory(cfg, 0.0, max_layers=8)
    layers = REF_SAMPLE_LAYERS
    if probe_info["layers"] < probe_info["Hv"]:
        t8 = probe_info["probe_s"]
        t16 = cpu_reference_step_factory(cfg, 0.0, max_layers=16)[1]["probe_s"]
        per_layer = max(t16 - t8, 1e-4) / 8.0
        fixed = max(t8 - 8.0 * per_layer, 0.0)
        if n * (fixed + per_layer * REF_SAMPLE_LAYERS) > 300.0:
            layers = int(max(64, (300.0 / n - fixed) / per_layer))
    step, info = cpu_reference_step_factory(cfg, 0.0, max_layers=layers)
    for _ in range(args.warmup):
        step()
    tot_t, tot_p = 0.0, 0
    for _ in range(args.steps):
        dt, p = step()
        tot_t += dt
        tot_p += p
    v = tot_p / tot_t / 1e9
    sample = ("forward + error + backward of a %d-layer y-slab of the %d^3 grid against %d projections per step"
              % (info["layers"], info["W"], info["Pc"]))
    emit({"impl": "reference", "metric": "GUPS per sub-iteration (voxel x projection pairs / s)", "value": v,
          "unit": "GUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
          "ms_per_step": 1000.0 * tot_t / args.steps, "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "f32", "data": "synthetic",
          "config": {"workload": args.config + ": " + cfg["desc"], "arith": "reference OpenCL kernels, IEEE fp32",
                     "storage": "fp32"},
          "cpu_baseline": {"value": v, "unit": "GUPS", "cores": info["cores"], "kind": info["kind"],
                           "sample": sample},
          "e2e": {"value": v, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return 0


def run_ours(args, cfg, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    args.storage = args.storage or "fp32"
    prob = Problem(cfg, args.arith, args.storage, local, cfg["seed"] + 1000 * rank)
    stream = prob.stream
    K, Wm = args.steps, args.warmup
    for _ in range(Wm):
        prob.subiteration()
    stream.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
    clocks = ClockSampler(local)
    clocks.start()
    for k in range(K):
        prob.subiteration(events=evs[k])
    stream.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = evs[0][0].elapsed_time(evs[K - 1][3])
    fwd = [e[0].elapsed_time(e[1]) for e in evs]
    err = [e[1].elapsed_time(e[2]) for e in evs]
    bwd = [e[2].elapsed_time(e[3]) for e in evs]
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    pairs_step = prob.nvox * prob.Pc
    value = pairs_step * K * world / (total_ms / 1000.0) / 1e9

    # ---- e2e: host buffers through the C ABI; uploads overlapped on a copy stream
    from xpulse_recon_b200 import _lib
    L = prob.L
    nbytes = prob.npix * prob.images[0].element_size()
    pinned = []
    for s in range(prob.S):
        hp = C.c_void_p()
        _lib.check(L.xpr_alloc_pinned(prob.ctx.handle, nbytes, C.byref(hp)), "alloc_pinned")
        host = prob.images[s].view(torch.uint8).cpu().numpy()  # keep alive across the copy
        C.memmove(hp, host.ctypes.data, nbytes)
        pinned.append(hp)
    # the raw leg: intensities I / I0 (float32) go up instead, and -log runs on the device
    raw_bytes = prob.npix * 4
    pinned_raw = []
    for s in range(prob.S):
        hp = C.c_void_p()
        _lib.check(L.xpr_alloc_pinned(prob.ctx.handle, raw_bytes, C.byref(hp)), "alloc_pinned")
        host = prob.raw_host[s].numpy()
        C.memmove(hp, host.ctypes.data, raw_bytes)
        pinned_raw.append(hp)
    res_host = C.c_void_p()
    _lib.check(L.xpr_alloc_pinned(prob.ctx.handle, 8, C.byref(res_host)), "alloc_pinned")
    dbuf = [torch.empty_like(prob.images[0]) for _ in range(2)]
    rbuf = [torch.empty(prob.npix, dtype=torch.float32, device=prob.device) for _ in range(2)]
    copy_stream = torch.cuda.Stream(device=prob.device)
    cs = C.c_void_p(copy_stream.cuda_stream)
    up_done = [torch.cuda.Event() for _ in range(2)]
    used = [torch.cuda.Event() for _ in range(2)]

    def e2e_steps(n, timed, raw=False):
        """n sub-iterations with each subset's images uploaded from page-locked host memory
        (double-buffered on a copy stream) and the residual read back; raw: the uploads are
        the raw intensities and the -log preprocessing runs on the device in the step."""
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        src, dst, size = (pinned_raw, rbuf, raw_bytes) if raw else (pinned, dbuf, nbytes)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        start.record(prob.stream)
        s0 = prob.sit_next
        _lib.check(L.xpr_upload(prob.ctx.handle, dst[0].data_ptr(), src[s0], size, cs), "upload")
        up_done[0].record(copy_stream)
        for k in range(n):
            b = k % 2
            if k + 1 < n:  # prefetch the next subset while this one computes
                nb = (k + 1) % 2
                if k >= 1:
                    copy_stream.wait_event(used[nb])
                nxt = (prob.sit_next + 1) % prob.S
                _lib.check(L.xpr_upload(prob.ctx.handle, dst[nb].data_ptr(), src[nxt], size, cs), "upload")
                up_done[nb].record(copy_stream)
            prob.stream.wait_event(up_done[b])
            if raw:
                _lib.check(L.xpr_preprocess_apply(prob.ctx.handle, rbuf[b].data_ptr(), dbuf[b].data_ptr(),
                                                  prob.storage, prob.npix, 0, None, 1, prob.sp), "preprocess")
            prob.subiteration(images=dbuf[b])
            used[b].record(prob.stream)
            _lib.check(L.xpr_download(prob.ctx.handle, res_host, prob.residual.data_ptr(), 8, prob.sp), "download")
        end.record(prob.stream)
        prob.stream.synchronize()
        return start.elapsed_time(end)

    e2e_steps(min(2, K), False)
    e2e_ms = e2e_steps(K, True)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = pairs_step * K * world / (e2e_ms / 1000.0) / 1e9
    e2e_steps(min(2, K), False, raw=True)
    raw_ms = e2e_steps(K, True, raw=True)
    if dist:
        t = torch.tensor([raw_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        raw_ms = float(t.item())
    e2e_raw_value = pairs_step * K * world / (raw_ms / 1000.0) / 1e9
    for hp in pinned + pinned_raw:
        L.xpr_free_pinned(prob.ctx.handle, hp)
    L.xpr_free_pinned(prob.ctx.handle, res_host)

    # ---- roofline of the dominant kernel
    f_ms, b_ms = statistics.mean(fwd), statistics.mean(bwd)
    dom = "backward" if b_ms >= f_ms else "forward"
    dom_ms = max(f_ms, b_ms)
    isz = prob.images[0].element_size()
    if dom == "forward":
        alg_bytes = 4 * prob.nvox + 4 * prob.npix
    else:
        alg_bytes = 8 * prob.nvox + isz * prob.npix
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = alg_bytes / (dom_ms / 1000.0) / 1e9
    traffic = None
    if args.config in ("c2", "c2slab") and args.storage == "fp32":
        traffic = MEASURED_TRAFFIC_PER_VOXEL[args.arith][dom] * prob.nvox
    sm_mhz = (clk or {}).get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = NOMINAL_FP32_LANES * 2 * float(sm_mhz) * 1e6 / 1e12
    step_ms = total_ms / K
    line = {
        "metric": "GUPS per sub-iteration (voxel x projection pairs / s)",
        "value": value, "unit": "GUPS", "n_gpus": world, "steps": K, "warmup": Wm,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.config + ": " + cfg["desc"], "grid": [prob.W, prob.y1 - prob.y0, prob.W],
                   "projections": prob.P, "sit": prob.S, "per_subiteration": prob.Pc, "arith": args.arith,
                   "storage": args.storage, "l2": "inputs larger than L2 (%.2f GB volume, %.0f MB subset)"
                   % (4 * prob.nvox / 1e9, isz * prob.npix / 1e6), "parallelism": "independent volume per rank"},
        "e2e": {"value": e2e_value, "unit": "GUPS", "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": 8,
                "what": "steady-state sub-iterations: each step uploads its subset's preprocessed images from "
                        "page-locked host memory and reads the residual back"},
        "e2e_raw": {"value": e2e_raw_value, "unit": "GUPS", "h2d_bytes_per_step": raw_bytes,
                    "d2h_bytes_per_step": 8,
                    "what": "as e2e, but each step uploads the raw intensities I / I0 and runs the -log "
                            "preprocessing on the device inside the step"},
        "gpu_launches": 3 * K,
        "kernels_ms": {"forward": f_ms, "error": statistics.mean(err), "backward": b_ms},
        "kernel_gups": {"forward": pairs_step / (f_ms / 1000.0) / 1e9, "backward": pairs_step / (b_ms / 1000.0) / 1e9},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "algorithmic_bytes": alg_bytes,
                     "note": "issue/atomic-bound (not a dense contraction, not HBM-bound): see compute; "
                             "traffic scaled from an ncu capture of the 256-layer slab by voxel count"},
        "compute": {"flops_per_pair": FLOPS_PER_PAIR, "achieved_tflops": FLOPS_PER_PAIR * pairs_step / (step_ms / 1000) / 1e12,
                    "peak_fp32_tflops": fp32_peak, "frac": FLOPS_PER_PAIR * pairs_step / (step_ms / 1000) / 1e12 / fp32_peak,
                    "peak_source": "nominal: 148 SM x 128 FP32 lanes x 2 x median SM clock",
                    "note": "44 algorithmic flop per pair (the reference's operations), not the executed "
                            "instructions: see profile"},
        "profile": MEASURED_PROFILE[args.arith],
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(cfg, args.cpu_seconds)
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    if rank == 0:
        emit(line)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ----------------------------------------------------------------------------- batched (c4)
def run_batched(args, cfg, rank, world, local):
    """Many small reconstructions in one batched run (xpr_batch: persistent launches over
    all problems, the whole it x sit run captured into a CUDA graph, autotuned schedule),
    BF16 image / ratio storage; beside it the plain FP32 path (one problem at a time,
    one xpr_subiteration per sub-iteration) on a sample of the same problems."""
    import torch
    from xpulse_recon_b200 import _lib
    from xpulse_recon_b200.batch import Batch, Problem as BProblem, torch_dtype
    from xpulse_recon_b200.projector import Context, geometry
    torch.cuda.set_device(local)
    L = _lib.lib()
    ctx = Context(local)
    rng = np.random.default_rng(cfg["seed"] + 1000 * rank)
    storage = {"fp32": _lib.F32, "bf16": _lib.BF16, "fp16": _lib.F16}[args.storage or "bf16"]
    arith = _lib.STRICT if args.arith == "strict" else _lib.FAST
    S, it, M, P = cfg["sit"], cfg["it"], cfg["modules"], cfg["projections"]
    Wd, Hd = cfg["dwidth"], cfg["dheight"]
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    probs, plain_imgs = [], []
    for i in range(cfg["batch"]):
        so, sd = float(rng.uniform(80, 120)), float(rng.uniform(800, 1200))
        rpy = rng.uniform(-cfg["rpy"], cfg["rpy"], 3 * M).astype(np.float32)
        pd_all, g = geometry(so=so, sd=sd, px=cfg["px"], dwidth=Wd, dheight=Hd, projections=P, sit=S,
                             module_number=M, mod_rpy=rpy)
        W, Hv, Pc = int(g["vwidth"]), int(g["vheight"]), int(g["concurrent"])
        phantom = make_phantom(cfg, g["vx"], W, Hv, "cuda", int(rng.integers(1 << 30)))
        sums = torch.zeros(P * Wd * Hd, dtype=torch.int32, device="cuda")
        d = _lib.Launch()
        d.vmax[:] = [W, Hv, W]
        d.origin[:] = list(g["orig"])
        d.voxel[:] = [g["vx"]] * 3
        d.det_w, d.rows, d.n_angles, d.modules, d.arith = Wd, Hd, P, M, _lib.FAST
        dpd = torch.from_numpy(pd_all).cuda()
        _lib.check(L.xpr_forward(ctx.handle, phantom.data_ptr(), sums.data_ptr(), dpd.data_ptr(), P * M,
                                 C.byref(d), sp), "forward")
        p = sums.to(torch.int64).bitwise_and(0xFFFFFFFF).to(torch.float32) / float(1 << 22)
        gen = torch.Generator(device="cuda").manual_seed(int(rng.integers(1 << 30)))
        raw = (torch.poisson(cfg["i0"] * torch.exp(-p), generator=gen) / cfg["i0"]).view(P, Hd, Wd)
        order = torch.tensor([s + k * S for s in range(S) for k in range(Pc)], device="cuda")
        raw_sub = raw[order].reshape(-1).contiguous()
        del sums, p, raw, phantom
        pd = torch.from_numpy(np.ascontiguousarray(pd_all.reshape(P, M, 20)[order.cpu().numpy()].reshape(-1, 20)))
        imgs = torch.empty(raw_sub.numel(), dtype=torch_dtype(storage), device="cuda")
        _lib.check(L.xpr_preprocess_apply(ctx.handle, raw_sub.data_ptr(), imgs.data_ptr(), storage, raw_sub.numel(),
                                          0, None, 1, sp), "preprocess")
        if i < cfg["plain_sample"]:
            f32 = torch.empty(raw_sub.numel(), dtype=torch.float32, device="cuda")
            _lib.check(L.xpr_preprocess_apply(ctx.handle, raw_sub.data_ptr(), f32.data_ptr(), _lib.F32,
                                              raw_sub.numel(), 0, None, 1, sp), "preprocess")
            plain_imgs.append(f32)
        del raw_sub
        probs.append(BProblem(vol=torch.ones(W * Hv * W, dtype=torch.float32, device="cuda"), images=imgs,
                              projdata=pd.cuda(), det_w=Wd, det_h=Hd, per_subset=Pc, modules=M, sit=S, it=it,
                              vwidth=W, vheight=Hv, voxel=float(g["vx"]), orig=tuple(g["orig"]),
                              seed=int(rng.integers(1 << 31)), weight=1.0, weight_factor=0.9))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b = Batch(ctx, probs, arith=arith, storage=storage, use_graph=True, autotune=True)
    tune_s = time.perf_counter() - t0
    steps = b.steps
    pairs_step = sum(p.vwidth * p.vheight * p.vwidth * p.per_subset for p in probs)
    runs_w = max(1, -(-args.warmup // steps))
    runs_t = max(1, -(-args.steps // steps))
    for _ in range(runs_w):
        b.run()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(runs_t):
        b.run()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    n_steps = runs_t * steps
    value = pairs_step * n_steps / (ms / 1000.0) / 1e9
    # the plain FP32 path on a sample of the same problems, one at a time
    plain_ms, plain_pairs = 0.0, 0
    for i, f32 in enumerate(plain_imgs):
        p = probs[i]
        q = BProblem(vol=torch.ones_like(p.vol), images=f32, projdata=p.projdata, det_w=Wd, det_h=Hd,
                     per_subset=p.per_subset, modules=M, sit=S, it=it, vwidth=p.vwidth, vheight=p.vheight,
                     voxel=p.voxel, orig=p.orig, seed=p.seed)
        q.run_alone(ctx, arith, _lib.F32)  # warm
        torch.cuda.synchronize()
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        q.run_alone(ctx, arith, _lib.F32)
        z.record()
        torch.cuda.synchronize()
        plain_ms += a.elapsed_time(z)
        plain_pairs += p.vwidth * p.vheight * p.vwidth * p.per_subset * p.it * p.sit
    plain = plain_pairs / (plain_ms / 1000.0) / 1e9 if plain_ms else None
    sch = b.schedule()

    # the same sample: alone in the batch's storage, and batched in FP32 / the batch's storage
    def timed(fn):
        fn()
        torch.cuda.synchronize()
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        z.record()
        torch.cuda.synchronize()
        return a.elapsed_time(z)

    sample = []
    for i, f32 in enumerate(plain_imgs):
        p = probs[i]
        sample.append((p, BProblem(vol=torch.ones_like(p.vol), images=f32, projdata=p.projdata, det_w=Wd, det_h=Hd,
                                   per_subset=p.per_subset, modules=M, sit=S, it=it, vwidth=p.vwidth,
                                   vheight=p.vheight, voxel=p.voxel, orig=p.orig, seed=p.seed)))
    breakdown = {}
    if sample:
        alone_st = sum(timed(lambda p=p: p.run_alone(ctx, arith, storage)) for p, _ in sample)
        bq = Batch(ctx, [q for _, q in sample], arith=arith, storage=_lib.F32, use_graph=True, autotune=True)
        batch_f32 = timed(bq.run)
        bq.close()
        bs = Batch(ctx, [p for p, _ in sample], arith=arith, storage=storage, use_graph=True, autotune=True)
        batch_st = timed(bs.run)
        bs.close()
        g = lambda ms: plain_pairs / (ms / 1000.0) / 1e9  # noqa: E731
        breakdown = {"alone_fp32": plain, "alone_storage": g(alone_st), "batched_fp32": g(batch_f32),
                     "batched_storage": g(batch_st)}
    line = {"metric": "GUPS per sub-iteration (voxel x projection pairs / s)", "value": value, "unit": "GUPS",
            "n_gpus": world, "steps": n_steps, "warmup": runs_w * steps, "ms_per_step": ms / n_steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"bf16": "bf16 storage, f32 compute", "fp16": "fp16 storage, f32 compute",
                      "fp32": "f32"}[{_lib.BF16: "bf16", _lib.F16: "fp16", _lib.F32: "fp32"}[storage]],
            "data": "synthetic", "config": {"workload": "c4: " + cfg["desc"], "problems": len(probs),
                                            "steps_per_run": steps, "l2": "inputs larger than L2 (%.1f GB)"
                                            % (sum(p.vol.numel() * 4 for p in probs) / 1e9)},
            "module_pairs_gups": value * M, "schedule": sch, "autotune_s": tune_s,
            "plain_fp32": {"value": plain, "unit": "GUPS", "sample": "%d of the %d problems, each alone, FP32, "
                           "one xpr_subiteration per sub-iteration" % (len(plain_imgs), len(probs))},
            "speedup_vs_plain_fp32": (value / plain) if plain else None, "sample_gups": breakdown,
            "gpu_launches": 3 * n_steps, "clocks": clk}
    if rank == 0:
        emit(line)
    b.close()
    return 0


# ----------------------------------------------------------------------------- serving (c5)
def simulate_raw(ctx, cfg, edge, P, seed):
    """Raw intensities (P, D, D) of a seeded ellipsoid phantom of `edge` voxels in a grid
    of D = 1.5 edge, projected by this library's forward (FAST) with Poisson noise."""
    import torch
    from xpulse_recon_b200 import _lib
    from xpulse_recon_b200.projector import geometry
    L = _lib.lib()
    D = int(round(1.5 * edge))
    pd_all, g = geometry(px=cfg["px"], dwidth=D, dheight=D, projections=P, sit=1)
    W, Hv = int(g["vwidth"]), int(g["vheight"])
    pcfg = dict(phantom=edge, ellipsoids=cfg["ellipsoids"], background=cfg["background"])
    phantom = make_phantom(pcfg, g["vx"], W, Hv, "cuda", seed)
    sums = torch.zeros(P * D * D, dtype=torch.int32, device="cuda")
    d = _lib.Launch()
    d.vmax[:] = [W, Hv, W]
    d.origin[:] = list(g["orig"])
    d.voxel[:] = [g["vx"]] * 3
    d.det_w, d.rows, d.n_angles, d.modules, d.arith = D, D, P, 1, _lib.FAST
    dpd = torch.from_numpy(pd_all).cuda()
    _lib.check(L.xpr_forward(ctx.handle, phantom.data_ptr(), sums.data_ptr(), dpd.data_ptr(), P, C.byref(d),
                             C.c_void_p(torch.cuda.current_stream().cuda_stream)), "forward")
    p = sums.to(torch.int64).bitwise_and(0xFFFFFFFF).to(torch.float32) / float(1 << 22)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    raw = torch.poisson(cfg["i0"] * torch.exp(-p), generator=gen) / cfg["i0"]
    out = torch.empty((P, D, D), dtype=torch.float32, pin_memory=True)  # a client's page-locked buffer
    out.copy_(raw.view(P, D, D))
    del sums, p, raw, phantom
    return out.numpy(), W * Hv * W


def run_serving(args, cfg, rank, world, local):
    """Open loop: requests submitted at Poisson arrival times, latency percentiles from
    the server's own clock.  Closed loop: every request submitted at once, served GUPS
    from the makespan, against the plain FP32 path (each request alone through the
    whole-run entry point, uploads included) on one request of each kind."""
    import torch
    from xpulse_recon_b200 import _lib
    from xpulse_recon_b200.projector import Context
    from xpulse_recon_b200.serve import DONE, Server
    torch.cuda.set_device(local)
    ctx = Context(local)
    rng = np.random.default_rng(cfg["seed"])
    kinds = [(e, P) for e in cfg["edges"] for P in cfg["projections_set"]]
    data = {}
    for i, (e, P) in enumerate(kinds):
        data[(e, P)] = simulate_raw(ctx, cfg, e, P, cfg["seed"] * 100 + i)
    torch.cuda.synchronize()
    n = cfg["requests"]
    reqs = []
    for i in range(n):
        e = cfg["edges"][rng.integers(len(cfg["edges"]))]
        P = cfg["projections_set"][rng.integers(len(cfg["projections_set"]))]
        params = {"recon": {"method": "naive", "it": cfg["it"], "sit": cfg["sit"], "seed": int(rng.integers(1 << 31)),
                            "mlog": True, "weight": 1.0, "weight_factor": 0.9},
                  "geometry": {"so": 100.0, "sd": 1000.0, "angle": 360.0}, "detector": {"px": cfg["px"]}}
        reqs.append((params, (e, P)))
    arrivals = np.cumsum(rng.exponential(1.0 / cfg["rate"], n))
    # page-locked result buffers (a serving client's own); requests of one volume size share
    # one, as the benchmark reads no result
    out_by_edge = {e: torch.empty(max(data[k][1] for k in kinds if k[0] == e), dtype=torch.float32,
                                  pin_memory=True).numpy() for e in cfg["edges"]}
    out_of = {k: out_by_edge[k[0]][:data[k][1]] for k in kinds}
    outs = [out_of[k] for _, k in reqs]
    pairs_of = {k: data[k][1] * k[1] for k in kinds}  # N x P per reconstruction (it 1)
    total_pairs = sum(pairs_of[k] for _, k in reqs) * cfg["it"]

    arith = _lib.STRICT if args.arith == "strict" else _lib.FAST

    def serve(storage, open_loop, image_storage=None):
        srv = Server(ctx, arith=arith, storage=storage, image_storage=image_storage)
        # warm the kernels and the allocator on one small request
        w = srv.submit(reqs[0][0], data[reqs[0][1]][0])
        srv.wait(w, 120.0)
        t0 = time.perf_counter()
        tickets = []
        for i, (params, k) in enumerate(reqs):
            if open_loop:
                dt = arrivals[i] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
            tickets.append(srv.submit(params, data[k][0], outs[i]))
        infos = [srv.wait(t, 600.0) for t in tickets]
        ok = all(i.state == DONE for i in infos)
        lat = np.array([i.done_s - i.submit_s for i in infos])
        span = max(i.done_s for i in infos) - min(i.submit_s for i in infos)
        st = srv.stats()
        srv.close()
        failed = [i for i in infos if i.state != DONE]
        return {"ok": ok, "failed": len(failed), "errors": sorted({int(i.error) for i in failed}),
                "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "mean_s": float(lat.mean()), "gups": total_pairs / span / 1e9, "makespan_s": span,
                "ticks": int(st.ticks), "peak_device_gb": st.peak_bytes / 1e9}

    res = {}
    clocks = ClockSampler(local)
    clocks.start()
    for name, st, ist in (("fp32", _lib.F32, None), ("bf16", _lib.BF16, _lib.F16)):
        res[name] = {"open_loop": serve(st, True, ist)}
    clk = clocks.stop()
    # the plain FP32 path: one request of each kind alone through xpr_reconstruct_host
    L = _lib.lib()
    L.xpr_reconstruct_host.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.c_uint64, C.POINTER(C.c_double)]
    plain_pairs, plain_s = 0, 0.0
    for k in kinds:
        raw, N = data[k]
        params = {"recon": {"method": "naive", "it": cfg["it"], "sit": cfg["sit"], "seed": 7, "mlog": True,
                            "arith": args.arith},
                  "geometry": {"so": 100.0, "sd": 1000.0, "angle": 360.0}, "detector": {"px": cfg["px"]}}
        out = np.empty(N, np.float32)
        P, H, W = raw.shape
        t = time.perf_counter()
        rc = L.xpr_reconstruct_host(json.dumps(params).encode(), np.ascontiguousarray(raw).ctypes.data, P, W, H,
                                    out.ctypes.data, out.size, C.byref(C.c_double()))
        plain_s += time.perf_counter() - t
        plain_pairs += pairs_of[k] * cfg["it"]
        assert rc == 0
    plain = plain_pairs / plain_s / 1e9

    # the plain FP32 path under the same arrivals: one request at a time, first come first
    # served, each through xpr_reconstruct_host (the reference's one-scan-per-run model);
    # on the first plain_requests requests (it falls behind the arrivals, so the whole
    # stream would take many minutes)
    n_plain = min(n, cfg.get("plain_requests", n))

    def plain_open_loop():
        import queue
        import threading
        jobs, lat = queue.Queue(), []

        def worker():
            while True:
                item = jobs.get()
                if item is None:
                    return
                t_sub, params, k = item
                raw, N = data[k]
                P, H, W = raw.shape
                out = out_of[k]
                rc = L.xpr_reconstruct_host(json.dumps(params).encode(), raw.ctypes.data, P, W, H, out.ctypes.data,
                                            out.size, C.byref(C.c_double()))
                lat.append(time.perf_counter() - t_sub if rc == 0 else float("nan"))

        th = threading.Thread(target=worker)
        th.start()
        t0 = time.perf_counter()
        for i, (params, k) in enumerate(reqs[:n_plain]):
            dt = arrivals[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            p2 = json.loads(json.dumps(params))
            p2["recon"]["arith"] = args.arith
            jobs.put((time.perf_counter(), p2, k))
        jobs.put(None)
        th.join()
        span = time.perf_counter() - t0
        lat = np.array(lat)
        pairs = sum(pairs_of[k] for _, k in reqs[:n_plain]) * cfg["it"]
        return {"ok": bool(np.isfinite(lat).all()), "requests": n_plain, "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                "gups": pairs / span / 1e9, "makespan_s": span}

    res["plain_fp32"] = {"open_loop": plain_open_loop()}
    best = res["bf16"]["open_loop"]["gups"]
    line = {"metric": "GUPS served (voxel x projection pairs / s), with p50 / p99 request latency",
            "value": best, "unit": "GUPS", "n_gpus": world, "steps": n, "warmup": 1,
            "ms_per_step": 1000.0 * res["bf16"]["open_loop"]["makespan_s"] / n, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 ratio / fp16 image storage, f32 compute",
            "data": "synthetic",
            "config": {"workload": "c5: " + cfg["desc"], "requests": n, "rate_per_s": cfg["rate"],
                       "arith": args.arith},
            "serving": res, "plain_fp32_e2e": {"value": plain, "unit": "GUPS",
                                               "sample": "one request of each of the %d kinds, alone, through "
                                                         "xpr_reconstruct_host (host images in, volume out)" % len(kinds)},
            "speedup_vs_plain_fp32": best / plain,
            "e2e": {"value": best, "unit": "GUPS", "h2d_bytes_per_step": int(np.mean([data[k][0].nbytes for _, k in reqs])),
                    "d2h_bytes_per_step": int(np.mean([4 * data[k][1] for _, k in reqs]))},
            "clocks": clk}
    if rank == 0:
        emit(line)
    return 0


# ----------------------------------------------------------------------------- slab-sharded
def run_sharded(args, cfg, rank, world, local):
    """One c2 reconstruction split into y-slabs over the ranks (xpulse_recon_b200.shard):
    per sub-iteration a slab forward into the detector rows the slab reaches, a
    point-to-point NCCL exchange of the u32 sums over the rows shared with other ranks,
    the error on the rank's rows and a slab backward.  Total work is fixed as N grows
    (strong scaling)."""
    import datetime

    import torch
    import torch.distributed as dist
    from xpulse_recon_b200.shard import GpuOps, SlabReconstruction
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        dist.barrier()  # every rank takes part in the communicator's first call
    args.storage = args.storage or "fp32"
    prob = Problem(cfg, args.arith, args.storage, local, cfg["seed"])  # the same measured data on every rank
    images = torch.cat(prob.images)
    del prob.vol, prob.sums, prob.ratio, prob.phantom
    torch.cuda.empty_cache()
    K, Wm = args.steps, args.warmup
    steps = Wm + K + 1
    ops = GpuOps(prob.ctx, prob.arith, prob.storage)
    r = SlabReconstruction(ops, None, prob.pd_all, prob.g, it=-(-steps // prob.S), sit=prob.S, seed=cfg["seed"],
                           rank=rank, world=world, images=images, shape=(prob.P, prob.Hd, prob.Wd))
    for k in range(Wm + 1):  # step 0 has no forward: warm-up starts with it
        r.step(k)
    torch.cuda.synchronize()
    sent0 = r.exchanged_bytes
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    e0.record()
    for k in range(Wm + 1, Wm + 1 + K):
        r.step(k)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    pairs_step = prob.W * prob.Hv * prob.W * prob.Pc
    value = pairs_step * K / (ms / 1000.0) / 1e9
    line = {"metric": "GUPS per sub-iteration (voxel x projection pairs / s)", "value": value, "unit": "GUPS",
            "n_gpus": world, "steps": K, "warmup": Wm + 1, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config + ": " + cfg["desc"], "parallelism": "y-slab sharding, %d ranks, "
                       "u32 sums of the shared detector rows exchanged point to point" % world,
                       "arith": args.arith, "storage": args.storage, "l2": "inputs larger than L2",
                       "row_window": [r.r0, r.r1]},
            "exchange_bytes_per_step": (r.exchanged_bytes - sent0) / K, "gpu_launches": 3 * K,
            "clocks": clk}
    if rank == 0:
        emit(line)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ----------------------------------------------------------------------------- out-of-core (c3)
def host_available_bytes():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def run_outofcore(args, cfg, rank, world, local):
    """Whole reconstructions through the drop-in entry point (xpr_reconstruct_host: host
    projections in, host volume out) with each memory mode; the streaming modes under a
    device-memory cap smaller than the volume."""
    import torch
    from xpulse_recon_b200 import _lib
    from xpulse_recon_b200.projector import Context, geometry
    P, Wd, Hd = cfg["projections"], cfg["dwidth"], cfg["dheight"]
    # host memory: projections and volume here, and the streaming modes' pinned copies of both
    need = 2 * (4 * P * Wd * Hd) + 2 * (4 * Wd * Hd * Wd)
    avail = host_available_bytes()
    if avail and need > avail // 2:
        emit({"metric": "GUPS per sub-iteration (voxel x projection pairs / s)", "value": None,
              "unavailable": "needs %.1f GB of host memory, %.1f GB available" % (need / 1e9, avail / 1e9)})
        return 0
    torch.cuda.set_device(local)
    L = _lib.lib()
    ctx = Context(local)
    pd_all, g = geometry(so=cfg["so"], sd=cfg["sd"], px=cfg["px"], dwidth=Wd, dheight=Hd, projections=P, sit=1)
    W, Hv = int(g["vwidth"]), int(g["vheight"])
    N = W * Hv * W
    phantom = make_phantom(cfg, g["vx"], W, Hv, "cuda", cfg["seed"])
    raw = np.empty((P, Hd, Wd), np.float32)
    gen = torch.Generator(device="cuda").manual_seed(cfg["seed"])
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    chunk = 50
    for a in range(0, P, chunk):  # simulate a chunk of projections at a time (bounded device memory)
        n = min(chunk, P - a)
        sums = torch.zeros(n * Wd * Hd, dtype=torch.int32, device="cuda")
        d = _lib.Launch()
        d.vmax[:] = [W, Hv, W]
        d.origin[:] = list(g["orig"])
        d.voxel[:] = [g["vx"]] * 3
        d.det_w, d.rows, d.n_angles, d.modules, d.arith = Wd, Hd, n, 1, _lib.FAST
        dpd = torch.from_numpy(np.ascontiguousarray(pd_all[a:a + n])).cuda()
        _lib.check(L.xpr_forward(ctx.handle, phantom.data_ptr(), sums.data_ptr(), dpd.data_ptr(), n, C.byref(d), sp),
                   "forward")
        p = sums.to(torch.int64).bitwise_and(0xFFFFFFFF).to(torch.float32) / float(1 << 22)
        raw[a:a + n] = (torch.poisson(cfg["i0"] * torch.exp(-p), generator=gen) / cfg["i0"]).view(n, Hd, Wd).cpu()
        del sums, p
    del phantom
    torch.cuda.empty_cache()
    ctx.close()
    L.xpr_reconstruct_host.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.c_uint64, C.POINTER(C.c_double)]
    out = np.empty(N, np.float32)
    results = {}
    pairs = N * (P // cfg["sit"]) * cfg["sit"] * cfg["it"]
    clocks = ClockSampler(local)
    clocks.start()
    for m in cfg["methods"]:
        params = {"recon": {"method": m, "it": cfg["it"], "sit": cfg["sit"], "seed": 11, "mlog": True,
                            "mem_cap": 0 if m == "naive" else cfg["mem_cap"]},
                  "geometry": {"so": cfg["so"], "sd": cfg["sd"], "angle": 360.0}, "detector": {"px": cfg["px"]}}
        secs = C.c_double()
        t = time.perf_counter()
        rc = L.xpr_reconstruct_host(json.dumps(params).encode(), raw.ctypes.data, P, Wd, Hd, out.ctypes.data, N,
                                    C.byref(secs))
        wall = time.perf_counter() - t
        results[m] = {"rc": rc, "iterations_s": secs.value, "wall_s": wall,
                      "gups_iterations": pairs / max(secs.value, 1e-9) / 1e9, "gups_e2e": pairs / wall / 1e9,
                      "finite": float(np.isfinite(out).mean())}
    clk = clocks.stop()
    best = max(results[m]["gups_e2e"] for m in cfg["methods"] if m != "naive")
    line = {"metric": "GUPS per sub-iteration (voxel x projection pairs / s)", "value": best, "unit": "GUPS",
            "n_gpus": 1, "steps": cfg["sit"] * cfg["it"], "warmup": 0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "c3h: " + cfg["desc"], "grid": [W, Hv, W], "mem_cap_bytes": cfg["mem_cap"]},
            "methods": results, "clocks": clk,
            "e2e": {"value": best, "unit": "GUPS", "h2d_bytes_per_step": int(raw.nbytes // cfg["sit"]),
                    "d2h_bytes_per_step": int(4 * N // cfg["sit"])}}
    emit(line)
    return 0


def main():
    args = parse_args()
    cfg = CONFIGS[args.config]
    if args.arith is None:
        args.arith = "fast" if "batch" in cfg else "strict"
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, cfg, rank, world)
    if "batch" in cfg:
        return run_batched(args, cfg, rank, world, local)
    if cfg.get("serve"):
        return run_serving(args, cfg, rank, world, local)
    if args.shard or (world > 1 and not args.replicas):
        return run_sharded(args, cfg, rank, world, local)
    if cfg.get("outofcore"):
        return run_outofcore(args, cfg, rank, world, local)
    return run_ours(args, cfg, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
