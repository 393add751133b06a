"""Seeded synthetic data at the benchmark configurations' sizes, made on the CPU.

The reference ships no datasets; these stand in for scans with the shapes, sizes and
value ranges its benchmark configurations state:

* c1 -- a 128^3 phantom of 10 ellipsoids (attenuation uniform in [0, 0.02) per mm,
  voxel 0.01 mm) centred in the 192^3 grid the reference derives from a 192 x 192
  detector (px 0.1 mm, so 100, sd 1000, rx = sx = sy = 0); 180 projections over 360
  degrees; intensities I = Poisson(1e5 exp(-p)) / 1e5.
* c2 slab -- the c2 geometry (768 x 768 detector, 720 projections, rx 1.5 px, sx -2,
  sy 3 mm) restricted to a y-slab of central layers of its 768^3 grid; the phantom is
  the slab of a 512^3 phantom of 40 ellipsoids plus a 5 % Gaussian-textured background.

Line integrals p are the oracle's fixed-point forward projection (FAST contract, grid
origin without jitter) of the phantom along the reference's rays (source -> pixel of
its projection matrices), so the data need no GPU and are the same on every machine.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

I0 = 1e5

C1 = dict(dwidth=192, dheight=192, projections=180, sit=10, px=0.1, so=100.0, sd=1000.0, rx=0.0, sx=0.0, sy=0.0)
C1_PHANTOM = dict(edge=128, ellipsoids=10, background=0.0, seed=1)
C1_RECON = dict(it=1, sit=10, weight=1.0, weight_factor=0.9, seed=77)

C2 = dict(dwidth=768, dheight=768, projections=720, sit=10, px=0.1, so=100.0, sd=1000.0, rx=1.5, sx=-2.0, sy=3.0)
C2_PHANTOM = dict(edge=512, ellipsoids=40, background=0.05, seed=2)
C2_RECON = dict(it=3, sit=10, weight=1.0, weight_factor=0.9, seed=78)


def _gauss_kernel(sigma=4.0, half=12):
    k = np.exp(-0.5 * (np.arange(-half, half + 1, dtype=np.float64) / sigma) ** 2)
    return k / k.sum()


def _smooth_axis(a, k, axis):
    """'same'-size convolution along one axis with zero padding."""
    half = len(k) // 2
    pad = [(0, 0)] * a.ndim
    pad[axis] = (half, half)
    ap = np.pad(a, pad)
    out = np.zeros_like(a)
    n = a.shape[axis]
    for i, w in enumerate(k):
        sl = [slice(None)] * a.ndim
        sl[axis] = slice(i, i + n)
        out += w * ap[tuple(sl)]
    return out


def ellipsoid_phantom(W, Hv, vx, edge, ellipsoids, background, seed, y0=0, y1=None):
    """Attenuation per voxel (mu * vx) of a seeded phantom in the central edge^3 region of
    the (y, z, x) grid W x Hv x W: ellipsoids with centres uniform in the phantom's
    inscribed cylinder, semi-axes uniform in [3 %, 25 %] of its edge, uniform random
    orientation, mu uniform in [0, 0.02) per mm; optionally a background of
    `background` x the mean mu, textured by Gaussian-smoothed (sigma 4 voxels) noise and
    clipped at 0.  Only layers [y0, y1) are returned, as float32[y1 - y0, W, W]."""
    y1 = Hv if y1 is None else y1
    rng = np.random.default_rng(seed)
    vol = np.zeros((y1 - y0, W, W), np.float64)
    centre = np.array([W / 2.0, Hv / 2.0, W / 2.0])  # x, y, z in voxels
    mus = []
    for _ in range(ellipsoids):
        while True:
            cx, cz = rng.uniform(-edge / 2, edge / 2, 2)
            if cx * cx + cz * cz <= (edge / 2) ** 2:
                break
        cy = rng.uniform(-edge / 2, edge / 2)
        axes = rng.uniform(0.03, 0.25, 3) * edge
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        mu = rng.uniform(0.0, 0.02)
        mus.append(mu)
        c = centre + np.array([cx, cy, cz])
        r = axes.max()
        lo = np.maximum(np.floor(c - r).astype(int), [0, y0, 0])
        hi = np.minimum(np.ceil(c + r).astype(int) + 1, [W, y1, W])
        if (hi <= lo).any():
            continue
        ys = np.arange(lo[1], hi[1]) + 0.5 - c[1]
        zs = np.arange(lo[2], hi[2]) + 0.5 - c[2]
        xs = np.arange(lo[0], hi[0]) + 0.5 - c[0]
        Y, Z, X = np.meshgrid(ys, zs, xs, indexing="ij")
        P = np.stack([X, Y, Z], axis=-1) @ q
        inside = ((P / axes) ** 2).sum(-1) <= 1.0
        vol[lo[1] - y0:hi[1] - y0, lo[2]:hi[2], lo[0]:hi[0]] += inside * (mu * vx)
    if background > 0:
        k = _gauss_kernel()
        half = len(k) // 2
        p0 = (Hv - edge) // 2
        a, b = max(p0, y0), min(p0 + edge, y1)
        if a < b:
            ga, gb = max(p0, a - half), min(p0 + edge, b + half)  # noise layers that reach [a, b)
            noise = np.random.default_rng(seed + 7919).standard_normal((gb - ga, edge, edge))
            for ax in range(3):
                noise = _smooth_axis(noise, k, ax)
            noise = noise[a - ga:b - ga]
            noise /= noise.std()
            level = background * float(np.mean(mus)) * vx
            x0 = (W - edge) // 2
            vol[a - y0:b - y0, x0:x0 + edge, x0:x0 + edge] += np.clip(level * (1.0 + noise), 0.0, None)
    return vol.astype(np.float32)


def project(vol, pd_all, go, Wd, Hd, box):
    """Line integrals p (float64[P, Hd, Wd]) of `vol` (the box's voxels) for every
    ProjData entry (one module), through the oracle's fixed-point forward."""
    P = pd_all.shape[0]
    sums = np.zeros(P * Wd * Hd, np.uint32)
    L, keep = O.make_launch(box[0], box[1], [float(v) for v in go.orig], [go.vx] * 3, Wd, Hd, 0, P, 1,
                            arith=O.FAST)
    O.forward(np.ascontiguousarray(vol.ravel()), sums, np.ascontiguousarray(pd_all), L)
    return (sums.astype(np.float64) / float(1 << 22)).reshape(P, Hd, Wd)


def noisy(p, seed):
    """Raw intensities I / I0 with Poisson noise at I0 photons per pixel."""
    rng = np.random.default_rng(seed)
    return (rng.poisson(I0 * np.exp(-p)) / I0).astype(np.float32)


def c1_raw():
    """(raw float32[180, 192, 192], geometry params, pd_all, GeomOut) of the c1 scan."""
    gp = O.geom_params(**C1)
    pd_all, go = O.geometry(gp)
    W, Hv = int(go.vwidth), int(go.vheight)
    vol = ellipsoid_phantom(W, Hv, go.vx, **C1_PHANTOM)
    p = project(vol, pd_all, go, C1["dwidth"], C1["dheight"], ((0, 0, 0), (W, Hv, W)))
    return noisy(p, 101), gp, pd_all, go


def c2_slab_raw(layers=32):
    """(raw float32[720, 768, 768], gp, pd_all, go, (y0, y1)): projections of the central
    `layers` layers of the c2 phantom, the slab the test reconstructs."""
    gp = O.geom_params(**C2)
    pd_all, go = O.geometry(gp)
    W, Hv = int(go.vwidth), int(go.vheight)
    y0 = Hv // 2 - layers // 2
    y1 = y0 + layers
    vol = ellipsoid_phantom(W, Hv, go.vx, y0=y0, y1=y1, **C2_PHANTOM)
    p = project(vol, pd_all, go, C2["dwidth"], C2["dheight"], ((0, y0, 0), (W, y1, W)))
    return noisy(p, 202), gp, pd_all, go, (y0, y1)


def preprocess(raw):
    """-log(clamp(v, eps, 1 - eps)) by the oracle (data_loader.hpp:48-101, no normalise)."""
    imgs = np.ascontiguousarray(raw, np.float32).ravel().copy()
    O.lib().orc_preprocess(imgs, imgs.size, 0, 0.0, 0.0, 1)
    return imgs.reshape(raw.shape)
