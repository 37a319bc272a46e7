"""Seeded synthetic images of the image-TV workloads (no dataset is involved).

* ``noise``    -- i.i.d. N(0, 1) pixels.
* ``phantom``  -- a piecewise-constant phantom: 20 random axis-aligned
  rectangles and 10 random disks, each painted with an intensity drawn from
  U[0, 1] over a zero background, plus Gaussian noise of std ``sigma``.
* ``phantom3d`` -- the same in 3D with boxes and balls.
All draws come from ``numpy.random.default_rng(seed)``.
"""

from __future__ import annotations

import numpy as np


def noise(shape, seed=0, dtype=np.float32):
    return np.random.default_rng(seed).normal(size=shape).astype(dtype)


def _phantom_one(rng, H, W):
    img = np.zeros((H, W))
    ii = np.arange(H)[:, None]
    jj = np.arange(W)[None, :]
    for _ in range(20):
        h = rng.integers(max(1, H // 16), max(2, H // 3) + 1)
        w = rng.integers(max(1, W // 16), max(2, W // 3) + 1)
        i0 = rng.integers(0, max(1, H - h + 1))
        j0 = rng.integers(0, max(1, W - w + 1))
        img[i0:i0 + h, j0:j0 + w] = rng.uniform()
    for _ in range(10):
        r = rng.uniform(min(H, W) / 32, min(H, W) / 6)
        ci, cj = rng.uniform(0, H), rng.uniform(0, W)
        img[(ii - ci) ** 2 + (jj - cj) ** 2 <= r * r] = rng.uniform()
    return img


def phantom(batch, H, W, seed=0, sigma=0.1, dtype=np.float32, clean=False):
    """(batch, H, W) phantoms plus N(0, sigma^2) noise; with clean=True also
    returns the noiseless phantoms."""
    rng = np.random.default_rng(seed)
    ph = np.stack([_phantom_one(rng, H, W) for _ in range(batch)])
    noisy = ph + sigma * rng.normal(size=ph.shape)
    if clean:
        return noisy.astype(dtype), ph.astype(dtype)
    return noisy.astype(dtype)


def phantom3d(batch, D, H, W, seed=0, sigma=0.1, dtype=np.float32):
    rng = np.random.default_rng(seed)
    out = np.zeros((batch, D, H, W))
    kk = np.arange(D)[:, None, None]
    ii = np.arange(H)[None, :, None]
    jj = np.arange(W)[None, None, :]
    for b in range(batch):
        vol = out[b]
        for _ in range(12):
            d, h, w = (rng.integers(max(1, n // 8), max(2, n // 3) + 1) for n in (D, H, W))
            k0, i0, j0 = rng.integers(0, max(1, D - d + 1)), rng.integers(0, max(1, H - h + 1)), \
                rng.integers(0, max(1, W - w + 1))
            vol[k0:k0 + d, i0:i0 + h, j0:j0 + w] = rng.uniform()
        for _ in range(6):
            r = rng.uniform(min(D, H, W) / 16, min(D, H, W) / 5)
            c = rng.uniform(0, 1, 3) * np.array([D, H, W])
            vol[(kk - c[0]) ** 2 + (ii - c[1]) ** 2 + (jj - c[2]) ** 2 <= r * r] = rng.uniform()
    out = out + sigma * rng.normal(size=out.shape)
    return out.astype(dtype)


def pixel_weights(shape, seed=0, lo=0.5, hi=1.5, dtype=np.float64):
    return np.random.default_rng(seed).uniform(lo, hi, size=shape).astype(dtype)
