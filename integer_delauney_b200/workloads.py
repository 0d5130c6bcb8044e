"""Seeded synthetic seed sets with the shapes and distributions of the
benchmark configurations (no dataset is involved anywhere).

  uniform(W, H, n, seed)          n distinct uniform integer points
  clustered(W, H, n, seed, ...)   n distinct points from isotropic Gaussian
                                  blobs, rounded, clipped, deduplicated
  batched_images(count, seed)     per-image (W, H, seeds) with sides
                                  log-uniform in 64..1024 and density
                                  uniform in 0.1%..2% of pixels

Points are returned in a shuffled (not sorted) order, as callers pass them.
"""
from __future__ import annotations

import math

import numpy as np


def uniform(W: int, H: int, n: int, seed: int = 0, margin: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if n > (W - 2 * margin) * (H - 2 * margin):
        raise ValueError("more seeds than pixels")
    got = np.zeros((0,), dtype=np.int64)
    span_w = W - 2 * margin
    while got.size < n:
        k = int((n - got.size) * 1.2) + 16
        xs = rng.integers(margin, W - margin, size=k, dtype=np.int64)
        ys = rng.integers(margin, H - margin, size=k, dtype=np.int64)
        lin = (ys - margin) * span_w + (xs - margin)
        got = np.concatenate([got, lin])
        _, first = np.unique(got, return_index=True)
        got = got[np.sort(first)]
    got = got[:n]
    out = np.stack([got % span_w + margin, got // span_w + margin], axis=1).astype(np.int32)
    rng.shuffle(out)
    return np.ascontiguousarray(out)


def clustered(W: int, H: int, n: int, seed: int = 0, blobs: int = 64, sigma: float = 40.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, [W, H], size=(blobs, 2))
    got = np.zeros((0,), dtype=np.int64)
    while got.size < n:
        k = max(4096, int((n - got.size) * 1.3))
        c = centres[rng.integers(0, blobs, size=k)]
        p = np.rint(c + rng.normal(0.0, sigma, size=(k, 2))).astype(np.int64)
        p[:, 0] = np.clip(p[:, 0], 0, W - 1)
        p[:, 1] = np.clip(p[:, 1], 0, H - 1)
        got = np.concatenate([got, p[:, 1] * W + p[:, 0]])
        _, first = np.unique(got, return_index=True)
        got = got[np.sort(first)]
    got = got[:n]
    out = np.stack([got % W, got // W], axis=1).astype(np.int32)
    rng.shuffle(out)
    return np.ascontiguousarray(out)


def batched_images(count: int = 512, seed: int = 0, side_lo: int = 64, side_hi: int = 1024,
                   dens_lo: float = 0.001, dens_hi: float = 0.02):
    """List of (W, H, seeds) for the batched configuration."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        W = int(round(math.exp(rng.uniform(math.log(side_lo), math.log(side_hi)))))
        H = int(round(math.exp(rng.uniform(math.log(side_lo), math.log(side_hi)))))
        dens = rng.uniform(dens_lo, dens_hi)
        n = max(3, int(math.ceil(dens * W * H)))
        out.append((W, H, uniform(W, H, n, seed=int(rng.integers(1 << 31)))))
    return out
