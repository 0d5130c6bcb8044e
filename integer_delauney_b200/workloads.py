"""Seeded synthetic seed sets with the shapes and distributions of the
benchmark configurations (no dataset is involved anywhere).

  uniform(W, H, n, seed)          n distinct uniform integer points
  clustered(W, H, n, seed, ...)   n distinct points from isotropic Gaussian
                                  blobs, rounded, clipped, deduplicated
  batched_images(count, seed)     per-image (W, H, seeds) with sides
                                  log-uniform in 64..1024 and density
                                  uniform in 0.1%..2% of pixels
  incremental(...)                a uniform base set and insert batches of
                                  new distinct points, a fixed share of each
                                  inside a hotspot square
  serving_trace(...)              Poisson arrivals of new triangulations and
                                  insert batches, and fresh_points() for the
                                  inserts' seeds

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


def incremental(W: int = 2048, H: int = 2048, base: int = 50_000, batches: int = 100, per_batch: int = 1_000,
                hot_frac: float = 0.3, hot: int = 256, seed: int = 0):
    """(base (base, 2), [batch (per_batch, 2), ...]) for the incremental
    configuration: every point distinct from all earlier ones; in each batch
    round(hot_frac * per_batch) points are uniform in a hot x hot square
    placed by the seed, the rest uniform on the canvas."""
    rng = np.random.default_rng(seed)
    b0 = uniform(W, H, base, seed=seed)
    taken = set((b0[:, 1].astype(np.int64) * W + b0[:, 0]).tolist())
    hx = int(rng.integers(0, W - hot + 1))
    hy = int(rng.integers(0, H - hot + 1))
    out = []
    n_hot = int(round(hot_frac * per_batch))
    for _ in range(batches):
        pts = []
        for want, (x0, y0, w, h) in ((n_hot, (hx, hy, hot, hot)), (per_batch - n_hot, (0, 0, W, H))):
            got = 0
            while got < want:
                k = (want - got) * 2 + 8
                xs = rng.integers(x0, x0 + w, size=k)
                ys = rng.integers(y0, y0 + h, size=k)
                for x, y in zip(xs.tolist(), ys.tolist()):
                    key = y * W + x
                    if key in taken:
                        continue
                    taken.add(key)
                    pts.append((x, y))
                    got += 1
                    if got == want:
                        break
        b = np.array(pts, dtype=np.int32)
        rng.shuffle(b)
        out.append(np.ascontiguousarray(b))
    return b0, out


def serving_trace(rate: float = 1000.0, seconds: float = 60.0, frac_new: float = 0.7, side=(128, 4096),
                  density=(0.0005, 0.01), insert=(100, 5000), seed: int = 0):
    """Poisson request stream for the serving configuration: a list of
    (arrival_s, kind, params) with kind "new" -> (width, height, n_seeds,
    point_seed) and kind "insert" -> (n_seeds, pick, point_seed), pick in
    [0, 1) choosing the target among the diagrams resident at that time.
    Sides are log-uniform in `side`, density uniform in `density`, insert
    sizes uniform integers in `insert`."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    lo, hi = math.log(side[0]), math.log(side[1])
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        if rng.random() < frac_new:
            W = int(round(math.exp(rng.uniform(lo, hi))))
            H = int(round(math.exp(rng.uniform(lo, hi))))
            n = max(3, int(math.ceil(rng.uniform(*density) * W * H)))
            out.append((t, "new", (W, H, n, int(rng.integers(1 << 31)))))
        else:
            out.append((t, "insert", (int(rng.integers(insert[0], insert[1] + 1)), float(rng.random()),
                                      int(rng.integers(1 << 31)))))
    return out


def fresh_points(W: int, H: int, n: int, taken_keys: np.ndarray, seed: int) -> np.ndarray:
    """n distinct uniform points of a W x H canvas whose keys y * W + x are
    not in the sorted int64 array `taken_keys` (fewer if the canvas is full)."""
    taken_keys = np.asarray(taken_keys, dtype=np.int64)
    rng = np.random.default_rng(seed)
    free = W * H - len(taken_keys)
    n = min(n, max(free, 0))
    got = np.zeros(0, dtype=np.int64)
    while len(got) < n:
        k = rng.integers(0, W * H, size=(n - len(got)) * 2 + 16, dtype=np.int64)
        if len(taken_keys):
            at = np.minimum(np.searchsorted(taken_keys, k), len(taken_keys) - 1)
            k = k[taken_keys[at] != k]
        got = np.concatenate([got, k])
        _, first = np.unique(got, return_index=True)
        got = got[np.sort(first)]
    got = got[:n]
    return np.ascontiguousarray(np.stack([got % W, got // W], axis=1).astype(np.int32))
