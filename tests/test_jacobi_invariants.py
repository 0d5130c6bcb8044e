"""Properties of the reference Jacobi iteration that the propagation kernels'
work lists rely on, checked on the CPU pass by pass (no GPU needed).

The reference pass (src/cuda/voronoi.cu:32-53, geometry_device.cuh:22-66)
gives each owned-or-unowned cell the best of its own owner and its four
neighbours' owners: smallest squared distance, ties to the higher id.  The
cell-list tile rounds and the persistent kernel list, for pass t + 1, only
cells that can still change:

* from scratch, pass 0 can change only the 4-neighbours of the seeds (a seed
  itself is at distance 0, which nothing beats);
* a cell changes in pass t + 1 only if one of its 4-neighbours changed in
  pass t -- not merely itself: the best of its owner and unchanged
  neighbours is already its owner.

A small vectorised pass in this file is first pinned to the oracle's
fixed point (oracle.voronoi, itself pinned to the reference elsewhere), then
every pass of its trajectory is checked against both rules.
"""
import numpy as np
import pytest

import oracle
from tests.conftest import random_seeds

FAR = np.int64(1) << 40


def _pass(lab, xs, ys):
    """One synchronous reference pass over an (H, W) grid of seed ids (-1: unowned)."""
    H, W = lab.shape
    yy, xx = np.mgrid[0:H, 0:W]

    def dist(ids):
        ok = ids >= 0
        safe = np.where(ok, ids, 0)
        d = (xx - xs[safe]).astype(np.int64) ** 2 + (yy - ys[safe]).astype(np.int64) ** 2
        return np.where(ok, d, FAR)

    best = lab.copy()
    bd = dist(lab)
    for dy, dx in ((0, -1), (0, 1), (-1, 0), (1, 0)):
        n = np.full_like(lab, -1)
        ys0, ys1 = max(0, dy), H + min(0, dy)
        xs0, xs1 = max(0, dx), W + min(0, dx)
        # n[y, x] = lab[y + dy, x + dx] where that cell exists
        n[ys0 - dy:ys1 - dy, xs0 - dx:xs1 - dx] = lab[ys0:ys1, xs0:xs1]
        nd = dist(n)
        better = (n >= 0) & ((nd < bd) | ((nd == bd) & (n > best)))
        best = np.where(better, n, best)
        bd = np.where(better, nd, bd)
    return best


def _neighbours(mask):
    """Cells with a 4-neighbour in `mask` (the cells themselves not included)."""
    out = np.zeros_like(mask)
    out[1:, :] |= mask[:-1, :]
    out[:-1, :] |= mask[1:, :]
    out[:, 1:] |= mask[:, :-1]
    out[:, :-1] |= mask[:, 1:]
    return out


def _clustered(W, H, n, seed, blobs=4, sigma=6.0):
    rng = np.random.default_rng(seed)
    centres = rng.uniform([0, 0], [W, H], size=(blobs, 2))
    pts = centres[rng.integers(0, blobs, size=4 * n)] + rng.normal(0, sigma, size=(4 * n, 2))
    pts = np.clip(np.rint(pts), [0, 0], [W - 1, H - 1]).astype(np.int64)
    _, first = np.unique(pts[:, 1] * W + pts[:, 0], return_index=True)
    return pts[np.sort(first)][:n]


@pytest.mark.parametrize("W,H,n,seed,layout", [
    (48, 32, 12, 0, "uniform"), (64, 64, 40, 1, "uniform"), (97, 61, 150, 2, "uniform"),
    (96, 96, 60, 3, "clustered"), (128, 80, 25, 4, "clustered"),
])
def test_changes_spread_only_from_changed_neighbours(W, H, n, seed, layout):
    pts = random_seeds(W, H, n, seed) if layout == "uniform" else _clustered(W, H, n, seed)
    s = oracle.sort_seeds(pts, W, H)
    xs, ys = (np.asarray(v, dtype=np.int64) for v in oracle._xy(s))
    lab = np.full((H, W), -1, dtype=np.int64)
    lab[ys, xs] = np.arange(len(xs))
    seeds = lab >= 0

    changed_before = None
    passes = 0
    while True:
        nxt = _pass(lab, xs, ys)
        changed = nxt != lab
        if changed_before is None:
            # pass 0: only the seeds' 4-neighbours, never a seed
            assert not (changed & seeds).any()
            assert not (changed & ~_neighbours(seeds)).any()
        else:
            assert not (changed & ~_neighbours(changed_before)).any(), f"pass {passes}"
        lab = nxt
        passes += 1
        if not changed.any():
            break
        changed_before = changed
        assert passes < 4 * (W + H)

    want, want_passes = oracle.voronoi("reference", W, H, s)
    np.testing.assert_array_equal(lab, want[..., 0])
    assert passes == want_passes
