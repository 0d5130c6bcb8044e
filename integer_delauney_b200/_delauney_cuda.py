"""Drop-in replacement for the reference's compiled module ``delauney._delauney_cuda``.

Same classes, functions, argument names, defaults, return types and error
types as the pybind11 module of src/cuda/bindings.cpp:17-228; every call goes
through the C ABI of include/idelaunay.h into the sm_100a kernels.  PyTorch is
used only as plumbing: the current CUDA device and stream, and pinned host
buffers (its caching host allocator) that the results are copied into and
that the returned NumPy arrays wrap.

One addition per entry point: a keyword-only ``voronoi_mode`` selecting the
propagation semantics -- "reference" (default; the reference CUDA path's
Jacobi fixed point, bit for bit), "numpy" (bit for bit what
``delauney.reference.Voronoi`` computes) or "exact" (nearest seed, ties to
the higher id).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from ._capi import AUTO_BORDER_PADDING, DEFAULT_BORDER_PADDING, check, mode_id

_capi.load()   # fail at import time, like an unbuilt extension module

try:
    import torch
except ImportError:   # pragma: no cover - torch is part of the supported stack
    torch = None


def _device() -> int:
    if torch is not None and torch.cuda.is_available():
        return torch.cuda.current_device()
    return 0


def _bind(ctx) -> None:
    stream = 0
    if torch is not None and torch.cuda.is_available():
        stream = torch.cuda.current_stream().cuda_stream
    ctx.set_stream(stream)


def _context():
    ctx = _capi.context_for(_device())
    return ctx


def _host_buffer(shape, dtype=np.int32):
    """Pinned host array (torch's caching host allocator) viewed as NumPy."""
    if torch is not None and torch.cuda.is_available():
        t = torch.empty(tuple(shape), dtype=torch.int32 if dtype == np.int32 else torch.uint8, pin_memory=True)
        return t.numpy()
    return np.empty(shape, dtype=dtype)


def parse_seeds(seeds) -> np.ndarray:
    """(N, 2) int32 C-contiguous copy of an iterable of (x, y) pairs.

    Accepts any sequence of pairs or an (N, 2) integer array (the fast path of
    src/cuda/bindings/py_delaunay.hpp:279-304).  Coordinates that do not fit
    int32 are mapped to -1 so that bounds validation rejects them.
    """
    if isinstance(seeds, np.ndarray) and seeds.ndim == 2 and seeds.shape[1] == 2 and \
            np.issubdtype(seeds.dtype, np.integer):
        a = seeds
    else:
        try:
            a = np.asarray(list(seeds) if not isinstance(seeds, np.ndarray) else seeds)
        except TypeError:
            raise TypeError("seeds must be an iterable of (x, y) pairs") from None
        if a.size == 0:
            return np.zeros((0, 2), dtype=np.int32)
        if a.ndim != 2 or a.shape[1] != 2:
            raise TypeError("each seed must be an (x, y) pair")
        if not np.issubdtype(a.dtype, np.integer):
            if np.issubdtype(a.dtype, np.floating) and np.all(np.isfinite(a)) and np.all(a == np.floor(a)):
                a = a.astype(np.int64)
            else:
                raise TypeError("seed coordinates must be integers")
    if a.dtype != np.int32:
        a64 = a.astype(np.int64, copy=False)
        bad = (a64 < np.iinfo(np.int32).min) | (a64 > np.iinfo(np.int32).max)
        a = np.where(bad, -1, a64).astype(np.int32)
    return np.ascontiguousarray(a, dtype=np.int32)


def resolve_padding(border_padding: int) -> int:
    """binding_helpers.hpp:49-53; other negatives clamp to 0 (reference/triangulation.py:78)."""
    p = int(border_padding)
    if p == AUTO_BORDER_PADDING:
        return DEFAULT_BORDER_PADDING
    return max(0, p)


def build_output(tris: np.ndarray, grid: np.ndarray, as_arrays: bool):
    """(triangle_map | verts, grid) as binding_helpers.hpp:61-87 packs it."""
    if as_arrays:
        return np.ascontiguousarray(tris[:, 2:5], dtype=np.int32), grid
    rows = tris.tolist()
    return {tid: tuple(r) for tid, r in enumerate(rows)}, grid


def _fetch_triangles(ctx, n_tri: int) -> np.ndarray:
    out = np.empty((max(n_tri, 0), 5), dtype=np.int32)
    check(_capi.load().idl_get_triangles(ctx.handle, out.ctypes.data if n_tri else None, n_tri))
    return out


def _triangulate(width, height, seeds_arr, vgrid, border_padding, mode, timings=False, debug=False):
    lib = _capi.load()
    ctx = _context()
    P = resolve_padding(border_padding)
    grid = _host_buffer((height, width, 3))
    padded = None
    if debug:
        padded = np.zeros((height + 2 * P, width + 2 * P, 2), dtype=np.int32)
    tbuf = (ctypes.c_float * _capi.T_COUNT)() if timings else None
    n_tri = ctypes.c_int64(0)
    with ctx.lock:
        _bind(ctx)
        check(lib.idl_triangulate(ctx.handle, int(width), int(height),
                                  seeds_arr.ctypes.data if len(seeds_arr) else None, len(seeds_arr),
                                  vgrid.ctypes.data if vgrid is not None else None, int(border_padding),
                                  mode_id(mode), grid.ctypes.data, ctypes.byref(n_tri),
                                  ctypes.cast(tbuf, ctypes.c_void_p) if tbuf is not None else None,
                                  padded.ctypes.data if (padded is not None and P > 0) else None))
        tris = _fetch_triangles(ctx, int(n_tri.value))
    tdict = None
    if timings:
        tdict = {"detect_ms": float(tbuf[_capi.T_DETECT_MS]), "dedup_ms": float(tbuf[_capi.T_DEDUP_MS]),
                 "assign_ms": float(tbuf[_capi.T_ASSIGN_MS])}
    return tris, grid, tdict, padded


class Voronoi:
    """Stateless L2 Voronoi diagram (src/cuda/bindings/py_voronoi.hpp:9-25)."""

    def compute(self, width: int, height: int, seeds, *, voronoi_mode="reference") -> np.ndarray:
        """(height, width, 2) int32: (seed id, squared L2 distance) per cell."""
        s = parse_seeds(seeds)
        lib = _capi.load()
        ctx = _context()
        out = _host_buffer((max(int(height), 0), max(int(width), 0), 2))
        with ctx.lock:
            _bind(ctx)
            check(lib.idl_voronoi(ctx.handle, int(width), int(height), s.ctypes.data if len(s) else None, len(s),
                                  mode_id(voronoi_mode), out.ctypes.data if out.size else None, None))
        return out


def triangulate(width: int, height: int, seeds, border_padding: int = AUTO_BORDER_PADDING,
                as_arrays: bool = False, *, voronoi_mode="reference"):
    """The whole pipeline in one call (src/cuda/bindings/triangulate.hpp:15-43)."""
    s = parse_seeds(seeds)
    tris, grid, _, _ = _triangulate(width, height, s, None, border_padding, voronoi_mode)
    return build_output(tris, grid, as_arrays)


class GridTriangulation:
    """Triangles from a Voronoi grid (src/cuda/bindings/py_grid_triangulation.hpp:10-110)."""

    @staticmethod
    def _prepare(voronoi_grid, seed_positions):
        vg = np.ascontiguousarray(np.asarray(voronoi_grid), dtype=np.int32)
        if vg.ndim != 3 or vg.shape[2] != 2:
            raise ValueError("voronoi_grid must have shape (H, W, 2)")
        return vg, parse_seeds(seed_positions)

    def compute(self, voronoi_grid, seed_positions, border_padding: int = AUTO_BORDER_PADDING,
                as_arrays: bool = False, *, voronoi_mode="reference"):
        vg, s = self._prepare(voronoi_grid, seed_positions)
        H, W = vg.shape[:2]
        tris, grid, _, _ = _triangulate(W, H, s, vg, border_padding, voronoi_mode)
        return build_output(tris, grid, as_arrays)

    def compute_timed(self, voronoi_grid, seed_positions, border_padding: int = AUTO_BORDER_PADDING, *,
                      voronoi_mode="reference"):
        vg, s = self._prepare(voronoi_grid, seed_positions)
        H, W = vg.shape[:2]
        tris, grid, t, _ = _triangulate(W, H, s, vg, border_padding, voronoi_mode, timings=True)
        m, g = build_output(tris, grid, False)
        return m, g, t

    def compute_debug(self, voronoi_grid, seed_positions, border_padding: int = AUTO_BORDER_PADDING, *,
                      voronoi_mode="reference"):
        vg, s = self._prepare(voronoi_grid, seed_positions)
        H, W = vg.shape[:2]
        tris, grid, _, padded = _triangulate(W, H, s, vg, border_padding, voronoi_mode, debug=True)
        m, g = build_output(tris, grid, False)
        return m, g, padded
