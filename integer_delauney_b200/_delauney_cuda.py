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
    """(triangle_map | verts, grid) as binding_helpers.hpp:61-87 packs it.
    ``tris`` holds (x, y, a, b, c) rows, or for as_arrays already the (a, b, c)
    triples (idl_get_triangle_vertices)."""
    if as_arrays:
        if tris.shape[1] == 3:
            return tris, grid
        return np.ascontiguousarray(tris[:, 2:5], dtype=np.int32), grid
    rows = tris.tolist()
    return {tid: tuple(r) for tid, r in enumerate(rows)}, grid


def _fetch_triangles(ctx, n_tri: int) -> np.ndarray:
    # pageable: the count changes call to call, and a new pinned block of a
    # new size costs a page-locking allocation of milliseconds
    out = np.empty((max(n_tri, 0), 5), dtype=np.int32)
    check(_capi.load().idl_get_triangles(ctx.handle, out.ctypes.data if n_tri else None, n_tri))
    return out


def _fetch_vertices(ctx, n_tri: int) -> np.ndarray:
    """(n, 3) vertex triples, packed on the device (12 bytes per triangle cross PCIe)."""
    out = np.empty((max(n_tri, 0), 3), dtype=np.int32)
    check(_capi.load().idl_get_triangle_vertices(ctx.handle, out.ctypes.data if n_tri else None, n_tri))
    return out


def _triangulate(width, height, seeds_arr, vgrid, border_padding, mode, timings=False, debug=False,
                 vertices=False):
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
        tris = (_fetch_vertices if vertices else _fetch_triangles)(ctx, int(n_tri.value))
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
    tris, grid, _, _ = _triangulate(width, height, s, None, border_padding, voronoi_mode, vertices=as_arrays)
    return build_output(tris, grid, as_arrays)


def triangulate_batch(images, border_padding: int = AUTO_BORDER_PADDING, as_arrays: bool = False, *,
                      voronoi_mode="reference"):
    """Triangulate many independent images in one pass of the pipeline.

    ``images``: iterable of (width, height, seeds).  Returns a list with one
    (triangle_map | verts, grid) per image, each equal to
    ``triangulate(width, height, seeds, border_padding, as_arrays)``.  Not in
    the reference API (which has one image per call); see
    idl_triangulate_batch in include/idelaunay.h for the limits."""
    imgs = [(int(w), int(h), parse_seeds(s)) for w, h, s in images]
    n = len(imgs)
    if n == 0:
        return []
    dims = np.array([(w, h) for w, h, _ in imgs], dtype=np.int32)
    counts = np.array([len(s) for _, _, s in imgs], dtype=np.int64)
    seeds = np.ascontiguousarray(np.concatenate([s for _, _, s in imgs]) if counts.sum() else
                                 np.zeros((0, 2), np.int32), dtype=np.int32)
    px = [w * h for w, h, _ in imgs]
    grids = _host_buffer((max(sum(px), 0) * 3,))
    tri_counts = np.zeros(n, dtype=np.int64)
    lib = _capi.load()
    ctx = _context()
    with ctx.lock:
        _bind(ctx)
        check(lib.idl_triangulate_batch(ctx.handle, n, dims.ctypes.data, counts.ctypes.data,
                                        seeds.ctypes.data if len(seeds) else None, int(border_padding),
                                        mode_id(voronoi_mode), grids.ctypes.data, tri_counts.ctypes.data, None))
        tris = _fetch_triangles(ctx, int(tri_counts.sum()))
    out = []
    p0 = t0 = 0
    for (w, h, _), npx, nt in zip(imgs, px, tri_counts.tolist()):
        g = grids[p0 * 3:(p0 + npx) * 3].reshape(h, w, 3)
        out.append(build_output(tris[t0:t0 + nt], g, as_arrays))
        p0 += npx
        t0 += nt
    return out


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
        tris, grid, _, _ = _triangulate(W, H, s, vg, border_padding, voronoi_mode, vertices=as_arrays)
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


# ---------------------------------------------------------------------------
# Incremental triangulation (src/cuda/bindings/py_delaunay.hpp,
# src/cuda/bindings/py_device_array_view.hpp)
# ---------------------------------------------------------------------------

def _timings_dict(t) -> dict:
    """The keys of PyDelaunay::_timings_dict (py_delaunay.hpp:268-277)."""
    return {"bfs_ms": float(t[_capi.T_BFS_MS]), "bfs_iters": int(t[_capi.T_BFS_ITERS]),
            "detect_ms": float(t[_capi.T_DETECT_MS]), "dedup_ms": float(t[_capi.T_DEDUP_MS]),
            "assign_ms": float(t[_capi.T_ASSIGN_MS])}


def _points(points) -> np.ndarray:
    q = np.ascontiguousarray(np.asarray(points), dtype=np.int32)
    if q.ndim != 2 or q.shape[1] != 2:
        raise ValueError("points must have shape (N, 2)")
    return q


class DeviceArrayView:
    """Read-only ``__cuda_array_interface__`` (v3) onto one of a Delaunay
    object's device arrays (py_device_array_view.hpp:29-89).

    Holds a reference to its Delaunay, so the memory outlives every view; it
    raises RuntimeError once the Delaunay has moved to a new generation (any
    insert, finalise or finalise_device after the one that made the view)."""

    def __init__(self, owner, ptr: int, count: int, typestr: str, generation: int):
        self._owner = owner
        self._ptr = int(ptr)
        self._count = int(count)
        self._typestr = typestr
        self._generation = int(generation)

    def _check_fresh(self):
        if self._owner._generation() != self._generation:
            raise RuntimeError("device view is stale: the mesh was mutated after "
                               "finalise_device() produced this view")

    @property
    def __cuda_array_interface__(self) -> dict:
        self._check_fresh()
        return {"shape": (self._count,), "typestr": self._typestr, "data": (self._ptr, True),
                "strides": None, "version": 3}

    def _raw(self, keep):
        """An object exposing the same memory through a writable interface
        (torch refuses read-only ones), holding `keep` alive."""
        raw = type("_Raw", (), {"__cuda_array_interface__": {
            "shape": (self._count,), "typestr": self._typestr, "data": (self._ptr, False),
            "strides": None, "version": 3}})()
        raw._keep = keep
        return raw

    def to_torch(self):
        """The view as a torch tensor on the object's device, without a copy
        (1-D, int32 or uint8): for consumers that take tensors or DLPack --
        not in the reference, whose views stop at the CUDA array interface.
        The tensor keeps the Delaunay alive, but like the view it is only
        meaningful until the object's next insert or finalise.  torch has no
        read-only tensors: writes through it land in the object's arrays."""
        self._check_fresh()
        if torch is None:
            raise RuntimeError("to_torch() needs torch")
        dev = self._owner._device
        if not self._count:
            return torch.empty(0, dtype=torch.int32 if self._typestr == "<i4" else torch.uint8, device=f"cuda:{dev}")
        return torch.as_tensor(self._raw(self), device=f"cuda:{dev}")

    def __dlpack__(self, stream=None, **kwargs):
        """DLPack export (zero-copy, through ``to_torch``): ``torch.from_dlpack(view)``
        and other DLPack consumers read the device memory in place."""
        return self.to_torch().__dlpack__(stream=stream, **kwargs)

    def __dlpack_device__(self):
        return (2, int(self._owner._device))   # kDLCUDA, device ordinal

    def to_host(self) -> np.ndarray:
        """Host NumPy copy of the view's content."""
        self._check_fresh()
        dtype = np.int32 if self._typestr == "<i4" else np.uint8
        if torch is None:
            raise RuntimeError("to_host() needs torch for the device copy")
        out = np.empty(self._count, dtype=dtype)
        if self._count:
            inner = self._raw(None)   # the copy below only reads
            with torch.cuda.device(self._owner._device):
                torch.cuda.current_stream().synchronize()
                out[:] = torch.as_tensor(inner, device=f"cuda:{self._owner._device}").cpu().numpy()
        return out


class Delaunay:
    """Incremental Delaunay triangulator with device-resident state
    (src/cuda/delaunay.cuh:22-378, bound in py_delaunay.hpp:11-305).

    Seeds keep insertion-order ids internally; the triangle map and grids of
    insert / finalise and the Voronoi grid use the batch (x asc, y asc) ids,
    as the reference translates through ``sorted_rank``.  Triangle ids are the
    batch pipeline's canonical ids (rank of the sorted vertex triple), so
    they are dense after every call and independent of the insertion history.
    """

    def __init__(self, width: int, height: int, max_seeds: int, border_padding: int = AUTO_BORDER_PADDING, *,
                 voronoi_mode="reference"):
        import threading
        self._lib = _capi.load()
        self._h = None
        self._device = _device()
        self._lock = threading.Lock()
        h = ctypes.c_void_p()
        check(self._lib.idl_delaunay_create(self._device, int(width), int(height), int(max_seeds),
                                            int(border_padding), mode_id(voronoi_mode), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                self._lib.idl_delaunay_destroy(h)
            except Exception:   # pragma: no cover - interpreter shutdown
                pass

    # -- plumbing ------------------------------------------------------------
    def _call(self, name, *args):
        with self._lock:
            if torch is not None and torch.cuda.is_available():
                stream = torch.cuda.current_stream(self._device).cuda_stream
                check(self._lib.idl_delaunay_set_stream(self._h, stream))
            check(getattr(self._lib, name)(self._h, *args))

    def _info(self) -> np.ndarray:
        info = np.zeros(_capi.DI_COUNT, dtype=np.int64)
        check(self._lib.idl_delaunay_info(self._h, info.ctypes.data_as(_capi._pi64), _capi.DI_COUNT))
        return info

    def _generation(self) -> int:
        return int(self._info()[_capi.DI_GENERATION])

    def _tris(self, ids: int, count: int | None = None) -> np.ndarray:
        """Triangle rows (idl_delaunay_triangles format `ids`); `count`, when
        the caller already has the triangle count, saves the query call.
        Pageable memory: a pinned block of each new size would cost a
        page-locking allocation."""
        n = ctypes.c_int64(0)
        if count is None:
            self._call("idl_delaunay_triangles", ids, None, 0, ctypes.byref(n))
            count = n.value
        cols = 5 if ids == 0 else 3
        out = np.empty((count, cols), dtype=np.int32)
        if count:
            self._call("idl_delaunay_triangles", ids, out.ctypes.data, out.size, ctypes.byref(n))
        return out

    def _insert(self, seeds, values, timings: bool, order: str = "given"):
        if order not in ("given", "xy"):
            raise ValueError("order must be 'given' or 'xy'")
        s = parse_seeds(seeds)
        v = None
        if values is not None:
            v = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
            if len(v) != len(s):
                raise ValueError("values must have one entry per seed in the batch")
        t = (ctypes.c_float * _capi.T_COUNT)() if timings else None
        self._call("idl_delaunay_insert_ordered", s.ctypes.data if len(s) else None, len(s),
                   v.ctypes.data if (v is not None and len(v)) else None, 1 if order == "xy" else 0,
                   ctypes.cast(t, ctypes.c_void_p) if t is not None else None)
        return t

    def _finalise(self, as_arrays: bool, timings: bool):
        H, W = self.height, self.width
        grid = _host_buffer((H, W, 3))
        n = ctypes.c_int64(0)
        t = (ctypes.c_float * _capi.T_COUNT)() if timings else None
        self._call("idl_delaunay_finalise", grid.ctypes.data, ctypes.byref(n),
                   ctypes.cast(t, ctypes.c_void_p) if t is not None else None)
        # as_arrays: the vertex triples packed on the device (format 2), not
        # the five-column rows sliced on the host
        m, g = build_output(self._tris(2 if as_arrays else 0, int(n.value)), grid, as_arrays)
        return m, g, t

    # -- reference API ---------------------------------------------------------
    def insert(self, seeds, as_arrays: bool = False):
        """Append a batch and return (triangle_map | verts, grid (H, W, 3))."""
        self._insert(seeds, None, False)
        m, g, _ = self._finalise(as_arrays, False)
        return m, g

    def insert_timed(self, seeds, as_arrays: bool = False):
        t0 = self._insert(seeds, None, True)
        m, g, t1 = self._finalise(as_arrays, True)
        d = _timings_dict(t0)
        d["assign_ms"] = float(t1[_capi.T_ASSIGN_MS])
        d["detect_ms"] += float(t1[_capi.T_DETECT_MS])
        d["dedup_ms"] += float(t1[_capi.T_DEDUP_MS])
        return m, g, d

    def insert_deferred(self, seeds, values=None, *, order: str = "given") -> None:
        """Append a batch (and optionally its scalar values) without assigning pixels.

        ``order="xy"`` (an addition) numbers this batch's seeds in (x, y)
        order instead of the order given; into an empty object that yields
        the batch pipeline's result exactly."""
        self._insert(seeds, values, False, order)

    def insert_deferred_timed(self, seeds) -> dict:
        return _timings_dict(self._insert(seeds, None, True))

    def finalise(self, as_arrays: bool = False):
        m, g, _ = self._finalise(as_arrays, False)
        return m, g

    def finalise_timed(self, as_arrays: bool = False):
        m, g, t = self._finalise(as_arrays, True)
        return m, g, _timings_dict(t)

    def finalise_device(self):
        """(verts (N_tri, 3), pixel_tids, pixel_seed_ids, outside_hull_mask) with
        the three per-pixel arrays as device views (py_delaunay.hpp:65-91)."""
        n = ctypes.c_int64(0)
        p_t, p_s, p_m = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        gen = ctypes.c_uint64(0)
        self._call("idl_delaunay_finalise_device", ctypes.byref(n), ctypes.byref(p_t), ctypes.byref(p_s),
                   ctypes.byref(p_m), ctypes.byref(gen))
        verts = self._tris(2, int(n.value))
        count = self.width * self.height
        return (verts, DeviceArrayView(self, p_t.value or 0, count, "<i4", gen.value),
                DeviceArrayView(self, p_s.value or 0, count, "<i4", gen.value),
                DeviceArrayView(self, p_m.value or 0, count, "|u1", gen.value))

    def _adopt(self, context, image: int) -> None:
        """Take image `image` of the last idl_voronoi_batch on `context` as
        this (empty) object's state (see idl_delaunay_adopt)."""
        self._call("idl_delaunay_adopt", context.handle, int(image))

    def _finalise_device_count(self) -> int:
        """finalise_device() without the triangle copy: the count only."""
        n = ctypes.c_int64(0)
        self._call("idl_delaunay_finalise_device", ctypes.byref(n), None, None, None, None)
        return int(n.value)

    def get_triangles(self) -> np.ndarray:
        """(N_tri, 3) vertex ids in INSERTION order, rows in triangle-id order."""
        return self._tris(1)

    def get_edges(self) -> np.ndarray:
        n = ctypes.c_int64(0)
        self._call("idl_delaunay_edges", None, 0, ctypes.byref(n))
        out = np.empty((n.value, 2), dtype=np.int32)
        if n.value:
            self._call("idl_delaunay_edges", out.ctypes.data, out.size, ctypes.byref(n))
        return out

    def edge_scores(self, min_length: float = 0.0) -> np.ndarray:
        n = ctypes.c_int64(0)
        self._call("idl_delaunay_edge_scores", float(min_length), None, 0, ctypes.byref(n))
        out = np.empty(n.value, dtype=np.float32)
        if n.value:
            self._call("idl_delaunay_edge_scores", float(min_length), out.ctypes.data, out.size, ctypes.byref(n))
        return out

    def select_midpoints(self, min_length: float, count: int, threshold: float = 0.0) -> np.ndarray:
        cap = max(int(count), 0)
        out = np.empty((cap, 2), dtype=np.int32)
        n = ctypes.c_int64(0)
        self._call("idl_delaunay_select_midpoints", float(min_length), int(count), float(threshold),
                   out.ctypes.data if cap else None, out.size, ctypes.byref(n))
        return out[: n.value].copy()

    def in_circumsphere(self, points, t):
        q = _points(points)
        tt = np.ascontiguousarray(np.asarray(t, dtype=np.float64).reshape(-1))
        if len(tt) != len(q):
            raise ValueError("t must have one entry per point")
        mask = np.zeros(len(q), dtype=np.uint8)
        tids = np.full(len(q), -1, dtype=np.int32)
        if len(q):
            self._call("idl_delaunay_in_circumsphere", q.ctypes.data, tt.ctypes.data, len(q), mask.ctypes.data,
                       tids.ctypes.data)
        return mask.astype(bool), tids

    def locate(self, points) -> np.ndarray:
        q = _points(points)
        out = np.full(len(q), -1, dtype=np.int32)
        if len(q):
            self._call("idl_delaunay_locate", q.ctypes.data, len(q), out.ctypes.data)
        return out

    def get_seeds(self) -> np.ndarray:
        out = np.empty((self.seed_count, 2), dtype=np.int32)
        self._call("idl_delaunay_seeds", out.ctypes.data if out.size else None, None, None)
        return out

    def get_values(self) -> np.ndarray:
        n = ctypes.c_int64(0)
        self._call("idl_delaunay_seeds", None, None, ctypes.byref(n))
        out = np.empty(n.value, dtype=np.float32)
        if n.value:
            self._call("idl_delaunay_seeds", None, out.ctypes.data, ctypes.byref(n))
        return out

    @property
    def sorted_rank(self) -> np.ndarray:
        out = np.empty(self.seed_count, dtype=np.int32)
        if out.size:
            self._call("idl_delaunay_sorted_rank", out.ctypes.data)
        return out

    def get_voronoi_grid(self) -> np.ndarray:
        out = _host_buffer((self.height, self.width, 2))
        self._call("idl_delaunay_voronoi", out.ctypes.data)
        return out

    # -- additions (no counterpart in the reference) ------------------------
    def reset(self, width: int, height: int, max_seeds: int, border_padding: int = AUTO_BORDER_PADDING) -> None:
        """Empty the object and reuse its device memory for another canvas
        (ValueError if it does not fit).  Outstanding device views go stale."""
        self._call("idl_delaunay_reset", int(width), int(height), int(max_seeds), int(border_padding))

    def use_workspace(self, context) -> None:
        """Take scratch memory from ``context`` (an ``_capi.Context`` on the
        same device) instead of the object's own; None goes back to its own.
        Objects sharing a context must not run at the same time."""
        self._workspace = context            # keeps the context alive while in use
        self._call("idl_delaunay_set_workspace", context.handle if context is not None else None)

    @property
    def device_bytes(self) -> int:
        """Device memory held by the object, workspace included."""
        return int(self._info()[_capi.DI_DEVICE_BYTES])

    @property
    def seed_count(self) -> int:
        return int(self._info()[_capi.DI_SEED_COUNT])

    @property
    def width(self) -> int:
        return int(self._info()[_capi.DI_WIDTH])

    @property
    def height(self) -> int:
        return int(self._info()[_capi.DI_HEIGHT])

    @property
    def border_padding(self) -> int:
        return int(self._info()[_capi.DI_BORDER_PADDING])

    @property
    def has_pending(self) -> bool:
        return bool(self._info()[_capi.DI_HAS_PENDING])
