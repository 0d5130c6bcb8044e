"""CPU oracle for the integer Delaunay hot path -- test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this package, always as the checker (or the timed CPU baseline), never as the
product.  The product path (``integer_delauney_b200``) never imports it and
fails loudly when its CUDA library is missing.

The numerics live in ``idl_oracle.c`` (plain C, OpenMP), which restates the
reference algorithm function by function; each C function cites the
reference file:line it follows.  This module is a thin ctypes wrapper plus the
seed validation/sort of ``src/cuda/bindings/binding_helpers.hpp:23-46``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MODE_REFERENCE = 0   # voronoi.cu Jacobi fixed point
MODE_SWEEP = 1       # reference/voronoi.py four-direction sweep
MODE_NEAREST = 2     # exact nearest seed, ties to the higher id
MODES = {"reference": MODE_REFERENCE, "numpy": MODE_SWEEP, "exact": MODE_NEAREST}

DEFAULT_BORDER_PADDING = 16

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liboracle.so in place (gcc + make)."""
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "idl_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "CC=gcc"], check=True)
    return path


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle.so")
    if not os.path.exists(path):
        build()
    L = ctypes.CDLL(path)
    i64, i32 = ctypes.c_int64, ctypes.c_int
    L.or_voronoi_jacobi.restype = i64
    L.or_voronoi_jacobi.argtypes = [i32, i32, _i32p, _i32p, _i32p, i64]
    L.or_voronoi_sweep.restype = i64
    L.or_voronoi_sweep.argtypes = [i32, i32, _i32p, _i32p, _i32p, i64]
    L.or_voronoi_nearest.restype = None
    L.or_voronoi_nearest.argtypes = [i32, i32, _i32p, _i32p, i32, _i32p]
    L.or_voronoi.restype = i64
    L.or_voronoi.argtypes = [i32, i32, i32, _i32p, _i32p, i32, _i32p]
    L.or_detect.restype = i64
    L.or_detect.argtypes = [i32, i32, _i32p, _i32p, _i32p, i32, _i32p, i64]
    L.or_block_rule.restype = i32
    L.or_block_rule.argtypes = [i32, i32, i32, i32, _i32p, _i32p, _i32p]
    L.or_window_cap.restype = i32
    L.or_window_cap.argtypes = [_i32p, i64, _i32p, _i32p]
    L.or_assign.restype = None
    L.or_assign.argtypes = [i32, i32, _i32p, _i32p, i32, _i32p, i64, _i32p]
    L.or_assign_rows.restype = None
    L.or_assign_rows.argtypes = [i32, i32, _i32p, _i32p, i32, _i32p, i64, i32, i32, _i32p]
    L.or_assign_bbox_rows.restype = None
    L.or_assign_bbox_rows.argtypes = [i32, i32, _i32p, _i32p, _i32p, i64, i32, i32, _i32p]
    L.or_triangulate.restype = i64
    L.or_triangulate.argtypes = [i32, i32, _i32p, _i32p, i32, i32, i32, ctypes.c_void_p,
                                 _i32p, _i32p, i64, ctypes.POINTER(ctypes.c_int64)]
    L.or_num_threads.restype = i32
    L.or_set_threads.argtypes = [i32]
    _LIB = L
    return L


def num_threads() -> int:
    return int(lib().or_num_threads())


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def mode_id(mode) -> int:
    if isinstance(mode, str):
        return MODES[mode]
    return int(mode)


def sort_seeds(seeds, W: int, H: int) -> np.ndarray:
    """Validate and sort seeds by (x, y); binding_helpers.hpp:23-46.

    Raises ValueError with the reference's messages: out of bounds first (in
    input order), then empty, then duplicates.
    """
    arr = np.asarray(seeds, dtype=np.int64).reshape(-1, 2) if len(seeds) else np.zeros((0, 2), np.int64)
    oob = (arr[:, 0] < 0) | (arr[:, 0] >= W) | (arr[:, 1] < 0) | (arr[:, 1] >= H)
    if oob.any():
        raise ValueError("seed coordinate out of bounds")
    if len(arr) == 0:
        raise ValueError("seeds must not be empty")
    order = np.lexsort((arr[:, 1], arr[:, 0]))
    s = arr[order].astype(np.int32)
    if len(s) > 1 and np.any((np.diff(s[:, 0]) == 0) & (np.diff(s[:, 1]) == 0)):
        raise ValueError("duplicate seed positions are not allowed")
    return np.ascontiguousarray(s)


def _xy(sorted_seeds):
    s = np.ascontiguousarray(np.asarray(sorted_seeds, dtype=np.int32).reshape(-1, 2))
    return np.ascontiguousarray(s[:, 0]), np.ascontiguousarray(s[:, 1])


def voronoi(mode, W: int, H: int, sorted_seeds) -> tuple[np.ndarray, int]:
    """(H, W, 2) int32 (seed id, squared distance) and the pass count."""
    xs, ys = _xy(sorted_seeds)
    out = np.empty((H, W, 2), dtype=np.int32)
    passes = lib().or_voronoi(mode_id(mode), W, H, xs, ys, len(xs), out)
    return out, int(passes)


def jacobi_from(W: int, H: int, xs, ys, labels: np.ndarray) -> tuple[np.ndarray, int]:
    """Run the reference Jacobi from an arbitrary starting label grid."""
    lab = np.ascontiguousarray(labels, dtype=np.int32).copy()
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    passes = lib().or_voronoi_jacobi(W, H, xs, ys, lab, 0)
    return lab, int(passes)


def sweep_from(W: int, H: int, xs, ys, labels: np.ndarray) -> tuple[np.ndarray, int]:
    lab = np.ascontiguousarray(labels, dtype=np.int32).copy()
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    iters = lib().or_voronoi_sweep(W, H, xs, ys, lab, 0)
    return lab, int(iters)


def nearest(W: int, H: int, xs, ys) -> np.ndarray:
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    lab = np.empty((H, W), dtype=np.int32)
    lib().or_voronoi_nearest(W, H, xs, ys, len(xs), lab)
    return lab


def block_rule(a, b, c, d, xs, ys):
    out = np.zeros((2, 3), dtype=np.int32)
    k = lib().or_block_rule(int(a), int(b), int(c), int(d),
                            np.ascontiguousarray(xs, dtype=np.int32),
                            np.ascontiguousarray(ys, dtype=np.int32), out)
    return [tuple(int(v) for v in out[i]) for i in range(k)]


def detect(labels: np.ndarray, xs, ys, shift: int = 0) -> np.ndarray:
    """Deduplicated (N_tri, 5) int32 (x, y, orig_a, orig_b, orig_c)."""
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    H, W = lab.shape
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    cap = max(16, 4 * len(xs) + 64)
    while True:
        out = np.empty((cap, 5), dtype=np.int32)
        nt = lib().or_detect(W, H, lab, xs, ys, int(shift), out, cap)
        if nt >= 0:
            return out[:nt].copy()
        cap = -nt


def assign(W: int, H: int, xs, ys, tris: np.ndarray) -> np.ndarray:
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 5)
    out = np.empty((H, W), dtype=np.int32)
    lib().or_assign(W, H, xs, ys, len(xs), t, len(t), out)
    return out


def window_cap(tris: np.ndarray, xs, ys) -> int:
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 5)
    return int(lib().or_window_cap(t, len(t), np.ascontiguousarray(xs, dtype=np.int32),
                                   np.ascontiguousarray(ys, dtype=np.int32)))


def assign_rows(W: int, H: int, xs, ys, tris: np.ndarray, y0: int, y1: int) -> np.ndarray:
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 5)
    out = np.empty((y1 - y0, W), dtype=np.int32)
    lib().or_assign_rows(W, H, xs, ys, len(xs), t, len(t), y0, y1, out)
    return out


def assign_bbox(W: int, H: int, xs, ys, tris: np.ndarray, y0: int = 0, y1=None) -> np.ndarray:
    """assign() evaluated per triangle over its bounding box (same result,
    cost proportional to the triangles' box areas); rows [y0, y1)."""
    y1 = H if y1 is None else y1
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 5)
    out = np.empty((y1 - y0, W), dtype=np.int32)
    lib().or_assign_bbox_rows(W, H, xs, ys, t, len(t), int(y0), int(y1), out)
    return out


def triangulate(W: int, H: int, sorted_seeds, P: int = DEFAULT_BORDER_PADDING,
                mode="reference", vgrid=None):
    """The batch pipeline of triangulation.cu:143-365.

    Returns (tris (N_tri, 5) int32, grid (H, W, 3) int32, propagation passes).
    """
    xs, ys = _xy(sorted_seeds)
    n = len(xs)
    out = np.empty((H, W, 3), dtype=np.int32)
    passes = ctypes.c_int64(0)
    vg = None
    vptr = None
    if vgrid is not None:
        vg = np.ascontiguousarray(vgrid, dtype=np.int32)
        vptr = vg.ctypes.data_as(ctypes.c_void_p)
    cap = max(16, 4 * n + 64)
    while True:
        tris = np.empty((cap, 5), dtype=np.int32)
        nt = lib().or_triangulate(W, H, xs, ys, n, int(P), mode_id(mode), vptr, out, tris, cap,
                                  ctypes.byref(passes))
        if nt >= 0:
            return tris[:nt].copy(), out, int(passes.value)
        cap = -nt


def incremental(W: int, H: int, batches, P: int = DEFAULT_BORDER_PADDING):
    """The reference's incremental Delaunay, restated on the CPU.

    Seeds keep insertion-order ids; each batch is written into the padded
    label grid and the Jacobi iteration continues from the previous fixed
    point (src/cuda/delaunay.cu:184-268, src/cuda/delaunay_voronoi.cu:12-108).
    Triangles are detected on the insertion-id grid (the block rule's
    lowest-id tie-break sees insertion ids, triangle_detect.cuh:75-166) and
    reported the batch way: vertex ids through sorted_rank
    (src/cuda/delaunay_output.cu:39-84), triangle id = rank of the sorted
    triple, pixel = highest id of the triangles containing it.

    Returns dict(rank, tris (N_tri, 5) batch ids, tris_ins (N_tri, 3)
    insertion ids, grid (H, W, 3), labels (padded, insertion ids), passes).
    """
    Wd, Hd = W + 2 * P, H + 2 * P
    lab = np.full((Hd, Wd), -1, dtype=np.int32)
    xs = np.zeros(0, dtype=np.int32)
    ys = np.zeros(0, dtype=np.int32)
    passes = []
    for b in batches:
        b = np.asarray(b, dtype=np.int32).reshape(-1, 2)
        if len(b) == 0:
            continue
        n0 = len(xs)
        xs = np.concatenate([xs, b[:, 0]])
        ys = np.concatenate([ys, b[:, 1]])
        lab[b[:, 1] + P, b[:, 0] + P] = np.arange(n0, n0 + len(b), dtype=np.int32)
        lab, k = jacobi_from(Wd, Hd, xs + P, ys + P, lab)
        passes.append(k)
    n = len(xs)
    order = np.lexsort((ys, xs))
    rank = np.empty(n, dtype=np.int32)
    rank[order] = np.arange(n, dtype=np.int32)
    raw = detect(lab, xs + P, ys + P, P) if n >= 3 else np.zeros((0, 5), np.int32)
    tris = raw.copy()
    if len(raw):
        tris[:, 2:5] = rank[raw[:, 2:5]]
        key = np.sort(tris[:, 2:5], axis=1)
        o = np.lexsort((key[:, 2], key[:, 1], key[:, 0]))
        tris = tris[o]
        raw = raw[o]
    sx, sy = xs[order], ys[order]
    tgrid = assign_bbox(W, H, sx, sy, tris) if n else np.full((H, W), -1, np.int32)
    inner = lab[P:P + H, P:P + W]
    grid = np.empty((H, W, 3), dtype=np.int32)
    ok = inner >= 0
    grid[:, :, 0] = np.where(ok, rank[np.maximum(inner, 0)], -1) if n else -1
    yy, xx = np.mgrid[0:H, 0:W]
    if n:
        d = (xx - xs[np.maximum(inner, 0)]) ** 2 + (yy - ys[np.maximum(inner, 0)]) ** 2
        grid[:, :, 1] = np.where(ok, d, -1)
    else:
        grid[:, :, 1] = -1
    grid[:, :, 2] = tgrid
    return {"rank": rank, "tris": tris, "tris_ins": np.ascontiguousarray(raw[:, 2:5]), "grid": grid,
            "labels": lab, "passes": passes, "xs": xs, "ys": ys}


# ---------------------------------------------------------------------------
# The reference's own CUDA batch path (oracle/_ref/libref_cuda.so, built by
# oracle/build_ref.sh).  Present only where it was built; needs a GPU to run.
# ---------------------------------------------------------------------------
_REF = None
REF_PATH = os.path.join(_HERE, "_ref", "libref_cuda.so")


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def _ref():
    global _REF
    if _REF is None:
        L = ctypes.CDLL(REF_PATH)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_voronoi.restype = ctypes.c_int
        L.ref_voronoi.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, _i32p]
        L.ref_triangulate.restype = ctypes.c_int
        L.ref_triangulate.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_int, _i32p, _i32p, ctypes.c_int64,
                                      ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
        _REF = L
    return _REF


def ref_voronoi(W: int, H: int, sorted_seeds) -> np.ndarray:
    """Reference voronoi.cu run on the GPU: (H, W, 2) int32."""
    s = np.ascontiguousarray(np.asarray(sorted_seeds, dtype=np.int32).reshape(-1, 2))
    out = np.empty((H, W, 2), dtype=np.int32)
    if _ref().ref_voronoi(W, H, s, len(s), out) != 0:
        raise RuntimeError(_ref().ref_last_error().decode())
    return out


def ref_triangulate(W: int, H: int, sorted_seeds, P: int = DEFAULT_BORDER_PADDING, vgrid=None, padded=False):
    """Reference cuda_compute_triangulation on the GPU.

    Returns (tris (N, 5) int32 as the reference numbers them, grid (H, W, 3),
    padded grid or None).  The (x, y) and vertex order of each triangle come
    from whichever duplicate the reference's unstable sort kept.
    """
    s = np.ascontiguousarray(np.asarray(sorted_seeds, dtype=np.int32).reshape(-1, 2))
    out = np.empty((H, W, 3), dtype=np.int32)
    cap = 4 * len(s) + 64
    vg = None if vgrid is None else np.ascontiguousarray(vgrid, dtype=np.int32)
    pad = np.empty((H + 2 * P, W + 2 * P, 2), dtype=np.int32) if (padded and P > 0) else None
    while True:
        tris = np.empty((cap, 5), dtype=np.int32)
        n = ctypes.c_int64(0)
        rc = _ref().ref_triangulate(W, H, s, len(s), vg.ctypes.data if vg is not None else None, int(P), out,
                                    tris, cap, ctypes.byref(n), pad.ctypes.data if pad is not None else None)
        if rc == 2:
            cap = int(n.value)
            continue
        if rc != 0:
            raise RuntimeError(_ref().ref_last_error().decode())
        return tris[:n.value].copy(), out, pad


def _ref_dl_lib():
    L = _ref()
    if not getattr(L, "_idl_dl_bound", False):
        vp = ctypes.c_void_p
        L.ref_dl_create.restype = vp
        L.ref_dl_create.argtypes = [ctypes.c_int] * 4
        L.ref_dl_destroy.restype = None
        L.ref_dl_destroy.argtypes = [vp]
        L.ref_dl_seed_count.restype = ctypes.c_int
        L.ref_dl_seed_count.argtypes = [vp]
        L.ref_dl_insert_deferred.restype = ctypes.c_int
        L.ref_dl_insert_deferred.argtypes = [vp, _i32p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.ref_dl_finalise.restype = ctypes.c_int
        L.ref_dl_finalise.argtypes = [vp, _i32p, _i32p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        L.ref_dl_voronoi_grid.restype = ctypes.c_int
        L.ref_dl_voronoi_grid.argtypes = [vp, _i32p]
        L.ref_dl_triangles.restype = ctypes.c_int
        L.ref_dl_triangles.argtypes = [vp, _i32p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        L.ref_dl_sorted_rank.restype = ctypes.c_int
        L.ref_dl_sorted_rank.argtypes = [vp, _i32p]
        L._idl_dl_bound = True
    return L


class RefDelaunay:
    """The reference's own incremental ``Delaunay`` class (src/cuda/delaunay.cuh),
    run on the GPU through oracle/_ref/libref_cuda.so.

    Seeds are passed in insertion order, exactly as the reference binding
    (src/cuda/bindings/py_delaunay.hpp) hands them to ``insert_deferred``.
    """

    def __init__(self, W: int, H: int, max_seeds: int, P: int = DEFAULT_BORDER_PADDING):
        self.W, self.H = int(W), int(H)
        self._L = _ref_dl_lib()
        self._h = self._L.ref_dl_create(self.W, self.H, int(max_seeds), int(P))
        if not self._h:
            raise RuntimeError(self._L.ref_last_error().decode())

    def close(self):
        if self._h:
            self._L.ref_dl_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, rc):
        if rc == 1:
            raise RuntimeError(self._L.ref_last_error().decode())
        return rc

    @property
    def seed_count(self) -> int:
        return int(self._L.ref_dl_seed_count(self._h))

    def insert_deferred(self, seeds) -> int:
        """Returns the Jacobi passes the reference ran for this batch."""
        s = np.ascontiguousarray(np.asarray(seeds, dtype=np.int32).reshape(-1, 2))
        it = ctypes.c_int(0)
        self._check(self._L.ref_dl_insert_deferred(self._h, s, len(s), ctypes.byref(it)))
        return int(it.value)

    def _tris(self, fn, *head):
        cap = 4 * max(self.seed_count, 1) + 64
        while True:
            out = np.empty((cap, 5), dtype=np.int32)
            n = ctypes.c_int64(0)
            rc = self._check(fn(self._h, *head, out, cap, ctypes.byref(n)))
            if rc == 2:
                cap = int(n.value)
                continue
            return out[:n.value].copy()

    def finalise(self):
        """(tris (N_tri, 5) int32 in the reference's slot order, grid (H, W, 3))."""
        grid = np.empty((self.H, self.W, 3), dtype=np.int32)
        tris = self._tris(self._L.ref_dl_finalise, grid)
        return tris, grid

    def insert(self, seeds):
        self.insert_deferred(seeds)
        return self.finalise()

    def get_voronoi_grid(self) -> np.ndarray:
        out = np.empty((self.H, self.W, 2), dtype=np.int32)
        self._check(self._L.ref_dl_voronoi_grid(self._h, out))
        return out

    def get_triangles(self) -> np.ndarray:
        """(N_tri, 5): canonical (x, y) in image coordinates and insertion ids."""
        return self._tris(self._L.ref_dl_triangles)

    @property
    def sorted_rank(self) -> np.ndarray:
        out = np.empty(self.seed_count, dtype=np.int32)
        self._check(self._L.ref_dl_sorted_rank(self._h, out))
        return out


def ref_triangulate_stock(W: int, H: int, seeds, P: int = DEFAULT_BORDER_PADDING):
    """The reference's stock triangulate() on the GPU: host validation and
    (x, y) sort, then cuda_compute_triangulation building its own padded
    diagram (src/cuda/bindings/triangulate.hpp:15-43).  Seeds in caller order.
    Returns (tris (N, 5) int32, grid (H, W, 3) int32)."""
    L = _ref()
    if not getattr(L, "_idl_stock_bound", False):
        L.ref_triangulate_stock.restype = ctypes.c_int
        L.ref_triangulate_stock.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int,
                                            _i32p, _i32p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        L._idl_stock_bound = True
    s = np.ascontiguousarray(np.asarray(seeds, dtype=np.int32).reshape(-1, 2))
    out = np.empty((H, W, 3), dtype=np.int32)
    cap = 4 * len(s) + 64
    while True:
        tris = np.empty((cap, 5), dtype=np.int32)
        n = ctypes.c_int64(0)
        rc = L.ref_triangulate_stock(W, H, s, len(s), int(P), out, tris, cap, ctypes.byref(n))
        if rc == 2:
            cap = int(n.value)
            continue
        if rc != 0:
            raise RuntimeError(L.ref_last_error().decode())
        return tris[:n.value].copy(), out
