"""ctypes binding of the C ABI in include/idelaunay.h.

Loads the in-tree libidelaunay.so.  There is no fallback: if the library is
missing, importing anything that needs it raises ImportError naming the build
command, the same way ``from delauney import _delauney_cuda`` fails when the
reference's extension was not built.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libidelaunay.so")

IDL_OK = 0
IDL_ERR_INVALID = 1
IDL_ERR_CUDA = 2
IDL_ERR_STATE = 3
IDL_ERR_INTERNAL = 4
IDL_ERR_BUDGET = 5
IDL_ERR_NOT_RESIDENT = 6

MODE_REFERENCE = 0
MODE_NUMPY = 1
MODE_EXACT = 2
MODES = {"reference": MODE_REFERENCE, "numpy": MODE_NUMPY, "exact": MODE_EXACT}

AUTO_BORDER_PADDING = -1
DEFAULT_BORDER_PADDING = 16

T_DETECT_MS, T_DEDUP_MS, T_ASSIGN_MS, T_BFS_MS, T_BFS_ITERS, T_COUNT = range(6)

_vp = ctypes.c_void_p
_i32 = ctypes.c_int
_i64 = ctypes.c_int64
_pi64 = ctypes.POINTER(ctypes.c_int64)

# name -> (restype, argtypes); every declaration of include/idelaunay.h
SIGNATURES = {
    "idl_last_error": (ctypes.c_char_p, []),
    "idl_version": (_i32, []),
    "idl_launch_count": (ctypes.c_longlong, []),
    "idl_alloc_count": (ctypes.c_longlong, []),
    "idl_selftest_grid_barrier": (_i32, [_vp, _i32, ctypes.c_uint]),
    "idl_context_create": (_i32, [_i32, ctypes.POINTER(_vp)]),
    "idl_context_destroy": (_i32, [_vp]),
    "idl_context_set_stream": (_i32, [_vp, _vp]),
    "idl_context_synchronize": (_i32, [_vp]),
    "idl_context_set_schedule": (_i32, [_vp, _i32]),
    "idl_context_set_tile": (_i32, [_vp, _i32, ctypes.POINTER(_i32)]),
    "idl_context_pass_trace": (_i32, [_vp, _vp, _vp, _vp, _i32, ctypes.POINTER(_i32)]),
    "idl_context_set_tail_rounds": (_i32, [_vp, _i32]),
    "idl_context_workspace_bytes": (_i32, [_vp, _pi64]),
    "idl_context_set_profiling": (_i32, [_vp, _i32]),
    "idl_context_last_profile": (_i32, [_vp, ctypes.POINTER(ctypes.c_double), _i32]),
    "idl_voronoi": (_i32, [_vp, _i32, _i32, _vp, _i64, _i32, _vp, _pi64]),
    "idl_triangulate": (_i32, [_vp, _i32, _i32, _vp, _i64, _vp, _i32, _i32, _vp, _pi64, _vp, _vp]),
    "idl_get_triangles": (_i32, [_vp, _vp, _i64]),
    "idl_get_triangle_vertices": (_i32, [_vp, _vp, _i64]),
    "idl_triangulate_device": (_i32, [_vp, _i32, _i32, _vp, _i64, _i32, _i32, _vp, _pi64]),
    "idl_triangles_device": (_i32, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "idl_voronoi_noalloc": (_i32, [_i32, _i32, _vp, _i64, _i32, _vp, _vp, _pi64]),
    # batched triangulation
    "idl_triangulate_batch": (_i32, [_vp, _i32, _vp, _vp, _vp, _i32, _i32, _vp, _vp, _vp]),
    "idl_triangulate_batch_device": (_i32, [_vp, _i32, _vp, _vp, _vp, _i32, _i32, _vp, _vp]),
    "idl_voronoi_batch": (_i32, [_vp, _i32, _vp, _vp, _vp, _i32, _i32]),
    # incremental triangulation
    "idl_delaunay_create": (_i32, [_i32, _i32, _i32, _i64, _i32, _i32, ctypes.POINTER(_vp)]),
    "idl_delaunay_destroy": (_i32, [_vp]),
    "idl_delaunay_reset": (_i32, [_vp, _i32, _i32, _i64, _i32]),
    "idl_delaunay_set_workspace": (_i32, [_vp, _vp]),
    "idl_delaunay_adopt_group": (_i32, [_vp, _vp, _i32, _vp]),
    "idl_delaunay_adopt": (_i32, [_vp, _vp, _i32]),
    "idl_delaunay_set_stream": (_i32, [_vp, _vp]),
    "idl_delaunay_insert": (_i32, [_vp, _vp, _i64, _vp, _vp]),
    "idl_delaunay_insert_ordered": (_i32, [_vp, _vp, _i64, _vp, _i32, _vp]),
    "idl_delaunay_finalise": (_i32, [_vp, _vp, _pi64, _vp]),
    "idl_delaunay_finalise_device": (_i32, [_vp, _pi64, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                            ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_uint64)]),
    "idl_delaunay_triangles": (_i32, [_vp, _i32, _vp, _i64, _pi64]),
    "idl_delaunay_edges": (_i32, [_vp, _vp, _i64, _pi64]),
    "idl_delaunay_edge_scores": (_i32, [_vp, ctypes.c_double, _vp, _i64, _pi64]),
    "idl_delaunay_select_midpoints": (_i32, [_vp, ctypes.c_double, _i32, ctypes.c_float, _vp, _i64, _pi64]),
    "idl_delaunay_locate": (_i32, [_vp, _vp, _i64, _vp]),
    "idl_delaunay_in_circumsphere": (_i32, [_vp, _vp, _vp, _i64, _vp, _vp]),
    "idl_delaunay_seeds": (_i32, [_vp, _vp, _vp, _pi64]),
    "idl_delaunay_sorted_rank": (_i32, [_vp, _vp]),
    "idl_delaunay_voronoi": (_i32, [_vp, _vp]),
    "idl_delaunay_info": (_i32, [_vp, _pi64, _i32]),
    # serving
    "idl_server_clock_ns": (_i64, []),
    "idl_server_create": (_i32, [_i32, _i64, _i32, _i32, _i32, ctypes.POINTER(_vp)]),
    "idl_server_destroy": (_i32, [_vp]),
    "idl_server_set_schedule": (_i32, [_vp, _i32, _i32]),
    "idl_server_set_tile": (_i32, [_vp, _i32]),
    "idl_server_submit_new": (_i32, [_vp, _i32, _i32, _vp, _i64, _i32, _vp, _i64, _pi64, _pi64]),
    "idl_server_submit_insert": (_i32, [_vp, _i64, _vp, _i64, _i32, _vp, _i64, _pi64]),
    "idl_server_wait": (_i32, [_vp, _i64, ctypes.c_double, _pi64, _vp, _i64]),
    "idl_server_drain": (_i32, [_vp]),
    "idl_server_recycle": (_i32, [_vp, _i64, ctypes.POINTER(_i32)]),
    "idl_server_info": (_i32, [_vp, _pi64, _i32]),
    "idl_server_resident": (_i32, [_vp, _pi64, _i64, _pi64]),
}

# idl_server_wait result row and idl_server_info slots
(SR_STATUS, SR_KIND, SR_DIAGRAM, SR_SEEDS, SR_TRIANGLES, SR_ARRIVAL_NS, SR_START_NS, SR_DONE_NS, SR_COUNT) = range(9)
(SI_USED_BYTES, SI_BUDGET_BYTES, SI_RESIDENT, SI_POOLED, SI_QUEUED, SI_GROUPS, SI_GROUPED, SI_NEW_OBJECTS,
 SI_REUSED_OBJECTS, SI_EVICTED, SI_FREED_OBJECTS, SI_COUNT) = range(12)

# idl_delaunay_info slots
(DI_SEED_COUNT, DI_WIDTH, DI_HEIGHT, DI_BORDER_PADDING, DI_HAS_PENDING, DI_GENERATION, DI_MAX_SEEDS, DI_MODE,
 DI_HAS_VALUES, DI_DEVICE_BYTES, DI_COUNT) = range(11)

_lib = None
_lib_lock = threading.Lock()


def load():
    """Load libidelaunay.so (once) and declare every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run `python -m integer_delauney_b200.build` "
                "(nvcc, sm_100a) first")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().idl_last_error()
    return msg.decode(errors="replace") if msg else ""


def check(status: int) -> None:
    """Map a status code to the reference's exception types."""
    if status == IDL_OK:
        return
    msg = last_error()
    if status == IDL_ERR_INVALID:
        raise ValueError(msg)
    if status == IDL_ERR_BUDGET:
        raise MemoryError(msg)
    if status == IDL_ERR_NOT_RESIDENT:
        raise KeyError(msg)
    raise RuntimeError(msg)


def mode_id(mode) -> int:
    if isinstance(mode, str):
        try:
            return MODES[mode]
        except KeyError:
            raise ValueError(f"voronoi_mode must be one of {sorted(MODES)}, not {mode!r}") from None
    return int(mode)


def ptr(a) -> int | None:
    """Raw data pointer of a numpy array or torch tensor (None for None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


class Context:
    """One idl_context: a device, a stream and the grow-only workspace."""

    def __init__(self, device: int = -1):
        self._lib = load()
        h = _vp()
        check(self._lib.idl_context_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.lock = threading.RLock()

    def set_stream(self, stream_handle: int | None) -> None:
        check(self._lib.idl_context_set_stream(self.handle, _vp(stream_handle or 0)))

    def synchronize(self) -> None:
        check(self._lib.idl_context_synchronize(self.handle))

    def set_schedule(self, dense_rounds: int) -> None:
        """Propagation schedule from scratch (idl_context_set_schedule)."""
        check(self._lib.idl_context_set_schedule(self.handle, int(dense_rounds)))

    def set_tile(self, shape: int) -> int:
        """Tile shape of the tile rounds (idl_context_set_tile); returns the number of shapes."""
        n = _i32(0)
        check(self._lib.idl_context_set_tile(self.handle, int(shape), ctypes.byref(n)))
        return int(n.value)

    def set_profiling(self, enable: bool) -> None:
        check(self._lib.idl_context_set_profiling(self.handle, 1 if enable else 0))

    PROFILE_KEYS = ("seeds_ms", "propagate_ms", "detect_ms", "dedup_ms", "assign_ms", "compose_ms", "rounds",
                    "tiles", "passes", "tile_w", "tile_h", "steps_per_round", "canvas_px", "image_px",
                    "n_triangles", "prop_bytes")

    def last_profile(self) -> dict:
        buf = (ctypes.c_double * len(self.PROFILE_KEYS))()
        check(self._lib.idl_context_last_profile(self.handle, buf, len(self.PROFILE_KEYS)))
        return {k: float(buf[i]) for i, k in enumerate(self.PROFILE_KEYS)}

    def pass_trace(self) -> list[tuple[int, float, int]]:
        """(work-list micro-tiles, microseconds, passes advanced) of each
        work-list generation of the persistent kernel in the last profiled run
        (idl_context_pass_trace)."""
        n = _i32(0)
        check(self._lib.idl_context_pass_trace(self.handle, None, None, None, 0, ctypes.byref(n)))
        ns = np.zeros(n.value, dtype=np.int64)
        tiles = np.zeros(n.value, dtype=np.int32)
        steps = np.zeros(n.value, dtype=np.int32)
        check(self._lib.idl_context_pass_trace(self.handle, ns.ctypes.data, tiles.ctypes.data, steps.ctypes.data,
                                               n.value, ctypes.byref(n)))
        return [(int(t), round(float(v) / 1e3, 2), int(k)) for t, v, k in zip(tiles, ns, steps)]

    def set_tail_rounds(self, max_list: int) -> None:
        """Work-list length at or below which the persistent kernel advances a
        round of passes per barrier (idl_context_set_tail_rounds; 0 = never)."""
        check(self._lib.idl_context_set_tail_rounds(self.handle, int(max_list)))

    def workspace_bytes(self) -> int:
        v = ctypes.c_int64(0)
        check(self._lib.idl_context_workspace_bytes(self.handle, ctypes.byref(v)))
        return int(v.value)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.idl_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts: dict[int, Context] = {}
_ctx_lock = threading.Lock()


def context_for(device: int) -> Context:
    with _ctx_lock:
        c = _contexts.get(device)
        if c is None:
            c = Context(device)
            _contexts[device] = c
        return c
