"""Serving: a request loop over diagrams kept resident on one GPU.

Two kinds of request arrive at any time:
  * ``new``    -- triangulate W x H with a seed set and keep the diagram
                  resident (an incremental ``Delaunay`` whose seeds are
                  inserted in (x, y) order, so its grid and triangles equal
                  ``triangulate(W, H, seeds)`` bit for bit);
  * ``insert`` -- add a batch of seeds to a resident diagram and bring its
                  triangles and pixel arrays up to date.

The loop itself is native (csrc/server.cu, idl_server_* in the C ABI): worker
threads with a CUDA stream each, continuous batching (a request that cannot
run yet -- its diagram busy, its memory not free -- is passed over for later
ones), queued new diagrams propagated several per launch, admission against a
device-memory budget with least-recently-used eviction into a pool of objects
that are recycled instead of freed (the policy is csrc/scheduler.h).  This
module is the Python face of it: ``Server.submit_*`` is one C call that copies
the seeds and returns at once; ``Ticket.result()`` is one call that waits.
No Python runs while requests execute.

Results are identical whether a request runs alone or in the mix: each
diagram's work runs on one stream at a time, in the order its requests were
submitted, and no kernel reads another diagram's memory.
"""
from __future__ import annotations

import collections
import ctypes
import threading
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _capi

SIZE_CLASS = 128            # object canvases are rounded up to multiples of this
SEED_HEADROOM = 50_000      # seed capacity beyond the initial set, for inserts
GROUP_MAX = 16              # new diagrams propagated together in one launch, at most


@dataclass
class Result:
    request_id: int
    kind: str
    diagram_id: int
    n_seeds: int
    n_triangles: int
    arrival: float          # seconds on the time.monotonic() clock
    start: float
    done: float
    verts: Optional[np.ndarray] = None     # (N_tri, 3) batch seed ids, when fetched
    grid: Optional[np.ndarray] = None      # (H, W, 3), when fetched

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def _class_dims(width: int, height: int):
    r = lambda v: (int(v) + SIZE_CLASS - 1) // SIZE_CLASS * SIZE_CLASS
    return r(width), r(height)


def estimate_bytes(width: int, height: int, max_seeds: int, padding: int, workspace: bool = True) -> int:
    """Device footprint of a diagram: label planes, padded raster, pixel
    outputs and seed arrays, plus (``workspace``) the scratch a triangulation
    of it grows (micro-tile lists and bitmaps, hash table, triangle rows).
    Without the workspace this is what the server charges for a fresh object
    (capacity() of csrc/scheduler.h)."""
    Wd, Hd = width + 2 * padding, height + 2 * padding
    pitch = (Wd + 31) // 32 * 32
    fixed = pitch * Hd * 8 + Wd * Hd * 4 + width * height * 9 + max_seeds * 32
    if not workspace:
        return int(fixed)
    n_mt = ((Wd + 7) // 8) * ((Hd + 7) // 8)
    hash_cap = 1 << max(10, int(8 * max_seeds + 1024 - 1).bit_length())
    work = (n_mt * 8 + n_mt // 4 + 16 * (Wd + Hd) + 56 * hash_cap + 48 * max_seeds + Wd * Hd // 8 +
            3 * ((Wd + 127) // 32 + 1) * 4 * Hd)
    return int(fixed + work)


#: Largest request the server's slot workspaces are reserved for.
MAX_SIDE = 4096
MAX_REQUEST_SEEDS = 200_000


def slot_reserve(padding: int) -> int:
    """Budget the server reserves per worker slot (slot_reserve() of
    csrc/scheduler.h): a diagram workspace, and a batch context triangulating
    a full group (one atlas of MAX_SIDE^2 padded: label planes, raster,
    composed grids, seed arrays)."""
    Wd = Hd = MAX_SIDE + 2 * padding
    pitch = (Wd + 31) // 32 * 32
    scratch = (estimate_bytes(MAX_SIDE, MAX_SIDE, MAX_REQUEST_SEEDS, padding) -
               estimate_bytes(MAX_SIDE, MAX_SIDE, MAX_REQUEST_SEEDS, padding, workspace=False))
    return 2 * scratch + pitch * Hd * 8 + MAX_SIDE * MAX_SIDE * 16 + 32 * MAX_REQUEST_SEEDS


_KIND = {0: "new", 1: "insert"}


class Ticket:
    """A submitted request.  ``diagram_id`` is usable for inserts at once;
    ``result()`` waits for the request and returns its ``Result`` or raises
    its error (MemoryError: never fits the budget; KeyError: diagram not
    resident; ValueError: invalid input; RuntimeError: CUDA failure)."""

    def __init__(self, server: "Server", request_id: int, diagram_id: int, fetch: bool,
                 grid: Optional[np.ndarray]):
        self._srv = server
        self.request_id = request_id
        self.diagram_id = diagram_id
        self._fetch = fetch
        self._grid = grid
        self._res: Optional[Result] = None
        self._exc: Optional[BaseException] = None
        self._collected = False

    def _collect(self, timeout: Optional[float]) -> None:
        if self._collected:
            return
        lib, h = self._srv._lib, self._srv._handle()
        t = -1.0 if timeout is None else float(timeout)
        row = (ctypes.c_int64 * _capi.SR_COUNT)()
        tris = np.empty((0, 5), np.int32)
        if self._fetch:
            probe = ctypes.c_int32(0)     # capacity 0: learn the triangle count, leave the request in place
            st = lib.idl_server_wait(h, self.request_id, t, row, ctypes.addressof(probe), 0)
            if st == _capi.IDL_ERR_INVALID and row[_capi.SR_STATUS] == _capi.IDL_OK and \
                    row[_capi.SR_TRIANGLES] > 0:
                tris = np.empty((row[_capi.SR_TRIANGLES], 5), np.int32)
                st = lib.idl_server_wait(h, self.request_id, t, row, tris.ctypes.data, tris.size)
        else:
            st = lib.idl_server_wait(h, self.request_id, t, row, None, 0)
        if st == _capi.IDL_ERR_STATE and "timeout" in _capi.last_error():
            raise TimeoutError(_capi.last_error())
        self._collected = True
        try:
            _capi.check(st)
        except BaseException as e:   # noqa: BLE001 - kept for result()/exception()
            self._exc = e
            self._grid = None
            return
        ns = 1e-9
        self._res = Result(self.request_id, _KIND[int(row[_capi.SR_KIND])], int(row[_capi.SR_DIAGRAM]),
                           int(row[_capi.SR_SEEDS]), int(row[_capi.SR_TRIANGLES]), row[_capi.SR_ARRIVAL_NS] * ns,
                           row[_capi.SR_START_NS] * ns, row[_capi.SR_DONE_NS] * ns,
                           np.ascontiguousarray(tris[:, 2:5]) if self._fetch else None, self._grid)
        self._grid = None

    def result(self, timeout: Optional[float] = None) -> Result:
        self._collect(timeout)
        if self._exc is not None:
            raise self._exc
        return self._res

    def exception(self, timeout: Optional[float] = None) -> Optional[BaseException]:
        self._collect(timeout)
        return self._exc

    def done(self) -> bool:
        if not self._collected:
            try:
                self._collect(0.0)
            except TimeoutError:
                return False
        return True


class Server:
    """Native continuous-batching request loop on one GPU (module docstring).

    ``arrival`` (submit_*): the request's arrival in seconds of
    time.monotonic(), for latency accounting when requests are replayed on a
    schedule; default now."""

    def __init__(self, device: Optional[int] = None, budget_bytes: int = 40 << 30, slots: int = 4,
                 border_padding: int = _capi.AUTO_BORDER_PADDING, mode: str = "reference"):
        import torch
        from . import _delauney_cuda as cu
        self._cu = cu
        self._lib = _capi.load()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.budget = int(budget_bytes)
        self.padding = cu.resolve_padding(border_padding)
        self._dims: dict[int, tuple] = {}       # diagram id -> (W, H), for fetched inserts
        self._dims_lock = threading.Lock()
        self._news = 0
        h = ctypes.c_void_p()
        _capi.check(self._lib.idl_server_create(self.device, self.budget, int(slots), self.padding,
                                                _capi.mode_id(mode), ctypes.byref(h)))
        self._h = h.value

    def set_tile(self, shape: int) -> None:
        """Tile shape (Context.set_tile) of the grouped new diagrams'
        propagation; set before the first request (idl_server_set_tile)."""
        _capi.check(self._lib.idl_server_set_tile(self._handle(), int(shape)))

    def set_schedule(self, group_rounds: int, insert_rounds: int) -> None:
        """Propagation schedules (Context.set_schedule) of the grouped new
        diagrams and of inserts (-1 for inserts: tile rounds from the new
        seeds' tiles, no device-wide persistent kernel).  Before the first
        request."""
        _capi.check(self._lib.idl_server_set_schedule(self._handle(), int(group_rounds), int(insert_rounds)))

    def _handle(self) -> int:
        if self._h is None:
            raise RuntimeError("server is closed")
        return self._h

    @staticmethod
    def _arrival_ns(arrival: Optional[float]) -> int:
        return 0 if arrival is None else int(round(arrival * 1e9))

    # -- public API --------------------------------------------------------
    def submit_new(self, width: int, height: int, seeds, fetch: bool = False,
                   arrival: Optional[float] = None) -> Ticket:
        s = self._cu.parse_seeds(seeds)
        grid = np.empty((int(height), int(width), 3), np.int32) if fetch else None
        rid, did = ctypes.c_int64(), ctypes.c_int64()
        _capi.check(self._lib.idl_server_submit_new(
            self._handle(), int(width), int(height), s.ctypes.data if len(s) else None, len(s), int(fetch),
            grid.ctypes.data if fetch else None, self._arrival_ns(arrival), ctypes.byref(rid), ctypes.byref(did)))
        with self._dims_lock:
            self._dims[did.value] = (int(width), int(height))
            self._news += 1
            prune = self._news % 4096 == 0
        if prune:                               # forget diagrams the server no longer holds
            live = set(self.resident())
            with self._dims_lock:
                self._dims = {k: v for k, v in self._dims.items() if k in live or k >= did.value}
        return Ticket(self, rid.value, did.value, fetch, grid)

    def submit_insert(self, diagram_id: int, seeds, fetch: bool = False,
                      arrival: Optional[float] = None) -> Ticket:
        """Raises KeyError at once if the diagram is not resident."""
        s = self._cu.parse_seeds(seeds)
        grid = None
        if fetch:
            with self._dims_lock:
                dims = self._dims.get(diagram_id)
            if dims is None:
                raise KeyError(f"diagram {diagram_id} is not resident")
            W, H = dims
            grid = np.empty((H, W, 3), np.int32)
        rid = ctypes.c_int64()
        _capi.check(self._lib.idl_server_submit_insert(
            self._handle(), int(diagram_id), s.ctypes.data if len(s) else None, len(s), int(fetch),
            grid.ctypes.data if fetch else None, self._arrival_ns(arrival), ctypes.byref(rid)))
        return Ticket(self, rid.value, int(diagram_id), fetch, grid)

    def resident(self) -> list[int]:
        """Ids of the diagrams currently resident (created, not evicted), and
        of those whose creation is queued."""
        n = ctypes.c_int64(0)
        _capi.check(self._lib.idl_server_resident(self._handle(), None, 0, ctypes.byref(n)))
        ids = np.empty(max(1, n.value + 64), np.int64)
        _capi.check(self._lib.idl_server_resident(self._handle(), ids.ctypes.data_as(_capi._pi64), len(ids),
                                                  ctypes.byref(n)))
        return ids[:min(n.value, len(ids))].tolist()

    def info(self) -> dict:
        v = (ctypes.c_int64 * _capi.SI_COUNT)()
        _capi.check(self._lib.idl_server_info(self._handle(), v, _capi.SI_COUNT))
        keys = ("used_bytes", "budget_bytes", "resident", "pooled", "queued", "groups", "grouped_requests",
                "new_objects", "reused_objects", "evicted", "freed_objects")
        return dict(zip(keys, (int(x) for x in v)))

    @property
    def stats(self) -> collections.Counter:
        i = self.info()
        return collections.Counter({k: i[k] for k in ("groups", "grouped_requests", "new_objects",
                                                      "reused_objects", "evicted", "freed_objects")})

    def memory_used(self) -> int:
        return self.info()["used_bytes"]

    def drain(self) -> None:
        """Wait until every submitted request has finished."""
        _capi.check(self._lib.idl_server_drain(self._handle()))

    def recycle(self, diagram_id: int) -> bool:
        """Retire an idle diagram now, keeping its object for reuse."""
        ok = ctypes.c_int(0)
        _capi.check(self._lib.idl_server_recycle(self._handle(), int(diagram_id), ctypes.byref(ok)))
        if ok.value:
            with self._dims_lock:
                self._dims.pop(int(diagram_id), None)
        return bool(ok.value)

    @staticmethod
    def clock() -> float:
        """The server's clock (time.monotonic() on Linux), in seconds."""
        return _capi.load().idl_server_clock_ns() * 1e-9

    def close(self) -> None:
        """Run what is queued, stop the workers and free every object."""
        if self._h is not None:
            h, self._h = self._h, None
            _capi.check(self._lib.idl_server_destroy(h))

    def __del__(self):
        try:
            self.close()
        except Exception:   # noqa: BLE001 - interpreter teardown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_serial(requests, border_padding: int = _capi.AUTO_BORDER_PADDING, budget_bytes: int = 40 << 30):
    """The plain loop the server is measured against: the same requests, one
    at a time on the current stream, each diagram a fresh ``Delaunay`` (freed
    oldest-first when the budget is exceeded), a result read back per request.

    ``requests``: iterable of ("new", width, height, seeds) or
    ("insert", index_of_new_request, seeds).  Returns per-request
    (n_seeds, n_triangles)."""
    from . import _delauney_cuda as cu
    P = cu.resolve_padding(border_padding)
    live: "collections.OrderedDict[int, tuple]" = collections.OrderedDict()
    used = 0
    out = []
    for i, r in enumerate(requests):
        if r[0] == "new":
            _, w, h, s = r
            s = cu.parse_seeds(s)
            cap = len(s) + SEED_HEADROOM
            need = estimate_bytes(w, h, cap, P)
            while live and used + need > budget_bytes:
                _, (o, b) = live.popitem(last=False)
                used -= b
                del o
            obj = cu.Delaunay(w, h, cap, P)
            obj.insert_deferred(s, order="xy")
            live[i] = (obj, need)
            used += need
            out.append((len(s), obj._finalise_device_count()))
        else:
            _, j, s = r
            if j not in live:
                out.append((0, -1))
                continue
            obj = live[j][0]
            live.move_to_end(j)
            obj.insert_deferred(s)
            out.append((obj.seed_count, obj._finalise_device_count()))
    return out
