"""Serving: a request loop over diagrams kept resident on one GPU.

Two kinds of request arrive at any time:
  * ``new``    -- triangulate W x H with a seed set and keep the diagram
                  resident (an incremental ``Delaunay`` whose seeds are
                  inserted in (x, y) order, so its grid and triangles equal
                  ``triangulate(W, H, seeds)`` bit for bit);
  * ``insert`` -- add a batch of seeds to a resident diagram and bring its
                  triangles and pixel arrays up to date.

Continuous batching.  ``slots`` worker threads each own a CUDA stream.  A
request is admitted as soon as a slot is free and its memory fits the device
budget: a request that cannot be admitted (its diagram is busy, or its memory
does not fit yet) is passed over for later ones instead of blocking the queue,
so work from many requests is on the device at once.  The C ABI releases the
GIL for the whole of every call, so slots overlap their host work too.

Memory.  Every resident diagram, and every idle object kept for reuse, is
charged to ``budget_bytes`` with its real device footprint; so is each slot's
scratch workspace (hash table, work lists, triangle rows), which all the
diagrams a slot runs share and which is reserved for the largest request.  Objects are
allocated in size classes and recycled (``Delaunay.reset``) when diagrams are
evicted, so a steady stream of requests allocates and frees almost nothing;
eviction takes the least recently used idle diagram.  A request whose own
footprint exceeds the budget fails with ``MemoryError``.

Results are identical whether a request runs alone or in the mix: each
diagram's work runs on one stream at a time, in the order its requests were
submitted, and no kernel reads another diagram's memory.
"""
from __future__ import annotations

import collections
import ctypes
import itertools
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
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
    arrival: float
    start: float
    done: float
    verts: Optional[np.ndarray] = None     # (N_tri, 3) batch seed ids, when fetched
    grid: Optional[np.ndarray] = None      # (H, W, 3), when fetched

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class _Request:
    rid: int
    kind: str
    arrival: float
    future: Future
    diagram_id: int
    width: int = 0
    height: int = 0
    seeds: Optional[np.ndarray] = None
    fetch: bool = False
    need: int = 0


@dataclass
class _Diagram:
    did: int
    obj: object = None
    bytes: int = 0
    busy: bool = False
    pins: int = 0
    last_used: float = 0.0
    cap: tuple = ()
    n_seeds: int = 0


@dataclass
class _Pooled:
    obj: object
    bytes: int
    cap: tuple = field(default_factory=tuple)


def _class_dims(width: int, height: int):
    r = lambda v: (int(v) + SIZE_CLASS - 1) // SIZE_CLASS * SIZE_CLASS
    return r(width), r(height)


def _capacity(width: int, height: int, max_seeds: int, padding: int) -> tuple:
    """The four allocations of a Delaunay object created for this canvas:
    label planes, padded raster, pixel outputs (bytes) and seed slots."""
    Wd, Hd = width + 2 * padding, height + 2 * padding
    return ((Wd + 31) // 32 * 32 * Hd * 8, Wd * Hd * 4, width * height * 9, max_seeds)


def _fits(cap: tuple, width: int, height: int, max_seeds: int, padding: int) -> bool:
    """Whether an object with allocations `cap` can be reset to this canvas
    (the rule of idl_delaunay_reset: areas, not sides, must fit)."""
    need = _capacity(width, height, max_seeds, padding)
    return all(n <= c for n, c in zip(need, cap))


def estimate_bytes(width: int, height: int, max_seeds: int, padding: int, workspace: bool = True) -> int:
    """Device footprint of a diagram: label planes, padded raster, pixel
    outputs and seed arrays, plus (``workspace``) the scratch a triangulation
    of it grows (micro-tile lists and bitmaps, hash table, triangle rows)."""
    Wd, Hd = width + 2 * padding, height + 2 * padding
    pitch = (Wd + 31) // 32 * 32
    fixed = pitch * Hd * 8 + Wd * Hd * 4 + width * height * 9 + max_seeds * 32
    if not workspace:
        return int(fixed)
    n_mt = ((Wd + 7) // 8) * ((Hd + 7) // 8)
    hash_cap = 1 << max(10, int(8 * max_seeds + 1024 - 1).bit_length())
    work = n_mt * 8 + n_mt // 4 + 16 * (Wd + Hd) + 32 * hash_cap + 48 * max_seeds + Wd * Hd // 8
    return int(fixed + work)


#: Largest request the server's slot workspaces are reserved for.
MAX_SIDE = 4096
MAX_REQUEST_SEEDS = 200_000


def slot_reserve(padding: int) -> int:
    """Budget reserved per server slot for its shared scratch workspace."""
    return (estimate_bytes(MAX_SIDE, MAX_SIDE, MAX_REQUEST_SEEDS, padding) -
            estimate_bytes(MAX_SIDE, MAX_SIDE, MAX_REQUEST_SEEDS, padding, workspace=False))


class Server:
    """Continuous-batching request loop on one GPU (see the module docstring)."""

    def __init__(self, device: Optional[int] = None, budget_bytes: int = 40 << 30, slots: int = 4,
                 border_padding: int = _capi.AUTO_BORDER_PADDING):
        import torch
        from . import _delauney_cuda as cu
        self._torch = torch
        self._cu = cu
        self._lib = _capi.load()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.budget = int(budget_bytes)
        self.padding = cu.resolve_padding(border_padding)
        self._cv = threading.Condition()
        self._queue: collections.deque[_Request] = collections.deque()
        self._diagrams: dict[int, _Diagram] = {}
        self._pool: list[_Pooled] = []
        # each slot: a workspace for diagrams and one for its grouped propagations
        self._used = 2 * max(1, int(slots)) * slot_reserve(self.padding)
        self._ids = itertools.count()
        self._dids = itertools.count()
        self._closed = False
        self.stats = collections.Counter()
        self._threads = [threading.Thread(target=self._worker, name=f"idl-slot-{i}", daemon=True)
                         for i in range(max(1, int(slots)))]
        for t in self._threads:
            t.start()

    # -- public API --------------------------------------------------------
    def submit_new(self, width: int, height: int, seeds, fetch: bool = False,
                   arrival: Optional[float] = None) -> Future:
        """Queue a new diagram; the returned future carries ``diagram_id``
        (usable for inserts at once) and resolves to a ``Result``."""
        s = self._cu.parse_seeds(seeds)
        did = next(self._dids)
        cap = len(s) + SEED_HEADROOM
        need = estimate_bytes(*_class_dims(width, height), cap, self.padding, workspace=False)
        fut: Future = Future()
        req = _Request(next(self._ids), "new", time.perf_counter() if arrival is None else arrival, fut, did,
                       int(width), int(height), s, fetch, need)
        fut.diagram_id = did
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            self._diagrams[did] = _Diagram(did, pins=1)
            self._queue.append(req)
            self._cv.notify()
        return fut

    def submit_insert(self, diagram_id: int, seeds, fetch: bool = False,
                      arrival: Optional[float] = None) -> Future:
        s = self._cu.parse_seeds(seeds)
        fut: Future = Future()
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            d = self._diagrams.get(diagram_id)
            if d is None:
                raise KeyError(f"diagram {diagram_id} is not resident")
            d.pins += 1
            self._queue.append(_Request(next(self._ids), "insert",
                                        time.perf_counter() if arrival is None else arrival, fut, diagram_id,
                                        seeds=s, fetch=fetch))
            self._cv.notify()
        return fut

    def resident(self) -> list[int]:
        """Ids of the diagrams currently resident (created, not evicted)."""
        with self._cv:
            return [k for k, d in self._diagrams.items() if d.obj is not None or d.pins]

    def memory_used(self) -> int:
        with self._cv:
            return self._used

    def drain(self) -> None:
        """Wait until every submitted request has finished."""
        with self._cv:
            while self._queue or any(d.busy for d in self._diagrams.values()):
                self._cv.wait(0.05)

    def close(self) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        with self._cv:
            for d in self._diagrams.values():
                d.obj = None
            self._diagrams.clear()
            self._pool.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- scheduling (called with the lock held) ----------------------------
    def _take_pooled(self, req: _Request) -> Optional[_Pooled]:
        """Smallest pooled object the request fits in, if it is not more than
        twice the request's own footprint."""
        cap = len(req.seeds) + SEED_HEADROOM
        best = None
        for i, p in enumerate(self._pool):
            if p.bytes <= 2 * req.need and _fits(p.cap, req.width, req.height, cap, self.padding) and \
                    (best is None or p.bytes < self._pool[best].bytes):
                best = i
        return self._pool.pop(best) if best is not None else None

    def _place(self, req: _Request, to_free: list):
        """Find memory for a new diagram: a pooled object, fresh budget, or
        budget freed by retiring idle diagrams (least recently used first)
        into the pool and, if that is not enough, dropping pooled objects.
        Returns (ok, pooled object or None)."""
        pooled = self._take_pooled(req)
        if pooled is not None:
            return True, pooled
        if self._used + req.need <= self.budget:
            return True, None
        idle = sorted((d for d in self._diagrams.values() if d.obj is not None and not d.busy and d.pins == 0),
                      key=lambda d: d.last_used)
        for d in idle:
            del self._diagrams[d.did]
            self._pool.append(_Pooled(d.obj, d.bytes, d.cap))
            d.obj = None
            self.stats["evicted"] += 1
            pooled = self._take_pooled(req)
            if pooled is not None:
                return True, pooled
        self._pool.sort(key=lambda p: p.bytes, reverse=True)
        while self._pool and self._used + req.need > self.budget:
            p = self._pool.pop(0)
            self._used -= p.bytes
            to_free.append(p.obj)
            self.stats["freed_objects"] += 1
        return self._used + req.need <= self.budget, None

    def _next(self, to_free: list) -> Optional[tuple]:
        while True:
            for i, req in enumerate(self._queue):
                d = self._diagrams.get(req.diagram_id)
                if d is None:                           # target evicted or its creation failed
                    del self._queue[i]
                    req.future.set_exception(KeyError(f"diagram {req.diagram_id} is not resident"))
                    break
                if req.kind == "new":
                    if req.need > self.budget:
                        del self._queue[i]
                        del self._diagrams[req.diagram_id]
                        req.future.set_exception(MemoryError(
                            f"request needs {req.need} bytes, over the {self.budget}-byte budget"))
                        break
                    ok, pooled = self._place(req, to_free)
                    if not ok:
                        continue
                    if pooled is None:
                        self._used += req.need          # charged now, corrected after creation
                    del self._queue[i]
                    d.busy = True
                    return "new", [(req, pooled)] + self._group_more(req, to_free)
                if d.busy or d.obj is None:
                    continue                            # busy, or its creation has not run yet
                del self._queue[i]
                d.busy = True
                return "insert", [(req, None)]
            else:
                if self._closed and not self._queue:
                    return None
                if self._queue and not any(d.busy for d in self._diagrams.values()):
                    # nothing in flight can free memory any more: a new
                    # diagram that does not fit now never will
                    for i, req in enumerate(self._queue):
                        if req.kind == "new":
                            del self._queue[i]
                            del self._diagrams[req.diagram_id]
                            req.future.set_exception(MemoryError(
                                f"request needs {req.need} bytes; the budget of {self.budget} bytes has "
                                f"{self.budget - self._used} left with nothing to evict"))
                            break
                    else:
                        self._cv.wait(0.1)
                    continue
                self._cv.wait()

    def _group_more(self, first: _Request, to_free: list) -> list:
        """Further queued new diagrams to propagate in the same launch as
        `first`, while they fit the group limits and the memory budget."""
        out = []
        area = (first.width + 2 * self.padding + 1) * (first.height + 2 * self.padding + 1)
        seeds = len(first.seeds)
        limit_area = (MAX_SIDE + 2 * self.padding + 1) ** 2
        i = 0
        while i < len(self._queue) and len(out) + 1 < GROUP_MAX:
            req = self._queue[i]
            if req.kind != "new" or req.need > self.budget:
                i += 1
                continue
            a = (req.width + 2 * self.padding + 1) * (req.height + 2 * self.padding + 1)
            if area + a > limit_area or seeds + len(req.seeds) > MAX_REQUEST_SEEDS:
                i += 1
                continue
            ok, pooled = self._place(req, to_free)
            if not ok:
                break
            if pooled is None:
                self._used += req.need
            del self._queue[i]
            self._diagrams[req.diagram_id].busy = True
            out.append((req, pooled))
            area += a
            seeds += len(req.seeds)
        return out

    # -- execution ------------------------------------------------------------
    def _worker(self):
        torch = self._torch
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream(self.device)
        workspace = _capi.Context(self.device)   # scratch shared by every diagram this slot runs
        batch = _capi.Context(self.device)       # atlas of the new diagrams this slot propagates together
        lib = _capi.load()
        while True:
            to_free: list = []
            with self._cv:
                got = self._next(to_free)
            to_free.clear()                             # objects are freed outside the lock
            if got is None:
                return
            kind, items = got
            with torch.cuda.stream(stream):
                src = None
                if kind == "new":
                    # one propagation launch for the whole group; a request
                    # the batch rejects fails alone on the per-diagram path
                    start = time.perf_counter()
                    batch.set_stream(stream.cuda_stream)
                    reqs = [r for r, _ in items]
                    dims = np.array([(r.width, r.height) for r in reqs], dtype=np.int32)
                    counts = np.array([len(r.seeds) for r in reqs], dtype=np.int64)
                    seeds = np.ascontiguousarray(np.concatenate([r.seeds for r in reqs]), dtype=np.int32)
                    st = lib.idl_voronoi_batch(batch.handle, len(reqs), dims.ctypes.data, counts.ctypes.data,
                                               seeds.ctypes.data, self.padding, _capi.MODE_REFERENCE)
                    src = batch if st == _capi.IDL_OK else None
                    with self._cv:
                        self.stats["groups"] += 1
                        self.stats["grouped_requests"] += len(reqs)
                else:
                    start = time.perf_counter()
                for k, (req, pooled) in enumerate(items):
                    self._execute(req, pooled, start, workspace, (src, k) if src is not None else None,
                                  stream.cuda_stream)

    def _execute(self, req: _Request, pooled: Optional[_Pooled], start: float, workspace, adopt,
                 stream_handle: int) -> None:
        try:
            res = self._run(req, pooled, start, workspace, adopt, stream_handle)
            req.future.set_result(res)
        except BaseException as e:   # noqa: BLE001 - delivered to the caller
            with self._cv:
                dd = self._diagrams.get(req.diagram_id)
                if req.kind == "new" and dd is not None and dd.obj is None:
                    self._used -= pooled.bytes if pooled is not None else req.need
                    del self._diagrams[req.diagram_id]
            req.future.set_exception(e)
        finally:
            with self._cv:
                d = self._diagrams.get(req.diagram_id)
                if d is not None:
                    d.busy = False
                    d.pins -= 1
                    d.last_used = time.perf_counter()
                self._cv.notify_all()

    def _run(self, req: _Request, pooled: Optional[_Pooled], start: float, workspace, adopt=None,
             stream_handle: int = 0) -> Result:
        """One request on this slot's stream.  The calls go to the C ABI
        directly (one per step), so a request costs the interpreter little."""
        cu, lib, ck = self._cu, self._lib, _capi.check
        d = self._diagrams[req.diagram_id]
        if req.kind == "new":
            cap = len(req.seeds) + SEED_HEADROOM
            if pooled is not None:
                obj = pooled.obj
                charged = pooled.bytes
                self.stats["reused_objects"] += 1
            else:
                Wc, Hc = _class_dims(req.width, req.height)
                obj = cu.Delaunay(Wc, Hc, cap, self.padding)
                alloc_cap = _capacity(Wc, Hc, cap, self.padding)
                charged = req.need
                self.stats["new_objects"] += 1
        else:
            obj = d.obj
        h = obj._h
        ck(lib.idl_delaunay_set_stream(h, stream_handle or None))
        ck(lib.idl_delaunay_set_workspace(h, workspace.handle))
        obj._workspace = workspace
        s = req.seeds
        if req.kind == "new":
            ck(lib.idl_delaunay_reset(h, req.width, req.height, cap, self.padding))
            if adopt is not None:
                ck(lib.idl_delaunay_adopt(h, adopt[0].handle, adopt[1]))
            else:
                ck(lib.idl_delaunay_insert_ordered(h, s.ctypes.data if len(s) else None, len(s), None, 1, None))
            seeds_after = len(s)
        else:
            ck(lib.idl_delaunay_insert_ordered(h, s.ctypes.data if len(s) else None, len(s), None, 0, None))
            seeds_after = d.n_seeds + len(s)
        verts = grid = None
        if req.fetch:
            verts, grid = obj.finalise(as_arrays=True)
            grid = np.array(grid, copy=True)
            n_tri = len(verts)
        else:
            n = ctypes.c_int64(0)
            ck(lib.idl_delaunay_finalise_device(h, ctypes.byref(n), None, None, None, None))
            n_tri = int(n.value)
        if req.kind == "new":
            actual = max(obj.device_bytes, charged)
            with self._cv:
                d.obj = obj
                d.bytes = actual
                d.cap = pooled.cap if pooled is not None else alloc_cap
                self._used += actual - charged
        d.n_seeds = seeds_after
        done = time.perf_counter()
        return Result(req.rid, req.kind, req.diagram_id, seeds_after, n_tri, req.arrival, start, done,
                      verts, grid)

    def recycle(self, diagram_id: int) -> None:
        """Retire a diagram now, keeping its object for reuse."""
        with self._cv:
            d = self._diagrams.get(diagram_id)
            if d is None or d.busy or d.pins:
                return
            del self._diagrams[diagram_id]
            if d.obj is not None:
                self._pool.append(_Pooled(d.obj, d.bytes, d.cap))
            self._cv.notify_all()


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
