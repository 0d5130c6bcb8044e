"""Spreading independent images and diagrams over several GPUs.

Every image of a batch and every served diagram is independent of the others,
so the library scales across the GPUs of a node as replicas: whole images or
diagrams are assigned to devices and each device runs them alone, with no
collective and no data crossing between GPUs.  (A single image needs no
spatial split: the largest canvas, 4128^2 padded, holds well under 1 GB.)

  * ``partition`` -- greedy least-loaded assignment (largest item first to the
    lightest part), deterministic; used for batches and for the ranks of a
    multi-process job (``rank_shard``).
  * ``triangulate_batch_devices`` -- ``triangulate_batch`` with the images
    spread over devices by pixel count, one worker thread per device; the
    results come back in input order and equal the single-device call's.
  * ``ServerPool`` -- one native server (``serving.Server``) per device: a new
    diagram goes to the device with the least work assigned so far, an insert
    to its diagram's device.  Diagram ids are the pool's own.
"""
from __future__ import annotations

import threading
from typing import Callable, Iterable, Optional, Sequence

from . import _capi


def partition(weights: Sequence[float], n_parts: int) -> list[list[int]]:
    """Indices of ``weights`` split into ``n_parts`` lists of about equal total
    weight: items in descending weight (ties by index) each go to the part with
    the least weight so far (ties by part number).  Every index appears in
    exactly one part; each part lists its indices in ascending order."""
    if n_parts < 1:
        raise ValueError("n_parts must be at least 1")
    load = [0.0] * n_parts
    parts: list[list[int]] = [[] for _ in range(n_parts)]
    for i in sorted(range(len(weights)), key=lambda k: (-float(weights[k]), k)):
        p = min(range(n_parts), key=lambda q: (load[q], q))
        parts[p].append(i)
        load[p] += float(weights[i])
    return [sorted(p) for p in parts]


def rank_shard(weights: Sequence[float], rank: int, world: int) -> list[int]:
    """The indices rank ``rank`` of ``world`` processes takes (``partition``);
    every rank computes the same split without communicating."""
    if not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    return partition(weights, world)[rank]


def _devices(devices: Optional[Iterable[int]]) -> list[int]:
    if devices is None:
        import torch
        return list(range(torch.cuda.device_count()))
    out = [int(d) for d in devices]
    if not out:
        raise ValueError("at least one device is needed")
    return out


def triangulate_batch_devices(images, devices: Optional[Iterable[int]] = None,
                              border_padding: int = _capi.AUTO_BORDER_PADDING, as_arrays: bool = False):
    """``triangulate_batch`` over several devices: images are assigned by
    padded pixel count (``partition``), each device triangulates its share in
    one batch on its own thread, and the results return in input order --
    each equal to ``triangulate(W, H, seeds)`` on one device."""
    import torch
    from . import _delauney_cuda as cu
    imgs = list(images)
    devs = _devices(devices)
    P = cu.resolve_padding(border_padding)
    weights = [(int(w) + 2 * P) * (int(h) + 2 * P) for w, h, _ in imgs]
    parts = partition(weights, len(devs))
    out: list = [None] * len(imgs)
    errors: list[BaseException] = []

    def run(dev: int, idx: list[int]) -> None:
        try:
            with torch.cuda.device(dev):
                res = cu.triangulate_batch([imgs[i] for i in idx], P, as_arrays)
                torch.cuda.current_stream().synchronize()
            for i, r in zip(idx, res):
                out[i] = r
        except BaseException as e:   # noqa: BLE001 - re-raised on the caller's thread
            errors.append(e)

    threads = [threading.Thread(target=run, args=(d, idx)) for d, idx in zip(devs, parts) if idx]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return out


class PoolTicket:
    """A request submitted to a ``ServerPool``: ``diagram_id`` is the pool's
    id; ``result()`` returns the device server's ``Result`` with that id."""

    def __init__(self, ticket, diagram_id: int, device: int):
        self._t = ticket
        self.diagram_id = diagram_id
        self.device = device

    def result(self, timeout: Optional[float] = None):
        r = self._t.result(timeout)
        r.diagram_id = self.diagram_id
        return r

    def exception(self, timeout: Optional[float] = None):
        return self._t.exception(timeout)

    def done(self) -> bool:
        return self._t.done()


class ServerPool:
    """Native servers on several devices behind one submit/collect interface.

    A new diagram goes to the device with the least work assigned so far
    (padded pixels of its new diagrams plus seeds of its inserts), ties to the
    lower device number; an insert goes to the device its diagram lives on.
    Each device has its own memory budget.  ``make_server(device)`` builds a
    device's server (default ``serving.Server`` with the given settings)."""

    def __init__(self, devices: Optional[Iterable[int]] = None, budget_bytes: int = 40 << 30, slots: int = 8,
                 border_padding: int = _capi.AUTO_BORDER_PADDING, mode: str = "reference",
                 make_server: Optional[Callable[[int], object]] = None):
        devs = _devices(devices)
        if make_server is None:
            from .serving import Server

            def make_server(dev: int):
                return Server(device=dev, budget_bytes=budget_bytes, slots=slots, border_padding=border_padding,
                              mode=mode)
        self.devices = devs
        self._servers = [make_server(d) for d in devs]
        self._load = [0] * len(devs)
        self._home: dict[int, tuple[int, int]] = {}    # pool diagram id -> (server index, its diagram id)
        self._next = 0
        self._lock = threading.Lock()
        auto = border_padding == _capi.AUTO_BORDER_PADDING
        self._pad = _capi.DEFAULT_BORDER_PADDING if auto else max(0, int(border_padding))

    def submit_new(self, width: int, height: int, seeds, fetch: bool = False,
                   arrival: Optional[float] = None) -> PoolTicket:
        with self._lock:   # a submit is one quick call: held so the id is known before any insert
            k = min(range(len(self._servers)), key=lambda q: (self._load[q], q))
            t = self._servers[k].submit_new(width, height, seeds, fetch=fetch, arrival=arrival)
            self._load[k] += (int(width) + 2 * self._pad) * (int(height) + 2 * self._pad)
            did = self._next
            self._next += 1
            self._home[did] = (k, t.diagram_id)
        return PoolTicket(t, did, self.devices[k])

    def submit_insert(self, diagram_id: int, seeds, fetch: bool = False,
                      arrival: Optional[float] = None) -> PoolTicket:
        """Raises KeyError if the pool never created that diagram or its
        device server no longer holds it."""
        with self._lock:
            home = self._home.get(int(diagram_id))
            if home is None:
                raise KeyError(f"diagram {diagram_id} is not resident")
            k, local = home
            self._load[k] += len(seeds)
        t = self._servers[k].submit_insert(local, seeds, fetch=fetch, arrival=arrival)
        return PoolTicket(t, int(diagram_id), self.devices[k])

    def resident(self) -> list[int]:
        out = []
        with self._lock:
            homes = dict(self._home)
        live = [set(s.resident()) for s in self._servers]
        for did, (k, local) in homes.items():
            if local in live[k]:
                out.append(did)
        return sorted(out)

    def drain(self) -> None:
        for s in self._servers:
            s.drain()

    @property
    def stats(self) -> dict:
        total: dict = {}
        for s in self._servers:
            for key, v in dict(s.stats).items():
                total[key] = total.get(key, 0) + v
        return total

    def loads(self) -> list[int]:
        """Work assigned to each device so far (padded pixels + insert seeds)."""
        with self._lock:
            return list(self._load)

    def close(self) -> None:
        for s in self._servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
