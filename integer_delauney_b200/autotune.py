"""Autotuning of the propagation schedule and tile shape.

From scratch, the reference-semantics propagation runs its first passes as
tile rounds (several passes per HBM round trip over every tile that can still
change) and hands the tail to the persistent sparse kernel.  Two knobs decide
its speed, never its result:

* the schedule (idl_context_set_schedule): how many tile rounds run before the
  sparse kernel takes over (0 = sparse kernel only, -1 = tile rounds to
  convergence);
* the tile shape (idl_context_set_tile), one of twelve:
  0-3 are register tile rounds (inner tile / passes per round trip:
  48 x 48 / 8, 48 x 112 / 8, 56 x 56 / 4, 40 x 104 / 12), one launch per
  round; 4-7 are the same shapes with every round in one cooperative launch;
  8-11 are shared-memory tile rounds that step only the 8 x 8 cells still
  changing (48 x 48 / 8, 56 x 56 / 4, 112 x 48 / 8, 96 x 96 / 16).  Larger
  tiles waste less work on halos, more passes per round trip suit thin
  fronts crossing empty space, fewer suit dense seed sets.

Where each pays depends on the seed density and layout: dense, uniform seed
sets change most of the canvas for the first few passes, clustered ones leave
long thin fronts.  ``tune`` times one representative input under every
candidate (schedule, shape) on the device and keeps the fastest for that
input's class (canvas size and density on a log scale, and how much of the
canvas the seeds occupy), so a stream of similar inputs is tuned once.  Every
candidate gives the same result bit for bit; only the time differs.
"""
from __future__ import annotations

import math
from typing import Iterable, Optional

import numpy as np

from . import _capi

SCHEDULES = (0, 1, 2, 3, 4, 6, -1)
_cache: dict[tuple, tuple[int, int]] = {}
# the timings of the last tuning run: {(schedule, shape): best ms of the repeats}
last_report: dict[tuple[int, int], float] = {}


def occupancy(width: int, height: int, seeds) -> float:
    """Share of the canvas's 64 x 64 cells that hold at least one seed: near 1
    for uniform seed sets, small for clustered ones (long fronts through empty
    space), which favour other schedules at the same size and density."""
    s = np.asarray(seeds, dtype=np.int64).reshape(-1, 2)
    cw = (int(width) + 63) // 64
    ch = (int(height) + 63) // 64
    if len(s) == 0:
        return 0.0
    cells = np.unique((s[:, 1] // 64) * cw + s[:, 0] // 64)
    return len(cells) / float(cw * ch)


def input_class(width: int, height: int, n_seeds: int, occ: float = 1.0) -> tuple:
    """Inputs in one class share a tuned schedule: canvas pixels and seeds per
    pixel, each bucketed by powers of two, and the seed occupancy in quarters."""
    px = max(1, int(width) * int(height))
    return (int(math.log2(px)), int(math.log2(max(1, int(n_seeds)) / px * 1e6 + 1)), min(4, int(occ * 4)))


def candidates(n_shapes: int, schedules: Iterable[int] = SCHEDULES) -> list[tuple[int, int]]:
    """Every (schedule, shape) pair; the sparse-only schedule has no tile rounds,
    so it is tried once."""
    out = []
    for sched in schedules:
        for shape in ([0] if sched == 0 else range(n_shapes)):
            out.append((int(sched), int(shape)))
    return out


def apply(ctx: _capi.Context, choice: tuple[int, int]) -> None:
    ctx.set_schedule(choice[0])
    ctx.set_tile(choice[1])


def tune(width: int, height: int, seeds, border_padding: int = _capi.AUTO_BORDER_PADDING,
         schedules: Iterable[int] = SCHEDULES, repeats: int = 3, context: Optional[_capi.Context] = None,
         force: bool = False) -> tuple[int, int]:
    """Pick the fastest (schedule, tile shape) for inputs like this one, set it
    on ``context`` (the current device's default context if None) and return
    it.  Times idl_triangulate_device with CUDA events on the current stream."""
    import torch
    s = np.ascontiguousarray(np.asarray(seeds, dtype=np.int32).reshape(-1, 2))
    key = input_class(width, height, len(s), occupancy(width, height, s))
    ctx = context or _capi.context_for(torch.cuda.current_device())
    if key in _cache and not force:
        apply(ctx, _cache[key])
        return _cache[key]
    lib = _capi.load()
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    d_seeds = torch.from_numpy(s).cuda()
    d_out = torch.empty((int(height), int(width), 3), dtype=torch.int32, device="cuda")
    n_shapes = ctx.set_tile(0)

    def run():
        _capi.check(lib.idl_triangulate_device(ctx.handle, int(width), int(height), d_seeds.data_ptr(), len(s),
                                               int(border_padding), _capi.MODE_REFERENCE, d_out.data_ptr(), None))

    best, best_ms = None, float("inf")
    last_report.clear()
    for choice in candidates(n_shapes, schedules):
        apply(ctx, choice)
        run()                                   # warm-up: workspace at its high-water mark
        times = []
        for _ in range(max(1, repeats)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = min(times)
        last_report[choice] = ms
        if ms < best_ms:
            best, best_ms = choice, ms
    _cache[key] = best
    apply(ctx, best)
    return best
