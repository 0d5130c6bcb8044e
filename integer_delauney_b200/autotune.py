"""Autotuning of the propagation schedule.

From scratch, the reference-semantics propagation runs its first passes as
tile rounds (8 passes per HBM round trip over every tile that can still
change) and hands the tail to the persistent sparse kernel
(idl_context_set_schedule).  Where the switch pays depends on the seed
density and layout: dense, uniform seed sets change most of the canvas for
the first few passes, clustered ones leave long thin fronts.  ``tune`` times
one representative input under each candidate schedule on the device and
keeps the fastest for that input's class (canvas size and density, both on a
log scale), so a stream of similar inputs is tuned once.  Every schedule gives
the same result bit for bit; only the time differs.
"""
from __future__ import annotations

import math
from typing import Iterable, Optional

import numpy as np

from . import _capi

CANDIDATES = (0, 1, 2, 3)
_cache: dict[tuple, int] = {}


def input_class(width: int, height: int, n_seeds: int) -> tuple:
    """Inputs in one class share a tuned schedule: canvas pixels and seeds per
    pixel, each bucketed by powers of two."""
    px = max(1, int(width) * int(height))
    return (int(math.log2(px)), int(math.log2(max(1, int(n_seeds)) / px * 1e6 + 1)))


def tune(width: int, height: int, seeds, border_padding: int = _capi.AUTO_BORDER_PADDING,
         candidates: Iterable[int] = CANDIDATES, repeats: int = 3, context: Optional[_capi.Context] = None,
         force: bool = False) -> int:
    """Pick the fastest propagation schedule for inputs like this one, set it
    on ``context`` (the current device's default context if None) and return
    it.  Times idl_triangulate_device with CUDA events on the current stream."""
    import torch
    s = np.ascontiguousarray(np.asarray(seeds, dtype=np.int32).reshape(-1, 2))
    key = input_class(width, height, len(s))
    ctx = context or _capi.context_for(torch.cuda.current_device())
    if key in _cache and not force:
        ctx.set_schedule(_cache[key])
        return _cache[key]
    lib = _capi.load()
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    d_seeds = torch.from_numpy(s).cuda()
    d_out = torch.empty((int(height), int(width), 3), dtype=torch.int32, device="cuda")

    def run():
        _capi.check(lib.idl_triangulate_device(ctx.handle, int(width), int(height), d_seeds.data_ptr(), len(s),
                                               int(border_padding), _capi.MODE_REFERENCE, d_out.data_ptr(), None))

    best, best_ms = None, float("inf")
    for sched in candidates:
        ctx.set_schedule(sched)
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
        if ms < best_ms:
            best, best_ms = sched, ms
    _cache[key] = best
    ctx.set_schedule(best)
    return best
