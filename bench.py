"""Benchmark: Mpixel/s of Voronoi + Delaunay + per-pixel assignment, bit-exact.

Workload (one step = one image through the whole pipeline):
  4096 x 4096 image, 200 000 distinct uniform random seeds (seeded), border
  padding 16 (detection canvas 4128 x 4128), reference-CUDA Voronoi
  semantics -- the plain GPU drop-in configuration.  A clustered variant
  (64 Gaussian blobs, sigma 40 px) of the same size is timed too and reported
  beside it.

  value  device-resident throughput: seeds already on the device, (H, W, 3)
         output left on the device (idl_triangulate_device), CUDA events on the
         library's stream around K steps.
  e2e    the public drop-in call triangulate(W, H, seeds, as_arrays=True) with
         seeds in pinned host memory: host->device copy of the seeds, all
         stages, device->host copy of the (H, W, 3) grid and the triangles.

Also on the same line: the same step in exact semantics ("exact"); the
incremental workload (2048 x 2048, 50 000 seeds + 100 inserts of 1 000) in
reference and exact semantics; the batched workload (512 images in one call
against the per-image loop); and the serving workload (Poisson request stream
against the server, and a fixed prefix against the plain serial loop).

Multi-GPU (torchrun): every rank triangulates its own image per step (replicas,
no collective on the data path); the time is the max over ranks.

`--impl reference` times the reference's own CUDA triangulate, compiled from
its sources for sm_100a (oracle/_ref), through its stock host path on the same
full workload, on rank 0 only (the oracle port on the host cores if that build
is absent).  The same measurement appears on this arm's line as `ref_cuda`,
beside `cpu_baseline` (the oracle port on all host cores: the 512 x 512 CPU
configuration measured outright, the 4096 x 4096 image extrapolated from a
sample of assignment rows and marked so).
"""
from __future__ import annotations

import argparse
import ctypes
import gc
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = H = 4096
N_SEEDS = 200_000
PADDING = 16
MODE = "reference"
METRIC = "Mpixel/s Voronoi+Delaunay+assign (bit-exact)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def reduce_max(value: float, world: int) -> float:
    """Max of a per-rank timing over all ranks (identity for one rank)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# dram__bytes_read.sum + dram__bytes_write.sum of the dominant stage's kernels
# for one step of this workload (uniform seeds), from ncu --set full captures:
# the three cell-list tile rounds (72.6 + 29.1, 72.6 + 33.2, 72.6 + 33.5 MB) and
# the persistent kernel's tail (113.7 + 30.6 MB)
TRAFFIC_PER_LAUNCH = {"propagate_ms": 72.6e6 + 29.1e6 + 72.6e6 + 33.2e6 + 72.6e6 + 33.5e6 + 113.7e6 + 30.6e6}


class ClockSampler:
    """SM clock and throttle reasons of one GPU, polled through NVML (read
    only) every few milliseconds while the timed region runs, plus one sample
    on entry and one on exit so that even a short region is covered."""

    PERIOD_S = 0.002
    # NVML clocks-event reason bits (nvml.h): the ones a bench line must report.
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap"}

    def __init__(self, index: int):
        self.index = index
        self.sm = []
        self.mask = 0
        self.max_mhz = None
        self.nv = None
        self.stop = threading.Event()

    def _sample(self):
        nv = self.nv
        self.sm.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
        self.mask |= int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))

    def _loop(self):
        while not self.stop.wait(self.PERIOD_S):
            try:
                self._sample()
            except Exception:
                return

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self._sample()
            self.thread = threading.Thread(target=self._loop, daemon=True)
            self.thread.start()
        except Exception:
            self.nv = None
        return self

    def __exit__(self, *exc):
        if self.nv is None:
            return
        self.stop.set()
        self.thread.join(timeout=2)
        try:
            self._sample()
            self.nv.nvmlShutdown()
        except Exception:
            pass

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        reasons = sorted(nm for bit, nm in self.REASONS.items() if self.mask & bit)
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.sm)}


def cpu_baseline(sample_rows: int = 0):
    """The reference algorithm on the host cores (the oracle port of
    src/cuda/voronoi.cu + triangulation.cu, OpenMP): full Jacobi + detection
    on the padded 4096 x 4096 canvas, the reference's per-pixel assignment on
    a sample of rows, extrapolated to the image; and the whole pipeline,
    measured outright, on the 512 x 512 / 2 000-seed CPU configuration.
    Returns the cpu_baseline object."""
    import oracle
    from integer_delauney_b200.workloads import uniform

    threads = oracle.num_threads()
    rows = sample_rows or max(4, min(64, threads))
    seeds = uniform(W, H, N_SEEDS, seed=0)
    s = oracle.sort_seeds(seeds, W, H)
    xs, ys = np.ascontiguousarray(s[:, 0]), np.ascontiguousarray(s[:, 1])
    Wd, Hd = W + 2 * PADDING, H + 2 * PADDING
    t0 = time.perf_counter()
    lab = np.full((Hd, Wd), -1, dtype=np.int32)
    lab[ys + PADDING, xs + PADDING] = np.arange(len(s), dtype=np.int32)
    lab, passes = oracle.jacobi_from(Wd, Hd, xs + PADDING, ys + PADDING, lab)
    t1 = time.perf_counter()
    tris = oracle.detect(lab, xs + PADDING, ys + PADDING, PADDING)
    t2 = time.perf_counter()
    y0 = H // 2 - rows // 2
    oracle.assign_rows(W, H, xs, ys, tris, y0, y0 + rows)
    t3 = time.perf_counter()
    est = (t1 - t0) + (t2 - t1) + (t3 - t2) * (H / rows)
    desc = (f"oracle port, {threads} threads: full Jacobi ({passes} passes) + detection on the "
            f"{Wd}x{Hd} canvas, reference per-pixel assignment on {rows} of {H} rows, extrapolated to "
            f"{H} rows")
    # the CPU configuration, whole pipeline, no extrapolation
    c1 = oracle.sort_seeds(uniform(512, 512, 2000, seed=0), 512, 512)
    c1_s = []
    for _ in range(3):
        t = time.perf_counter()
        oracle.triangulate(512, 512, c1, PADDING, "reference")
        c1_s.append(time.perf_counter() - t)
    c1_t = statistics.median(c1_s)
    return {"value": W * H / est / 1e6, "unit": "Mpixel/s", "cores": threads, "kind": "port", "sample": desc,
            "extrapolated": True, "estimated_s": est, "measured_s": t3 - t0,
            "cpu_config": {"workload": f"triangulate 512x512, 2000 uniform seeds, P={PADDING}, whole pipeline "
                                       f"measured", "s": c1_t, "mpix_s": 512 * 512 / c1_t / 1e6}}


def ref_cuda_baseline(seeds: np.ndarray, reps: int, warmup: int = 1):
    """The reference's own CUDA triangulate compiled from its sources for
    sm_100a (oracle/_ref/libref_cuda.so, built by oracle/build_ref.sh): its
    stock path (src/cuda/bindings/triangulate.hpp:15-43 -> triangulation.cu:
    143-365) with host seeds in and the (H, W, 3) grid and triangles out, on
    this GPU and one host core, wall clock per call (the path synchronises
    itself).  Returns (ms per call list, triangle count) or None when the
    library was not built."""
    import oracle
    if not oracle.ref_available():
        return None
    for _ in range(warmup):
        oracle.ref_triangulate_stock(W, H, seeds, PADDING)
    ms = []
    n_tri = 0
    for _ in range(reps):
        t = time.perf_counter()
        tris, _ = oracle.ref_triangulate_stock(W, H, seeds, PADDING)
        ms.append((time.perf_counter() - t) * 1e3)
        n_tri = len(tris)
    return ms, n_tri


REF_CUDA_DESC = ("the reference's own triangulate compiled from its sources for sm_100a "
                 "(src/cuda/voronoi.cu + triangulation.cu via its stock host path): host loops on one "
                 "core, kernels on this GPU; host seeds in, (H, W, 3) grid and triangles out; wall clock")


def run_reference(args, rank, world):
    """The reference arm: the reference's own CUDA path on the full
    4096 x 4096 / 200 000-seed workload, every step measured (no sample);
    the oracle port on the host cores when the reference build is absent."""
    if rank != 0:
        return
    from integer_delauney_b200.workloads import uniform
    seeds = uniform(W, H, N_SEEDS, seed=0)
    r = ref_cuda_baseline(seeds, args.steps, args.warmup)
    if r is not None:
        ms_list, n_tri = r
        ms = statistics.median(ms_list)
        value = W * H / (ms / 1e3) / 1e6
        base = {"value": value, "unit": "Mpixel/s", "cores": 1, "kind": "reference",
                "sample": f"full workload every step ({args.steps} steps); " + REF_CUDA_DESC,
                "ms_per_call": ms_list, "triangles": n_tri}
    else:
        vals, secs = [], []
        base = {}
        for _ in range(args.warmup):
            cpu_baseline(args.ref_rows)
        for _ in range(args.steps):
            base = cpu_baseline(args.ref_rows)
            vals.append(base["value"])
            secs.append(base["estimated_s"])
        value = statistics.median(vals)
        ms = statistics.median(secs) * 1e3
        base["value"] = value
    line = {
        "metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": f"triangulate {W}x{H}, {N_SEEDS} uniform seeds, P={PADDING}, reference mode",
                   "parallelism": f"replicas x{world}"},
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": "Mpixel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def incremental_case(cu, torch, rank, mode="reference"):
    """2048 x 2048, 50 000 uniform seeds, then 100 insert batches of 1 000
    new seeds (30 % in a 256 x 256 hotspot).  Each batch is timed through the
    public call a caller makes: insert() (propagate, topology, assignment and
    the (H, W, 3) grid copied to host memory), wall clock per batch; then the
    same batches through insert_deferred() and one finalise() (three runs on
    fresh objects, median).  Triangles come
    back as arrays (as_arrays=True): a 300 000-entry dict costs more host time
    than the whole device update."""
    from integer_delauney_b200.workloads import incremental
    Wi = Hi = 2048
    base, batches = incremental(Wi, Hi, 50_000, 100, 1_000, seed=rank)
    cap = len(base) + sum(len(b) for b in batches)

    def fresh():
        d = cu.Delaunay(Wi, Hi, cap, PADDING, voronoi_mode=mode)
        d.insert_deferred(base)
        d.finalise()
        return d

    d = fresh()
    m = g = None
    for b in batches[:3]:                 # warm-up on a throwaway object, holding results as the timed loop
        m, g = d.insert(b, as_arrays=True)   # does, so the pinned output blocks it alternates between are cached
    d = fresh()
    torch.cuda.synchronize()
    gc.collect()
    gc.disable()                             # no collector pauses inside the timed loops
    lat = []
    allocs = []
    from integer_delauney_b200 import _capi
    lib = _capi.load()
    t_all = time.perf_counter()
    for b in batches:
        a0 = lib.idl_alloc_count()
        t0 = time.perf_counter()
        m, g = d.insert(b, as_arrays=True)
        lat.append(time.perf_counter() - t0)
        allocs.append(lib.idl_alloc_count() - a0)
    t_all = time.perf_counter() - t_all
    n_tri = len(m)
    # the deferred form three times, each on a fresh object: one run is at
    # the mercy of host-side hiccups (tens of ms), the median is not
    t_defs = []
    for _ in range(3):
        d2 = fresh()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for b in batches:
            d2.insert_deferred(b)
        d2.finalise(as_arrays=True)
        t_defs.append(time.perf_counter() - t0)
        del d2
    t_def = statistics.median(t_defs)
    gc.enable()
    lat_ms = sorted(x * 1e3 for x in lat)
    return {"workload": f"Delaunay {Wi}x{Hi}, {len(base)} uniform seeds + {len(batches)} x {len(batches[0])} "
                        f"(30% in a 256x256 hotspot), P={PADDING}, {mode} mode",
            "insert_ms_mean": t_all * 1e3 / len(batches), "insert_ms_p50": lat_ms[len(lat_ms) // 2],
            "insert_ms_p99": lat_ms[min(len(lat_ms) - 1, int(0.99 * len(lat_ms)))],
            "slowest_inserts": [[int(i), round(lat[i] * 1e3, 2), int(allocs[i])] for i in np.argsort(lat)[::-1][:4]],
            "inserts_that_allocated": [int(i) for i in np.flatnonzero(np.array(allocs) > 0)][:10],
            "insert_mpix_s": Wi * Hi * len(batches) / t_all / 1e6,
            "deferred_total_ms": t_def * 1e3, "deferred_runs_ms": [round(x * 1e3, 2) for x in t_defs],
            "triangles_final": n_tri,
            "d2h_bytes_per_insert": Wi * Hi * 12}


def batched_case(torch, lib, ctx, stream, rank):
    """512 images, sides log-uniform in 64..1024, density 0.1..2 %: one
    idl_triangulate_batch_device call against the plain per-image loop of
    idl_triangulate_device (one call and one count read-back per image), both
    on device-resident seeds and outputs, both timed with CUDA events."""
    from integer_delauney_b200 import _capi
    from integer_delauney_b200.workloads import batched_images
    imgs = batched_images(512, seed=rank)
    dims = np.array([(w, h) for w, h, _ in imgs], dtype=np.int32)
    counts = np.array([len(sd) for _, _, sd in imgs], dtype=np.int64)
    seeds = torch.from_numpy(np.concatenate([sd for _, _, sd in imgs])).cuda()
    px = dims[:, 0].astype(np.int64) * dims[:, 1]
    out = torch.empty(int(px.sum()) * 3, dtype=torch.int32, device="cuda")
    tri_counts = np.zeros(len(imgs), dtype=np.int64)
    s_off = np.concatenate([[0], np.cumsum(counts)])
    p_off = np.concatenate([[0], np.cumsum(px)])
    mode = _capi.mode_id(MODE)

    def batch():
        _capi.check(lib.idl_triangulate_batch_device(ctx.handle, len(imgs), dims.ctypes.data, counts.ctypes.data,
                                                     seeds.data_ptr(), PADDING, mode, out.data_ptr(),
                                                     tri_counts.ctypes.data))

    n_tri = ctypes.c_int64(0)

    def loop():
        for i, (w, h, _) in enumerate(imgs):
            _capi.check(lib.idl_triangulate_device(ctx.handle, w, h, seeds.data_ptr() + int(s_off[i]) * 8,
                                                   int(counts[i]), PADDING, mode,
                                                   out.data_ptr() + int(p_off[i]) * 12, ctypes.byref(n_tri)))

    def timed(fn, reps):
        fn()
        fn()
        torch.cuda.synchronize()
        l0 = lib.idl_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, (lib.idl_launch_count() - l0) // reps

    ms_b, launches_b = timed(batch, 5)
    ms_l, launches_l = timed(loop, 2)
    exact = _capi.mode_id("exact")

    def batch_exact():
        _capi.check(lib.idl_triangulate_batch_device(ctx.handle, len(imgs), dims.ctypes.data, counts.ctypes.data,
                                                     seeds.data_ptr(), PADDING, exact, out.data_ptr(),
                                                     tri_counts.ctypes.data))

    def loop_exact():
        for i, (w, h, _) in enumerate(imgs):
            _capi.check(lib.idl_triangulate_device(ctx.handle, w, h, seeds.data_ptr() + int(s_off[i]) * 8,
                                                   int(counts[i]), PADDING, exact,
                                                   out.data_ptr() + int(p_off[i]) * 12, ctypes.byref(n_tri)))

    ms_bx, _ = timed(batch_exact, 5)
    ms_lx, _ = timed(loop_exact, 2)
    total = float(px.sum())
    return {"workload": f"{len(imgs)} images, sides log-uniform 64..1024, density 0.1..2 %, "
                        f"{int(counts.sum())} seeds, {int(total)} pixels, P={PADDING}, reference mode",
            "batch_ms": ms_b, "batch_mpix_s": total / (ms_b / 1e3) / 1e6, "batch_launches": int(launches_b),
            "loop_ms": ms_l, "loop_mpix_s": total / (ms_l / 1e3) / 1e6, "loop_launches": int(launches_l),
            "speedup_vs_loop": ms_l / ms_b,
            "exact_mode": {"batch_ms": ms_bx, "batch_mpix_s": total / (ms_bx / 1e3) / 1e6, "loop_ms": ms_lx,
                           "speedup_vs_loop": ms_lx / ms_bx}}


def serving_case(torch, rank, seconds, slots=8):
    """Serving: (1) a Poisson stream (1 000 req/s for `seconds`, 70 % new
    triangulations of side log-uniform 128..4096 and density 0.05..1 %, 30 %
    inserts of 100..5 000 seeds into a uniformly chosen resident diagram,
    40 GB admission budget) replayed in real time against the server:
    latency p50/p99 from arrival to result, also at 500 req/s (a rate the
    server sustains, for a p99 without queueing); (2) throughput with every request
    of a fixed 2 000-request prefix submitted at once, server against the
    plain serial loop over the same requests.  The server is the native loop
    (idl_server_*): submission copies the seeds and returns, latency runs from
    the scheduled arrival to the worker's completion timestamp."""
    from integer_delauney_b200.serving import Server, run_serial
    from integer_delauney_b200.workloads import fresh_points, serving_trace, uniform
    budget = 40 << 30
    trace = serving_trace(1000.0, seconds, seed=rank)

    def keys_of(W, pts):
        return np.sort(pts[:, 1].astype(np.int64) * W + pts[:, 0])

    def realtime(rate):
        """Replay a Poisson trace at `rate` req/s in real time; the new
        requests' seed sets are generated before the clock starts, the
        inserts' (which depend on the target) on the fly."""
        tr = trace if rate == 1000.0 else serving_trace(rate, seconds, seed=rank)
        pre = {i: uniform(prm[0], prm[1], prm[2], seed=prm[3]) for i, (t, kind, prm) in enumerate(tr)
               if kind == "new"}
        srv = Server(budget_bytes=budget, slots=slots, border_padding=PADDING)
        # warm-up, untimed: new diagrams from another stretch of the same
        # distribution until the budget is full, so the timed replay sees the
        # steady state (objects recycled, not allocated)
        warm = [prm for _, kind, prm in serving_trace(rate, 4.0, seed=rank + 1000) if kind == "new"]
        for W_, H_, n_, ps_ in warm:
            srv.submit_new(W_, H_, uniform(W_, H_, n_, seed=ps_))
        srv.drain()
        warm_stats = dict(srv.stats)
        gc.collect()
        gc.freeze()                          # no collector pauses inside the timed replay
        gc.disable()
        info = {}          # diagram id -> (W, H, sorted keys)
        dims = {}          # diagram id -> (W, H), kept after eviction
        ids = []           # the same ids, for uniform picks
        futs = []
        failed_submit = 0
        late = 0.0
        t0 = time.monotonic() + 0.05         # the server's clock: arrivals are passed in on it
        for i, (t, kind, prm) in enumerate(tr):
            at = t0 + t
            now = time.monotonic()
            if at > now:
                time.sleep(at - now)
            else:
                late = max(late, now - at)
            if kind == "new":
                W, H, n, ps = prm
                pts = pre.pop(i)
                f = srv.submit_new(W, H, pts, arrival=at)
                info[f.diagram_id] = (W, H, keys_of(W, pts))
                dims[f.diagram_id] = (W, H)
                ids.append(f.diagram_id)
                futs.append(f)
                continue
            n, pick, ps = prm
            if i % 32 == 0:                     # drop the diagrams the server has evicted
                live = set(srv.resident())
                ids = [d for d in ids if d in live]
                for d in [d for d in info if d not in live]:
                    del info[d]
            for attempt in range(8):            # a pick may have been evicted meanwhile
                if not ids:
                    break
                j = int(pick * len(ids)) if attempt == 0 else int(np.random.default_rng(ps + attempt).integers(
                    len(ids)))
                did = ids[j]
                W, H, k = info[did]
                pts = fresh_points(W, H, n, k, ps)
                try:
                    futs.append(srv.submit_insert(did, pts, arrival=at))
                except KeyError:
                    ids[j] = ids[-1]
                    ids.pop()
                    del info[did]
                    continue
                info[did] = (W, H, np.sort(np.concatenate([k, keys_of(W, pts)])))
                break
            else:
                failed_submit += 1
        srv.drain()
        t_end = time.monotonic()
        gc.enable()
        gc.unfreeze()
        lat, n_new, n_ins, errors = [], 0, 0, 0
        parts = {"new": ([], []), "insert": ([], [])}     # kind -> (queue wait ms, service ms)
        slow = []
        for f in futs:
            e = f.exception()
            if e is not None:
                errors += 1
                continue
            r = f.result()
            lat.append(r.latency * 1e3)
            n_new += r.kind == "new"
            n_ins += r.kind == "insert"
            parts[r.kind][0].append((r.start - r.arrival) * 1e3)
            parts[r.kind][1].append((r.done - r.start) * 1e3)
            slow.append((r.latency * 1e3, r.kind, dims.get(r.diagram_id), r.n_seeds,
                         (r.start - r.arrival) * 1e3, (r.done - r.start) * 1e3, r.arrival - t0))
        stats = {k: v - warm_stats.get(k, 0) for k, v in srv.stats.items()}
        mem = srv.memory_used()
        srv.close()
        lat.sort()

        def pct(q, v=lat):
            v = sorted(v)
            return v[min(len(v) - 1, int(q * len(v)))] if v else None

        breakdown = {k: {"wait_p50_ms": pct(0.5, w), "wait_p99_ms": pct(0.99, w), "service_p50_ms": pct(0.5, sv),
                         "service_p99_ms": pct(0.99, sv)} for k, (w, sv) in parts.items()}
        slow.sort(key=lambda x: -x[0])
        slowest = [{"ms": round(a, 2), "kind": b, "dims": c, "seeds": d, "wait_ms": round(e, 2),
                    "service_ms": round(f_, 2), "arrival_s": round(g, 3)} for a, b, c, d, e, f_, g in slow[:6]]

        return {"rate_req_s": rate, "requests": len(tr), "completed": len(lat), "new": n_new, "inserts": n_ins,
                "errors": errors, "not_submitted": failed_submit, "wall_s": t_end - t0,
                "throughput_req_s": len(lat) / (t_end - t0), "p50_ms": pct(0.5), "p99_ms": pct(0.99),
                "max_ms": lat[-1] if lat else None, "submit_lag_max_s": late, "memory_bytes_end": mem,
                "warmup_new_diagrams": len(warm), "objects": stats, "breakdown": breakdown, "slowest": slowest}

    # (2) saturated: the same fixed requests through the server and the plain loop
    reqs, meta = [], []
    for t, kind, prm in trace[:2000]:
        if kind == "new":
            W, H, n, ps = prm
            pts = uniform(W, H, n, seed=ps)
            meta.append((W, H, keys_of(W, pts)))
            reqs.append(("new", W, H, pts))
        else:
            n, pick, ps = prm
            news = [i for i, r in enumerate(reqs) if r[0] == "new"][-100:]
            if not news:
                continue
            j = news[int(pick * len(news))]
            W, H, k = meta[j]
            pts = fresh_points(W, H, n, k, ps)
            meta[j] = (W, H, np.sort(np.concatenate([k, keys_of(W, pts)])))
            meta.append(None)              # meta stays index-aligned with reqs
            reqs.append(("insert", j, pts))
    def saturate(n_slots, schedule=None, tile=None):
        torch.cuda.synchronize()
        srv = Server(budget_bytes=budget, slots=n_slots, border_padding=PADDING)
        if schedule is not None:
            srv.set_schedule(*schedule)
        if tile is not None:
            srv.set_tile(tile)
        t1 = time.perf_counter()
        fut_of = {}
        sfuts = []
        for i, r in enumerate(reqs):
            if r[0] == "new":
                f = srv.submit_new(r[1], r[2], r[3])
                fut_of[i] = f
            else:
                try:
                    f = srv.submit_insert(fut_of[r[1]].diagram_id, r[2])
                except KeyError:
                    continue
            sfuts.append(f)
        srv.drain()
        dt = time.perf_counter() - t1
        ok = sum(1 for f in sfuts if f.exception() is None)
        srv.close()
        return dt, ok

    saturate(slots)                         # warm-up, untimed: the device memory pool grows once
    # group propagation as tile rounds to convergence on cell lists (plain
    # launches, so workers overlap) against the default hybrid schedule
    variants = {}
    for name, sched, tile in (("groups_hybrid_tiles0", (1, -1), 0), ("groups_cells9", (-1, -1), 9),
                              ("groups_tiles0", (-1, -1), 0)):
        t_v, ok_v = saturate(slots, sched, tile)
        variants[name] = ok_v / t_v
    t_srv, srv_ok = saturate(slots)
    t_one, one_ok = saturate(1)
    t_pk, pk_ok = saturate(slots, (1, 1))      # inserts in the persistent kernel instead of tile rounds
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    out = run_serial(reqs, PADDING, budget)
    torch.cuda.synchronize()
    t_ser = time.perf_counter() - t1
    ser_ok = sum(1 for o in out if o[1] >= 0)
    saturated = {"requests": len(reqs), "slots": slots,
                 "server_s": t_srv, "server_req_s": srv_ok / t_srv, "server_ok": srv_ok,
                 "server_1slot_req_s": one_ok / t_one,
                 "server_insert_persistent_kernel_req_s": pk_ok / t_pk,
                 "serial_s": t_ser, "serial_req_s": ser_ok / t_ser, "serial_ok": ser_ok,
                 "speedup_vs_serial": (srv_ok / t_srv) / (ser_ok / t_ser),
                 "speedup_vs_1slot": (srv_ok / t_srv) / (one_ok / t_one),
                 "group_schedule_variants_req_s": variants}
    rt = [realtime(1000.0), realtime(500.0)]
    return {"workload": f"Poisson 1000 req/s for {seconds:g} s: 70% new (side log-U 128..4096, density "
                        f"0.05..1%), 30% inserts of 100..5000 seeds into resident diagrams; 40 GB budget; "
                        f"P={PADDING}, reference mode; results stay on the device",
            "realtime": rt[0], "realtime_500": rt[1], "saturated": saturated}


def run_ours(args, rank, world):
    import torch

    from integer_delauney_b200 import _capi
    from integer_delauney_b200 import _delauney_cuda as cu
    from integer_delauney_b200.workloads import clustered, uniform

    dev = rank % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    if args.incremental_only:
        print(json.dumps({"incremental": incremental_case(cu, torch, rank),
                          "incremental_exact": incremental_case(cu, torch, rank, "exact")}), flush=True)
        return
    lib = _capi.load()
    ctx = _capi.context_for(dev)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)

    def device_case(seeds_np):
        d_seeds = torch.from_numpy(seeds_np).cuda()
        d_out = torch.empty((H, W, 3), dtype=torch.int32, device="cuda")
        return d_seeds, d_out

    def step_device(d_seeds, d_out, mode=MODE):
        _capi.check(lib.idl_triangulate_device(ctx.handle, W, H, d_seeds.data_ptr(), d_seeds.shape[0], PADDING,
                                               _capi.mode_id(mode), d_out.data_ptr(), None))

    def time_device(seeds_np, steps, warmup, profile=False, mode=MODE):
        d_seeds, d_out = device_case(seeds_np)
        for _ in range(warmup):
            step_device(d_seeds, d_out, mode)
        ctx.set_profiling(profile)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        profs = []
        launches0 = lib.idl_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as clk:
            e0.record(stream)
            for _ in range(steps):
                step_device(d_seeds, d_out, mode)
                if profile:
                    profs.append(ctx.last_profile())
            e1.record(stream)
            torch.cuda.synchronize()
        launches = lib.idl_launch_count() - launches0
        ms = reduce_max(e0.elapsed_time(e1), world)
        ctx.set_profiling(False)
        return ms, profs, clk.summary(), launches

    seeds_u = uniform(W, H, N_SEEDS, seed=rank)
    if args.device_only and args.seeds == "clustered":
        seeds_u = clustered(W, H, N_SEEDS, seed=rank)
    # propagation schedule for this input class, picked by timing the
    # candidates (untimed; every schedule gives the same result)
    from integer_delauney_b200 import autotune
    if args.schedule is not None:
        schedule = (args.schedule, args.tile)
        autotune.apply(ctx, schedule)
    else:
        schedule = autotune.tune(W, H, seeds_u, PADDING, context=ctx)
    tuned_u = {f"{s},{t}": round(v, 3) for (s, t), v in autotune.last_report.items()}
    ctx.set_stream(stream.cuda_stream)
    # headline: K plain steps; the per-stage events are recorded in a second
    # timed run, since profiling reads counters back between stages
    head_mode = args.voronoi_mode if args.device_only else MODE
    ms, _, clocks, launches = time_device(seeds_u, args.steps, args.warmup, profile=False, mode=head_mode)
    value = world * W * H * args.steps / (ms / 1e3) / 1e6
    _, profs, _, _ = time_device(seeds_u, args.steps, 1, profile=True, mode=head_mode)

    # stage breakdown and roofline of the dominant stage
    keys = ["seeds_ms", "propagate_ms", "detect_ms", "dedup_ms", "assign_ms", "compose_ms"]
    stage = {k: statistics.mean(p[k] for p in profs) for k in keys}
    p0 = profs[-1]
    hbm, peak_kind = _peaks()
    # propagation: 8 B per cell update (4-byte label in, label out), counted
    # by the library over the tiles the schedule actually processed
    prop_bytes = statistics.mean(p["prop_bytes"] for p in profs)
    prop_gbs = prop_bytes / (stage["propagate_ms"] / 1e3) / 1e9
    canvas = p0["canvas_px"]
    detect_gbs = 4.0 * canvas / (stage["detect_ms"] / 1e3) / 1e9
    assign_gbs = 8.0 * W * H / (stage["assign_ms"] / 1e3) / 1e9
    compose_gbs = 20.0 * W * H / (stage["compose_ms"] / 1e3) / 1e9
    dominant = max(keys, key=lambda k: stage[k])
    roof = {"propagate_ms": prop_gbs, "detect_ms": detect_gbs, "assign_ms": assign_gbs,
            "compose_ms": compose_gbs}
    dom_kernel = dominant if dominant in roof else "propagate_ms"
    achieved = roof[dom_kernel]

    if args.device_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "Mpixel/s", "ms_per_step": ms / args.steps,
                              "voronoi_mode": head_mode,
                              "stages_ms": {k[:-3]: round(v, 4) for k, v in stage.items()},
                              "schedule": schedule, "autotune_ms": tuned_u, "passes": p0["passes"],
                              "sparse_pass_trace": ctx.pass_trace() if head_mode == "reference" else [],
                              "gpu_launches": int(launches),
                              "roofline_achieved_gbs": achieved, "clocks": clocks}), flush=True)
        return

    # clustered variant (same size), device path, with its own tuned schedule
    seeds_c = clustered(W, H, N_SEEDS, seed=rank)
    schedule_c = schedule if args.schedule is not None else autotune.tune(W, H, seeds_c, PADDING, context=ctx)
    tuned_c = {f"{s},{t}": round(v, 3) for (s, t), v in autotune.last_report.items()}
    ctx.set_stream(stream.cuda_stream)
    c_steps = max(1, args.steps // 2)
    ms_c, _, _, _ = time_device(seeds_c, c_steps, args.warmup)
    value_c = world * W * H * c_steps / (ms_c / 1e3) / 1e6
    _, profs_c, _, _ = time_device(seeds_c, c_steps, 1, profile=True)
    autotune.apply(ctx, schedule)

    # end to end through the public drop-in call, pinned host seeds
    pinned = torch.from_numpy(seeds_u).pin_memory()
    seeds_host = pinned.numpy()
    # warm up exactly as the timed loop runs, so that the pinned output
    # buffers the loop alternates between are already cached
    verts = grid = None
    for _ in range(max(2, args.warmup)):
        verts, grid = cu.triangulate(W, H, seeds_host, PADDING, as_arrays=True)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_tri = 0
    e_steps = max(1, args.steps)
    e0.record(stream)
    for _ in range(e_steps):
        verts, grid = cu.triangulate(W, H, seeds_host, PADDING, as_arrays=True)
        n_tri = len(verts)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e = reduce_max(e0.elapsed_time(e1), world)
    e2e = world * W * H * e_steps / (ms_e / 1e3) / 1e6

    inc = incremental_case(cu, torch, rank)
    inc_exact = incremental_case(cu, torch, rank, "exact")

    # the same 4096 x 4096 step in exact semantics (nearest seed, ties to the
    # higher id; history-independent), device-resident like the headline,
    # then its stages in a second, profiled run
    ms_x, _, _, _ = time_device(seeds_u, args.steps, args.warmup, mode="exact")
    ms_x /= args.steps
    _, profs_x, _, _ = time_device(seeds_u, args.steps, 1, profile=True, mode="exact")
    exact = {"workload": f"triangulate {W}x{H}, {N_SEEDS} uniform seeds, P={PADDING}, voronoi_mode=exact",
             "ms_per_step": ms_x, "mpix_s": world * W * H / (ms_x / 1e3) / 1e6,
             "stages_ms": {k[:-3]: round(statistics.mean(p[k] for p in profs_x), 4) for k in keys}}
    # the clustered seed set, exact semantics
    ms_xc, _, _, _ = time_device(seeds_c, c_steps, args.warmup, mode="exact")
    ms_xc /= c_steps
    _, profs_xc, _, _ = time_device(seeds_c, c_steps, 1, profile=True, mode="exact")
    exact["clustered_ms_per_step"] = ms_xc
    exact["clustered_mpix_s"] = world * W * H / (ms_xc / 1e3) / 1e6
    exact["clustered_stages_ms"] = {k[:-3]: round(statistics.mean(p[k] for p in profs_xc), 4) for k in keys}
    bat = batched_case(torch, lib, ctx, stream, rank)
    srv = serving_case(torch, rank, args.serve_seconds) if args.serve_seconds > 0 else None

    if rank != 0:
        return
    base = ref_cuda = None
    if not args.no_cpu_baseline:
        base = cpu_baseline(args.ref_rows)
        r = ref_cuda_baseline(seeds_u, 3)
        if r is not None:
            ms_r = statistics.median(r[0])
            ref_cuda = {"ms_per_call": ms_r, "mpix_s": W * H / (ms_r / 1e3) / 1e6, "calls": r[0],
                        "triangles": r[1], "what": REF_CUDA_DESC,
                        "ratio_e2e": (ms_r / (ms_e / e_steps)), "ratio_device": ms_r / (ms / args.steps)}
    if srv is not None:
        for k in ("realtime", "realtime_500"):
            print(json.dumps({"serving_" + k + "_slowest": srv[k].pop("slowest")}), file=sys.stderr, flush=True)
    line = {
        "metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"triangulate {W}x{H}, {N_SEEDS} uniform seeds (rng = rank), P={PADDING}, "
                               f"voronoi_mode={MODE}",
                   "global_batch": world, "parallelism": f"replicas x{world}",
                   "l2": "working set > L2 (label planes 2 x 68 MB, output 201 MB); no flush"},
        "stages_ms": {k[:-3]: round(v, 4) for k, v in stage.items()},
        "propagation": {"schedule_dense_rounds": schedule[0], "tile_shape": schedule[1], "autotune_ms": tuned_u,
                        "passes": p0["passes"],
                        "rounds": p0["rounds"],
                        "tiles": p0["tiles"],
                        "tile": [p0["tile_w"], p0["tile_h"]], "steps_per_round": p0["steps_per_round"]},
        "roofline": {"bound": "hbm", "kernel": dom_kernel[:-3], "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                     "traffic": TRAFFIC_PER_LAUNCH.get(dom_kernel),
                     "per_stage_gbs": {k[:-3]: v for k, v in roof.items()}},
        "clustered": {"value": value_c, "unit": "Mpixel/s", "ms_per_step": ms_c / c_steps,
                      "schedule": schedule_c, "autotune_ms": tuned_c, "passes": profs_c[-1]["passes"],
                      "rounds": profs_c[-1]["rounds"],
                      "stages_ms": {k[:-3]: round(statistics.mean(p[k] for p in profs_c), 4) for k in keys}},
        "e2e": {"value": e2e, "unit": "Mpixel/s", "ms_per_step": ms_e / e_steps,
                "h2d_bytes_per_step": int(seeds_u.nbytes),
                "d2h_bytes_per_step": int(W * H * 12 + n_tri * 20)},
        "incremental": inc,
        "incremental_exact": inc_exact,
        "exact": exact,
        "batched": bat,
        "serving": srv,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": base,
        "ref_cuda": ref_cuda,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-rows", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--device-only", action="store_true",
                    help="time only the device-resident 4096 x 4096 step (for profiler captures)")
    ap.add_argument("--schedule", type=int, default=None,
                    help="propagation schedule instead of the autotuned one (idl_context_set_schedule)")
    ap.add_argument("--tile", type=int, default=0, help="tile shape with --schedule (idl_context_set_tile)")
    ap.add_argument("--incremental-only", action="store_true",
                    help="time only the incremental workload (both semantics)")
    ap.add_argument("--seeds", choices=["uniform", "clustered"], default="uniform",
                    help="seed layout of the --device-only step")
    ap.add_argument("--voronoi-mode", choices=["reference", "exact"], default="reference",
                    help="propagation semantics of the --device-only step")
    ap.add_argument("--serve-seconds", type=float, default=10.0,
                    help="length of the real-time serving trace (0 skips the serving measurement)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
