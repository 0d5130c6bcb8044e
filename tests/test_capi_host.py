"""Host-side checks that need no GPU: the C ABI library's symbol table, the
drop-in layer's argument handling, the workload generators and the
multi-rank timing reduction of bench.py (gloo, world size 2)."""
import os
import re
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names.update(re.findall(r"^IDL_API\s+[\w\s\*]+?\b(idl_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    from integer_delauney_b200 import _capi
    lib = _capi.load()                       # loads without a GPU: no CUDA call is made
    declared = _declared_symbols()
    assert len(declared) >= 14
    for name in sorted(declared):
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(_capi.SIGNATURES) == declared, "ctypes signatures out of step with the header"
    assert lib.idl_version() >= 100
    assert lib.idl_launch_count() >= 0


def test_last_error_is_empty_before_any_failure():
    from integer_delauney_b200 import _capi
    assert isinstance(_capi.last_error(), str)


def test_status_codes_map_to_reference_exception_types():
    from integer_delauney_b200 import _capi
    _capi.check(_capi.IDL_OK)
    with pytest.raises(ValueError):
        _capi.check(_capi.IDL_ERR_INVALID)
    for st in (_capi.IDL_ERR_CUDA, _capi.IDL_ERR_STATE, _capi.IDL_ERR_INTERNAL):
        with pytest.raises(RuntimeError):
            _capi.check(st)
    with pytest.raises(MemoryError):            # serving: never fits the memory budget
        _capi.check(_capi.IDL_ERR_BUDGET)
    with pytest.raises(KeyError):               # serving: diagram not resident
        _capi.check(_capi.IDL_ERR_NOT_RESIDENT)


def test_server_clock_is_the_monotonic_clock():
    """Request timestamps are comparable with time.monotonic() (arrival
    times a client passes in)."""
    import time
    from integer_delauney_b200 import _capi
    lib = _capi.load()
    a = time.monotonic_ns()
    b = lib.idl_server_clock_ns()
    c = time.monotonic_ns()
    assert a - 1_000_000 <= b <= c + 1_000_000


def test_server_rejects_bad_arguments_before_touching_a_device():
    import ctypes
    from integer_delauney_b200 import _capi
    lib = _capi.load()
    h = ctypes.c_void_p()
    for slots, budget, mode in ((0, 1 << 30, 0), (65, 1 << 30, 0), (1, 0, 0), (1, 1 << 30, 1)):
        assert lib.idl_server_create(0, budget, slots, 16, mode, ctypes.byref(h)) == _capi.IDL_ERR_INVALID
        assert h.value is None
    assert lib.idl_server_destroy(None) == _capi.IDL_OK
    assert lib.idl_server_drain(None) == _capi.IDL_ERR_INVALID


def test_mode_names():
    from integer_delauney_b200 import _capi
    assert _capi.mode_id("reference") == 0 and _capi.mode_id("numpy") == 1 and _capi.mode_id("exact") == 2
    with pytest.raises(ValueError):
        _capi.mode_id("fast")


class TestParseSeeds:
    def setup_method(self):
        from integer_delauney_b200 import _delauney_cuda
        self.parse = _delauney_cuda.parse_seeds

    def test_list_of_tuples(self):
        a = self.parse([(1, 2), (3, 4)])
        assert a.dtype == np.int32 and a.shape == (2, 2) and a.flags.c_contiguous
        assert a.tolist() == [[1, 2], [3, 4]]

    def test_array_fast_path_and_generators(self):
        src = np.array([[5, 6], [7, 8]], dtype=np.int64)
        assert self.parse(src).tolist() == [[5, 6], [7, 8]]
        assert self.parse((p for p in [(1, 1)])).tolist() == [[1, 1]]
        assert self.parse([]).shape == (0, 2)

    def test_out_of_int32_maps_to_out_of_bounds(self):
        a = self.parse([(2**40, 3)])
        assert a[0, 0] == -1

    def test_bad_shapes(self):
        with pytest.raises(TypeError):
            self.parse([(1, 2, 3)])
        with pytest.raises(TypeError):
            self.parse([(1.5, 2)])


def test_padding_resolution_matches_reference():
    """binding_helpers.hpp:49-53 (-1 -> 16) and reference/triangulation.py:78 (clamp)."""
    from integer_delauney_b200 import _delauney_cuda
    r = _delauney_cuda.resolve_padding
    assert r(-1) == 16 and r(0) == 0 and r(5) == 5 and r(-5) == 0


class TestMaxBoundarySpacing:
    """tests/test_border_padding.py:37-53."""

    def test_inverts_the_bound(self):
        from integer_delauney_b200 import max_boundary_spacing
        for p in (1, 2, 8, 16, 32, 128, 10**6):
            s = max_boundary_spacing(p)
            assert s * s / 8 <= p and (s + 1) ** 2 / 8 > p

    def test_defaults(self):
        import integer_delauney_b200 as d
        assert d.DEFAULT_BORDER_PADDING == 16
        assert d.max_boundary_spacing(d.DEFAULT_BORDER_PADDING) >= 8
        assert d.max_boundary_spacing(0) == 0 and d.max_boundary_spacing(-1) == 0
        assert set(d.__all__) >= {"triangulate", "Voronoi", "GridTriangulation", "Delaunay",
                                  "DEFAULT_BORDER_PADDING", "max_boundary_spacing"}


def test_build_output_dict_and_arrays():
    from integer_delauney_b200._delauney_cuda import build_output
    tris = np.array([[1, 2, 0, 1, 2], [3, 4, 1, 2, 3]], dtype=np.int32)
    grid = np.zeros((2, 2, 3), np.int32)
    m, g = build_output(tris, grid, False)
    assert m == {0: (1, 2, 0, 1, 2), 1: (3, 4, 1, 2, 3)} and g is grid
    v, _ = build_output(tris, grid, True)
    assert v.tolist() == [[0, 1, 2], [1, 2, 3]] and v.dtype == np.int32


def test_workloads_are_distinct_and_seeded():
    from integer_delauney_b200 import workloads
    a = workloads.uniform(200, 100, 500, seed=1)
    b = workloads.uniform(200, 100, 500, seed=1)
    assert np.array_equal(a, b) and a.shape == (500, 2)
    assert len({(int(x), int(y)) for x, y in a}) == 500
    assert a[:, 0].max() < 200 and a[:, 1].max() < 100 and a.min() >= 0
    c = workloads.clustered(512, 512, 3000, seed=2, blobs=4, sigma=20.0)
    assert len({(int(x), int(y)) for x, y in c}) == 3000
    imgs = workloads.batched_images(8, seed=3)
    for W, H, s in imgs:
        assert 64 <= W <= 1024 and 64 <= H <= 1024
        assert 0.001 * W * H - 1 <= len(s) <= 0.02 * W * H + 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    out[rank] = bench.reduce_max(10.0 + rank, world)
    dist.destroy_process_group()


def test_bench_reduces_time_as_max_over_ranks():
    """The multi-GPU bench times each rank on its own device and reports the
    slowest; the reduction itself is plain torch.distributed (gloo here)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    assert out[0] == 11.0 and out[1] == 11.0
