"""Failure detection on the device without a GPU fault.

The persistent propagation kernel separates its passes with a grid-wide
barrier whose every wait is bounded; a wait that runs out raises the kernel's
error flag, every block returns, and the host reports IDL_ERR_INTERNAL
("grid barrier timed out").  idl_selftest_grid_barrier runs that barrier on
its own with a short poll limit and, on request, arrivals that never come (a
count nothing completes), so the wait really runs out.  No trap, assert, bad
address or endless loop is involved; the context must stay usable.
"""
import ctypes

import numpy as np
import pytest

import oracle
from integer_delauney_b200.workloads import uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from integer_delauney_b200 import _capi
    return _capi


def triangulate_on(capi, ctx, W, H, seeds):
    lib = capi.load()
    out = np.empty((H, W, 3), dtype=np.int32)
    n_tri = ctypes.c_int64(0)
    s = np.ascontiguousarray(seeds, dtype=np.int32)
    capi.check(lib.idl_triangulate(ctx.handle, W, H, s.ctypes.data, len(s), None, 16, capi.MODE_REFERENCE,
                                   out.ctypes.data, ctypes.byref(n_tri), None, None))
    return out


def test_barrier_completes_when_every_block_arrives(capi):
    ctx = capi.Context(0)
    assert capi.load().idl_selftest_grid_barrier(ctx.handle, 0, 1 << 20) == capi.IDL_OK


@pytest.mark.parametrize("missing", [1, 7])
def test_barrier_wait_runs_out_and_the_context_survives(capi, missing):
    lib = capi.load()
    ctx = capi.Context(0)
    rc = lib.idl_selftest_grid_barrier(ctx.handle, missing, 1 << 12)
    assert rc == capi.IDL_ERR_INTERNAL
    assert "grid barrier timed out" in capi.last_error()
    # the same context and device still work: the barrier completes again and
    # a triangulation through the persistent kernel equals the oracle
    assert lib.idl_selftest_grid_barrier(ctx.handle, 0, 1 << 20) == capi.IDL_OK
    W, H = 300, 200
    seeds = uniform(W, H, 900, seed=missing)
    got = triangulate_on(capi, ctx, W, H, seeds)
    _, want, _ = oracle.triangulate(W, H, oracle.sort_seeds(seeds, W, H), 16, "reference")
    np.testing.assert_array_equal(got, want)


def test_selftest_rejects_bad_arguments(capi):
    lib = capi.load()
    ctx = capi.Context(0)
    assert lib.idl_selftest_grid_barrier(ctx.handle, -1, 100) == capi.IDL_ERR_INVALID
    assert lib.idl_selftest_grid_barrier(ctx.handle, 0, 0) == capi.IDL_ERR_INVALID
    assert lib.idl_selftest_grid_barrier(None, 0, 100) == capi.IDL_ERR_INVALID
