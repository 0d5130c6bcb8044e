"""The allocation-free Voronoi entry point (idl_voronoi_noalloc).

It exists for callers that cannot call cudaMalloc -- code on a latency budget
that an allocation's stall or device synchronisation would break, processes
held to a fixed device-memory quota or pool, hosts embedding the library under
their own allocator.  Its workspace is one static device array shared by every
call, so this checks, through the C ABI, that two calls in a row on different
inputs each reproduce what the ordinary entry point (idl_voronoi, via
Voronoi().compute) and the CPU oracle return, bit for bit -- the second call
must not see anything the first one left in the shared array -- and that
once the device's array is set up a call makes no allocation at all (the
library's own allocation counter, idl_alloc_count, does not move).

Kept in a file of its own that pytest collects last, so that a run stopping at
the first failure has already run every other test; it passes alone in a fresh
process as well as after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

import oracle
from tests.conftest import random_seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
cu = pytest.importorskip("integer_delauney_b200._delauney_cuda")
from integer_delauney_b200 import _capi  # noqa: E402


def _noalloc(W, H, seeds, mode):
    lib = _capi.load()
    d_seeds = torch.from_numpy(np.ascontiguousarray(seeds, dtype=np.int32)).cuda()
    d_out = torch.empty((H, W, 2), dtype=torch.int32, device="cuda")
    passes = ctypes.c_int64(0)
    stream = torch.cuda.current_stream().cuda_stream
    _capi.check(lib.idl_voronoi_noalloc(W, H, d_seeds.data_ptr(), len(seeds), _capi.mode_id(mode),
                                        d_out.data_ptr(), ctypes.c_void_p(stream), ctypes.byref(passes)))
    torch.cuda.current_stream().synchronize()
    return d_out.cpu().numpy(), int(passes.value)


@pytest.mark.parametrize("mode", ["reference", "numpy"])
def test_noalloc_matches_voronoi_on_two_calls_in_a_row(mode):
    lib = _capi.load()
    cases = [(512, 512, 2000, 0), (300, 200, 900, 1)]   # the second call is smaller than the first
    for i, (W, H, n, seed) in enumerate(cases):
        seeds = random_seeds(W, H, n, seed)
        want = cu.Voronoi().compute(W, H, seeds, voronoi_mode=mode)
        a0 = lib.idl_alloc_count()
        got, passes = _noalloc(W, H, seeds, mode)
        if i > 0:       # the first call on a device may set up its workspace view
            assert lib.idl_alloc_count() == a0, "the no-allocation entry point allocated"
        np.testing.assert_array_equal(got, want)
        o, _ = oracle.voronoi(mode, W, H, oracle.sort_seeds(seeds, W, H))
        np.testing.assert_array_equal(got, o)
        assert passes >= 1


def test_noalloc_rejects_sizes_beyond_its_workspace():
    lib = _capi.load()
    d_seeds = torch.zeros((1, 2), dtype=torch.int32, device="cuda")
    d_out = torch.empty((2, 2), dtype=torch.int32, device="cuda")
    rc = lib.idl_voronoi_noalloc(2048, 16, d_seeds.data_ptr(), 1, 0, d_out.data_ptr(), None, None)
    assert rc == _capi.IDL_ERR_INVALID
    assert "1024" in _capi.last_error()
