"""GPU parity of the batch path (Voronoi, triangulate, GridTriangulation).

Every case runs the product through its C ABI (the drop-in Python layer) and
compares with the oracle on the same seeded input, bit for bit: labels,
squared distances, the triangle list (ids, witnesses and vertex order are
deterministic in both) and per-pixel triangle ids.  Where the reference's own
CUDA code was built (oracle/_ref), it is run on the same GPU and compared too.
"""
import numpy as np
import pytest

import oracle
from tests.conftest import clustered_seeds, random_seeds

pytestmark = pytest.mark.gpu

cu = pytest.importorskip("integer_delauney_b200._delauney_cuda")


def _tris_array(tm):
    return np.asarray([tm[k] for k in range(len(tm))], dtype=np.int32).reshape(-1, 5)


def _check_against_oracle(W, H, seeds, P, mode):
    s = oracle.sort_seeds(seeds, W, H)
    o_tris, o_grid, _ = oracle.triangulate(W, H, s, P, mode)
    tm, grid = cu.triangulate(W, H, seeds, P, voronoi_mode=mode)
    tris = _tris_array(tm)
    np.testing.assert_array_equal(grid[..., 0], o_grid[..., 0], err_msg="seed ids")
    np.testing.assert_array_equal(grid[..., 1], o_grid[..., 1], err_msg="squared distances")
    assert tris.shape == o_tris.shape
    np.testing.assert_array_equal(tris, o_tris, err_msg="triangle list")
    np.testing.assert_array_equal(grid[..., 2], o_grid[..., 2], err_msg="pixel triangle ids")


# ---------------------------------------------------------------------------
# stage (a)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("mode", ["reference", "numpy", "exact"])
@pytest.mark.parametrize("W,H,n,seed", [
    (5, 5, 1, 0), (5, 1, 2, 1), (1, 5, 2, 2), (10, 10, 3, 3), (33, 17, 20, 4), (64, 64, 20, 5),
    (128, 128, 400, 6), (100, 70, 300, 7), (257, 129, 700, 8), (512, 512, 2000, 0),
])
def test_voronoi_matches_oracle(mode, W, H, n, seed):
    seeds = random_seeds(W, H, n, seed)
    s = oracle.sort_seeds(seeds, W, H)
    want, passes = oracle.voronoi(mode, W, H, s)
    got = cu.Voronoi().compute(W, H, seeds, voronoi_mode=mode)
    assert got.shape == (H, W, 2) and got.dtype == np.int32
    np.testing.assert_array_equal(got, want)


def test_voronoi_clustered_matches_oracle():
    W = H = 384
    seeds = clustered_seeds(W, H, 3000, seed=3, blobs=6, sigma=12.0)
    s = oracle.sort_seeds(seeds, W, H)
    for mode in ("reference", "numpy", "exact"):
        want, _ = oracle.voronoi(mode, W, H, s)
        got = cu.Voronoi().compute(W, H, seeds, voronoi_mode=mode)
        np.testing.assert_array_equal(got, want)


def test_numpy_mode_equals_reference_numpy_golden(golden_dir):
    """voronoi_mode='numpy' is bit-equal to delauney.reference.Voronoi's output."""
    z = np.load(f"{golden_dir}/voronoi_numpy.npz")
    names = sorted({k.split("__")[0] for k in z.files})
    for name in names:
        W, H = (int(v) for v in z[f"{name}__wh"])
        seeds = z[f"{name}__seeds"]
        got = cu.Voronoi().compute(W, H, seeds, voronoi_mode="numpy")
        np.testing.assert_array_equal(got, z[f"{name}__grid"], err_msg=name)
        # on these inputs the NumPy reference also meets the exact contract
        got = cu.Voronoi().compute(W, H, seeds, voronoi_mode="exact")
        np.testing.assert_array_equal(got, z[f"{name}__grid"], err_msg=name + " (exact)")


# ---------------------------------------------------------------------------
# stages (a) + (b) + (d)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("mode", ["reference", "numpy", "exact"])
@pytest.mark.parametrize("W,H,n,seed,P", [
    (10, 10, 3, 1, 0), (30, 30, 4, 2, 16), (64, 64, 20, 3, 0), (64, 64, 40, 4, 16), (96, 80, 120, 5, 8),
    (200, 150, 600, 6, 16), (300, 200, 2000, 7, 32), (128, 96, 300, 8, 1),
])
def test_triangulate_matches_oracle(mode, W, H, n, seed, P):
    _check_against_oracle(W, H, random_seeds(W, H, n, seed), P, mode)


def test_triangulate_config1_matches_oracle():
    """The CPU configuration: 512 x 512, 2 000 uniform seeds (rng 0), P = 16."""
    _check_against_oracle(512, 512, random_seeds(512, 512, 2000, 0), 16, "reference")


def test_triangulate_clustered_matches_oracle():
    W = H = 320
    _check_against_oracle(W, H, clustered_seeds(W, H, 1500, seed=9, blobs=5, sigma=10.0), 16, "reference")


def test_grid_triangulation_with_caller_grid_at_zero_padding(golden_dir):
    """At P = 0 the caller's grid drives detection and fills channels 0/1."""
    z = np.load(f"{golden_dir}/triangulation_numpy.npz")
    names = sorted({k.split("__")[0] for k in z.files})
    for name in names:
        W, H, P = (int(v) for v in z[f"{name}__whp"])
        seeds = z[f"{name}__seeds"]
        vg = z[f"{name}__vgrid"]
        s = oracle.sort_seeds(seeds, W, H)
        o_tris, o_grid, _ = oracle.triangulate(W, H, s, 0, "numpy", vgrid=vg)
        tm, grid = cu.GridTriangulation().compute(vg, seeds, 0)
        np.testing.assert_array_equal(_tris_array(tm), o_tris, err_msg=name)
        np.testing.assert_array_equal(grid, o_grid, err_msg=name)


def test_as_arrays_and_dict_agree():
    W, H = 120, 90
    seeds = random_seeds(W, H, 150, 11)
    verts, g1 = cu.triangulate(W, H, seeds, as_arrays=True)
    tm, g2 = cu.triangulate(W, H, seeds)
    assert verts.shape == (len(tm), 3) and verts.dtype == np.int32
    for tid, (_x, _y, a, b, c) in tm.items():
        assert tuple(verts[tid]) == (a, b, c)
    np.testing.assert_array_equal(g1, g2)


def test_triangulate_equals_voronoi_plus_grid_triangulation():
    """triangulate == Voronoi + GridTriangulation (tests/test_triangulate.py:56-68)."""
    for (W, H, n, P) in [(64, 64, 20, -1), (128, 96, 60, 0), (256, 256, 500, 8), (300, 200, 2000, 32)]:
        seeds = random_seeds(W, H, n, W + n)
        vg = cu.Voronoi().compute(W, H, seeds)
        a_map, a_grid = cu.GridTriangulation().compute(vg, seeds, P)
        b_map, b_grid = cu.triangulate(W, H, seeds, P)
        assert a_map == b_map
        np.testing.assert_array_equal(a_grid, b_grid)


def test_compute_timed_and_debug():
    W, H = 100, 80
    seeds = random_seeds(W, H, 100, 12)
    vg = cu.Voronoi().compute(W, H, seeds)
    m, g, t = cu.GridTriangulation().compute_timed(vg, seeds)
    assert set(t) == {"detect_ms", "dedup_ms", "assign_ms"}
    assert all(v >= 0.0 for v in t.values())
    m2, g2, padded = cu.GridTriangulation().compute_debug(vg, seeds, 8)
    assert padded.shape == (H + 16, W + 16, 2)
    s = oracle.sort_seeds(seeds, W, H)
    want, _ = oracle.voronoi("reference", W + 16, H + 16, s + 8)
    np.testing.assert_array_equal(padded, want)


# ---------------------------------------------------------------------------
# errors (src/cuda/bindings/binding_helpers.hpp:23-46, triangulate.hpp:22-23)
# ---------------------------------------------------------------------------

def test_errors():
    with pytest.raises(ValueError, match="out of bounds"):
        cu.triangulate(10, 10, [(1, 1), (10, 3), (4, 4)])
    with pytest.raises(ValueError, match="empty"):
        cu.triangulate(10, 10, [])
    with pytest.raises(ValueError, match="duplicate"):
        cu.triangulate(10, 10, [(1, 1), (5, 5), (1, 1)])
    with pytest.raises(ValueError, match="positive"):
        cu.triangulate(0, 10, [(0, 0)])
    with pytest.raises(ValueError, match="out of bounds"):
        cu.Voronoi().compute(4, 4, [(10, 10)])
    with pytest.raises(ValueError, match="shape"):
        cu.GridTriangulation().compute(np.zeros((4, 4), np.int32), [(1, 1)])
    # out-of-bounds wins over duplicates, as in the reference's loop order
    with pytest.raises(ValueError, match="out of bounds"):
        cu.triangulate(10, 10, [(1, 1), (1, 1), (-1, 0)])
    # the context stays usable after errors
    tm, g = cu.triangulate(10, 10, [(1, 1), (8, 1), (4, 8)])
    assert g.shape == (10, 10, 3)


# ---------------------------------------------------------------------------
# the reference's own CUDA code, where it was built
# ---------------------------------------------------------------------------

ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@ref
@pytest.mark.parametrize("W,H,n,seed", [(64, 64, 20, 1), (128, 128, 400, 2), (512, 512, 2000, 0),
                                        (300, 200, 2000, 4)])
def test_voronoi_bit_exact_vs_reference_cuda(W, H, n, seed):
    seeds = random_seeds(W, H, n, seed)
    s = oracle.sort_seeds(seeds, W, H)
    want = oracle.ref_voronoi(W, H, s)
    got = cu.Voronoi().compute(W, H, seeds)
    np.testing.assert_array_equal(got, want)


@ref
@pytest.mark.parametrize("W,H,n,seed,P", [(64, 64, 20, 1, 0), (64, 64, 40, 2, 16), (256, 256, 500, 3, 8),
                                          (512, 512, 2000, 0, 16), (300, 200, 2000, 5, 32)])
def test_triangulate_vs_reference_cuda(W, H, n, seed, P):
    """Same Voronoi, same triangle set and numbering, same per-pixel ids.

    The reference's (x, y) witness and vertex order per triangle come from
    whichever duplicate its unstable sort kept, so those are compared as
    sorted triples; everything else bit for bit.
    """
    seeds = random_seeds(W, H, n, seed)
    s = oracle.sort_seeds(seeds, W, H)
    r_tris, r_grid, _ = oracle.ref_triangulate(W, H, s, P)
    tm, grid = cu.triangulate(W, H, seeds, P)
    tris = _tris_array(tm)
    assert len(tris) == len(r_tris)
    np.testing.assert_array_equal(np.sort(tris[:, 2:5], axis=1), np.sort(r_tris[:, 2:5], axis=1))
    np.testing.assert_array_equal(grid, r_grid)


def test_voronoi_large_canvas_matches_oracle():
    """A canvas large enough that the propagation kernel's per-block staging
    of next-pass work overflows into the global list in the early passes."""
    W, H = 8192, 4096
    seeds = random_seeds(W, H, 400_000, 12)
    s = oracle.sort_seeds(seeds, W, H)
    want, _ = oracle.voronoi("reference", W, H, s)
    got = cu.Voronoi().compute(W, H, seeds)
    np.testing.assert_array_equal(got, want)


@ref
@pytest.mark.parametrize("kind", ["uniform"])
def test_triangulate_4096_200k_vs_reference_cuda(kind):
    """The headline workload (4096 x 4096, 200 000 seeds, P = 16): grid bit
    for bit and the same triangle set as the reference's own CUDA path."""
    W = H = 4096
    seeds = random_seeds(W, H, 200_000, 0) if kind == "uniform" else clustered_seeds(W, H, 200_000, 0)
    s = oracle.sort_seeds(seeds, W, H)
    r_tris, r_grid, _ = oracle.ref_triangulate(W, H, s, 16)
    tm, grid = cu.triangulate(W, H, seeds, 16, as_arrays=True)
    assert len(tm) == len(r_tris)
    np.testing.assert_array_equal(np.sort(tm, axis=1), np.sort(r_tris[:, 2:5], axis=1))
    np.testing.assert_array_equal(grid, r_grid)


@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_propagation_schedules_agree(kind):
    """Tile rounds for the first passes and the persistent kernel for the
    tail, switched at any round, under every tile shape, give the Jacobi
    fixed point bit for bit; so does the Voronoi entry point, which has no
    padding."""
    from integer_delauney_b200 import _capi, autotune
    W, H = 700, 500
    seeds = random_seeds(W, H, 3000, 31) if kind == "uniform" else clustered_seeds(W, H, 3000, 31, blobs=5,
                                                                                     sigma=15.0)
    s = oracle.sort_seeds(seeds, W, H)
    o_tris, o_grid, _ = oracle.triangulate(W, H, s, 16)
    o_vor, _ = oracle.voronoi("reference", W, H, s)
    ctx = _capi.context_for(0)
    try:
        n_shapes = ctx.set_tile(0)
        assert n_shapes >= 4
        for sched, shape in autotune.candidates(n_shapes, (0, 1, 2, 5, -1)):
            ctx.set_schedule(sched)
            ctx.set_tile(shape)
            tm, grid = cu.triangulate(W, H, seeds, 16)
            np.testing.assert_array_equal(grid, o_grid, err_msg=f"schedule {sched}, tile {shape}")
            np.testing.assert_array_equal(_tris_array(tm), o_tris, err_msg=f"schedule {sched}, tile {shape}")
            np.testing.assert_array_equal(cu.Voronoi().compute(W, H, seeds), o_vor,
                                          err_msg=f"schedule {sched}, tile {shape}")
        choice = autotune.tune(W, H, seeds, 16, schedules=(0, 1, -1), repeats=1, context=ctx)
        assert choice in autotune.candidates(n_shapes, (0, 1, -1))
        with pytest.raises(ValueError):
            ctx.set_tile(n_shapes)
    finally:
        ctx.set_schedule(3)   # the context defaults
        ctx.set_tile(9)


def test_exact_mode_lattice_ties():
    """Seeds on a regular lattice make equidistant seeds everywhere (cells
    halfway between lattice rows, columns and diagonals): every tie must go to
    the higher id, in the column pass and across columns alike."""
    W, H = 301, 203
    xs, ys = np.meshgrid(np.arange(3, W, 6), np.arange(2, H, 4))
    seeds = np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)
    s = oracle.sort_seeds(seeds, W, H)
    want, _ = oracle.voronoi("exact", W, H, s)
    np.testing.assert_array_equal(cu.Voronoi().compute(W, H, seeds, voronoi_mode="exact"), want)


@pytest.mark.parametrize("W", [28000, 28001])
def test_exact_mode_row_pass_width_limit(W):
    """The lower-hull row pass handles canvases up to 28 000 columns; wider
    ones take the outward scan.  Both sides of the limit, a few rows, seeds
    with long empty stretches between them."""
    H = 3
    rng = np.random.default_rng(W)
    seeds = np.unique(np.stack([rng.integers(0, W, 40), rng.integers(0, H, 40)], 1), axis=0).astype(np.int32)
    s = oracle.sort_seeds(seeds, W, H)
    want, _ = oracle.voronoi("exact", W, H, s)
    np.testing.assert_array_equal(cu.Voronoi().compute(W, H, seeds, voronoi_mode="exact"), want)


@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_exact_mode_at_scale(kind):
    """Exact mode on a large canvas, dense and clustered (long scans through
    empty space), against the oracle's bucketed nearest-seed search; the
    result does not depend on the order the seeds are given in."""
    W, H = 1024, 768
    seeds = random_seeds(W, H, 8000, 41) if kind == "uniform" else clustered_seeds(W, H, 8000, 41, blobs=6,
                                                                                    sigma=25.0)
    s = oracle.sort_seeds(seeds, W, H)
    want, _ = oracle.voronoi("exact", W, H, s)
    got = cu.Voronoi().compute(W, H, seeds, voronoi_mode="exact")
    np.testing.assert_array_equal(got, want)
    perm = np.random.default_rng(0).permutation(len(seeds))
    np.testing.assert_array_equal(cu.Voronoi().compute(W, H, seeds[perm], voronoi_mode="exact"), want)
    o_tris, o_grid, _ = oracle.triangulate(W, H, s, 16, "exact")
    tm, grid = cu.triangulate(W, H, seeds, 16, voronoi_mode="exact")
    np.testing.assert_array_equal(grid, o_grid)
    np.testing.assert_array_equal(_tris_array(tm), o_tris)


def test_triangulate_device_equals_host_call_at_any_alignment():
    """idl_triangulate_device writes the same (H, W, 3) grid as the host call,
    whether the output pointer is 16-byte aligned (vector stores) or not, and
    nothing outside it."""
    import torch

    from integer_delauney_b200 import _capi
    W, H = 301, 77
    seeds = random_seeds(W, H, 500, 9)
    verts, grid = cu.triangulate(W, H, seeds, 16, as_arrays=True)
    tmap, grid_m = cu.triangulate(W, H, seeds, 16)
    # as_arrays' vertex triples (packed on the device) are the map's rows' ids
    np.testing.assert_array_equal(verts, np.array([tmap[t][2:5] for t in range(len(tmap))], dtype=np.int32))
    np.testing.assert_array_equal(grid, grid_m)
    lib = _capi.load()
    ctx = _capi.context_for(torch.cuda.current_device())
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    d_seeds = torch.from_numpy(np.ascontiguousarray(seeds, dtype=np.int32)).cuda()
    n = H * W * 3
    for off in (0, 1, 2, 3):
        buf = torch.full((n + 8,), -7, dtype=torch.int32, device="cuda")
        view = buf[off:off + n]
        _capi.check(lib.idl_triangulate_device(ctx.handle, W, H, d_seeds.data_ptr(), len(seeds), 16,
                                               _capi.MODE_REFERENCE, view.data_ptr(), None))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(view.cpu().numpy().reshape(H, W, 3), grid, err_msg=f"offset {off}")
        assert bool((buf[:off] == -7).all()) and bool((buf[off + n:] == -7).all())


@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_tail_rounds_agree(kind):
    """The persistent kernel's round mode (several Jacobi passes per grid
    barrier once its work list is short) gives the one-pass schedule's fixed
    point and pass count bit for bit: never, late, by default and from the
    first pass, from scratch and after tile rounds."""
    from integer_delauney_b200 import _capi
    W, H, P = 600, 420, 16
    seeds = random_seeds(W, H, 2500, 33) if kind == "uniform" else clustered_seeds(W, H, 2500, 33, blobs=4,
                                                                                     sigma=14.0)
    s = oracle.sort_seeds(seeds, W, H)
    o_tris, o_grid, _ = oracle.triangulate(W, H, s, P)
    _, o_passes = oracle.voronoi("reference", W + 2 * P, H + 2 * P, s + P)
    ctx = _capi.context_for(0)
    try:
        for sched, shape in ((0, 0), (3, 9), (1, 2)):
            ctx.set_schedule(sched)
            ctx.set_tile(shape)
            for rb in (0, 16, 4096, 1 << 30):
                ctx.set_tail_rounds(rb)
                ctx.set_profiling(True)
                tm, grid = cu.triangulate(W, H, seeds, P)
                passes = int(ctx.last_profile()["passes"])
                ctx.set_profiling(False)
                msg = f"schedule {sched}, tile {shape}, tail rounds below {rb}"
                np.testing.assert_array_equal(grid, o_grid, err_msg=msg)
                np.testing.assert_array_equal(_tris_array(tm), o_tris, err_msg=msg)
                assert passes == o_passes, msg
    finally:
        ctx.set_profiling(False)
        ctx.set_tail_rounds(4096)   # the context defaults
        ctx.set_schedule(3)
        ctx.set_tile(9)
