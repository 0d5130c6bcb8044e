"""The CPU oracle pinned against the reference (no GPU needed).

Golden vectors in tests/golden/ were produced by the reference's own NumPy
implementation (tests/golden/make_golden.py).  The known-answer cases restate
the expectations of the reference's test files, cited per test.
"""
import numpy as np
import pytest

import oracle
from tests.conftest import random_seeds


def _load(golden_dir, name):
    z = np.load(f"{golden_dir}/{name}")
    cases = sorted({k.split("__")[0] for k in z.files})
    return z, cases


# ---------------------------------------------------------------------------
# stage (a)
# ---------------------------------------------------------------------------

def test_sweep_oracle_equals_numpy_reference(golden_dir):
    """or_voronoi_sweep restates reference/voronoi.py:90-163 bit for bit."""
    z, cases = _load(golden_dir, "voronoi_numpy.npz")
    for c in cases:
        W, H = (int(v) for v in z[f"{c}__wh"])
        s = oracle.sort_seeds(z[f"{c}__seeds"], W, H)
        got, _ = oracle.voronoi("numpy", W, H, s)
        np.testing.assert_array_equal(got, z[f"{c}__grid"], err_msg=c)


def test_nearest_oracle_equals_numpy_reference(golden_dir):
    """The NumPy reference equals exact nearest-with-higher-id on every golden case."""
    z, cases = _load(golden_dir, "voronoi_numpy.npz")
    for c in cases:
        W, H = (int(v) for v in z[f"{c}__wh"])
        s = oracle.sort_seeds(z[f"{c}__seeds"], W, H)
        got, _ = oracle.voronoi("exact", W, H, s)
        np.testing.assert_array_equal(got, z[f"{c}__grid"], err_msg=c)


@pytest.mark.parametrize("name", ["single", "row_pair", "col_pair", "three", "four_square", "four_corners"])
def test_jacobi_oracle_on_reference_cuda_fixtures(golden_dir, name):
    """tests/test_voronoi_cuda.py:55-70: on these grids the reference CUDA
    Jacobi and the NumPy reference are element-wise identical."""
    z, _ = _load(golden_dir, "voronoi_numpy.npz")
    W, H = (int(v) for v in z[f"{name}__wh"])
    s = oracle.sort_seeds(z[f"{name}__seeds"], W, H)
    got, passes = oracle.voronoi("reference", W, H, s)
    np.testing.assert_array_equal(got, z[f"{name}__grid"])
    assert passes >= 1


def test_jacobi_differs_from_nearest_only_where_documented():
    """API_REFERENCE.md:101 / reference/voronoi.py:21-28: the CUDA fixed point
    is non-nearest at a small fraction of pixels, never closer than nearest."""
    W = H = 128
    s = oracle.sort_seeds(random_seeds(W, H, 400, 2), W, H)
    jac, _ = oracle.voronoi("reference", W, H, s)
    near, _ = oracle.voronoi("exact", W, H, s)
    diff = jac[..., 1] != near[..., 1]
    assert np.all(jac[..., 1] >= near[..., 1])
    assert 0 < diff.sum() < 0.01 * W * H


def test_jacobi_pass_count_matches_its_definition():
    """Passes = last changing pass + 1 (voronoi.cu:100-113 stops after a quiet pass)."""
    W, H = 64, 48
    s = oracle.sort_seeds(random_seeds(W, H, 30, 5), W, H)
    xs, ys = s[:, 0].copy(), s[:, 1].copy()
    lab = np.full((H, W), -1, np.int32)
    lab[ys, xs] = np.arange(len(s), dtype=np.int32)
    _, passes = oracle.jacobi_from(W, H, xs, ys, lab)
    # run one pass less from scratch: it must not have converged yet
    grid, p2 = oracle.voronoi("reference", W, H, s)
    assert p2 == passes


class TestVoronoiKnownAnswers:
    """tests/test_voronoi_ref.py:29-137 restated against every oracle mode."""

    @pytest.mark.parametrize("mode", ["reference", "numpy", "exact"])
    def test_squared_l2(self, mode):
        g, _ = oracle.voronoi(mode, 5, 5, oracle.sort_seeds([(2, 2)], 5, 5))
        yy, xx = np.mgrid[0:5, 0:5]
        np.testing.assert_array_equal(g[..., 1], (xx - 2) ** 2 + (yy - 2) ** 2)
        assert np.all(g[..., 0] == 0)

    @pytest.mark.parametrize("mode", ["reference", "numpy", "exact"])
    def test_id_order_and_ties(self, mode):
        g, _ = oracle.voronoi(mode, 5, 1, oracle.sort_seeds([(3, 0), (1, 0)], 5, 1))
        assert g[0, 1, 0] == 0 and g[0, 3, 0] == 1
        g, _ = oracle.voronoi(mode, 5, 1, oracle.sort_seeds([(0, 0), (4, 0)], 5, 1))
        assert list(g[0, :, 0]) == [0, 0, 1, 1, 1]      # tie at x=2 -> higher id
        assert list(g[0, :, 1]) == [0, 1, 4, 1, 0]
        g, _ = oracle.voronoi(mode, 5, 5, oracle.sort_seeds([(0, 2), (2, 0), (4, 2)], 5, 5))
        assert g[2, 2, 0] == 2                           # three-way tie -> highest id
        g, _ = oracle.voronoi(mode, 4, 4, oracle.sort_seeds([(0, 0)], 4, 4))
        assert g[3, 3, 1] == 18

    def test_errors(self):
        with pytest.raises(ValueError, match="empty"):
            oracle.sort_seeds([], 4, 4)
        with pytest.raises(ValueError, match="out of bounds"):
            oracle.sort_seeds([(10, 10)], 4, 4)
        with pytest.raises(ValueError, match="duplicate"):
            oracle.sort_seeds([(2, 2), (2, 2)], 5, 5)


# ---------------------------------------------------------------------------
# stages (b) and (d)
# ---------------------------------------------------------------------------

def _triplets(tris):
    return {tuple(sorted(int(v) for v in r[2:5])) for r in tris}


def _inside(p, tri, pts):
    a, b, c = (pts[i] for i in tri)

    def cr(o, u, v):
        return (u[0] - o[0]) * (v[1] - o[1]) - (u[1] - o[1]) * (v[0] - o[0])

    d = [cr(p, a, b), cr(p, b, c), cr(p, c, a)]
    return not (min(d) < 0 < max(d))


def _numpy_blocked(W, H, P, s):
    """Triples reference/triangulation.py:109-144 blocks globally: for every
    2x2 block of four distinct ids, the two triples of the rejected diagonal."""
    if P > 0:
        lab, _ = oracle.voronoi("numpy", W + 2 * P, H + 2 * P, s + P)
        lab = lab[..., 0]
    else:
        lab, _ = oracle.voronoi("numpy", W, H, s)
        lab = lab[..., 0]
    xs, ys = (s[:, 0] + P).astype(np.int32), (s[:, 1] + P).astype(np.int32)
    blocked = set()
    tl, tr, bl, br = lab[:-1, :-1], lab[:-1, 1:], lab[1:, :-1], lab[1:, 1:]
    quad = (tl != tr) & (tl != bl) & (tl != br) & (tr != bl) & (tr != br) & (bl != br)
    for y, x in zip(*np.nonzero(quad)):
        ids = [int(tl[y, x]), int(tr[y, x]), int(bl[y, x]), int(br[y, x])]
        chosen = {tuple(sorted(t)) for t in oracle.block_rule(*ids, xs, ys)}
        for k in range(4):
            t = tuple(sorted(ids[:k] + ids[k + 1:]))
            if t not in chosen:
                blocked.add(t)
    return blocked


def test_triangles_equal_numpy_reference(golden_dir):
    """Same Voronoi grid -> the triangle set of reference/triangulation.py,
    except triples that the NumPy path blocks globally as the rejected
    diagonal of some cocircular quad but a 3-region block elsewhere still
    witnesses: the CUDA rule (triangle_detect.cuh:75-166), which this library
    follows, emits those.

    Pixel ids are compared through the triangles' vertex triples (the NumPy
    reference numbers by discovery order, the CUDA path by sorted triple); a
    pixel may differ only where it lies inside both triangles (a shared edge
    or vertex: tests/test_incremental_padding.py:471-499 makes the same cut).
    """
    z, cases = _load(golden_dir, "triangulation_numpy.npz")
    for c in cases:
        W, H, P = (int(v) for v in z[f"{c}__whp"])
        seeds = z[f"{c}__seeds"]
        s = oracle.sort_seeds(seeds, W, H)
        tris, grid, _ = oracle.triangulate(W, H, s, P, "numpy", vgrid=z[f"{c}__vgrid"])
        ref = z[f"{c}__tris"]
        mine, theirs = _triplets(tris), _triplets(ref)
        assert theirs <= mine, c
        assert mine - theirs <= _numpy_blocked(W, H, P, s), c
        np.testing.assert_array_equal(grid[..., :2], z[f"{c}__tgrid"][..., :2], err_msg=c)
        lut_r = {i: tuple(sorted(int(v) for v in r[2:5])) for i, r in enumerate(ref)}
        lut_m = {i: tuple(sorted(int(v) for v in r[2:5])) for i, r in enumerate(tris)}
        pts = s.tolist()
        rt, mt = z[f"{c}__tgrid"][..., 2], grid[..., 2]
        for y, x in zip(*np.nonzero((rt >= 0) != (mt >= 0))):
            pytest.fail(f"{c}: pixel ({x},{y}) covered by one side only")
        for y, x in zip(*np.nonzero(rt >= 0)):
            a, b = lut_r[int(rt[y, x])], lut_m[int(mt[y, x])]
            if a != b:
                assert _inside((x, y), a, pts) and _inside((x, y), b, pts), (c, x, y)


def test_triangle_ids_are_sorted_triple_ranks():
    """triangulation.cu:254-256: tid = rank of the sorted vertex triple."""
    W, H = 96, 80
    s = oracle.sort_seeds(random_seeds(W, H, 120, 14), W, H)
    tris, _, _ = oracle.triangulate(W, H, s, 16, "reference")
    keys = [tuple(sorted(int(v) for v in r[2:5])) for r in tris]
    assert keys == sorted(keys) and len(set(keys)) == len(keys)


def test_block_rule():
    """triangle_detect.cuh:75-166: 3 distinct -> one triangle in first-seen
    order; 4 distinct -> the two triangles of one diagonal; any -1 -> none."""
    xs = np.array([0, 10, 0, 10, 5], np.int32)
    ys = np.array([0, 0, 10, 10, 20], np.int32)
    assert oracle.block_rule(1, 0, 1, 2, xs, ys) == [(1, 0, 2)]
    assert oracle.block_rule(0, 0, 0, 1, xs, ys) == []
    assert oracle.block_rule(0, -1, 1, 2, xs, ys) == []
    # square (0,0),(10,0),(0,10),(10,10): equal diagonals -> avoid the lowest id 0
    out = oracle.block_rule(0, 1, 2, 3, xs, ys)
    assert len(out) == 2
    shared = set(out[0]) & set(out[1])
    assert shared == {1, 2}


@pytest.mark.parametrize("quad", [
    [(60, 60), (180, 60), (60, 180), (180, 180)],
    [(60, 80), (200, 80), (200, 170), (60, 170)],
    [(80, 128), (128, 80), (176, 128), (128, 176)],
])
def test_cocircular_quads_give_two_triangles(quad):
    """tests/test_scipy_oracle.py:409-443: one diagonal, two triangles."""
    W = H = 256
    s = oracle.sort_seeds(quad, W, H)
    tris, _, _ = oracle.triangulate(W, H, s, 0, "exact")
    t = sorted(_triplets(tris))
    assert len(t) == 2 and len(set(t[0]) & set(t[1])) == 2


@pytest.mark.parametrize("name,W,H,seeds", [
    ("3-seeds-triangle", 30, 30, [(3, 3), (25, 5), (14, 25)]),
    ("4-seeds-quad", 30, 30, [(3, 3), (26, 3), (3, 26), (26, 26)]),
    ("grid-9-seeds", 40, 40, [(5, 5), (20, 3), (35, 5), (3, 20), (20, 20), (37, 20), (5, 35), (20, 37), (35, 35)]),
])
def test_every_pixel_in_its_max_tid_triangle(name, W, H, seeds):
    """tests/test_pixel_assignment_correctness.py:16-66: every pixel gets the
    highest id among the detected triangles containing it, else -1."""
    s = oracle.sort_seeds(seeds, W, H)
    tris, grid, _ = oracle.triangulate(W, H, s, 16, "reference")
    pts = s.tolist()
    for y in range(H):
        for x in range(W):
            best = -1
            for tid, r in enumerate(tris):
                if _inside((x, y), tuple(int(v) for v in r[2:5]), pts):
                    best = tid
            assert grid[y, x, 2] == best, (name, x, y)


def test_collinear_triangle_covers_its_line_within_the_window():
    """A detected collinear triple passes the closed test on its whole line
    (geometry_device.cuh:68-86 with all cross products 0); the reference
    reaches it only through seeds within window_cap (triangulation.cu:121-134)."""
    W, H = 64, 40
    seeds = [(5, 5), (10, 10), (15, 15), (50, 30)]
    s = oracle.sort_seeds(seeds, W, H)
    lab = np.full((H, W), 2, np.int32)
    lab[:20, :32] = 0
    lab[:20, 32:] = 1                               # only block (31, 19) sees ids 0, 1, 2 (collinear)
    xs, ys = s[:, 0].copy(), s[:, 1].copy()
    tris = oracle.detect(lab, xs, ys, 0)
    assert _triplets(tris) == {(0, 1, 2)}
    t = oracle.assign(W, H, xs, ys, tris)
    wc = oracle.window_cap(tris, xs, ys)
    on_line = np.zeros((H, W), bool)
    for k in range(min(W, H)):
        if max(abs(k - 5), abs(k - 5)) <= wc or max(abs(k - 15), abs(k - 15)) <= wc:
            on_line[k, k] = True
    np.testing.assert_array_equal(t == 0, on_line)


@pytest.mark.parametrize("W,H,n,kind", [(200, 150, 300, "uniform"), (512, 512, 2000, "uniform"),
                                        (300, 300, 500, "clustered"), (97, 61, 40, "uniform")])
def test_bounding_box_assignment_equals_windowed(W, H, n, kind):
    """assign_bbox (per triangle over its bounding box) is the reference's
    windowed per-pixel assignment (triangulation.cu:101-137) evaluated in
    another order: same grid, whole and by row bands."""
    from integer_delauney_b200.workloads import clustered, uniform
    seeds = uniform(W, H, n, seed=n) if kind == "uniform" else clustered(W, H, n, seed=n, blobs=4, sigma=10.0)
    s = oracle.sort_seeds(seeds, W, H)
    tris, grid, _ = oracle.triangulate(W, H, s, 16)
    want = oracle.assign(W, H, s[:, 0], s[:, 1], tris)
    np.testing.assert_array_equal(want, grid[:, :, 2])
    np.testing.assert_array_equal(oracle.assign_bbox(W, H, s[:, 0], s[:, 1], tris), want)
    y0, y1 = H // 3, H // 3 + 7
    np.testing.assert_array_equal(oracle.assign_bbox(W, H, s[:, 0], s[:, 1], tris, y0, y1), want[y0:y1])


def test_bounding_box_assignment_covers_collinear_triangles_like_the_window():
    """A collinear triangle passes the reference's closed test along its whole
    supporting line, within the seed window (triangulation.cu:101-137); the
    bounding-box form must give it the same pixels.  This incremental case
    holds such a triangle (seeds (220, 38), (221, 39), (222, 40))."""
    from integer_delauney_b200.workloads import uniform
    W, H, P = 300, 200, 16
    seeds = uniform(W, H, 2000, seed=2016)
    o = oracle.incremental(W, H, [seeds[i:i + 500] for i in range(0, 2000, 500)], P)
    order = np.lexsort((o["ys"], o["xs"]))
    sx, sy = o["xs"][order], o["ys"][order]
    t = o["tris"]
    v = t[:, 2:5]
    area = (sx[v[:, 1]] - sx[v[:, 0]]).astype(np.int64) * (sy[v[:, 2]] - sy[v[:, 0]]) - \
        (sy[v[:, 1]] - sy[v[:, 0]]).astype(np.int64) * (sx[v[:, 2]] - sx[v[:, 0]])
    assert (area == 0).any()
    np.testing.assert_array_equal(oracle.assign_bbox(W, H, sx, sy, t), oracle.assign(W, H, sx, sy, t))
