"""Incremental triangulation (``Delaunay``) on the GPU against the CPU oracle.

The oracle (``oracle.incremental``) restates the reference's incremental
trajectory: insertion-order ids, Jacobi continued from the previous fixed
point, detection on the insertion-id grid, outputs in batch ids.  Results are
compared bit for bit.  Behavioural cases follow the reference's own suites
(tests/test_incremental_cuda.py, test_incremental_deferred.py,
test_incremental_padding.py, test_finalise_device.py, test_scalar_field.py,
test_cuda_error_checking.py).
"""
import numpy as np
import pytest

import oracle
from integer_delauney_b200.workloads import uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from integer_delauney_b200 import _delauney_cuda
    return _delauney_cuda


def read_device(cai, dtype):
    """Copy a __cuda_array_interface__ out with the CUDA runtime directly, as
    a foreign consumer of the view would."""
    rt = pytest.importorskip("cuda.bindings.runtime")
    n = cai["shape"][0]
    out = np.empty(n, dtype=dtype)
    err, = rt.cudaMemcpy(out.ctypes.data, cai["data"][0], out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess
    return out


def split(seeds, sizes):
    out, i = [], 0
    for k in sizes:
        out.append(seeds[i:i + k])
        i += k
    return out


def run_incremental(cu, W, H, batches, P, max_seeds=None, deferred=False):
    d = cu.Delaunay(W, H, max_seeds or sum(len(b) for b in batches) + 8, P)
    m = g = None
    for b in batches:
        if deferred:
            d.insert_deferred(b)
        else:
            m, g = d.insert(b)
    if deferred:
        m, g = d.finalise()
    return d, m, g


def assert_matches_oracle(d, m, g, ref):
    np.testing.assert_array_equal(np.asarray(g), ref["grid"])
    rows = np.array([m[t] for t in range(len(m))], dtype=np.int32).reshape(-1, 5)
    np.testing.assert_array_equal(rows, ref["tris"])
    np.testing.assert_array_equal(d.get_triangles(), ref["tris_ins"])
    np.testing.assert_array_equal(d.sorted_rank, ref["rank"])
    np.testing.assert_array_equal(d.get_voronoi_grid(), ref["grid"][:, :, :2])


class TestAgainstOracle:
    @pytest.mark.parametrize("W,H,n,sizes,P", [
        (64, 64, 40, (10, 10, 20), 0),
        (64, 64, 60, (20, 20, 20), 16),
        (200, 150, 600, (100, 1, 299, 200), 16),
        (160, 120, 400, (400,), 5),
        (300, 200, 2000, (500, 500, 500, 500), 16),
    ])
    def test_bit_exact(self, cu, W, H, n, sizes, P):
        seeds = uniform(W, H, n, seed=n + P)
        batches = split(seeds, sizes)
        d, m, g = run_incremental(cu, W, H, batches, P)
        assert_matches_oracle(d, m, g, oracle.incremental(W, H, batches, P))

    def test_many_small_batches(self, cu):
        W, H = 256, 256
        seeds = uniform(W, H, 1500, seed=11)
        batches = split(seeds, [300] + [40] * 30)
        d, m, g = run_incremental(cu, W, H, batches, 16)
        assert_matches_oracle(d, m, g, oracle.incremental(W, H, batches, 16))

    def test_hotspot_refinement(self, cu):
        """Scaled-down incremental workload: a base set, then batches with 30 %
        of their seeds inside a hotspot square."""
        W = H = 512
        rng = np.random.default_rng(5)
        base = uniform(W, H, 3000, seed=5)
        taken = {(int(x), int(y)) for x, y in base}
        batches = [base]
        for _ in range(8):
            b = []
            while len(b) < 200:
                if rng.random() < 0.3:
                    x, y = rng.integers(192, 256, 2)
                else:
                    x, y = rng.integers(0, W), rng.integers(0, H)
                if (int(x), int(y)) not in taken:
                    taken.add((int(x), int(y)))
                    b.append((int(x), int(y)))
            batches.append(np.array(b, dtype=np.int32))
        d, m, g = run_incremental(cu, W, H, batches, 16)
        assert_matches_oracle(d, m, g, oracle.incremental(W, H, batches, 16))

    def test_sorted_single_batch_equals_batch_pipeline(self, cu):
        """Inserted in (x, y) order, insertion ids are the batch ids, so one
        insert from the empty state is the batch triangulation."""
        W, H = 200, 160
        s = oracle.sort_seeds(uniform(W, H, 700, seed=3), W, H)
        d, m, g = run_incremental(cu, W, H, [s], 16)
        tris, grid, _ = oracle.triangulate(W, H, s, 16)
        np.testing.assert_array_equal(np.asarray(g), grid)
        rows = np.array([m[t] for t in range(len(m))], dtype=np.int32).reshape(-1, 5)
        np.testing.assert_array_equal(rows, tris)


class TestApi:
    W, H = 64, 64

    def test_initial_state(self, cu):
        d = cu.Delaunay(self.W, self.H, 256, 0)
        assert d.seed_count == 0 and d.width == self.W and d.height == self.H
        assert d.border_padding == 0 and not d.has_pending
        vg = d.get_voronoi_grid()
        assert vg.shape == (self.H, self.W, 2) and vg.dtype == np.int32
        assert np.all(vg == -1)
        assert cu.Delaunay(self.W, self.H, 10).border_padding == 16

    def test_single_and_two_seeds_have_no_triangles(self, cu):
        d = cu.Delaunay(self.W, self.H, 256, 0)
        m, g = d.insert([(32, 32)])
        assert m == {} and g.shape == (self.H, self.W, 3)
        assert np.all(g[:, :, 0] == 0)
        yy, xx = np.mgrid[0:self.H, 0:self.W]
        np.testing.assert_array_equal(g[:, :, 1], (xx - 32) ** 2 + (yy - 32) ** 2)
        assert np.all(g[:, :, 2] == -1)
        m, g = d.insert([(10, 10)])
        assert m == {} and len(d.get_edges()) == 0

    def test_three_seeds_one_triangle(self, cu):
        d = cu.Delaunay(self.W, self.H, 256, 0)
        m, g = d.insert([(10, 10), (50, 10), (30, 50)])
        assert len(m) == 1
        assert sorted(m[0][2:]) == [0, 1, 2]
        assert set(np.unique(g[:, :, 2])) <= {-1, 0}

    def test_deferred_matches_immediate(self, cu):
        seeds = uniform(self.W, self.H, 120, seed=7)
        batches = split(seeds, (30, 30, 30, 30))
        d1, m1, g1 = run_incremental(cu, self.W, self.H, batches, 16)
        d2, m2, g2 = run_incremental(cu, self.W, self.H, batches, 16, deferred=True)
        assert m1 == m2
        np.testing.assert_array_equal(np.asarray(g1), np.asarray(g2))

    def test_has_pending_and_idempotent_finalise(self, cu):
        d = cu.Delaunay(self.W, self.H, 256, 0)
        d.insert_deferred(uniform(self.W, self.H, 30, seed=1))
        assert d.has_pending
        m1, g1 = d.finalise()
        assert not d.has_pending
        m2, g2 = d.finalise()
        assert m1 == m2 and np.array_equal(g1, g2)

    def test_get_triangles_between_deferred_inserts(self, cu):
        d = cu.Delaunay(self.W, self.H, 256, 0)
        d.insert_deferred(uniform(self.W, self.H, 40, seed=2))
        t = d.get_triangles()
        m, _ = d.finalise(as_arrays=True)
        np.testing.assert_array_equal(d.sorted_rank[t], m)

    def test_as_arrays_matches_dict(self, cu):
        d = cu.Delaunay(self.W, self.H, 256, 0)
        d.insert_deferred(uniform(self.W, self.H, 40, seed=4))
        verts, g1 = d.finalise(as_arrays=True)
        m, g2 = d.finalise()
        np.testing.assert_array_equal(verts, np.array([m[t][2:] for t in range(len(m))]))
        np.testing.assert_array_equal(g1, g2)

    def test_timings(self, cu):
        d = cu.Delaunay(self.W, self.H, 256, 0)
        m, g, t = d.insert_timed([(5, 5), (55, 5), (30, 30), (5, 55), (55, 55)])
        assert set(t) == {"bfs_ms", "bfs_iters", "detect_ms", "dedup_ms", "assign_ms"}
        assert 1 <= t["bfs_iters"] <= self.W + self.H
        assert all(v >= 0 for v in t.values())
        t2 = d.insert_deferred_timed([(40, 40)])
        assert set(t2) == set(t) and t2["assign_ms"] == 0.0
        _, _, t3 = d.finalise_timed()
        assert t3["assign_ms"] >= 0.0

    def test_validation(self, cu):
        d = cu.Delaunay(self.W, self.H, 8, 0)
        d.insert([(1, 1), (5, 5)])
        for bad, msg in [([(2, 2), (2, 2)], "within batch"), ([(1, 1)], "already exists"),
                         ([(-1, 3)], "out of bounds"), ([(self.W, 3)], "out of bounds"),
                         ([(3, self.H)], "out of bounds"), ([(i, 9) for i in range(7)], "max_seeds")]:
            with pytest.raises(ValueError, match=msg):
                d.insert(bad)
        assert d.seed_count == 2
        with pytest.raises(ValueError):
            d.insert_deferred([(3, 3)], values=[1.0, 2.0])
        d.insert_deferred([])
        assert d.seed_count == 2
        with pytest.raises(ValueError):
            cu.Delaunay(0, 10, 10)
        with pytest.raises(ValueError):
            cu.Delaunay(10, 10, 0)

    def test_allocation_failure_names_cudamalloc_and_source(self, cu):
        with pytest.raises(RuntimeError) as e:
            cu.Delaunay(200_000, 200_000, 1_000, 0)
        assert "cudaMalloc" in str(e.value) and "delaunay.cu" in str(e.value)
        d = cu.Delaunay(64, 64, 256, 0)
        m, g = d.insert([(10, 10), (50, 10), (30, 50)])
        assert len(m) > 0 and g.shape == (64, 64, 3)


class TestFinaliseDevice:
    W, H = 96, 80

    def _host(self, cu, seeds):
        d = cu.Delaunay(self.W, self.H, 512, -1)
        d.insert_deferred(seeds)
        verts, g = d.finalise(as_arrays=True)
        tids = g[:, :, 2].reshape(-1)
        return verts, g[:, :, 0].reshape(-1), (tids == -1).astype(np.uint8), np.where(tids == -1, 0, tids)

    @pytest.mark.parametrize("n", [10, 40, 150])
    def test_matches_finalise(self, cu, n):
        seeds = uniform(self.W, self.H, n, seed=n)
        d = cu.Delaunay(self.W, self.H, 512, -1)
        d.insert_deferred(seeds)
        verts, v_t, v_s, v_m = d.finalise_device()
        ref = self._host(cu, seeds)
        np.testing.assert_array_equal(verts, ref[0])
        for view, want, typ in ((v_t, ref[3], "<i4"), (v_s, ref[1], "<i4"), (v_m, ref[2], "|u1")):
            cai = view.__cuda_array_interface__
            assert cai["shape"] == (self.W * self.H,) and cai["typestr"] == typ
            assert cai["data"][1] is True and cai["version"] == 3
            np.testing.assert_array_equal(read_device(cai, want.dtype), want)
            np.testing.assert_array_equal(view.to_host(), want)
            # zero-copy handoff: a torch tensor and a DLPack import alias the same memory
            import torch
            t = view.to_torch()
            assert t.data_ptr() == cai["data"][0] and t.is_cuda and t.numel() == self.W * self.H
            np.testing.assert_array_equal(t.cpu().numpy(), want)
            u = torch.from_dlpack(view)
            assert u.data_ptr() == cai["data"][0]
            np.testing.assert_array_equal(u.cpu().numpy(), want)
            assert view.__dlpack_device__() == (2, torch.cuda.current_device())

    def test_stale_views_raise(self, cu):
        d = cu.Delaunay(self.W, self.H, 512, -1)
        seeds = uniform(self.W, self.H, 20, seed=2)
        _, a, b, c = (d.insert_deferred(seeds), *d.finalise_device())[1:]
        taken = {(int(x), int(y)) for x, y in seeds}
        d.insert_deferred([next((x, 0) for x in range(self.W) if (x, 0) not in taken)])
        for v in (a, b, c):
            with pytest.raises(RuntimeError):
                v.__cuda_array_interface__
            with pytest.raises(RuntimeError):
                v.to_host()
            with pytest.raises(RuntimeError):
                v.to_torch()
        _, t1, _, _ = d.finalise_device()
        _, t2, _, _ = d.finalise_device()
        with pytest.raises(RuntimeError):
            t1.__cuda_array_interface__
        t2.__cuda_array_interface__


W_SF, H_SF, P_SF = 240, 180, 16


def make_mesh(cu, n=400, seed=0):
    rng = np.random.default_rng(seed)
    pts = uniform(W_SF, H_SF, n, seed=seed)
    img = rng.random((H_SF, W_SF)).astype(np.float32)
    vals = img[pts[:, 1], pts[:, 0]]
    mesh = cu.Delaunay(W_SF, H_SF, 4000, P_SF)
    mesh.insert_deferred(pts, vals)
    return mesh, pts, vals


def host_scores(pts, vals, edges, min_length):
    d = pts[edges[:, 1]].astype(np.float64) - pts[edges[:, 0]].astype(np.float64)
    len2 = d[:, 0] ** 2 + d[:, 1] ** 2
    s = (np.abs(vals[edges[:, 0]].astype(np.float64) - vals[edges[:, 1]].astype(np.float64))
         * np.sqrt(len2)).astype(np.float32)
    s[len2 < min_length * min_length] = 0.0
    return s


def host_midpoints(pts, vals, edges, min_length, count, threshold, P=P_SF):
    """delaunay_scalar_field.cu:226-291, restated: best-first by (score desc,
    index asc), midpoint rounded half to even on the padded canvas, clamped to
    the image, dropped on seeds and on collisions (best rank kept)."""
    s = host_scores(pts, vals, edges, min_length)
    ok = (s > threshold) & (s > 0)
    order = sorted(np.flatnonzero(ok), key=lambda e: (-float(s[e]), int(e)))[:count]
    seeds = {(int(x), int(y)) for x, y in pts}
    Wd = W_SF + 2 * P
    best = {}
    for r, e in enumerate(order):
        a, b = edges[e]
        mx = int(np.rint(0.5 * (float(pts[a, 0] + P) + float(pts[b, 0] + P))))
        my = int(np.rint(0.5 * (float(pts[a, 1] + P) + float(pts[b, 1] + P))))
        mx = min(max(mx, P), Wd - 1 - P)
        my = min(max(my, P), H_SF + 2 * P - 1 - P)
        if (mx - P, my - P) in seeds:
            continue
        best.setdefault(my * Wd + mx, r)
    return np.array([(k % Wd - P, k // Wd - P) for k in sorted(best)], dtype=np.int32).reshape(-1, 2)


class TestScalarField:
    def test_edges_match_triangles(self, cu):
        mesh, pts, _ = make_mesh(cu, 300, seed=1)
        tris = mesh.get_triangles()
        want = set()
        for a, b, c in tris:
            for p, q in ((a, b), (b, c), (c, a)):
                want.add((min(p, q), max(p, q)))
        e = mesh.get_edges()
        assert [tuple(r) for r in e] == sorted(want)

    @pytest.mark.parametrize("min_length", [0.0, 2.0, 9.0])
    def test_edge_scores(self, cu, min_length):
        mesh, pts, vals = make_mesh(cu, 400, seed=2)
        got = mesh.edge_scores(min_length)
        np.testing.assert_array_equal(got, host_scores(pts, vals, mesh.get_edges(), min_length))

    def test_scores_need_values(self, cu):
        d = cu.Delaunay(W_SF, H_SF, 100, P_SF)
        d.insert_deferred(uniform(W_SF, H_SF, 30, seed=3))
        with pytest.raises(RuntimeError):
            d.edge_scores(0.0)
        with pytest.raises(RuntimeError):
            d.select_midpoints(2.0, 5)

    @pytest.mark.parametrize("count,threshold", [(1, 0.0), (25, 0.0), (400, 0.0), (5000, 0.0), (60, 3.0)])
    def test_select_midpoints(self, cu, count, threshold):
        mesh, pts, vals = make_mesh(cu, 400, seed=4)
        got = mesh.select_midpoints(2.0, count, threshold)
        want = host_midpoints(pts, vals, mesh.get_edges(), 2.0, count, threshold)
        np.testing.assert_array_equal(got, want)
        if len(got):
            mesh.insert_deferred(got, np.zeros(len(got), np.float32))

    def test_seeds_and_values(self, cu):
        mesh, pts, vals = make_mesh(cu, 100, seed=5)
        np.testing.assert_array_equal(mesh.get_seeds(), pts)
        np.testing.assert_array_equal(mesh.get_values(), vals)


class TestQueries:
    def _q(self, n, seed):
        rng = np.random.default_rng(seed)
        return np.stack([rng.integers(0, W_SF, n), rng.integers(0, H_SF, n)], axis=1).astype(np.int32)

    @pytest.mark.parametrize("n,nq", [(50, 200), (400, 9000)])
    def test_locate_matches_finalised_grid(self, cu, n, nq):
        mesh, _, _ = make_mesh(cu, n, seed=n)
        q = self._q(nq, n + 1)
        before = mesh.locate(q)
        _, g = mesh.finalise(as_arrays=True)
        np.testing.assert_array_equal(before, g[q[:, 1], q[:, 0], 2])
        assert len(mesh.locate(np.zeros((0, 2), np.int32))) == 0
        np.testing.assert_array_equal(mesh.locate([[-P_SF - 1, 0], [W_SF + P_SF, 0]]), [-1, -1])

    @pytest.mark.parametrize("t_val", [0.0, 1.0, 12.0, 1e6])
    def test_in_circumsphere(self, cu, t_val):
        mesh, pts, _ = make_mesh(cu, 400, seed=int(t_val) % 97 + 3)
        q = self._q(3000, 9)
        t = np.full(len(q), t_val)
        got, tids = mesh.in_circumsphere(q, t)
        np.testing.assert_array_equal(tids, mesh.locate(q))
        m, _ = mesh.finalise()
        srt = pts[np.lexsort((pts[:, 1], pts[:, 0]))].astype(np.float64) + P_SF
        want = np.zeros(len(q), bool)
        for i in np.flatnonzero(tids >= 0):
            (ax, ay), (bx, by), (cx, cy) = (srt[v] for v in m[int(tids[i])][2:])
            abx, aby, acx, acy = bx - ax, by - ay, cx - ax, cy - ay
            nz = abx * acy - aby * acx
            if nz * nz < 1e-12:
                ox, oy = (ax + bx + cx) / 3.0, (ay + by + cy) / 3.0
            else:
                ab2, ac2, den = abx * abx + aby * aby, acx * acx + acy * acy, 2.0 * (nz * nz)
                ox = ax + (ac2 * (-(nz * aby)) + ab2 * (acy * nz)) / den
                oy = ay + (ac2 * (nz * abx) + ab2 * (-(acx * nz))) / den
            r2 = max((vx - ox) * (vx - ox) + (vy - oy) * (vy - oy) for vx, vy in ((ax, ay), (bx, by), (cx, cy)))
            dx, dy = q[i, 0] + P_SF - ox, q[i, 1] + P_SF - oy
            want[i] = np.sqrt(dx * dx + dy * dy + t[i] * t[i]) < np.sqrt(r2)
        # the device may contract multiply-adds, so a point exactly on the
        # sphere (a vertex) can round either way; nothing else may differ
        seeds = {(int(x), int(y)) for x, y in pts}
        for i in np.flatnonzero(got != want):
            assert (int(q[i, 0]), int(q[i, 1])) in seeds, f"disagreed at {q[i]}"
        if t_val >= 1e6:
            assert not got.any()
        with pytest.raises(ValueError):
            mesh.in_circumsphere(q[:2], np.zeros(1))


def test_incremental_config_prefix_bit_exact(cu):
    """The incremental configuration at full size (2048 x 2048, 50 000 base
    seeds, 1 000-seed batches with a hotspot), first three batches, checked
    against the oracle after each batch."""
    from integer_delauney_b200.workloads import incremental
    base, batches = incremental(2048, 2048, 50_000, 3, 1_000, seed=0)
    d = cu.Delaunay(2048, 2048, 60_000, 16)
    d.insert_deferred(base)
    done = [base]
    for b in batches:
        m, g = d.insert(b)
        done.append(b)
    assert_matches_oracle(d, m, g, oracle.incremental(2048, 2048, done, 16))


def test_ordered_insert_equals_batch_pipeline(cu):
    """order='xy' numbers the batch by (x, y): into an empty object that is
    the batch pipeline's numbering, so its result, bit for bit; the values
    follow their seeds."""
    W, H = 230, 170
    s = uniform(W, H, 900, seed=21)
    vals = np.arange(len(s), dtype=np.float32)
    d = cu.Delaunay(W, H, 2000, 16)
    d.insert_deferred(s, vals, order="xy")
    v, g = d.finalise(as_arrays=True)
    v1, g1 = cu.triangulate(W, H, s, 16, as_arrays=True)
    np.testing.assert_array_equal(v, v1)
    np.testing.assert_array_equal(g, g1)
    order = np.lexsort((s[:, 1], s[:, 0]))
    np.testing.assert_array_equal(d.get_seeds(), s[order])
    np.testing.assert_array_equal(d.get_values(), vals[order])
    np.testing.assert_array_equal(d.sorted_rank, np.arange(len(s)))


def test_rejected_insert_changes_nothing(cu):
    W, H = 120, 90
    s = uniform(W, H, 200, seed=22)
    d = cu.Delaunay(W, H, 400, 16)
    d.insert_deferred(s[:150])
    m0, g0 = d.finalise(as_arrays=True)
    bad = np.concatenate([s[150:160], s[10:11]])           # repeats an existing seed
    with pytest.raises(ValueError, match="already exists"):
        d.insert(bad)
    with pytest.raises(ValueError, match="within batch"):
        d.insert(np.concatenate([s[150:160], s[155:156]]))
    with pytest.raises(ValueError, match="out of bounds"):
        d.insert(np.concatenate([s[150:160], [[W, 0]]]))
    assert d.seed_count == 150
    m1, g1 = d.finalise(as_arrays=True)
    np.testing.assert_array_equal(m0, m1)
    np.testing.assert_array_equal(g0, g1)
    np.testing.assert_array_equal(d.locate(s[:50]), g0[s[:50, 1], s[:50, 0], 2])


@pytest.mark.parametrize("sizes,P", [((300, 200, 1, 499), 16), ((1000,), 0), ((100,) * 10, 16)])
def test_exact_mode_equals_full_recompute_after_every_insert(cu, sizes, P):
    """In exact mode the incremental object is history-independent: after
    each insert it equals the exact batch triangulation of all its seeds."""
    W, H = 320, 240
    seeds = uniform(W, H, sum(sizes), seed=len(sizes) + P)
    d = cu.Delaunay(W, H, 2000, P, voronoi_mode="exact")
    done = 0
    for k in sizes:
        m, g = d.insert(seeds[done:done + k])
        done += k
        m1, g1 = cu.triangulate(W, H, seeds[:done], P, voronoi_mode="exact")
        assert m == m1
        np.testing.assert_array_equal(g, g1)
        np.testing.assert_array_equal(d.get_voronoi_grid(), g1[:, :, :2])
    s = oracle.sort_seeds(seeds, W, H)
    o_tris, o_grid, _ = oracle.triangulate(W, H, s, P, "exact")
    np.testing.assert_array_equal(g, o_grid)
    np.testing.assert_array_equal(np.array([m[t] for t in range(len(m))]).reshape(-1, 5), o_tris)
    np.testing.assert_array_equal(d.sorted_rank[d.get_triangles()], o_tris[:, 2:5])


def test_insert_as_tile_rounds_equals_sparse_kernel(cu):
    """A workspace context with schedule < 0 runs an insert's continued
    propagation as tile rounds from the new seeds' tiles; the result equals the
    persistent sparse kernel's (the default) after every insert, bit for bit
    -- both are the synchronous Jacobi fixed point continued from the last."""
    from integer_delauney_b200 import _capi
    from integer_delauney_b200.workloads import fresh_points
    W, H = 733, 517
    base = uniform(W, H, 2500, seed=21)
    ctx = _capi.Context(0)
    ctx.set_schedule(-1)
    a = cu.Delaunay(W, H, 9000, 16)
    b = cu.Delaunay(W, H, 9000, 16)
    b.use_workspace(ctx)
    keys = np.sort(base[:, 1].astype(np.int64) * W + base[:, 0])
    batches = [base]
    for i, n in enumerate((1, 40, 600, 1500)):
        add = fresh_points(W, H, n, keys, seed=100 + i)
        if i == 2:                                  # a dense hotspot in one corner
            add = fresh_points(90, 70, n // 2, np.zeros(0, np.int64), seed=300)
            k2 = add[:, 1].astype(np.int64) * W + add[:, 0]
            add = add[~np.isin(k2, keys)]
        batches.append(add)
        keys = np.sort(np.concatenate([keys, add[:, 1].astype(np.int64) * W + add[:, 0]]))
    for add in batches:
        a.insert_deferred(add)
        b.insert_deferred(add)
        np.testing.assert_array_equal(a.get_voronoi_grid(), b.get_voronoi_grid())
    va, ga = a.finalise(as_arrays=True)
    vb, gb = b.finalise(as_arrays=True)
    np.testing.assert_array_equal(va, vb)
    np.testing.assert_array_equal(ga, gb)


def test_vertex_arrays_equal_the_map_vertices(cu):
    """finalise(as_arrays=True) and finalise_device return the vertex triples
    packed on the device (idl_delaunay_triangles format 2); they equal the
    (a, b, c) columns of finalise's map, before and after further inserts."""
    W, H = 300, 200
    seeds = uniform(W, H, 900, seed=5)
    d = cu.Delaunay(W, H, 2000, 16)
    for part in (seeds[:500], seeds[500:]):
        d.insert_deferred(part)
        m, g = d.finalise()
        verts, g2 = d.finalise(as_arrays=True)
        want = np.array([m[t][2:5] for t in range(len(m))], dtype=np.int32).reshape(-1, 3)
        np.testing.assert_array_equal(verts, want)
        np.testing.assert_array_equal(g2, g)
        v_dev = d.finalise_device()[0]
        np.testing.assert_array_equal(v_dev, want)
        m2, g3 = d.insert(np.zeros((0, 2), dtype=np.int32), as_arrays=True)
        np.testing.assert_array_equal(m2, want)
