"""Serving: every request's result is the same when it runs alone as when it
runs in the mix on the server (many slots, overlapping streams, admission by
memory budget, recycled objects), bit for bit."""
import numpy as np
import pytest

from integer_delauney_b200.workloads import fresh_points, uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from integer_delauney_b200 import _delauney_cuda
    return _delauney_cuda


def _requests(seed=0, n_new=14):
    rng = np.random.default_rng(seed)
    news, inserts = [], []
    for i in range(n_new):
        W, H = int(rng.integers(40, 700)), int(rng.integers(40, 700))
        n = int(max(3, rng.uniform(0.001, 0.02) * W * H))
        pts = uniform(W, H, n, seed=1000 + i)
        news.append((W, H, pts))
        keys = np.sort(pts[:, 1].astype(np.int64) * W + pts[:, 0])
        for j in range(int(rng.integers(0, 3))):
            add = fresh_points(W, H, int(rng.integers(10, 400)), keys, seed=5000 + 10 * i + j)
            keys = np.sort(np.concatenate([keys, add[:, 1].astype(np.int64) * W + add[:, 0]]))
            inserts.append((i, add))
    return news, inserts


def _alone(cu, news, inserts, P=16):
    """Each diagram on its own, one request at a time."""
    out_new, out_ins = [], []
    objs = []
    for W, H, pts in news:
        d = cu.Delaunay(W, H, len(pts) + 2000, P)
        order = np.lexsort((pts[:, 1], pts[:, 0]))
        d.insert_deferred(np.ascontiguousarray(pts[order]))
        out_new.append(d.finalise(as_arrays=True))
        objs.append(d)
    for i, add in inserts:
        objs[i].insert_deferred(add)
        out_ins.append(objs[i].finalise(as_arrays=True))
    return out_new, out_ins


def _mixed(news, inserts, budget=40 << 30, slots=4):
    from integer_delauney_b200.serving import Server
    with Server(budget_bytes=budget, slots=slots, border_padding=16) as srv:
        fn = [srv.submit_new(W, H, pts, fetch=True) for W, H, pts in news]
        fi = [srv.submit_insert(fn[i].diagram_id, add, fetch=True) for i, add in inserts]
        srv.drain()
        stats = dict(srv.stats)
        return [f.result() for f in fn], [f.result() for f in fi], stats


def _same(a, b):
    np.testing.assert_array_equal(a[0], b.verts)
    np.testing.assert_array_equal(np.asarray(a[1]), b.grid)


def test_alone_equals_mixed(cu):
    news, inserts = _requests(0)
    a_new, a_ins = _alone(cu, news, inserts)
    m_new, m_ins, _ = _mixed(news, inserts)
    for a, m in zip(a_new, m_new):
        _same(a, m)
    for a, m in zip(a_ins, m_ins):
        _same(a, m)


def test_new_requests_equal_the_batch_pipeline(cu):
    news, _ = _requests(1, n_new=6)
    m_new, _, _ = _mixed(news, [])
    for (W, H, pts), r in zip(news, m_new):
        v, g = cu.triangulate(W, H, pts, 16, as_arrays=True)
        np.testing.assert_array_equal(v, r.verts)
        np.testing.assert_array_equal(g, r.grid)


def test_small_budget_recycles_objects_and_keeps_results(cu):
    from integer_delauney_b200.serving import SEED_HEADROOM, estimate_bytes, slot_reserve
    news = [(200, 180, uniform(200, 180, 300, seed=i)) for i in range(12)]
    # two slots' reserves; room for three diagrams besides
    budget = 3 * estimate_bytes(256, 256, 300 + SEED_HEADROOM, 16, workspace=False) + 2 * slot_reserve(16)
    a_new, _ = _alone(cu, news, [])
    m_new, _, stats = _mixed(news, [], budget=budget, slots=2)
    for a, m in zip(a_new, m_new):
        _same(a, m)
    assert stats.get("evicted", 0) > 0 and stats.get("reused_objects", 0) > 0


def test_over_budget_and_unknown_diagram(cu):
    from integer_delauney_b200.serving import Server
    with Server(budget_bytes=1 << 20, slots=1) as srv:
        f = srv.submit_new(512, 512, uniform(512, 512, 100, seed=1))
        with pytest.raises(MemoryError):
            f.result(timeout=60)
        with pytest.raises(KeyError):
            srv.submit_insert(12345, [(1, 1)])


def test_adopt_from_a_batch_equals_ordered_insert(cu):
    """idl_voronoi_batch + idl_delaunay_adopt (one propagation launch for
    several new diagrams) leaves each object exactly as an ordered insert of
    its seeds would; the object then takes inserts as usual."""
    from integer_delauney_b200 import _capi
    news, inserts = _requests(3, n_new=6)
    ctx = _capi.Context(0)
    lib = _capi.load()
    dims = np.array([(W, H) for W, H, _ in news], dtype=np.int32)
    counts = np.array([len(p) for _, _, p in news], dtype=np.int64)
    seeds = np.ascontiguousarray(np.concatenate([p for _, _, p in news]), dtype=np.int32)
    _capi.check(lib.idl_voronoi_batch(ctx.handle, len(news), dims.ctypes.data, counts.ctypes.data,
                                      seeds.ctypes.data, 16, 0))
    for k, (W, H, pts) in enumerate(news):
        a = cu.Delaunay(W, H, len(pts) + 500, 16)
        a._adopt(ctx, k)
        b = cu.Delaunay(W, H, len(pts) + 500, 16)
        b.insert_deferred(pts, order="xy")
        for x, y in ((a, b),):
            np.testing.assert_array_equal(x.get_voronoi_grid(), y.get_voronoi_grid())
            np.testing.assert_array_equal(x.get_seeds(), y.get_seeds())
        va, ga = a.finalise(as_arrays=True)
        vb, gb = b.finalise(as_arrays=True)
        np.testing.assert_array_equal(va, vb)
        np.testing.assert_array_equal(ga, gb)
        for i, add in inserts:
            if i == k:
                a.insert_deferred(add)
                b.insert_deferred(add)
        np.testing.assert_array_equal(a.finalise(as_arrays=True)[1], b.finalise(as_arrays=True)[1])
    with pytest.raises(ValueError):
        cu.Delaunay(7, 7, 10, 16)._adopt(ctx, 0)          # size differs from the batch image


def test_adopt_group_equals_adopting_one_by_one(cu):
    """idl_delaunay_adopt_group (every image of a group in one launch and one
    wait) leaves each object exactly as idl_delaunay_adopt of its image does."""
    import ctypes
    import torch
    from integer_delauney_b200 import _capi
    news, _ = _requests(5, n_new=6)
    ctx = _capi.Context(0)
    lib = _capi.load()
    stream = torch.cuda.current_stream().cuda_stream
    ctx.set_stream(stream)
    dims = np.array([(W, H) for W, H, _ in news], dtype=np.int32)
    counts = np.array([len(p) for _, _, p in news], dtype=np.int64)
    seeds = np.ascontiguousarray(np.concatenate([p for _, _, p in news]), dtype=np.int32)
    _capi.check(lib.idl_voronoi_batch(ctx.handle, len(news), dims.ctypes.data, counts.ctypes.data,
                                      seeds.ctypes.data, 16, 0))
    group = [cu.Delaunay(W, H, len(p) + 50, 16) for W, H, p in news]
    order = [4, 1, 5, 0, 3, 2]                      # any order of the group's images
    for o in group:
        _capi.check(lib.idl_delaunay_set_stream(o._h, stream))
    handles = (ctypes.c_void_p * len(order))(*[group[k]._h.value for k in order])
    images = (ctypes.c_int * len(order))(*order)
    _capi.check(lib.idl_delaunay_adopt_group(handles, images, len(order), ctx.handle))
    for k, (W, H, pts) in enumerate(news):
        one = cu.Delaunay(W, H, len(pts) + 50, 16)
        one._adopt(ctx, k)
        np.testing.assert_array_equal(group[k].get_voronoi_grid(), one.get_voronoi_grid())
        np.testing.assert_array_equal(group[k].get_seeds(), one.get_seeds())
        va, ga = group[k].finalise(as_arrays=True)
        vb, gb = one.finalise(as_arrays=True)
        np.testing.assert_array_equal(va, vb)
        np.testing.assert_array_equal(ga, gb)
    twice = (ctypes.c_void_p * 2)(group[0]._h.value, group[0]._h.value)
    assert lib.idl_delaunay_adopt_group(twice, (ctypes.c_int * 2)(0, 0), 2, ctx.handle) == _capi.IDL_ERR_INVALID
    assert lib.idl_delaunay_adopt_group(handles, images, 17, ctx.handle) == _capi.IDL_ERR_INVALID


def test_exact_mode_server_equals_exact_triangulate(cu):
    from integer_delauney_b200.serving import Server
    news, inserts = _requests(4, n_new=5)
    with Server(budget_bytes=40 << 30, slots=3, border_padding=16, mode="exact") as srv:
        fn = [srv.submit_new(W, H, pts, fetch=True) for W, H, pts in news]
        fi = [(i, srv.submit_insert(fn[i].diagram_id, add, fetch=True)) for i, add in inserts]
        got_new = [f.result(timeout=120) for f in fn]
        got_ins = [(i, f.result(timeout=120)) for i, f in fi]
    for (W, H, pts), r in zip(news, got_new):
        v, g = cu.triangulate(W, H, pts, 16, voronoi_mode="exact", as_arrays=True)
        np.testing.assert_array_equal(v, r.verts)
        np.testing.assert_array_equal(g, r.grid)
    # exact mode is history-independent: after an insert the diagram equals
    # the exact triangulation of all its seeds, in insertion order of ids
    for (i, add), (_, r) in zip(inserts, got_ins):
        W, H, pts = news[i]
        d = cu.Delaunay(W, H, len(pts) + 5000, 16, voronoi_mode="exact")
        d.insert_deferred(pts, order="xy")
        for j, more in inserts:
            if j == i:
                d.insert_deferred(more)
                if more is add:
                    break
        v, g = d.finalise(as_arrays=True)
        np.testing.assert_array_equal(g, r.grid)
        np.testing.assert_array_equal(v, r.verts)


def test_many_client_threads(cu):
    """Clients submitting from several threads at once get the same results
    as one client submitting in order."""
    import threading
    from integer_delauney_b200.serving import Server
    news, _ = _requests(5, n_new=24)
    expect = [cu.triangulate(W, H, pts, 16, as_arrays=True) for W, H, pts in news]
    out = [None] * len(news)
    with Server(budget_bytes=40 << 30, slots=4, border_padding=16) as srv:
        def client(k):
            for i in range(k, len(news), 4):
                W, H, pts = news[i]
                out[i] = srv.submit_new(W, H, pts, fetch=True).result(timeout=120)
        ts = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        info = srv.info()
    for (v, g), r in zip(expect, out):
        np.testing.assert_array_equal(v, r.verts)
        np.testing.assert_array_equal(g, r.grid)
        assert r.arrival <= r.start <= r.done
    assert info["queued"] == 0 and info["resident"] == len(news)


def test_collect_once_recycle_and_timestamps(cu):
    import ctypes
    import time
    from integer_delauney_b200 import _capi
    from integer_delauney_b200.serving import Server
    lib = _capi.load()
    with Server(budget_bytes=40 << 30, slots=2, border_padding=16) as srv:
        at = time.monotonic() - 0.5                  # arrived half a second ago
        f = srv.submit_new(300, 200, uniform(300, 200, 400, seed=3), arrival=at)
        r = f.result(timeout=60)
        assert abs(r.arrival - at) < 1e-6 and r.latency >= 0.5
        assert r.n_seeds == 400 and r.n_triangles > 0 and r.kind == "new"
        row = (ctypes.c_int64 * _capi.SR_COUNT)()
        assert lib.idl_server_wait(srv._handle(), f.request_id, 1.0, row, None, 0) == _capi.IDL_ERR_INVALID
        g = srv.submit_insert(f.diagram_id, [(5, 7)])
        assert g.result(timeout=60).n_seeds == 401
        assert srv.recycle(f.diagram_id)
        assert f.diagram_id not in srv.resident()
        with pytest.raises(KeyError):
            srv.submit_insert(f.diagram_id, [(9, 9)])
        # the pooled object is reused by the next diagram of its size class
        h = srv.submit_new(310, 190, uniform(310, 190, 300, seed=4))
        h.result(timeout=60)
        assert srv.stats["reused_objects"] >= 1
        # a request with a seed out of bounds fails alone
        bad = srv.submit_new(100, 100, [(5, 5), (100, 3)])
        with pytest.raises(ValueError):
            bad.result(timeout=60)
        assert bad.diagram_id not in srv.resident()
