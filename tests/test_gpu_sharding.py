"""Batches and served diagrams spread over devices give the same results as
on one device.  This machine's tests run on one GPU, so the two "devices" of
each case are the same GPU twice: two batches on two host threads, two
independent servers behind one pool -- the routing and the merging of
results is what is checked."""
import numpy as np
import pytest

from integer_delauney_b200.workloads import batched_images, fresh_points, uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from integer_delauney_b200 import _delauney_cuda
    return _delauney_cuda


def test_batch_over_devices_equals_one_batch(cu):
    from integer_delauney_b200.sharding import triangulate_batch_devices
    imgs = batched_images(count=40, seed=9, side_hi=400)
    one = cu.triangulate_batch(imgs, 16, as_arrays=True)
    many = triangulate_batch_devices(imgs, devices=[0, 0], border_padding=16, as_arrays=True)
    assert len(many) == len(one)
    for (va, ga), (vb, gb) in zip(one, many):
        np.testing.assert_array_equal(va, vb)
        np.testing.assert_array_equal(ga, gb)


def test_server_pool_equals_single_diagrams(cu):
    from integer_delauney_b200.sharding import ServerPool
    rng = np.random.default_rng(4)
    news = []
    for i in range(8):
        W, H = int(rng.integers(60, 500)), int(rng.integers(60, 500))
        news.append((W, H, uniform(W, H, int(max(4, 0.01 * W * H)), seed=70 + i)))
    with ServerPool(devices=[0, 0], budget_bytes=8 << 30, slots=2, border_padding=16) as pool:
        tn = [pool.submit_new(W, H, p, fetch=True) for W, H, p in news]
        adds = []
        for i in (1, 4, 6):
            W, H, p = news[i]
            keys = np.sort(p[:, 1].astype(np.int64) * W + p[:, 0])
            adds.append((i, fresh_points(W, H, 50, keys, seed=900 + i)))
        ti = [(i, pool.submit_insert(tn[i].diagram_id, a, fetch=True)) for i, a in adds]
        got_new = [t.result(timeout=120) for t in tn]
        got_ins = [(i, t.result(timeout=120)) for i, t in ti]
        assert min(pool.loads()) > 0                       # both servers took work
    for (W, H, p), r in zip(news, got_new):
        v, g = cu.triangulate(W, H, p, 16, as_arrays=True)
        np.testing.assert_array_equal(v, r.verts)
        np.testing.assert_array_equal(g, r.grid)
    for (i, add), (_, r) in zip(adds, got_ins):
        W, H, p = news[i]
        d = cu.Delaunay(W, H, len(p) + 100, 16)
        d.insert_deferred(p, order="xy")
        d.insert_deferred(add)
        v, g = d.finalise(as_arrays=True)
        np.testing.assert_array_equal(v, r.verts)
        np.testing.assert_array_equal(g, r.grid)
        assert r.diagram_id == tn[i].diagram_id
