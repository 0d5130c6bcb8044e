"""Batched triangulation: every image of a batch equals the single-image
pipeline on that image alone, bit for bit (grids and triangle rows), and the
single-image pipeline equals the oracle (tests/test_gpu_batch.py)."""
import numpy as np
import pytest

import oracle
from integer_delauney_b200.workloads import batched_images, clustered, uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from integer_delauney_b200 import _delauney_cuda
    return _delauney_cuda


def mixed_images():
    imgs = [(5, 7, [(1, 1)]), (9, 4, [(0, 0), (8, 3)]), (16, 16, [(2, 2), (13, 3), (7, 12)]),
            (300, 40, uniform(300, 40, 150, seed=1)), (40, 300, uniform(40, 300, 150, seed=2)),
            (128, 128, clustered(128, 128, 400, seed=3, blobs=3, sigma=8.0)),
            (257, 193, uniform(257, 193, 900, seed=4)), (64, 64, uniform(64, 64, 4000, seed=5))]
    imgs += [(w, h, s) for w, h, s in batched_images(12, seed=6)]
    return imgs


@pytest.mark.parametrize("P", [16, 0, 5])
def test_each_image_equals_single_image_call(cu, P):
    imgs = mixed_images()
    got = cu.triangulate_batch(imgs, P)
    assert len(got) == len(imgs)
    for (w, h, s), (m, g) in zip(imgs, got):
        m1, g1 = cu.triangulate(w, h, s, P)
        assert m == m1
        np.testing.assert_array_equal(g, g1)


def test_matches_oracle(cu):
    imgs = mixed_images()[:8]
    got = cu.triangulate_batch(imgs, 16, as_arrays=True)
    for (w, h, s), (v, g) in zip(imgs, got):
        tris, grid, _ = oracle.triangulate(w, h, oracle.sort_seeds(s, w, h), 16)
        np.testing.assert_array_equal(g, grid)
        np.testing.assert_array_equal(v, tris[:, 2:5])


@pytest.mark.parametrize("P", [16, 0])
def test_exact_mode_each_image_equals_single_image_call(cu, P):
    """Exact semantics over the atlas: each image's nearest-seed search stays
    inside its own canvas, so every image equals the single-image exact
    pipeline (and, for the small ones, the oracle)."""
    imgs = mixed_images()
    got = cu.triangulate_batch(imgs, P, as_arrays=True, voronoi_mode="exact")
    for k, ((w, h, s), (v, g)) in enumerate(zip(imgs, got)):
        v1, g1 = cu.triangulate(w, h, s, P, as_arrays=True, voronoi_mode="exact")
        np.testing.assert_array_equal(v, v1)
        np.testing.assert_array_equal(g, g1)
        if k < 8:
            tris, grid, _ = oracle.triangulate(w, h, oracle.sort_seeds(s, w, h), P, "exact")
            np.testing.assert_array_equal(g, grid)
            np.testing.assert_array_equal(v, tris[:, 2:5])
    # the configuration's shape: many images of uneven size in one batch
    imgs = batched_images(64, seed=12)
    got = cu.triangulate_batch(imgs, P, as_arrays=True, voronoi_mode="exact")
    for (w, h, s), (v, g) in zip(imgs, got):
        v1, g1 = cu.triangulate(w, h, s, P, as_arrays=True, voronoi_mode="exact")
        np.testing.assert_array_equal(v, v1)
        np.testing.assert_array_equal(g, g1)


def test_batched_configuration_sample(cu):
    imgs = batched_images(96, seed=11)
    got = cu.triangulate_batch(imgs, -1, as_arrays=True)
    for (w, h, s), (v, g) in zip(imgs, got):
        v1, g1 = cu.triangulate(w, h, s, -1, as_arrays=True)
        np.testing.assert_array_equal(v, v1)
        np.testing.assert_array_equal(g, g1)


def test_errors_name_the_image(cu):
    good = (32, 32, [(1, 1), (5, 5), (9, 2)])
    with pytest.raises(ValueError, match="image 1: seed coordinate out of bounds"):
        cu.triangulate_batch([good, (16, 16, [(3, 3), (16, 2)])])
    with pytest.raises(ValueError, match="image 2: duplicate"):
        cu.triangulate_batch([good, good, (16, 16, [(3, 3), (3, 3)])])
    with pytest.raises(ValueError, match="image 0: seeds must not be empty"):
        cu.triangulate_batch([(16, 16, []), good])
    assert cu.triangulate_batch([]) == []
    # the context is still usable after the failures
    m, g = cu.triangulate_batch([good])[0]
    assert len(m) == 1 and g.shape == (32, 32, 3)
