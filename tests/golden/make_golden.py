"""Generate golden vectors from the reference's own NumPy implementation.

Run in a container where the reference source tree is available:

    python tests/golden/make_golden.py [path/to/integer_delauney/src]

It imports ``delauney.reference`` (reference/voronoi.py and
reference/triangulation.py) and records, for fixed seeded inputs, exactly what
it returns.  The outputs are committed as small .npz files beside this script
so that the CPU test suite can pin the oracle against the reference without
the reference being present.  Nothing here runs at test time.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _seeds(W, H, n, seed):
    rng = np.random.default_rng(seed)
    pts = set()
    while len(pts) < n:
        pts.add((int(rng.integers(0, W)), int(rng.integers(0, H))))
    # unsorted on purpose: the API sorts internally
    out = list(pts)
    rng.shuffle(out)
    return out


# Voronoi cases: the fixed grids of tests/test_voronoi_cuda.py:55-70 plus
# seeded random cases up to the C1 canvas size.
VORONOI_CASES = [
    ("single", 5, 5, [(2, 2)]),
    ("row_pair", 5, 1, [(0, 0), (4, 0)]),
    ("col_pair", 1, 5, [(0, 0), (0, 4)]),
    ("three", 10, 10, [(1, 1), (8, 1), (4, 8)]),
    ("four_square", 10, 10, [(1, 1), (8, 1), (1, 8), (8, 8)]),
    ("four_corners", 5, 5, [(0, 0), (4, 0), (0, 4), (4, 4)]),
    ("tie_three", 5, 5, [(0, 2), (2, 0), (4, 2)]),
    ("rand_64_20", 64, 64, _seeds(64, 64, 20, 1)),
    ("rand_128_400", 128, 128, _seeds(128, 128, 400, 2)),
    ("rand_100x70_300", 100, 70, _seeds(100, 70, 300, 3)),
    ("rand_200x150_1500", 200, 150, _seeds(200, 150, 1500, 4)),
]

# Triangulation cases: GridTriangulation on the NumPy Voronoi grid, with the
# small fixed sets of tests/test_triangulation_cuda.py:68-73,
# tests/test_pixel_assignment_correctness.py:39-66 and
# tests/test_scipy_oracle.py:322-327,418-422, plus seeded random sets.
TRI_CASES = [
    ("three_10", 10, 10, [(1, 1), (8, 1), (4, 8)], 0),
    ("square_10", 10, 10, [(1, 1), (8, 1), (1, 8), (8, 8)], 0),
    ("corners_5", 5, 5, [(0, 0), (4, 0), (0, 4), (4, 4)], 0),
    ("three_20", 20, 20, [(2, 5), (15, 2), (10, 14)], 0),
    ("tri_30", 30, 30, [(3, 3), (25, 5), (14, 25)], 16),
    ("quad_30", 30, 30, [(3, 3), (26, 3), (3, 26), (26, 26)], 16),
    ("grid9_40", 40, 40, [(5, 5), (20, 3), (35, 5), (3, 20), (20, 20), (37, 20),
                          (5, 35), (20, 37), (35, 35)], 16),
    ("rand15_50", 50, 50, [(4, 7), (12, 2), (23, 5), (38, 3), (46, 8), (2, 18), (15, 22),
                           (30, 19), (44, 21), (8, 33), (22, 35), (36, 30), (47, 38),
                           (10, 45), (40, 44)], 16),
    ("sq_quad_256", 256, 256, [(60, 60), (180, 60), (60, 180), (180, 180)], 0),
    ("rot_quad_256", 256, 256, [(80, 128), (128, 80), (176, 128), (128, 176)], 0),
    ("scipy6_256", 256, 256, [(80, 40), (170, 60), (60, 140), (190, 150), (120, 210),
                              (128, 100)], 16),
    ("rand_64_20_p0", 64, 64, _seeds(64, 64, 20, 11), 0),
    ("rand_64_40_p16", 64, 64, _seeds(64, 64, 40, 12), 16),
    ("rand_48_60_p8", 48, 48, _seeds(48, 48, 60, 13), 8),
    ("rand_96x80_120_p16", 96, 80, _seeds(96, 80, 120, 14), 16),
]


def reference_root() -> str:
    """The reference source tree: $IDL_REFERENCE_SRC, else BASELINE.json's reference_path."""
    env = os.environ.get("IDL_REFERENCE_SRC")
    if env:
        return env
    import json
    with open(os.path.join(HERE, "..", "..", "BASELINE.json")) as f:
        return json.load(f)["reference_path"]


def main(src):
    sys.path.insert(0, src)
    from delauney.reference.voronoi import Voronoi
    from delauney.reference.triangulation import GridTriangulation

    vd, gt = Voronoi(), GridTriangulation()

    vor = {}
    for name, W, H, seeds in VORONOI_CASES:
        vor[f"{name}__seeds"] = np.asarray(seeds, dtype=np.int32).reshape(-1, 2)
        vor[f"{name}__wh"] = np.asarray([W, H], dtype=np.int32)
        vor[f"{name}__grid"] = vd.compute(W, H, seeds)
    np.savez_compressed(os.path.join(HERE, "voronoi_numpy.npz"), **vor)

    tri = {}
    for name, W, H, seeds, P in TRI_CASES:
        vg = vd.compute(W, H, seeds)
        tm, tg = gt.compute(vg, seeds, border_padding=P)
        arr = np.asarray([tm[k] for k in range(len(tm))], dtype=np.int32).reshape(-1, 5)
        tri[f"{name}__seeds"] = np.asarray(seeds, dtype=np.int32).reshape(-1, 2)
        tri[f"{name}__whp"] = np.asarray([W, H, P], dtype=np.int32)
        tri[f"{name}__vgrid"] = vg
        tri[f"{name}__tris"] = arr
        tri[f"{name}__tgrid"] = tg
    np.savez_compressed(os.path.join(HERE, "triangulation_numpy.npz"), **tri)
    print("wrote", len(VORONOI_CASES), "voronoi and", len(TRI_CASES), "triangulation cases")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(reference_root(), "src"))
