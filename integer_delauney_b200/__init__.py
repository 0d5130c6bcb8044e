"""B200-native integer Delaunay: drop-in for the reference's ``delauney`` package.

Mirrors src/delauney/__init__.py of timdahmen/integer_delauney: the same
public names, with the CUDA classes resolved lazily from ``_delauney_cuda`` so
that importing the package works on a machine without a GPU.  A caller of the
reference switches with ``import integer_delauney_b200 as delauney``, or by
registering this package and its ``_delauney_cuda`` module under the names
``delauney`` and ``delauney._delauney_cuda`` in ``sys.modules`` before the
first import.
"""
from __future__ import annotations

import math

_CUDA_EXPORTS = {"Voronoi", "GridTriangulation", "Delaunay", "triangulate", "triangulate_batch"}

__all__ = list(_CUDA_EXPORTS) + ["DEFAULT_BORDER_PADDING", "max_boundary_spacing"]

#: Pixels of Voronoi canvas added on each side when a caller does not choose
#: (src/delauney/__init__.py:6-16).  A triangle is registered where three
#: Voronoi regions meet -- its circumcentre -- so border triangles need canvas
#: beyond the image to be seen at all.
DEFAULT_BORDER_PADDING = 16


def max_boundary_spacing(border_padding: int = DEFAULT_BORDER_PADDING) -> int:
    """Largest convex-hull boundary seed spacing s for which no triangle is missed.

    Inverts the bound border_padding >= s^2 / 8 (src/delauney/__init__.py:18-24):
    the largest integer s with s^2 <= 8 * border_padding, 0 for no padding.
    """
    if border_padding <= 0:
        return 0
    return math.isqrt(8 * int(border_padding))


def __getattr__(name):
    if name in _CUDA_EXPORTS:
        from . import _delauney_cuda as _cu
        globals().update({k: getattr(_cu, k) for k in _CUDA_EXPORTS if hasattr(_cu, k)})
        if name in globals():
            return globals()[name]
    raise AttributeError(f"module 'integer_delauney_b200' has no attribute {name!r}")
