"""Run the reference project's own test suite against this drop-in.

    python tests/reference_suite.py REFERENCE_TESTS_DIR REFERENCE_SRC_DIR [pytest args...]

REFERENCE_TESTS_DIR is the reference's tests/ directory and REFERENCE_SRC_DIR
its src/ directory (the parent of its ``delauney`` package), used as they are:
nothing is copied into this repository and no test is edited.  Before pytest
imports a test module, the module names the reference's tests use are bound to
this library:

* ``delauney``                  -> ``integer_delauney_b200`` (same public names:
                                   triangulate, Voronoi, GridTriangulation,
                                   Delaunay, DEFAULT_BORDER_PADDING,
                                   max_boundary_spacing)
* ``delauney._delauney_cuda``   -> ``integer_delauney_b200._delauney_cuda``
* ``delauney.reference``        -> the reference's own NumPy implementation,
                                   loaded from REFERENCE_SRC_DIR, which the
                                   reference's CUDA tests use as their oracle.

That is the switch a user of the reference makes (the drop-in registered under
the reference's module names), so a passing test is the reference's own
contract met as written.  Needs a CUDA device: the reference's GPU tests skip
themselves otherwise.  Not collected by this repository's pytest run (the file
name does not start with ``test_``).
"""
from __future__ import annotations

import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def install_aliases(reference_src: str) -> None:
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import integer_delauney_b200 as pkg
    from integer_delauney_b200 import _delauney_cuda
    sys.modules["delauney"] = pkg
    sys.modules["delauney._delauney_cuda"] = _delauney_cuda
    ref_dir = os.path.join(reference_src, "delauney", "reference")
    spec = importlib.util.spec_from_file_location("delauney.reference", os.path.join(ref_dir, "__init__.py"),
                                                  submodule_search_locations=[ref_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["delauney.reference"] = mod
    spec.loader.exec_module(mod)
    pkg.reference = mod


def main(argv: list[str]) -> int:
    if len(argv) < 2:
        print(__doc__, file=sys.stderr)
        return 2
    tests_dir, src_dir = argv[0], argv[1]
    install_aliases(src_dir)
    import pytest
    return int(pytest.main([tests_dir, "-p", "no:cacheprovider", "-q", "-rfEs", *argv[2:]]))


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
