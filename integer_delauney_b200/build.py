"""Build recipe for the library's CUDA code (libidelaunay.so, in-tree).

Every .cu under csrc/ is compiled for sm_100a only and linked into one shared
library next to this file, which the Python layer loads with ctypes.  No JIT
cache, no torch extension machinery: the built .so travels with the tree.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_NAME = "libidelaunay.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(HERE, "csrc", "*.h")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


def lib_path() -> str:
    return os.path.join(HERE, LIB_NAME)


def up_to_date() -> bool:
    out = lib_path()
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compile every csrc/*.cu into libidelaunay.so (objects in _build/)."""
    out = lib_path()
    if not force and up_to_date():
        return out
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc(), *ARCH_FLAGS, *NVCC_FLAGS, *(extra or []), "-I", os.path.join(ROOT, "include"),
               "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        text = p.communicate()[0].decode(errors="replace")
        if p.returncode != 0:
            failed.append(f"{src}:\n{text}")
        elif verbose and text.strip():
            print(text, file=sys.stderr)
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(failed))
    tmp = out + ".tmp"
    link = [nvcc(), *ARCH_FLAGS, "-shared", "-o", tmp, *objs, "-lcudart"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
