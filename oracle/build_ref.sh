#!/usr/bin/env bash
# Build the reference's own CUDA batch path for sm_100a into
# oracle/_ref/libref_cuda.so (parity pinning only; never part of the product).
#
# Sources: src/cuda/voronoi.cu and src/cuda/triangulation.cu of
# timdahmen/integer_delauney with the headers they include, compiled from a
# temporary copy (deleted on exit, never placed in this repository) because
# one line needs a portability edit: nvcc's front end rejects the braced-init
# range-for at src/cuda/triangle_csr.cuh:34, so it is rewritten as a loop over
# a local array with the same three values.  The host code's std::sqrtf
# (triangulation.cu:305, absent from libstdc++) is provided by a forced-include
# shim.  No reference source is copied into the repository; only the built
# .so lands in oracle/_ref/, which is git-ignored.
set -euo pipefail
REF="${1:-/root/reference}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
[ -d "$REF/src/cuda" ] || { echo "reference source tree not found at $REF" >&2; exit 1; }
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
for f in voronoi.cu voronoi.cuh triangulation.cu triangulation.cuh triangle_detect.cuh triangle_csr.cuh \
         geometry_device.cuh phase_timer.cuh cuda_check.cuh device_buffer.cuh; do
    cp "$REF/src/cuda/$f" "$TMP/"
done
sed -i 's/for (int32_t s : {t.orig_a, t.orig_b, t.orig_c})/const int32_t idl_vs_[3] = {t.orig_a, t.orig_b, t.orig_c}; for (int32_t s : idl_vs_)/' \
    "$TMP/triangle_csr.cuh"
grep -q "idl_vs_" "$TMP/triangle_csr.cuh" || { echo "portability edit did not apply" >&2; exit 1; }
cat > "$TMP/idl_compat.h" <<'H'
#include <cmath>
namespace std { inline float sqrtf(float x) { return ::sqrtf(x); } }
H
"$NVCC" -std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -shared \
    -include "$TMP/idl_compat.h" -I "$TMP" \
    "$TMP/voronoi.cu" "$TMP/triangulation.cu" "$HERE/ref_shim.cu" -o "$OUT/libref_cuda.so.tmp"
mv "$OUT/libref_cuda.so.tmp" "$OUT/libref_cuda.so"
echo "$OUT/libref_cuda.so"
