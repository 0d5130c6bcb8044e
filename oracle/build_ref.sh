#!/usr/bin/env bash
# Build the reference's own CUDA code for sm_100a into oracle/_ref/libref_cuda.so
# (parity pinning and the reference-CUDA timing leg only; never part of the
# product).
#
# Usage: oracle/build_ref.sh [REFERENCE_SOURCE_TREE]
# The source tree defaults to $IDL_REFERENCE_SRC, else to BASELINE.json's
# reference_path at the repository root.
#
# Sources: the batch path (src/cuda/voronoi.cu, src/cuda/triangulation.cu) and
# the incremental Delaunay class (src/cuda/delaunay.cu, delaunay_voronoi.cu,
# delaunay_topology.cu, delaunay_assign.cu, delaunay_output.cu,
# delaunay_query.cu, delaunay_scalar_field.cu) of timdahmen/integer_delauney
# with the headers they include, compiled from a temporary copy (deleted on
# exit, never placed in this repository) because one line needs a portability
# edit: nvcc's front end rejects the braced-init range-for at
# src/cuda/triangle_csr.cuh:34, so it is rewritten as a loop over a local array
# with the same three values.  The host code's std::sqrtf (triangulation.cu:305,
# absent from libstdc++) is provided by a forced-include shim.  No reference
# source is copied into the repository; only the built .so lands in
# oracle/_ref/, which is git-ignored.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT="$(dirname "$HERE")"
default_ref() {
    if [ -n "${IDL_REFERENCE_SRC:-}" ]; then echo "$IDL_REFERENCE_SRC"; return; fi
    python3 -c 'import json,sys; print(json.load(open(sys.argv[1])).get("reference_path", ""))' \
        "$ROOT/BASELINE.json" 2>/dev/null || true
}
REF="${1:-$(default_ref)}"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
[ -n "$REF" ] && [ -d "$REF/src/cuda" ] || { echo "reference source tree not found at '$REF'" >&2; exit 1; }
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
BATCH_SRC="voronoi.cu triangulation.cu"
INC_SRC="delaunay.cu delaunay_voronoi.cu delaunay_topology.cu delaunay_assign.cu delaunay_output.cu \
delaunay_query.cu delaunay_scalar_field.cu"
HEADERS="voronoi.cuh triangulation.cuh triangle_detect.cuh triangle_csr.cuh geometry_device.cuh phase_timer.cuh \
cuda_check.cuh device_buffer.cuh delaunay.cuh delaunay_locate.cuh"
for f in $BATCH_SRC $INC_SRC $HEADERS; do
    cp "$REF/src/cuda/$f" "$TMP/"
done
sed -i 's/for (int32_t s : {t.orig_a, t.orig_b, t.orig_c})/const int32_t idl_vs_[3] = {t.orig_a, t.orig_b, t.orig_c}; for (int32_t s : idl_vs_)/' \
    "$TMP/triangle_csr.cuh"
grep -q "idl_vs_" "$TMP/triangle_csr.cuh" || { echo "portability edit did not apply" >&2; exit 1; }
cat > "$TMP/idl_compat.h" <<'H'
#include <cmath>
namespace std { inline float sqrtf(float x) { return ::sqrtf(x); } }
H
cp "$HERE/ref_shim.cu" "$TMP/"
FLAGS=(-std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -include "$TMP/idl_compat.h" -I "$TMP")
OBJS=()
pids=()
for f in $BATCH_SRC $INC_SRC ref_shim.cu; do
    "$NVCC" "${FLAGS[@]}" -c "$TMP/$f" -o "$TMP/${f%.cu}.o" &
    pids+=($!)
    OBJS+=("$TMP/${f%.cu}.o")
done
for p in "${pids[@]}"; do wait "$p"; done
"$NVCC" -shared -gencode arch=compute_100a,code=sm_100a "${OBJS[@]}" -o "$OUT/libref_cuda.so.tmp"
mv "$OUT/libref_cuda.so.tmp" "$OUT/libref_cuda.so"
echo "$OUT/libref_cuda.so"
