// Device helpers shared by the propagation kernels (propagate.cu,
// sparse_jacobi.cu): the cell sentinels and the candidate rule.
#pragma once

#include "common.cuh"

namespace idl {

constexpr int32_t OUTSIDE = -2;        // a cell beyond the canvas edge (never an owner)
constexpr int32_t FAR = 0x7FFFFFFF;    // distance of an unowned or outside cell
constexpr unsigned FULL = 0xFFFFFFFFu;

// Offer candidate owner n to a cell holding (bl, bd): adopt it if strictly
// closer, or equally close with a higher id (src/cuda/geometry_device.cuh:22-28,
// src/delauney/reference/voronoi.py:136-154).  An unowned cell has bd = FAR,
// so any owner wins.  Negative n (unowned or outside) is never a candidate.
__device__ __forceinline__ void relax(int32_t& bl, int32_t& bd, int32_t n, int x, int y,
                                      const uint32_t* __restrict__ pos)
{
    if (n < 0 || n == bl) return;
    const int32_t nd = dist2(x, y, __ldg(&pos[n]));
    if (nd < bd || (nd == bd && n > bl)) {
        bl = n;
        bd = nd;
    }
}

}  // namespace idl

namespace idl {

// Owner keys.  During a from-scratch propagation in reference semantics the
// label planes hold, instead of the owner's id, its position packed as
// x << 15 | y (x, y < 32768, so keys are non-negative and below 2^30).  Seed
// ids there are the seeds' (x, y)-sorted order (per image of a batch atlas,
// and cells of different images never meet), so key order is id order and the
// tie rule "equal distance, higher id wins" reads "higher key wins"; the
// candidate's distance comes from its key with no seed-table load.  Negative
// labels (UNDEF, OUTSIDE, batch walls) keep their meaning.
__host__ __device__ inline int32_t key_from_pos(uint32_t p)
{
    return int32_t((uint32_t)pos_x(p) << 15 | (uint32_t)pos_y(p));
}
__host__ __device__ inline int key_x(int32_t k) { return k >> 15; }
__host__ __device__ inline int key_y(int32_t k) { return k & 0x7FFF; }

// Exact for a real key (below 2^31); for a negative label the value is
// meaningless but defined (unsigned wrap-around), and callers mask it out.
__device__ __forceinline__ int32_t key_dist2(int x, int y, int32_t k)
{
    const uint32_t dx = uint32_t(x - key_x(k)), dy = uint32_t(y - key_y(k));
    return int32_t(dx * dx + dy * dy);
}

// relax() on keys, without branches: candidate n (negative = none) replaces
// (bk, bd) if strictly closer, or equally close with a higher key.
__device__ __forceinline__ void relax_key(int32_t& bk, int32_t& bd, int32_t n, int x, int y)
{
    const int32_t nd = key_dist2(x, y, n);
    const bool better = n >= 0 && (nd < bd || (nd == bd && n > bk));
    bk = better ? n : bk;
    bd = better ? nd : bd;
}

// Work lists of the persistent propagation kernel hold 8 x 8 micro-tiles,
// packed as mx | my << 16.
constexpr int MICRO_TILE = 8;
__device__ __forceinline__ int32_t pack_mt(int mx, int my) { return mx | (my << 16); }

}  // namespace idl
