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
