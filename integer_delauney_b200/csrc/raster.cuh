// Device helpers of stage (d), shared by the single-image raster
// (raster.cu) and the batched one (batch.cu).  The rules they implement are
// documented at the top of raster.cu.
#pragma once

#include "context.cuh"

namespace idl {

__device__ __forceinline__ long long floor_div(long long p, long long q)   // q > 0
{
    return p >= 0 ? p / q : -((-p + q - 1) / q);
}
__device__ __forceinline__ long long ceil_div_ll(long long p, long long q) { return -floor_div(-p, q); }

// Longest side of one triangle as triangulation.cu:357-362 computes it: float
// dx, dy, dx*dx + dy*dy rounded per operation, sqrtf, truncation.
__device__ __forceinline__ int tri_max_side(const int32_t* v, const int32_t* __restrict__ xs,
                                            const int32_t* __restrict__ ys)
{
    const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
    int best = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float dx = (float)(xs[v[pa[k]]] - xs[v[pb[k]]]);
        const float dy = (float)(ys[v[pa[k]]] - ys[v[pb[k]]]);
        const float s = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        best = max(best, (int)__fsqrt_rn(s));
    }
    return best;
}

constexpr int BIG_ROWS = 64;

// The x-interval [xl, xr] of row y inside the closed triangle (a, b, c), in
// exact integers; false if the row misses it.
__device__ __forceinline__ bool tri_row_span(long long ax, long long ay, long long bx, long long by, long long cx,
                                             long long cy, long long y, int W, long long& xl, long long& xr)
{
    const long long area2 = (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
    const long long sgn = area2 > 0 ? 1 : -1;
    const long long A[3] = {sgn * (ay - by), sgn * (by - cy), sgn * (cy - ay)};
    const long long B[3] = {sgn * (bx - ax), sgn * (cx - bx), sgn * (ax - cx)};
    const long long C0[3] = {sgn * (ax * by - ay * bx), sgn * (bx * cy - by * cx), sgn * (cx * ay - cy * ax)};
    xl = 0;
    xr = W - 1;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const long long c = B[e] * y + C0[e];   // need A*x + c >= 0
        if (A[e] > 0) xl = max(xl, ceil_div_ll(-c, A[e]));
        else if (A[e] < 0) xr = min(xr, floor_div(c, -A[e]));
        else if (c < 0) return false;
    }
    return xl <= xr;
}

// Rasterise one triangle (vertex ids v, coordinates xs/ys) into a W x H grid
// of triangle ids with atomicMax; a group of G lanes shares the rows (`lane`
// is the caller's index in its group).  wc: the degenerate-case seed window
// (max(20, max_side + 3)).  With `big` set, a proper triangle spanning
// BIG_ROWS rows or more is appended to big (count *n_big) instead, for
// raster_rows_block.
template <int G = 32>
__device__ __forceinline__ void raster_one(const int32_t* v, int32_t tid, const int32_t* __restrict__ xs,
                                           const int32_t* __restrict__ ys, int W, int H, int wc,
                                           int32_t* __restrict__ tgrid, int lane, int32_t* big = nullptr,
                                           int32_t* n_big = nullptr)
{
    const long long ax = xs[v[0]], ay = ys[v[0]], bx = xs[v[1]], by = ys[v[1]], cx = xs[v[2]], cy = ys[v[2]];
    const long long area2 = (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
    if (area2 == 0) {
        // collinear: supporting line within the reference's seed window
        if (lane != 0) return;
        const long long lo_y = max(0ll, min(ay, min(by, cy)) - wc);
        const long long hi_y = min((long long)H - 1, max(ay, max(by, cy)) + wc);
        for (long long y = lo_y; y <= hi_y; ++y) {
            long long x_lo, x_hi;
            if (by == ay) {
                if (y != ay) continue;
                x_lo = 0; x_hi = W - 1;
            } else {
                const long long num = (bx - ax) * (y - ay);
                const long long den = by - ay;
                if (num % den != 0) continue;
                x_lo = x_hi = ax + num / den;
            }
            for (long long x = max(0ll, x_lo); x <= min((long long)W - 1, x_hi); ++x) {
                const bool near = (llabs(ax - x) <= wc && llabs(ay - y) <= wc) ||
                                  (llabs(bx - x) <= wc && llabs(by - y) <= wc) ||
                                  (llabs(cx - x) <= wc && llabs(cy - y) <= wc);
                if (near) atomicMax(&tgrid[(size_t)y * W + x], tid);
            }
        }
        return;
    }
    const long long sgn = area2 > 0 ? 1 : -1;
    const long long y0 = max(0ll, min(ay, min(by, cy)));
    const long long y1 = min((long long)H - 1, max(ay, max(by, cy)));
    if (big && y1 - y0 >= BIG_ROWS) {   // tall: its rows go to a whole block, lanes along each row
        if (lane == 0) big[atomicAdd(n_big, 1)] = tid;
        return;
    }
    // d_i(x, y) = A_i * x + B_i * y + C_i for edges (a,b), (b,c), (c,a):
    // cross(u - p, w - p) = (uy - wy) * px + (wx - ux) * py + (ux*wy - uy*wx)
    const long long A[3] = {sgn * (ay - by), sgn * (by - cy), sgn * (cy - ay)};
    const long long B[3] = {sgn * (bx - ax), sgn * (cx - bx), sgn * (ax - cx)};
    const long long C0[3] = {sgn * (ax * by - ay * bx), sgn * (bx * cy - by * cx), sgn * (cx * ay - cy * ax)};
    for (long long y = y0 + lane; y <= y1; y += G) {
        long long xl = 0, xr = W - 1;
        bool empty = false;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const long long c = B[e] * y + C0[e];   // need A*x + c >= 0
            if (A[e] > 0) xl = max(xl, ceil_div_ll(-c, A[e]));
            else if (A[e] < 0) xr = min(xr, floor_div(c, -A[e]));
            else if (c < 0) empty = true;
        }
        if (empty) continue;
        int32_t* row = tgrid + (size_t)y * W;
        for (long long x = xl; x <= xr; ++x) atomicMax(&row[x], tid);
    }
}

// The rows of one proper triangle split over a whole block: each warp takes a
// row, its lanes the row's pixels.
__device__ __forceinline__ void raster_rows_block(const int32_t* v, int32_t tid, const int32_t* __restrict__ xs,
                                                  const int32_t* __restrict__ ys, int W, int H,
                                                  int32_t* __restrict__ tgrid)
{
    const long long ax = xs[v[0]], ay = ys[v[0]], bx = xs[v[1]], by = ys[v[1]], cx = xs[v[2]], cy = ys[v[2]];
    const long long y0 = max(0ll, min(ay, min(by, cy)));
    const long long y1 = min((long long)H - 1, max(ay, max(by, cy)));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (long long y = y0 + warp; y <= y1; y += nwarps) {
        long long xl, xr;
        if (!tri_row_span(ax, ay, bx, by, cx, cy, y, W, xl, xr)) continue;
        int32_t* row = tgrid + (size_t)y * W;
        for (long long x = xl + lane; x <= xr; x += 32) atomicMax(&row[x], tid);
    }
}

}  // namespace idl
