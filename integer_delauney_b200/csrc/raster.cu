// Stage (d): which triangle contains each pixel.
//
// Reference semantics (src/cuda/triangulation.cu:101-137 with
// geometry_device.cuh:68-86): pixel (x, y) is the integer point (x, y); it
// belongs to the highest triangle id among the detected triangles whose closed
// point-in-triangle test accepts it, and to -1 if none does.  The reference
// finds candidates by looping over ALL seeds per pixel, keeping those within a
// Chebyshev window_cap = max(20, max_side + 3) (max_side: the longest side over
// all triangles, float-truncated, triangulation.cu:355-368), and testing their
// CSR triangles -- O(W*H*N) work.
//
// Here each triangle rasterises itself instead: for every row its vertices
// span, the exact integer x-interval of the closed triangle is found from the
// three edge functions in int64, and atomicMax writes the triangle id into
// every pixel of it.  The window never excludes a pixel of a non-degenerate
// triangle (any vertex of a triangle is within its longest side of every
// point inside it, and window_cap exceeds every side), so the result is the
// same set union, computed in O(covered pixels).
//
// Two details keep it bit-equal:
//  * The reference's test is float.  For pixel and seed coordinates in
//    [0, 4096) every product in it is an exact float below 2^24 and the sign
//    of the difference is exact, so float and int64 agree; beyond that the
//    int64 test is the exact one.
//  * A degenerate (collinear) triangle passes the closed test at every point
//    of its supporting line (all three cross products are 0) and nowhere else.
//    The reference then reaches it only through the window, so such a triangle
//    covers the points of its line within Chebyshev window_cap of one of its
//    vertices, clipped to the image.  That case is rasterised separately.
#include "context.cuh"

namespace idl {
namespace {

__device__ __forceinline__ long long floor_div(long long p, long long q)   // q > 0
{
    return p >= 0 ? p / q : -((-p + q - 1) / q);
}
__device__ __forceinline__ long long ceil_div_ll(long long p, long long q) { return -floor_div(-p, q); }

// Longest side as triangulation.cu:357-362 computes it: float dx, dy,
// dx*dx + dy*dy rounded per operation, sqrtf, truncation.
__global__ void k_max_side(const int32_t* __restrict__ tris, const Scalars* __restrict__ sc_in,
                           const int32_t* __restrict__ xs, const int32_t* __restrict__ ys, Scalars* __restrict__ sc)
{
    const long long nt = sc_in->n_triangles;
    int best = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nt;
         t += (long long)gridDim.x * blockDim.x) {
        const int32_t* v = tris + t * 5 + 2;
        const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float dx = (float)(xs[v[pa[k]]] - xs[v[pb[k]]]);
            const float dy = (float)(ys[v[pa[k]]] - ys[v[pb[k]]]);
            const float s = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
            const int l = (int)__fsqrt_rn(s);
            best = max(best, l);
        }
    }
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best > 0) atomicMax(&sc->max_side, best);
}

// One warp per triangle; lanes take rows.
__global__ void __launch_bounds__(256)
k_raster(const int32_t* __restrict__ tris, const Scalars* __restrict__ sc, const int32_t* __restrict__ xs,
         const int32_t* __restrict__ ys, int W, int H, int32_t* __restrict__ tgrid)
{
    const long long nt = sc->n_triangles;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nt; t += warps) {
        const int32_t* v = tris + t * 5 + 2;
        const long long ax = xs[v[0]], ay = ys[v[0]], bx = xs[v[1]], by = ys[v[1]], cx = xs[v[2]], cy = ys[v[2]];
        const long long area2 = (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
        const int32_t tid = (int32_t)t;
        if (area2 == 0) {
            // collinear: supporting line within the reference's seed window
            if (lane != 0) continue;
            const int wc = max(20, sc->max_side + 3);
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
            continue;
        }
        const long long sgn = area2 > 0 ? 1 : -1;
        // d_i(x, y) = A_i * x + B_i * y + C_i for edges (a,b), (b,c), (c,a):
        // cross(u - p, w - p) = (uy - wy) * px + (wx - ux) * py + (ux*wy - uy*wx)
        const long long A[3] = {sgn * (ay - by), sgn * (by - cy), sgn * (cy - ay)};
        const long long B[3] = {sgn * (bx - ax), sgn * (cx - bx), sgn * (ax - cx)};
        const long long C0[3] = {sgn * (ax * by - ay * bx), sgn * (bx * cy - by * cx), sgn * (cx * ay - cy * ax)};
        const long long y0 = max(0ll, min(ay, min(by, cy)));
        const long long y1 = min((long long)H - 1, max(ay, max(by, cy)));
        for (long long y = y0 + lane; y <= y1; y += 32) {
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
}

}  // namespace

void assign_pixels(Context& C, int W, int H, const int32_t* xs, const int32_t* ys, int32_t* tgrid, int64_t max_tri)
{
    IDL_CUDA(cudaMemsetAsync(tgrid, 0xFF, (size_t)W * H * sizeof(int32_t), C.stream));
    if (max_tri <= 0) return;
    IDL_CUDA(cudaMemsetAsync(&C.sc()->max_side, 0, sizeof(int32_t), C.stream));
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(max_tri, 256), C.num_sms * 8));
    k_max_side<<<g, 256, 0, C.stream>>>(C.tris.as<int32_t>(), C.sc(), xs, ys, C.sc());
    IDL_LAUNCH();
    const int gr = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(max_tri, 8), C.num_sms * 16));
    k_raster<<<gr, 256, 0, C.stream>>>(C.tris.as<int32_t>(), C.sc(), xs, ys, W, H, tgrid);
    IDL_LAUNCH();
}

}  // namespace idl
