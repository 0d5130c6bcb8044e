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
#include "raster.cuh"

namespace idl {
namespace {

__global__ void k_max_side(const int32_t* __restrict__ tris, const Scalars* __restrict__ sc_in,
                           const int32_t* __restrict__ xs, const int32_t* __restrict__ ys, Scalars* __restrict__ sc)
{
    const long long nt = sc_in->n_triangles;
    int best = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nt;
         t += (long long)gridDim.x * blockDim.x)
        best = max(best, tri_max_side(tris + t * 5 + 2, xs, ys));
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best > 0) atomicMax(&sc->max_side, best);
}

// A group of RASTER_GROUP lanes per triangle (four triangles per warp: a
// Delaunay triangle of a dense seed set spans a few rows); lanes take rows.
constexpr int RASTER_GROUP = 8;

__global__ void __launch_bounds__(256)
k_raster(const int32_t* __restrict__ tris, Scalars* __restrict__ sc, const int32_t* __restrict__ xs,
         const int32_t* __restrict__ ys, int W, int H, int32_t* __restrict__ tgrid, int32_t* __restrict__ big)
{
    const long long nt = sc->n_triangles;
    const int lane = threadIdx.x % RASTER_GROUP;
    const int wc = max(20, sc->max_side + 3);
    const long long groups = (long long)gridDim.x * (blockDim.x / RASTER_GROUP);
    for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / RASTER_GROUP; t < nt; t += groups)
        raster_one<RASTER_GROUP>(tris + t * 5 + 2, (int32_t)t, xs, ys, W, H, wc, tgrid, lane, big, &sc->n_big);
}

// The tall triangles k_raster set aside: one block per triangle.
__global__ void __launch_bounds__(256)
k_raster_big(const int32_t* __restrict__ tris, const Scalars* __restrict__ sc, const int32_t* __restrict__ xs,
             const int32_t* __restrict__ ys, int W, int H, int32_t* __restrict__ tgrid,
             const int32_t* __restrict__ big)
{
    const int nb = sc->n_big;
    for (int i = blockIdx.x; i < nb; i += gridDim.x) {
        const int32_t t = big[i];
        raster_rows_block(tris + (size_t)t * 5 + 2, t, xs, ys, W, H, tgrid);
    }
}

}  // namespace

void assign_pixels(Context& C, int W, int H, const int32_t* xs, const int32_t* ys, int32_t* tgrid, int64_t max_tri)
{
    IDL_CUDA(cudaMemsetAsync(tgrid, 0xFF, (size_t)W * H * sizeof(int32_t), C.stream));
    if (max_tri <= 0) return;
    IDL_CUDA(cudaMemsetAsync(&C.sc()->max_side, 0, 2 * sizeof(int32_t), C.stream));   // max_side, n_big
    C.rbig.ensure((size_t)max_tri * 4);
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(max_tri, 256), C.num_sms * 8));
    k_max_side<<<g, 256, 0, C.stream>>>(C.tris.as<int32_t>(), C.sc(), xs, ys, C.sc());
    IDL_LAUNCH();
    const int gr = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(max_tri, 256 / RASTER_GROUP),
                                                                C.num_sms * 16));
    k_raster<<<gr, 256, 0, C.stream>>>(C.tris.as<int32_t>(), C.sc(), xs, ys, W, H, tgrid, C.rbig.as<int32_t>());
    IDL_LAUNCH();
    k_raster_big<<<C.num_sms * 4, 256, 0, C.stream>>>(C.tris.as<int32_t>(), C.sc(), xs, ys, W, H, tgrid,
                                                      C.rbig.as<int32_t>());
    IDL_LAUNCH();
}

}  // namespace idl
