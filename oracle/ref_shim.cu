// C shim over the reference's own CUDA batch path, for parity pinning only.
//
// Test infrastructure: built by oracle/build_ref.sh together with the
// reference's src/cuda/voronoi.cu and src/cuda/triangulation.cu into
// oracle/_ref/libref_cuda.so, and loaded only by tests/ to compare the
// library's output with what the reference's CUDA code computes on the same
// GPU.  Seeds arrive already sorted by (x, y), as the reference's binding
// passes them (src/cuda/bindings/binding_helpers.hpp:23-46).
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "voronoi.cuh"
#include "triangulation.cuh"

static thread_local std::string g_err;

extern "C" __attribute__((visibility("default"))) const char* ref_last_error() { return g_err.c_str(); }

extern "C" __attribute__((visibility("default")))
int ref_voronoi(int W, int H, const int32_t* sorted_xy, int n, int32_t* out_grid)
{
    try {
        std::vector<Seed> seeds(n);
        for (int i = 0; i < n; ++i) seeds[i] = {sorted_xy[2 * i], sorted_xy[2 * i + 1]};
        std::vector<int32_t> out;
        cuda_compute_voronoi(W, H, seeds, out);
        std::memcpy(out_grid, out.data(), out.size() * sizeof(int32_t));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

extern "C" __attribute__((visibility("default")))
int ref_triangulate(int W, int H, const int32_t* sorted_xy, int n, const int32_t* vgrid, int P,
                    int32_t* out_grid, int32_t* tris_out, int64_t cap, int64_t* n_tri, int32_t* padded_out)
{
    try {
        std::vector<int32_t> xs(n), ys(n);
        for (int i = 0; i < n; ++i) { xs[i] = sorted_xy[2 * i]; ys[i] = sorted_xy[2 * i + 1]; }
        std::vector<TriangleEntry> tris;
        std::vector<int32_t> grid, padded;
        cuda_compute_triangulation(W, H, vgrid, xs, ys, tris, grid, nullptr, P, padded_out ? &padded : nullptr);
        std::memcpy(out_grid, grid.data(), grid.size() * sizeof(int32_t));
        *n_tri = (int64_t)tris.size();
        if ((int64_t)tris.size() > cap) return 2;
        for (size_t t = 0; t < tris.size(); ++t) {
            tris_out[t * 5 + 0] = tris[t].x;
            tris_out[t * 5 + 1] = tris[t].y;
            tris_out[t * 5 + 2] = tris[t].id_a;
            tris_out[t * 5 + 3] = tris[t].id_b;
            tris_out[t * 5 + 4] = tris[t].id_c;
        }
        if (padded_out && !padded.empty()) std::memcpy(padded_out, padded.data(), padded.size() * sizeof(int32_t));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}
