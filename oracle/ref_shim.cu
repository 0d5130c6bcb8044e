// C shim over the reference's own CUDA code, for parity pinning only.
//
// Test infrastructure: built by oracle/build_ref.sh together with the
// reference's src/cuda/voronoi.cu, src/cuda/triangulation.cu and the
// src/cuda/delaunay*.cu sources of its incremental Delaunay class into
// oracle/_ref/libref_cuda.so, and loaded only by tests/ and by bench.py's
// reference-CUDA timing leg to compare the library's output and speed with
// what the reference's CUDA code computes on the same GPU.  Seeds for the
// batch entry points arrive already sorted by (x, y), as the reference's
// binding passes them (src/cuda/bindings/binding_helpers.hpp:23-46); the
// incremental entry points take seeds in insertion order, as
// src/cuda/bindings/py_delaunay.hpp passes them to Delaunay::insert_deferred.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "voronoi.cuh"
#include "triangulation.cuh"
#include "delaunay.cuh"

#define REF_API extern "C" __attribute__((visibility("default")))

static thread_local std::string g_err;

REF_API const char* ref_last_error() { return g_err.c_str(); }

REF_API int ref_voronoi(int W, int H, const int32_t* sorted_xy, int n, int32_t* out_grid)
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

static int copy_tris(const std::vector<TriangleEntry>& tris, int32_t* out, int64_t cap, int64_t* n_tri)
{
    *n_tri = (int64_t)tris.size();
    if ((int64_t)tris.size() > cap) return 2;
    for (size_t t = 0; t < tris.size(); ++t) {
        out[t * 5 + 0] = tris[t].x;
        out[t * 5 + 1] = tris[t].y;
        out[t * 5 + 2] = tris[t].id_a;
        out[t * 5 + 3] = tris[t].id_b;
        out[t * 5 + 4] = tris[t].id_c;
    }
    return 0;
}

REF_API int ref_triangulate(int W, int H, const int32_t* sorted_xy, int n, const int32_t* vgrid, int P,
                            int32_t* out_grid, int32_t* tris_out, int64_t cap, int64_t* n_tri,
                            int32_t* padded_out)
{
    try {
        std::vector<int32_t> xs(n), ys(n);
        for (int i = 0; i < n; ++i) { xs[i] = sorted_xy[2 * i]; ys[i] = sorted_xy[2 * i + 1]; }
        std::vector<TriangleEntry> tris;
        std::vector<int32_t> grid, padded;
        cuda_compute_triangulation(W, H, vgrid, xs, ys, tris, grid, nullptr, P, padded_out ? &padded : nullptr);
        std::memcpy(out_grid, grid.data(), grid.size() * sizeof(int32_t));
        if (copy_tris(tris, tris_out, cap, n_tri)) return 2;
        if (padded_out && !padded.empty()) std::memcpy(padded_out, padded.data(), padded.size() * sizeof(int32_t));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// The reference's stock triangulate() path (src/cuda/bindings/triangulate.hpp:15-43)
// minus the Python object handling: validate and sort the seeds as
// binding_helpers.hpp:23-46 does (bounds, empty, (x, y) order, duplicates),
// then cuda_compute_triangulation with no caller diagram, which builds the
// padded Voronoi diagram itself.  Seeds in caller order; outputs as ref_triangulate.
REF_API int ref_triangulate_stock(int W, int H, const int32_t* xy, int n, int P,
                                  int32_t* out_grid, int32_t* tris_out, int64_t cap, int64_t* n_tri)
{
    try {
        if (W <= 0 || H <= 0) throw std::invalid_argument("width and height must be positive");
        std::vector<Seed> seeds;
        seeds.reserve(n);
        for (int i = 0; i < n; ++i) {
            const int x = xy[2 * i], y = xy[2 * i + 1];
            if (x < 0 || x >= W || y < 0 || y >= H) throw std::invalid_argument("seed coordinate out of bounds");
            seeds.push_back({x, y});
        }
        if (seeds.empty()) throw std::invalid_argument("seeds must not be empty");
        std::sort(seeds.begin(), seeds.end(),
                  [](const Seed& a, const Seed& b) { return a.x != b.x ? a.x < b.x : a.y < b.y; });
        for (size_t i = 1; i < seeds.size(); ++i)
            if (seeds[i].x == seeds[i - 1].x && seeds[i].y == seeds[i - 1].y)
                throw std::invalid_argument("duplicate seed positions are not allowed");
        std::vector<int32_t> xs(n), ys(n);
        for (int i = 0; i < n; ++i) { xs[i] = seeds[i].x; ys[i] = seeds[i].y; }
        std::vector<TriangleEntry> tris;
        std::vector<int32_t> grid;
        cuda_compute_triangulation(W, H, nullptr, xs, ys, tris, grid, nullptr, P);
        std::memcpy(out_grid, grid.data(), grid.size() * sizeof(int32_t));
        return copy_tris(tris, tris_out, cap, n_tri);
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// ---- the incremental Delaunay class (src/cuda/delaunay.cuh) ----

REF_API void* ref_dl_create(int W, int H, int max_seeds, int P)
{
    try {
        return new Delaunay(W, H, max_seeds, P);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

REF_API void ref_dl_destroy(void* h) { delete static_cast<Delaunay*>(h); }

REF_API int ref_dl_seed_count(void* h) { return static_cast<Delaunay*>(h)->seed_count(); }

// insert_deferred (delaunay.cu:236-285); xy in insertion order.  bfs_iters, if
// non-null, receives the Jacobi passes the reference ran.
REF_API int ref_dl_insert_deferred(void* h, const int32_t* xy, int k, int* bfs_iters)
{
    try {
        std::vector<int32_t> xs(k), ys(k);
        for (int i = 0; i < k; ++i) { xs[i] = xy[2 * i]; ys[i] = xy[2 * i + 1]; }
        InsertTimings t;
        static_cast<Delaunay*>(h)->insert_deferred(xs, ys, bfs_iters ? &t : nullptr);
        if (bfs_iters) *bfs_iters = t.bfs_iters;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// finalise (delaunay.cu:287-310): triangle map in sorted-rank vertex ids and
// the (H, W, 3) grid.  Returns 2 with *n_tri set when cap is too small.
REF_API int ref_dl_finalise(void* h, int32_t* grid_out, int32_t* tris_out, int64_t cap, int64_t* n_tri)
{
    try {
        std::vector<TriangleEntry> tris;
        std::vector<int32_t> grid;
        static_cast<Delaunay*>(h)->finalise(tris, grid);
        std::memcpy(grid_out, grid.data(), grid.size() * sizeof(int32_t));
        return copy_tris(tris, tris_out, cap, n_tri);
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// get_voronoi_grid (delaunay_output.cu:165-186): (H, W, 2) sorted-rank label
// and squared distance, cropped from the padded canvas.
REF_API int ref_dl_voronoi_grid(void* h, int32_t* out)
{
    try {
        std::vector<int32_t> g;
        static_cast<Delaunay*>(h)->get_voronoi_grid(g);
        std::memcpy(out, g.data(), g.size() * sizeof(int32_t));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// get_triangles (delaunay_output.cu:192-206): live triangles, insertion-order
// vertex ids, canonical position in image coordinates.
REF_API int ref_dl_triangles(void* h, int32_t* out, int64_t cap, int64_t* n_tri)
{
    try {
        std::vector<TriangleEntry> tris;
        static_cast<Delaunay*>(h)->get_triangles(tris);
        return copy_tris(tris, out, cap, n_tri);
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// sorted_rank (delaunay.cuh): insertion id -> (x, y)-sorted id.
REF_API int ref_dl_sorted_rank(void* h, int32_t* out)
{
    try {
        const auto& r = static_cast<Delaunay*>(h)->sorted_rank();
        std::memcpy(out, r.data(), r.size() * sizeof(int32_t));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}
