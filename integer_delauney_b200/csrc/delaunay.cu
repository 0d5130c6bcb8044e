// Stage (c): incremental triangulation -- one growing seed set whose Voronoi
// diagram, triangles and pixel assignment stay on the device between calls.
// Replaces the reference's class Delaunay (src/cuda/delaunay.cu,
// delaunay_voronoi.cu, delaunay_topology.cu, delaunay_assign.cu,
// delaunay_output.cu, delaunay_query.cu, delaunay_scalar_field.cu).
//
// State on the device, all sized at construction:
//   planes   two pitch x Hd int32 label planes of the padded canvas, holding
//            insertion-order seed ids (both planes equal between calls);
//   tgrid    Wd x Hd int32 triangle ids of the padded canvas;
//   seed arrays (max_seeds each): image x, y; packed canvas position; batch
//            rank and its inverse; canvas x, y in batch order; values;
//   pixel    W x H triangle id, batch seed id and outside mask for
//            finalise_device.
// Triangles and grow-only query scratch live in the embedded Context.
//
// An insert writes the new seeds into both planes and continues the Jacobi
// iteration from the previous fixed point (delaunay_voronoi.cu:60-108) with the
// persistent sparse kernel, whose first work list is just the micro-tiles
// around the new seeds: everything else is already a fixed point.  Topology
// (detection + canonical numbering) and the raster are recomputed lazily, when
// something reads them, from the whole canvas: detection of a 2080 x 2080
// canvas is a few tens of microseconds on the device, so a per-insert dirty
// region and slot registry (delaunay_topology.cu:185-414) would only add host
// work, and canonical numbering keeps triangle ids dense and history-free.
#include "context.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

namespace idl {

struct DelaunayState {
    Context own;                  // scratch of this object unless a shared workspace is set
    Context* ws = nullptr;        // shared workspace context (idl_delaunay_set_workspace)
    cudaStream_t stream = nullptr;
    int device = 0;
    int W = 0, H = 0, P = 0, Wd = 0, Hd = 0, pitch = 0;
    int64_t max_seeds = 0;
    int mode = IDL_MODE_REFERENCE;
    int64_t N = 0;
    uint64_t generation = 0;
    bool pending = false;
    bool rank_dirty = false, topo_dirty = false, raster_dirty = false, edges_dirty = true;
    bool have_values = false;
    int64_t n_tri = 0, n_edges = 0;

    // device memory owned by this object (allocated in create; reset re-lays
    // the same allocations out for another canvas that fits)
    size_t planes_bytes = 0, tgrid_bytes = 0, pix_bytes = 0;
    int64_t seed_cap = 0;
    int32_t* planes = nullptr;
    int32_t* tgrid = nullptr;
    int32_t* seedmem = nullptr;
    void* pixmem = nullptr;
    int32_t *ix = nullptr, *iy = nullptr, *rank = nullptr, *inv = nullptr, *sx = nullptr, *sy = nullptr;
    uint32_t* pos = nullptr;
    float* values = nullptr;
    int32_t *pix_tid = nullptr, *pix_sid = nullptr;
    uint8_t* pix_out = nullptr;

    // grow-only scratch, stream-ordered on the object's stream
    DevBuf stage, edge_keys, edge_tmp, sort_tmp, num_sel, scores, score_keys, score_sorted, qbuf, qout, batch, verr;
    DevBuf spos;          // exact mode: canvas positions of the seeds in (x, y) order

    template <class F>
    void each_scratch(F&& f)
    {
        DevBuf* all[] = {&stage, &edge_keys, &edge_tmp, &sort_tmp, &num_sel, &scores, &score_keys, &score_sorted,
                         &qbuf, &qout, &batch, &verr, &spos};
        for (DevBuf* b : all) f(*b);
    }
    DelaunayState()
    {
        each_scratch([this](DevBuf& b) { b.stream = &stream; });
    }

    // host mirrors (insertion order, image coordinates)
    std::vector<int32_t> hx, hy;
    std::vector<float> hvals;

    Canvas canvas() const { return Canvas{Wd, Hd, pitch}; }

    // The context whose scratch (and stream) this object's work uses, bound to
    // this object: its label planes point at ours, and if another object used
    // it last, the triangle rows it holds are not ours, so topology is redone
    // when next needed (the raster, ranks and seeds live in our own memory).
    //
    // The binding of the planes is undone when the entry point returns
    // (unbind), so a context lent as a workspace keeps its own label buffers
    // for its other users.
    Context& ctx()
    {
        Context& c = ws ? *ws : own;
        if (!ws && !own.scalars.ptr) ensure_scalars(own);
        if (c.stream != stream) {
            // the context's last user queued work on another stream: let it
            // finish before this object's work (and stream-ordered frees of
            // the scratch) are ordered on ours
            if (ws) IDL_CUDA(cudaStreamSynchronize(c.stream));
            c.stream = stream;
        }
        if (bound != &c) {
            unbind();
            saved[0] = c.lab[0];
            saved[1] = c.lab[1];
            bound = &c;
        }
        const size_t plane = (size_t)pitch * Hd;
        c.lab[0].borrow(planes, plane * 4);
        c.lab[1].borrow(planes + plane, plane * 4);
        if (c.owner != this) {
            c.owner = this;
            topo_dirty = true;
        }
        return c;
    }

    void unbind() noexcept
    {
        if (!bound) return;
        bound->lab[0] = saved[0];
        bound->lab[1] = saved[1];
        bound = nullptr;
    }
    Context* bound = nullptr;     // context whose label buffers currently point at our planes
    DevBuf saved[2];              // its own label buffers meanwhile

    // Device memory of the object comes from the stream-ordered allocator:
    // freeing it never waits for the whole device, which matters when many
    // objects on many streams come and go (a server recycling diagrams).
    void free_owned() noexcept
    {
        if (planes) cudaFreeAsync(planes, stream);
        if (tgrid) cudaFreeAsync(tgrid, stream);
        if (seedmem) cudaFreeAsync(seedmem, stream);
        if (pixmem) cudaFreeAsync(pixmem, stream);
        planes = tgrid = seedmem = nullptr;
        pixmem = nullptr;
        each_scratch([](DevBuf& b) { b.drop(); });
    }
    // Marks the end of the object's work queued so far on its stream.  A
    // stream change makes the new stream wait for it (a device-side wait on
    // this object's own work, not on the rest of the old stream's), so the
    // object's data -- and the stream-ordered frees of its scratch -- stay
    // ordered after everything it did before.
    cudaEvent_t last_use = nullptr;
    void note_use() noexcept
    {
        if (!last_use) return;
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != device) cudaSetDevice(device);
        cudaEventRecord(last_use, stream);
        if (cur >= 0 && cur != device) cudaSetDevice(cur);
    }

    ~DelaunayState()
    {
        unbind();
        if (ws && ws->owner == this) ws->owner = nullptr;
        free_owned();
        if (last_use) cudaEventDestroy(last_use);
    }
};

}  // namespace idl

struct idl_delaunay : idl::DelaunayState {};

namespace idl {
namespace {

// ---- kernels ------------------------------------------------------------

// New seeds take ids first_id, first_id + 1, ... in both planes
// (write_seeds_kernel, delaunay_voronoi.cu:12-25).
__global__ void k_put_seeds(int32_t* __restrict__ a, int32_t* __restrict__ b, int pitch,
                            const uint32_t* __restrict__ pos, int64_t k, int64_t first_id)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const uint32_t p = pos[i];
    const size_t o = (size_t)pos_y(p) * pitch + pos_x(p);
    a[o] = (int32_t)(first_id + i);
    b[o] = (int32_t)(first_id + i);
}

// ---- batch validation (before any change), on the raster as scratch ----
// Out-of-bounds seeds are recorded and skipped; each in-bounds seed's cell
// is reset to "no seed yet".
__global__ void k_v_bounds(const int32_t* __restrict__ xy, int64_t k, int W, int H, int P, int Wd,
                           int32_t* __restrict__ mark, unsigned long long* __restrict__ err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const int32_t x = xy[2 * i], y = xy[2 * i + 1];
    if (x < 0 || y < 0 || x >= W || y >= H) {
        atomicMin(&err[0], (unsigned long long)i);
        return;
    }
    mark[(size_t)(y + P) * Wd + x + P] = 0x7FFFFFFF;
}

// Each cell remembers the first batch index that names it.
__global__ void k_v_first(const int32_t* __restrict__ xy, int64_t k, int W, int H, int P, int Wd,
                          int32_t* __restrict__ mark)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const int32_t x = xy[2 * i], y = xy[2 * i + 1];
    if (x < 0 || y < 0 || x >= W || y >= H) return;
    atomicMin(&mark[(size_t)(y + P) * Wd + x + P], (int32_t)i);
}

// err[1]: first index repeating an earlier one of the batch; err[2]: first
// index at a position the diagram already has a seed on.
__global__ void k_v_check(const int32_t* __restrict__ xy, int64_t k, int W, int H, int P, int Wd, int pitch,
                          const int32_t* __restrict__ mark, const int32_t* __restrict__ plane,
                          const uint32_t* __restrict__ pos, int64_t n_old, unsigned long long* __restrict__ err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const int32_t x = xy[2 * i], y = xy[2 * i + 1];
    if (x < 0 || y < 0 || x >= W || y >= H) return;
    if (mark[(size_t)(y + P) * Wd + x + P] != (int32_t)i) atomicMin(&err[1], (unsigned long long)i);
    const int32_t l = plane[(size_t)(y + P) * pitch + x + P];
    if (l >= 0 && l < n_old && pos[l] == pack_pos(x + P, y + P)) atomicMin(&err[2], (unsigned long long)i);
}

// One block per row of an image's padded canvas: the atlas labels of that
// image, as local ids, into both of the object's planes.
__global__ void k_adopt(const int32_t* __restrict__ atlas, int apitch, int ox, int oy, long long seed_off, int Wd,
                        int32_t* __restrict__ a, int32_t* __restrict__ b, int pitch)
{
    const int r = blockIdx.x;
    const int32_t* src = atlas + (size_t)(oy + r) * apitch + ox;
    const size_t o = (size_t)r * pitch;
    for (int c = threadIdx.x; c < Wd; c += blockDim.x) {
        const int32_t l = src[c];
        const int32_t v = l >= 0 ? (int32_t)(l - seed_off) : UNDEF;
        a[o + c] = v;
        b[o + c] = v;
    }
}

// Exact mode: plane a holds (x, y)-rank labels; move them to plane b and
// put the insertion ids into plane a.
__global__ void k_exact_planes(int32_t* __restrict__ a, int32_t* __restrict__ b, int pitch, int Wd,
                               const int32_t* __restrict__ inv)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= Wd) return;
    const size_t o = (size_t)y * pitch + x;
    const int32_t l = a[o];
    b[o] = l;
    a[o] = l >= 0 ? __ldg(&inv[l]) : l;
}

__global__ void k_split(const int32_t* __restrict__ xy, int64_t k, int32_t* __restrict__ x, int32_t* __restrict__ y)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    x[i] = xy[2 * i];
    y[i] = xy[2 * i + 1];
}

// A group of objects adopting images of one batch: per image the label rows
// (as k_adopt) and the seed coordinates and packed positions (as the copies
// and k_pack_pos of idl_delaunay_adopt), all in one launch; blockIdx.y picks
// the image.
constexpr int ADOPT_GROUP_MAX = 16;
struct AdoptItem {
    const int32_t* atlas;
    const int32_t* sxs;
    const int32_t* sys;
    int32_t* a;
    int32_t* b;
    int32_t* ix;
    int32_t* iy;
    uint32_t* pos;
    long long seed_off, n;
    int apitch, ox, oy, Wd, Hd, pitch, P;
};
struct AdoptGroup {
    AdoptItem it[ADOPT_GROUP_MAX];
};

__global__ void k_adopt_group(AdoptGroup g)
{
    const AdoptItem& m = g.it[blockIdx.y];
    for (int r = blockIdx.x; r < m.Hd; r += gridDim.x) {
        const int32_t* src = m.atlas + (size_t)(m.oy + r) * m.apitch + m.ox;
        const size_t o = (size_t)r * m.pitch;
        for (int c = threadIdx.x; c < m.Wd; c += blockDim.x) {
            const int32_t l = src[c];
            const int32_t v = l >= 0 ? (int32_t)(l - m.seed_off) : UNDEF;
            m.a[o + c] = v;
            m.b[o + c] = v;
        }
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m.n;
         i += (long long)gridDim.x * blockDim.x) {
        const int32_t x = m.sxs[m.seed_off + i], y = m.sys[m.seed_off + i];
        m.ix[i] = x;
        m.iy[i] = y;
        m.pos[i] = pack_pos(x + m.P, y + m.P);
    }
}

__global__ void k_pack_pos(const int32_t* __restrict__ x, const int32_t* __restrict__ y, int64_t k, int P,
                           uint32_t* __restrict__ pos)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) pos[i] = pack_pos(x[i] + P, y[i] + P);
}

__global__ void k_permute(const float* __restrict__ in, const int32_t* __restrict__ rank, int64_t k,
                          float* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) out[rank[i]] = in[i];
}

__device__ __forceinline__ void cell_out(const int32_t* __restrict__ lab, int pitch, int P, int x, int y,
                                         const uint32_t* __restrict__ pos, const int32_t* __restrict__ rank,
                                         int32_t& sid, int32_t& d)
{
    const int32_t l = lab[(size_t)(y + P) * pitch + x + P];
    sid = l >= 0 ? __ldg(&rank[l]) : UNDEF;
    d = l >= 0 ? dist2(x + P, y + P, __ldg(&pos[l])) : -1;
}

// (H, W, 3): batch seed id, squared distance, triangle id
// (Delaunay::build_outputs_, delaunay_output.cu:86-110).
__global__ void k_out3(const int32_t* __restrict__ lab, int pitch, int P, int W, int H,
                       const uint32_t* __restrict__ pos, const int32_t* __restrict__ rank,
                       const int32_t* __restrict__ tgrid, int Wd, int32_t* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    int32_t sid, d;
    cell_out(lab, pitch, P, x, y, pos, rank, sid, d);
    int32_t* o = out + ((size_t)y * W + x) * 3;
    o[0] = sid;
    o[1] = d;
    o[2] = tgrid[(size_t)(y + P) * Wd + x + P];
}

// (H, W, 2): batch seed id, squared distance (delaunay_output.cu:162-184).
__global__ void k_out2(const int32_t* __restrict__ lab, int pitch, int P, int W, int H,
                       const uint32_t* __restrict__ pos, const int32_t* __restrict__ rank, int32_t* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    int32_t sid, d;
    cell_out(lab, pitch, P, x, y, pos, rank, sid, d);
    out[((size_t)y * W + x) * 2] = sid;
    out[((size_t)y * W + x) * 2 + 1] = d;
}

// finalise_device's three arrays (crop_pixel_arrays_kernel,
// delaunay_output.cu:120-144).
__global__ void k_crop(const int32_t* __restrict__ lab, int pitch, int P, int W, int H,
                       const int32_t* __restrict__ rank, const int32_t* __restrict__ tgrid, int Wd,
                       int32_t* __restrict__ tid_out, int32_t* __restrict__ sid_out, uint8_t* __restrict__ mask_out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const int32_t l = lab[(size_t)(y + P) * pitch + x + P];
    const size_t d = (size_t)y * W + x;
    sid_out[d] = l >= 0 ? __ldg(&rank[l]) : l;
    const int32_t t = tgrid[(size_t)(y + P) * Wd + x + P];
    mask_out[d] = t == NO_TRIANGLE ? 1 : 0;
    tid_out[d] = t == NO_TRIANGLE ? 0 : t;
}

// Vertex ids of the canonical triangle rows mapped back to insertion ids.
__global__ void k_tris_insertion(const int32_t* __restrict__ tris, int64_t n, const int32_t* __restrict__ inv,
                                 int32_t* __restrict__ out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
#pragma unroll
    for (int j = 0; j < 3; ++j) out[t * 3 + j] = __ldg(&inv[tris[t * 5 + 2 + j]]);
}

// (a, b, c) of each (x, y, a, b, c) row, batch seed ids unchanged.
__global__ void k_tris_batch_verts(const int32_t* __restrict__ tris, int64_t n, int32_t* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * 3) return;
    const int64_t t = i / 3;
    out[i] = tris[t * 5 + 2 + (i - t * 3)];
}

// Three undirected edge keys a * n + b (a < b, insertion ids) per triangle
// (build_edge_keys_kernel, delaunay_scalar_field.cu:34-56).
__global__ void k_edge_keys(const int32_t* __restrict__ tris, int64_t n_tri, const int32_t* __restrict__ inv,
                            int64_t n_seeds, unsigned long long* __restrict__ keys)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tri) return;
    int32_t v[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) v[j] = __ldg(&inv[tris[t * 5 + 2 + j]]);
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const int32_t p = min(v[e], v[(e + 1) % 3]), q = max(v[e], v[(e + 1) % 3]);
        keys[t * 3 + e] = (unsigned long long)p * (unsigned long long)n_seeds + (unsigned long long)q;
    }
}

__global__ void k_edge_unpack(const unsigned long long* __restrict__ keys, int64_t n_edges, int64_t n_seeds,
                              int32_t* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_edges) return;
    const unsigned long long k = keys[i];
    out[i * 2] = (int32_t)(k / (unsigned long long)n_seeds);
    out[i * 2 + 1] = (int32_t)(k % (unsigned long long)n_seeds);
}

// |dv| * |ab| in double, rounded to float; 0 below min_length
// (score_edges_kernel, delaunay_scalar_field.cu:84-103).
__global__ void k_edge_scores(const unsigned long long* __restrict__ keys, int64_t n_edges, int64_t n_seeds,
                              const int32_t* __restrict__ x, const int32_t* __restrict__ y,
                              const float* __restrict__ values, double min_len2, float* __restrict__ scores)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_edges) return;
    const unsigned long long k = keys[e];
    const int32_t a = (int32_t)(k / (unsigned long long)n_seeds), b = (int32_t)(k % (unsigned long long)n_seeds);
    const double dx = (double)x[a] - (double)x[b];
    const double dy = (double)y[a] - (double)y[b];
    const double len2 = dx * dx + dy * dy;
    if (len2 < min_len2) {
        scores[e] = 0.f;
        return;
    }
    const double dv = fabs((double)values[a] - (double)values[b]);
    scores[e] = (float)(dv * sqrt(len2));
}

// Best-first sort key: complemented score bits over the edge index; edges at
// or below the threshold get the all-ones high word (pack_score_keys_kernel,
// delaunay_scalar_field.cu:105-127).
__global__ void k_score_keys(const float* __restrict__ scores, int64_t n, float threshold,
                             unsigned long long* __restrict__ keys)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float s = scores[i];
    uint32_t hi = 0xFFFFFFFFu;
    if (s > threshold && s > 0.f) hi = ~__float_as_uint(s);
    keys[i] = ((unsigned long long)hi << 32) | (uint32_t)i;
}

// Midpoints of the first `take` edges in sorted key order, on the padded
// canvas, rounded half to even (lrint) and clamped to the image
// (midpoints_from_sorted_kernel, delaunay_scalar_field.cu:129-160): the padded
// pixel index, or -1 where the pixel already holds a seed (its cell's label
// is a seed at that very position).
__global__ void k_midpoints(const unsigned long long* __restrict__ sorted, int take,
                            const unsigned long long* __restrict__ edge_keys, int64_t n_seeds,
                            const int32_t* __restrict__ x, const int32_t* __restrict__ y, int P, int Wd, int Hd,
                            int pitch, const int32_t* __restrict__ plane, const uint32_t* __restrict__ pos,
                            long long* __restrict__ out)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= take) return;
    const uint32_t e = (uint32_t)(sorted[r] & 0xFFFFFFFFull);
    const unsigned long long k = edge_keys[e];
    const int32_t a = (int32_t)(k / (unsigned long long)n_seeds), b = (int32_t)(k % (unsigned long long)n_seeds);
    int mx = (int)lrint(0.5 * ((double)(x[a] + P) + (double)(x[b] + P)));
    int my = (int)lrint(0.5 * ((double)(y[a] + P) + (double)(y[b] + P)));
    mx = min(max(mx, P), Wd - 1 - P);
    my = min(max(my, P), Hd - 1 - P);
    const int32_t l = plane[(size_t)my * pitch + mx];
    const bool seeded = l >= 0 && pos[l] == pack_pos(mx, my);
    out[r] = seeded ? -1ll : (long long)my * Wd + mx;
}

// Containing triangle of each query (image coordinates), read from the
// padded raster, which holds the highest id over every triangle containing
// the pixel.
__global__ void k_locate(const int32_t* __restrict__ q, int64_t n, int P, int Wd, int Hd,
                         const int32_t* __restrict__ tgrid, int32_t* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = q[i * 2] + P, y = q[i * 2 + 1] + P;
    out[i] = (x < 0 || y < 0 || x >= Wd || y >= Hd) ? NO_TRIANGLE : tgrid[(size_t)y * Wd + x];
}

// Lifted in-circle predicate (in_circumsphere_kernel,
// delaunay_query.cu:33-104): circumcentre in the reference's operation order
// on padded coordinates, radius = farthest vertex, distances compared (not
// their squares), all in double.
__global__ void k_circumsphere(const int32_t* __restrict__ q, const double* __restrict__ qt, int64_t n, int P,
                               int Wd, int Hd, const int32_t* __restrict__ tgrid, const int32_t* __restrict__ tris,
                               const int32_t* __restrict__ sx, const int32_t* __restrict__ sy,
                               uint8_t* __restrict__ mask, int32_t* __restrict__ tid_out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    mask[i] = 0;
    const int x = q[i * 2] + P, y = q[i * 2 + 1] + P;
    if (x < 0 || y < 0 || x >= Wd || y >= Hd) {
        tid_out[i] = NO_TRIANGLE;
        return;
    }
    const int32_t tid = tgrid[(size_t)y * Wd + x];
    tid_out[i] = tid;
    if (tid == NO_TRIANGLE) return;
    const int32_t* t = tris + (size_t)tid * 5;
    const double ax = sx[t[2]], ay = sy[t[2]];
    const double bx = sx[t[3]], by = sy[t[3]];
    const double cx = sx[t[4]], cy = sy[t[4]];
    const double abx = bx - ax, aby = by - ay;
    const double acx = cx - ax, acy = cy - ay;
    const double nz = abx * acy - aby * acx;
    double ox, oy;
    if (nz * nz < 1e-12) {
        ox = (ax + bx + cx) / 3.0;
        oy = (ay + by + cy) / 3.0;
    } else {
        const double ab2 = abx * abx + aby * aby;
        const double ac2 = acx * acx + acy * acy;
        const double den = 2.0 * (nz * nz);
        const double num_x = ac2 * (-(nz * aby)) + ab2 * (acy * nz);
        const double num_y = ac2 * (nz * abx) + ab2 * (-(acx * nz));
        ox = ax + num_x / den;
        oy = ay + num_y / den;
    }
    const double r2 = fmax(fmax((ax - ox) * (ax - ox) + (ay - oy) * (ay - oy),
                                (bx - ox) * (bx - ox) + (by - oy) * (by - oy)),
                           (cx - ox) * (cx - ox) + (cy - oy) * (cy - oy));
    const double dx = (double)x - ox, dy = (double)y - oy, tt = qt[i];
    mask[i] = sqrt(dx * dx + dy * dy + tt * tt) < sqrt(r2) ? 1 : 0;
}

// ---- host helpers ---------------------------------------------------------

inline unsigned blocks(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

struct Timer {
    Context& C;
    bool on;
    cudaEvent_t a = nullptr, b = nullptr;
    Timer(Context& c, bool enabled) : C(c), on(enabled)
    {
        if (!on) return;
        IDL_CUDA(cudaEventCreate(&a));
        IDL_CUDA(cudaEventCreate(&b));
        IDL_CUDA(cudaEventRecord(a, C.stream));
    }
    float stop()
    {
        if (!on) return 0.f;
        IDL_CUDA(cudaEventRecord(b, C.stream));
        IDL_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        IDL_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    }
    ~Timer()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

void ensure_rank(DelaunayState& D)
{
    if (!D.rank_dirty) return;
    rank_seeds_device(D.ctx(), D.W, D.H, D.ix, D.iy, D.N, D.P, D.rank, D.inv, D.sx, D.sy);
    D.rank_dirty = false;
}

void ensure_topology(DelaunayState& D, float* timings)
{
    if (!D.topo_dirty) return;
    ensure_rank(D);
    Context& C = D.ctx();
    if (D.N < 3) {
        D.n_tri = 0;
    } else {
        cudaEvent_t e[3] = {};
        if (timings)
            for (auto& ev : e) IDL_CUDA(cudaEventCreate(&ev));
        try {
            if (timings) IDL_CUDA(cudaEventRecord(e[0], C.stream));
            if (D.mode == IDL_MODE_EXACT)   // plane 1 holds the labels as (x, y) ranks
                detect_triangles(C, D.canvas(), D.planes + (size_t)D.pitch * D.Hd, D.spos.as<uint32_t>(), D.N,
                                 D.P, timings ? e[1] : nullptr, nullptr);
            else
                detect_triangles(C, D.canvas(), D.planes, D.pos, D.N, D.P, timings ? e[1] : nullptr, D.rank);
            if (timings) IDL_CUDA(cudaEventRecord(e[2], C.stream));
            D.n_tri = C.host_sc->n_triangles;   // from detection's own read-back
            if (timings) {
                IDL_CUDA(cudaEventSynchronize(e[2]));
                float a = 0.f, b = 0.f;
                IDL_CUDA(cudaEventElapsedTime(&a, e[0], e[1]));
                IDL_CUDA(cudaEventElapsedTime(&b, e[1], e[2]));
                timings[IDL_T_DETECT_MS] += a;
                timings[IDL_T_DEDUP_MS] += b;
            }
        } catch (...) {
            for (auto& ev : e)
                if (ev) cudaEventDestroy(ev);
            throw;
        }
        for (auto& ev : e)
            if (ev) cudaEventDestroy(ev);
    }
    D.topo_dirty = false;
}

// The padded canvas raster: every pixel's highest containing triangle id
// (the batch rule of triangulation.cu:101-137 over the whole triangle set).
void ensure_raster(DelaunayState& D, float* timings)
{
    if (!D.raster_dirty) return;
    ensure_topology(D, timings);
    Context& C = D.ctx();
    Timer T(C, timings != nullptr);
    assign_pixels(C, D.Wd, D.Hd, D.sx, D.sy, D.tgrid, D.n_tri);
    const float ms = T.stop();
    if (timings) timings[IDL_T_ASSIGN_MS] += ms;
    D.raster_dirty = false;
}

void ensure_edges(DelaunayState& D)
{
    ensure_topology(D, nullptr);
    if (!D.edges_dirty) return;
    Context& C = D.ctx();
    D.n_edges = 0;
    if (D.n_tri > 0) {
        const int64_t m = D.n_tri * 3;
        D.edge_tmp.ensure((size_t)m * 8);
        D.edge_keys.ensure((size_t)m * 8);
        D.num_sel.ensure(8);
        auto* raw = D.edge_tmp.as<unsigned long long>();
        auto* srt = D.edge_keys.as<unsigned long long>();
        k_edge_keys<<<blocks(D.n_tri), 256, 0, C.stream>>>(C.tris.as<int32_t>(), D.n_tri, D.inv, D.N, raw);
        IDL_LAUNCH();
        const unsigned long long top = (unsigned long long)D.N * (unsigned long long)D.N;
        int end_bit = 1;
        while (end_bit < 64 && (top >> end_bit) != 0) ++end_bit;
        size_t need_sort = 0, need_uniq = 0;
        IDL_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, need_sort, raw, srt, (int)m, 0, end_bit, C.stream));
        IDL_CUDA(cub::DeviceSelect::Unique(nullptr, need_uniq, srt, raw, D.num_sel.as<int>(), (int)m, C.stream));
        D.sort_tmp.ensure(std::max(need_sort, need_uniq));
        size_t tb = D.sort_tmp.bytes;
        IDL_CUDA(cub::DeviceRadixSort::SortKeys(D.sort_tmp.ptr, tb, raw, srt, (int)m, 0, end_bit, C.stream));
        tb = D.sort_tmp.bytes;
        IDL_CUDA(cub::DeviceSelect::Unique(D.sort_tmp.ptr, tb, srt, raw, D.num_sel.as<int>(), (int)m, C.stream));
        int n = 0;
        IDL_CUDA(cudaMemcpyAsync(&n, D.num_sel.ptr, sizeof(int), cudaMemcpyDeviceToHost, C.stream));
        IDL_CUDA(cudaStreamSynchronize(C.stream));
        std::swap(D.edge_tmp, D.edge_keys);   // unique keys now in edge_keys
        D.n_edges = n;
    }
    D.edges_dirty = false;
}

void compute_scores(DelaunayState& D, double min_length)
{
    D.scores.ensure((size_t)std::max<int64_t>(1, D.n_edges) * 4);
    k_edge_scores<<<blocks(D.n_edges), 256, 0, D.ctx().stream>>>(D.edge_keys.as<unsigned long long>(), D.n_edges, D.N,
                                                             D.ix, D.iy, D.values, min_length * min_length,
                                                             D.scores.as<float>());
    IDL_LAUNCH();
}

const int32_t* upload_queries(DelaunayState& D, const int32_t* pts, int64_t n)
{
    D.qbuf.ensure((size_t)n * 2 * 4);
    IDL_CUDA(cudaMemcpyAsync(D.qbuf.ptr, pts, (size_t)n * 2 * 4, cudaMemcpyHostToDevice, D.ctx().stream));
    return D.qbuf.as<int32_t>();
}

// Objects allocate from the device's default stream-ordered pool; keep what
// they free in the pool (no release threshold) so the next object reuses it
// without a trip to the driver.  This changes only this process's pool.
void keep_pool_memory(int dev)
{
    static std::once_flag once[64];
    std::call_once(once[dev & 63], [dev] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    });
}

// Lay the object's allocations out for a width x height canvas with padding P
// and room for max_seeds seeds, and reset it to the empty state.  The caller
// has checked that everything fits.
void layout(DelaunayState& d, int width, int height, int64_t max_seeds, int P)
{
    d.W = width;
    d.H = height;
    d.P = P;
    d.Wd = width + 2 * P;
    d.Hd = height + 2 * P;
    d.pitch = (d.Wd + 31) / 32 * 32;
    d.max_seeds = max_seeds;
    int32_t* s = d.seedmem;
    const int64_t cap = d.seed_cap;
    d.ix = s;
    d.iy = s + cap;
    d.pos = reinterpret_cast<uint32_t*>(s + 2 * cap);
    d.rank = s + 3 * cap;
    d.inv = s + 4 * cap;
    d.sx = s + 5 * cap;
    d.sy = s + 6 * cap;
    d.values = reinterpret_cast<float*>(s + 7 * cap);
    d.pix_tid = static_cast<int32_t*>(d.pixmem);
    d.pix_sid = d.pix_tid + (size_t)width * height;
    d.pix_out = reinterpret_cast<uint8_t*>(d.pix_sid + (size_t)width * height);
    const size_t plane = (size_t)d.pitch * d.Hd;
    d.N = 0;
    d.pending = false;
    d.rank_dirty = d.topo_dirty = d.raster_dirty = false;
    d.edges_dirty = true;
    d.have_values = false;
    d.n_tri = d.n_edges = 0;
    d.hx.clear();
    d.hy.clear();
    d.hvals.clear();
    IDL_CUDA(cudaMemsetAsync(d.planes, 0xFF, plane * 2 * sizeof(int32_t), d.stream));
    IDL_CUDA(cudaMemsetAsync(d.tgrid, 0xFF, (size_t)d.Wd * d.Hd * sizeof(int32_t), d.stream));
    IDL_CUDA(cudaMemsetAsync(d.values, 0, (size_t)max_seeds * sizeof(float), d.stream));
}

void check_handle(const idl_delaunay* d)
{
    if (!d) invalid("Delaunay handle must not be NULL");
}

// Every entry point ends by undoing the workspace binding and noting the
// object's last work on its stream.
struct Unbinder {
    DelaunayState* d;
    ~Unbinder()
    {
        d->unbind();
        d->note_use();
    }
};

}  // namespace
}  // namespace idl

using namespace idl;

extern "C" {

int idl_delaunay_create(int device, int width, int height, int64_t max_seeds, int border_padding, int mode,
                        idl_delaunay** out)
{
    IDL_API_BEGIN
    if (!out) invalid("out must not be NULL");
    *out = nullptr;
    if (width <= 0 || height <= 0 || max_seeds <= 0) invalid("dimensions and max_seeds must be positive");
    if (max_seeds > MAX_SEEDS) invalid("max_seeds exceeds the 2097151 seeds this build can number");
    if (mode != IDL_MODE_REFERENCE && mode != IDL_MODE_EXACT)
        invalid("the incremental Delaunay supports voronoi_mode 'reference' and 'exact' in this build");
    int dev = device;
    if (dev < 0) IDL_CUDA(cudaGetDevice(&dev));
    DeviceGuard g(dev);
    auto* d = new idl_delaunay();
    try {
        d->device = dev;
        d->own.device = dev;
        IDL_CUDA(cudaDeviceGetAttribute(&d->own.num_sms, cudaDevAttrMultiProcessorCount, dev));
        keep_pool_memory(dev);
        const int P = border_padding >= 0 ? border_padding : IDL_DEFAULT_BORDER_PADDING;
        const int64_t Wd = (int64_t)width + 2 * P, Hd = (int64_t)height + 2 * P;
        const int64_t pitch = (Wd + 31) / 32 * 32;
        // The canvas-sized buffers first: a canvas no GPU can hold fails here,
        // as a CUDA allocation error, before any size rule of this build.
        d->planes_bytes = (size_t)pitch * Hd * 2 * sizeof(int32_t);
        d->tgrid_bytes = (size_t)Wd * Hd * sizeof(int32_t);
        d->pix_bytes = (size_t)width * height * 9;
        d->seed_cap = max_seeds;
        for (int k = 0; k < 4; ++k) count_alloc();
        IDL_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d->planes), d->planes_bytes, d->stream));
        IDL_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d->tgrid), d->tgrid_bytes, d->stream));
        IDL_CUDA(cudaMallocAsync(&d->pixmem, d->pix_bytes, d->stream));
        IDL_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d->seedmem), (size_t)max_seeds * 8 * sizeof(int32_t),
                                 d->stream));
        if (Wd > MAX_CANVAS_SIDE || Hd > MAX_CANVAS_SIDE)
            invalid("padded canvas side exceeds the 32767 pixels this build addresses");
        d->mode = mode;
        layout(*d, width, height, max_seeds, P);
        // the allocations are ordered on the creating stream; a later
        // set_stream orders the object's new stream after them
        IDL_CUDA(cudaEventCreateWithFlags(&d->last_use, cudaEventDisableTiming));
        IDL_CUDA(cudaEventRecord(d->last_use, d->stream));
    } catch (...) {
        delete d;
        throw;
    }
    *out = d;
    IDL_API_END
}

int idl_delaunay_reset(idl_delaunay* d, int width, int height, int64_t max_seeds, int border_padding)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (width <= 0 || height <= 0 || max_seeds <= 0) invalid("dimensions and max_seeds must be positive");
    const int P = border_padding >= 0 ? border_padding : IDL_DEFAULT_BORDER_PADDING;
    const int64_t Wd = (int64_t)width + 2 * P, Hd = (int64_t)height + 2 * P;
    const int64_t pitch = (Wd + 31) / 32 * 32;
    if ((size_t)pitch * Hd * 8 > d->planes_bytes || (size_t)Wd * Hd * 4 > d->tgrid_bytes ||
        (size_t)width * height * 9 > d->pix_bytes || max_seeds > d->seed_cap)
        invalid("reset: the new canvas or seed capacity does not fit this object's allocations");
    DeviceGuard g(d->device);
    ++d->generation;
    layout(*d, width, height, max_seeds, P);
    IDL_API_END
}

int idl_delaunay_destroy(idl_delaunay* d)
{
    IDL_API_BEGIN
    if (!d) return IDL_OK;
    DeviceGuard g(d->device);
    // wait for this object's own work only (not the rest of its stream's)
    if (d->last_use) cudaEventSynchronize(d->last_use);
    else cudaStreamSynchronize(d->stream);
    delete d;
    IDL_API_END
}

int idl_delaunay_set_stream(idl_delaunay* d, void* stream)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    const cudaStream_t next = static_cast<cudaStream_t>(stream);
    // The new stream waits for the object's work so far on the old one.
    if (next != d->stream && d->last_use) {
        DeviceGuard g(d->device);
        IDL_CUDA(cudaStreamWaitEvent(next, d->last_use, 0));
    }
    d->stream = next;
    IDL_API_END
}

int idl_delaunay_set_workspace(idl_delaunay* d, idl_context* ws)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (ws && ws->device != d->device) invalid("the workspace context belongs to another device");
    d->ws = ws;
    IDL_API_END
}

int idl_delaunay_insert(idl_delaunay* d, const int32_t* xy, int64_t k, const float* values, float* timings)
{
    return idl_delaunay_insert_ordered(d, xy, k, values, 0, timings);
}

int idl_delaunay_insert_ordered(idl_delaunay* d, const int32_t* xy, int64_t k, const float* values, int order,
                                float* timings)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (timings)
        for (int i = 0; i < IDL_T_COUNT; ++i) timings[i] = 0.f;
    if (order != 0 && order != 1) invalid("order must be 0 (as given) or 1 (x, y)");
    if (k < 0) invalid("seed count must not be negative");
    if (k == 0) return IDL_OK;
    if (!xy) invalid("seeds must not be NULL");
    // validation before any change (delaunay.cu:190-212)
    if (d->N + k > d->max_seeds) invalid("insert would exceed max_seeds capacity");
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    const int64_t n0 = d->N;

    // upload, then validate on the device: bounds, repeats within the batch,
    // positions already seeded (a seed's own cell always holds its label)
    d->batch.ensure((size_t)k * 6 * 4);
    int32_t* b_xy = d->batch.as<int32_t>();
    int32_t* b_tx = b_xy + 2 * k;
    int32_t* b_ty = b_xy + 3 * k;
    int32_t* b_rank = b_xy + 4 * k;
    int32_t* b_inv = b_xy + 5 * k;
    d->verr.ensure(3 * sizeof(unsigned long long));
    unsigned long long* err = d->verr.as<unsigned long long>();
    IDL_CUDA(cudaMemcpyAsync(b_xy, xy, (size_t)k * 8, cudaMemcpyHostToDevice, C.stream));
    IDL_CUDA(cudaMemsetAsync(err, 0xFF, 3 * sizeof(unsigned long long), C.stream));
    const unsigned gk = blocks(k);
    k_v_bounds<<<gk, 256, 0, C.stream>>>(b_xy, k, d->W, d->H, d->P, d->Wd, d->tgrid, err);
    IDL_LAUNCH();
    k_v_first<<<gk, 256, 0, C.stream>>>(b_xy, k, d->W, d->H, d->P, d->Wd, d->tgrid);
    IDL_LAUNCH();
    k_v_check<<<gk, 256, 0, C.stream>>>(b_xy, k, d->W, d->H, d->P, d->Wd, d->pitch, d->tgrid, d->planes, d->pos,
                                        n0, err);
    IDL_LAUNCH();
    unsigned long long he[3];
    IDL_CUDA(cudaMemcpyAsync(he, err, sizeof(he), cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    d->raster_dirty = true;   // the raster served as scratch; it is rebuilt when next read
    if (he[0] != ~0ull) invalid("seed coordinate out of bounds");
    if (he[1] != ~0ull || he[2] != ~0ull)
        invalid(he[1] <= he[2] ? "duplicate seed positions within batch" : "seed position already exists");

    ++d->generation;
    // coordinates in insertion order, or (order 1) this batch in (x, y) order
    if (order == 0) {
        k_split<<<gk, 256, 0, C.stream>>>(b_xy, k, d->ix + n0, d->iy + n0);
        IDL_LAUNCH();
    } else {
        k_split<<<gk, 256, 0, C.stream>>>(b_xy, k, b_tx, b_ty);
        IDL_LAUNCH();
        rank_seeds_device(C, d->W, d->H, b_tx, b_ty, k, 0, b_rank, b_inv, d->ix + n0, d->iy + n0);
    }
    k_pack_pos<<<gk, 256, 0, C.stream>>>(d->ix + n0, d->iy + n0, k, d->P, d->pos + n0);
    IDL_LAUNCH();
    const size_t hn = d->hx.size();
    d->hx.resize(hn + k);
    d->hy.resize(hn + k);
    if (order == 0) {
        for (int64_t i = 0; i < k; ++i) {
            d->hx[hn + i] = xy[2 * i];
            d->hy[hn + i] = xy[2 * i + 1];
        }
    } else {
        IDL_CUDA(cudaMemcpyAsync(d->hx.data() + hn, d->ix + n0, (size_t)k * 4, cudaMemcpyDeviceToHost, C.stream));
        IDL_CUDA(cudaMemcpyAsync(d->hy.data() + hn, d->iy + n0, (size_t)k * 4, cudaMemcpyDeviceToHost, C.stream));
    }
    if (values) {
        const size_t vn = d->hvals.size();
        d->hvals.resize(vn + k);
        if (order == 0) {
            IDL_CUDA(cudaMemcpyAsync(d->values + n0, values, (size_t)k * 4, cudaMemcpyHostToDevice, C.stream));
            std::copy(values, values + k, d->hvals.begin() + vn);
        } else {
            float* b_val = reinterpret_cast<float*>(b_tx);   // free again after the rank
            IDL_CUDA(cudaMemcpyAsync(b_val, values, (size_t)k * 4, cudaMemcpyHostToDevice, C.stream));
            k_permute<<<gk, 256, 0, C.stream>>>(b_val, b_rank, k, d->values + n0);
            IDL_LAUNCH();
            IDL_CUDA(cudaMemcpyAsync(d->hvals.data() + vn, d->values + n0, (size_t)k * 4, cudaMemcpyDeviceToHost,
                                     C.stream));
        }
        d->have_values = true;
    }
    d->N += k;
    d->rank_dirty = d->topo_dirty = d->raster_dirty = d->edges_dirty = true;
    d->pending = true;

    Timer T(C, timings != nullptr);
    int64_t passes = 0;
    if (d->mode == IDL_MODE_EXACT) {
        // history-independent: the exact diagram of the whole seed set, in
        // (x, y) ranks (plane 1, which detection reads) and as insertion ids
        // (plane 0, which every other reader expects)
        ensure_rank(*d);
        d->spos.ensure((size_t)d->N * 4);
        k_pack_pos<<<blocks(d->N), 256, 0, C.stream>>>(d->sx, d->sy, d->N, 0, d->spos.as<uint32_t>());
        IDL_LAUNCH();
        propagate_exact(C, d->canvas(), d->spos.as<uint32_t>(), d->N);
        k_exact_planes<<<dim3(blocks(d->Wd), (unsigned)d->Hd), 256, 0, C.stream>>>(
            d->planes, d->planes + (size_t)d->pitch * d->Hd, d->pitch, d->Wd, d->inv);
        IDL_LAUNCH();
    } else {
        k_put_seeds<<<gk, 256, 0, C.stream>>>(d->planes, d->planes + (size_t)d->pitch * d->Hd, d->pitch,
                                              d->pos + n0, k, n0);
        IDL_LAUNCH();
        passes = propagate(C, d->mode, d->canvas(), d->pos, n0 + k, d->pos + n0, k);
    }
    const float bfs = T.stop();
    if (timings) {
        timings[IDL_T_BFS_MS] = bfs;
        timings[IDL_T_BFS_ITERS] = (float)passes;
        ensure_topology(*d, timings);
    }
    IDL_API_END
}

int idl_delaunay_adopt(idl_delaunay* d, idl_context* src, int image)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (!src) invalid("context must not be NULL");
    BatchImage bi;
    if (!batch_image(*src, image, bi)) invalid("the context holds no batch with that image");
    if (src->device != d->device) invalid("the batch was computed on another device");
    if (bi.W != d->W || bi.H != d->H || bi.P != d->P)
        invalid("the batch image's size or border padding differs from the object's");
    if (d->N != 0) invalid("adopt needs an empty object (reset it first)");
    if (d->mode != IDL_MODE_REFERENCE) invalid("adopt takes labels of reference semantics only");
    if (bi.n > d->max_seeds) invalid("insert would exceed max_seeds capacity");
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    const int32_t* atlas = src->lab[0].as<int32_t>();
    k_adopt<<<dim3((unsigned)d->Hd), 256, 0, C.stream>>>(atlas, bi.pitch, bi.ox, bi.oy, bi.seed_off, d->Wd,
                                                        d->planes, d->planes + (size_t)d->pitch * d->Hd, d->pitch);
    IDL_LAUNCH();
    const int64_t n = bi.n;
    IDL_CUDA(cudaMemcpyAsync(d->ix, src->xs.as<int32_t>() + bi.seed_off, (size_t)n * 4, cudaMemcpyDeviceToDevice,
                             C.stream));
    IDL_CUDA(cudaMemcpyAsync(d->iy, src->ys.as<int32_t>() + bi.seed_off, (size_t)n * 4, cudaMemcpyDeviceToDevice,
                             C.stream));
    k_pack_pos<<<blocks(n), 256, 0, C.stream>>>(d->ix, d->iy, n, d->P, d->pos);
    IDL_LAUNCH();
    d->hx.resize(n);
    d->hy.resize(n);
    IDL_CUDA(cudaMemcpyAsync(d->hx.data(), d->ix, (size_t)n * 4, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaMemcpyAsync(d->hy.data(), d->iy, (size_t)n * 4, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    ++d->generation;
    d->N = n;
    d->rank_dirty = d->topo_dirty = d->raster_dirty = d->edges_dirty = true;
    d->pending = true;
    IDL_API_END
}

int idl_delaunay_adopt_group(idl_delaunay* const* objs, const int* images, int n, idl_context* src)
{
    IDL_API_BEGIN
    if (!objs || !images) invalid("arguments must not be NULL");
    if (n < 1 || n > ADOPT_GROUP_MAX) invalid("a group holds 1 to 16 objects");
    if (!src) invalid("context must not be NULL");
    AdoptGroup g{};
    int64_t lo = INT64_MAX, hi = 0;
    int max_hd = 1;
    std::vector<BatchImage> bis(n);
    for (int k = 0; k < n; ++k) {
        idl_delaunay* d = objs[k];
        check_handle(d);
        BatchImage& bi = bis[k];
        if (!batch_image(*src, images[k], bi)) invalid("the context holds no batch with that image");
        if (src->device != d->device) invalid("the batch was computed on another device");
        if (bi.W != d->W || bi.H != d->H || bi.P != d->P)
            invalid("the batch image's size or border padding differs from the object's");
        if (d->N != 0) invalid("adopt needs an empty object (reset it first)");
        if (d->mode != IDL_MODE_REFERENCE) invalid("adopt takes labels of reference semantics only");
        if (bi.n > d->max_seeds) invalid("insert would exceed max_seeds capacity");
        if (d->stream != objs[0]->stream || d->device != objs[0]->device)
            invalid("the objects of a group must share one stream and device");
        for (int j = 0; j < k; ++j)
            if (objs[j] == d) invalid("an object appears twice in the group");
        AdoptItem& m = g.it[k];
        m.atlas = src->lab[0].as<int32_t>();
        m.sxs = src->xs.as<int32_t>();
        m.sys = src->ys.as<int32_t>();
        m.a = d->planes;
        m.b = d->planes + (size_t)d->pitch * d->Hd;
        m.ix = d->ix;
        m.iy = d->iy;
        m.pos = d->pos;
        m.seed_off = bi.seed_off;
        m.n = bi.n;
        m.apitch = bi.pitch;
        m.ox = bi.ox;
        m.oy = bi.oy;
        m.Wd = d->Wd;
        m.Hd = d->Hd;
        m.pitch = d->pitch;
        m.P = d->P;
        max_hd = std::max(max_hd, d->Hd);
        lo = std::min<int64_t>(lo, bi.seed_off);
        hi = std::max<int64_t>(hi, bi.seed_off + bi.n);
    }
    idl_delaunay* d0 = objs[0];
    DeviceGuard guard(d0->device);
    const cudaStream_t st = d0->stream;
    k_adopt_group<<<dim3((unsigned)std::min(max_hd, 1024), (unsigned)n), 256, 0, st>>>(g);
    IDL_LAUNCH();
    // host mirrors of every image's seeds: one copy of the group's range
    std::vector<int32_t> hx((size_t)(hi - lo)), hy((size_t)(hi - lo));
    if (hi > lo) {
        IDL_CUDA(cudaMemcpyAsync(hx.data(), src->xs.as<int32_t>() + lo, (size_t)(hi - lo) * 4,
                                 cudaMemcpyDeviceToHost, st));
        IDL_CUDA(cudaMemcpyAsync(hy.data(), src->ys.as<int32_t>() + lo, (size_t)(hi - lo) * 4,
                                 cudaMemcpyDeviceToHost, st));
    }
    IDL_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < n; ++k) {
        idl_delaunay* d = objs[k];
        const BatchImage& bi = bis[k];
        d->hx.assign(hx.begin() + (bi.seed_off - lo), hx.begin() + (bi.seed_off - lo + bi.n));
        d->hy.assign(hy.begin() + (bi.seed_off - lo), hy.begin() + (bi.seed_off - lo + bi.n));
        ++d->generation;
        d->N = bi.n;
        d->rank_dirty = d->topo_dirty = d->raster_dirty = d->edges_dirty = true;
        d->pending = true;
        d->note_use();
    }
    IDL_API_END
}

int idl_delaunay_finalise(idl_delaunay* d, int32_t* grid_out, int64_t* n_tri_out, float* timings)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (timings)
        for (int i = 0; i < IDL_T_COUNT; ++i) timings[i] = 0.f;
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    ensure_rank(*d);
    ensure_raster(*d, timings);
    if (d->pending) {
        d->pending = false;
        ++d->generation;
    }
    if (grid_out) {
        const size_t bytes = (size_t)d->W * d->H * 3 * 4;
        C.outgrid.ensure(bytes);
        if (d->N == 0) {
            IDL_CUDA(cudaMemsetAsync(C.outgrid.ptr, 0xFF, bytes, C.stream));
        } else {
            dim3 gr(blocks(d->W), d->H);
            k_out3<<<gr, 256, 0, C.stream>>>(d->planes, d->pitch, d->P, d->W, d->H, d->pos, d->rank, d->tgrid, d->Wd,
                                            C.outgrid.as<int32_t>());
            IDL_LAUNCH();
        }
        IDL_CUDA(cudaMemcpyAsync(grid_out, C.outgrid.ptr, bytes, cudaMemcpyDeviceToHost, C.stream));
    }
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    if (n_tri_out) *n_tri_out = d->n_tri;
    IDL_API_END
}

int idl_delaunay_finalise_device(idl_delaunay* d, int64_t* n_tri_out, const int32_t** tids,
                                 const int32_t** sids, const uint8_t** mask, uint64_t* generation_out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    ++d->generation;
    ensure_rank(*d);
    ensure_raster(*d, nullptr);
    d->pending = false;
    dim3 gr(blocks(d->W), d->H);
    k_crop<<<gr, 256, 0, C.stream>>>(d->planes, d->pitch, d->P, d->W, d->H, d->rank, d->tgrid, d->Wd, d->pix_tid,
                                     d->pix_sid, d->pix_out);
    IDL_LAUNCH();
    if (n_tri_out) *n_tri_out = d->n_tri;
    if (tids) *tids = d->pix_tid;
    if (sids) *sids = d->pix_sid;
    if (mask) *mask = d->pix_out;
    if (generation_out) *generation_out = d->generation;
    IDL_API_END
}

int idl_delaunay_triangles(idl_delaunay* d, int ids, int32_t* out, int64_t capacity, int64_t* n_out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (ids < 0 || ids > 2) invalid("ids must be 0 (batch rows), 1 (insertion order) or 2 (batch vertices)");
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    ensure_topology(*d, nullptr);
    if (n_out) *n_out = d->n_tri;
    if (!out || d->n_tri == 0) return IDL_OK;
    const int cols = ids == 0 ? 5 : 3;
    if (capacity < d->n_tri * cols) invalid("triangle buffer too small");
    if (ids == 0) {
        IDL_CUDA(cudaMemcpyAsync(out, C.tris.ptr, (size_t)d->n_tri * 5 * 4, cudaMemcpyDeviceToHost, C.stream));
    } else if (ids == 2) {
        d->stage.ensure((size_t)d->n_tri * 3 * 4);
        k_tris_batch_verts<<<blocks(d->n_tri * 3), 256, 0, C.stream>>>(C.tris.as<int32_t>(), d->n_tri,
                                                                      d->stage.as<int32_t>());
        IDL_LAUNCH();
        IDL_CUDA(cudaMemcpyAsync(out, d->stage.ptr, (size_t)d->n_tri * 3 * 4, cudaMemcpyDeviceToHost, C.stream));
    } else {
        d->stage.ensure((size_t)d->n_tri * 3 * 4);
        k_tris_insertion<<<blocks(d->n_tri), 256, 0, C.stream>>>(C.tris.as<int32_t>(), d->n_tri, d->inv,
                                                                 d->stage.as<int32_t>());
        IDL_LAUNCH();
        IDL_CUDA(cudaMemcpyAsync(out, d->stage.ptr, (size_t)d->n_tri * 3 * 4, cudaMemcpyDeviceToHost, C.stream));
    }
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    IDL_API_END
}

int idl_delaunay_edges(idl_delaunay* d, int32_t* out, int64_t capacity, int64_t* n_out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    ensure_edges(*d);
    if (n_out) *n_out = d->n_edges;
    if (!out || d->n_edges == 0) return IDL_OK;
    if (capacity < d->n_edges * 2) invalid("edge buffer too small");
    d->stage.ensure((size_t)d->n_edges * 2 * 4);
    k_edge_unpack<<<blocks(d->n_edges), 256, 0, C.stream>>>(d->edge_keys.as<unsigned long long>(), d->n_edges, d->N,
                                                            d->stage.as<int32_t>());
    IDL_LAUNCH();
    IDL_CUDA(cudaMemcpyAsync(out, d->stage.ptr, (size_t)d->n_edges * 2 * 4, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    IDL_API_END
}

int idl_delaunay_edge_scores(idl_delaunay* d, double min_length, float* out, int64_t capacity, int64_t* n_out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    DeviceGuard g(d->device);
    ensure_edges(*d);
    if (n_out) *n_out = d->n_edges;
    if (d->n_edges == 0) return IDL_OK;
    if (!d->have_values)
        throw Error(IDL_ERR_STATE, "edge_scores needs a value per seed; pass values to insert_deferred");
    if (!out) return IDL_OK;
    if (capacity < d->n_edges) invalid("score buffer too small");
    compute_scores(*d, min_length);
    IDL_CUDA(cudaMemcpyAsync(out, d->scores.ptr, (size_t)d->n_edges * 4, cudaMemcpyDeviceToHost, d->stream));
    IDL_CUDA(cudaStreamSynchronize(d->stream));
    IDL_API_END
}

int idl_delaunay_select_midpoints(idl_delaunay* d, double min_length, int count, float threshold, int32_t* out,
                                  int64_t capacity, int64_t* n_out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (n_out) *n_out = 0;
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    ensure_edges(*d);
    if (d->n_edges == 0 || count <= 0) return IDL_OK;
    if (!d->have_values)
        throw Error(IDL_ERR_STATE, "select_midpoints needs a value per seed; pass values to insert_deferred");
    const int64_t E = d->n_edges;
    compute_scores(*d, min_length);
    d->score_keys.ensure((size_t)E * 8);
    d->score_sorted.ensure((size_t)E * 8);
    k_score_keys<<<blocks(E), 256, 0, C.stream>>>(d->scores.as<float>(), E, threshold,
                                                  d->score_keys.as<unsigned long long>());
    IDL_LAUNCH();
    size_t need = 0;
    IDL_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, need, d->score_keys.as<unsigned long long>(),
                                            d->score_sorted.as<unsigned long long>(), (int)E, 0, 64, C.stream));
    d->sort_tmp.ensure(need);
    size_t tb = d->sort_tmp.bytes;
    IDL_CUDA(cub::DeviceRadixSort::SortKeys(d->sort_tmp.ptr, tb, d->score_keys.as<unsigned long long>(),
                                            d->score_sorted.as<unsigned long long>(), (int)E, 0, 64, C.stream));
    // the eligible edges sort first; take at most `count` of them
    const int64_t look = std::min<int64_t>(count, E);
    std::vector<unsigned long long> head((size_t)look);
    IDL_CUDA(cudaMemcpyAsync(head.data(), d->score_sorted.ptr, (size_t)look * 8, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    int take = 0;
    while (take < look && (head[take] >> 32) != 0xFFFFFFFFull) ++take;
    if (take == 0) return IDL_OK;
    d->stage.ensure((size_t)take * 8);
    k_midpoints<<<blocks(take), 256, 0, C.stream>>>(d->score_sorted.as<unsigned long long>(), take,
                                                    d->edge_keys.as<unsigned long long>(), d->N, d->ix, d->iy, d->P,
                                                    d->Wd, d->Hd, d->pitch, d->planes, d->pos,
                                                    d->stage.as<long long>());
    IDL_LAUNCH();
    std::vector<long long> pix((size_t)take);
    IDL_CUDA(cudaMemcpyAsync(pix.data(), d->stage.ptr, pix.size() * 8, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    // collisions keep the best-ranked edge; results ascend by padded pixel
    std::vector<std::pair<int64_t, int>> cand;
    cand.reserve(take);
    const int P = d->P;
    for (int r = 0; r < take; ++r)
        if (pix[r] >= 0) cand.emplace_back(pix[r], r);
    std::sort(cand.begin(), cand.end());
    std::vector<int32_t> res;
    for (size_t i = 0; i < cand.size(); ++i) {
        if (i > 0 && cand[i].first == cand[i - 1].first) continue;
        res.push_back((int32_t)(cand[i].first % d->Wd) - P);
        res.push_back((int32_t)(cand[i].first / d->Wd) - P);
    }
    const int64_t n = (int64_t)res.size() / 2;
    if (n_out) *n_out = n;
    if (out) {
        if (capacity < n * 2) invalid("midpoint buffer too small");
        std::copy(res.begin(), res.end(), out);
    }
    IDL_API_END
}

int idl_delaunay_locate(idl_delaunay* d, const int32_t* pts, int64_t n, int32_t* out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (n < 0) invalid("query count must not be negative");
    if (n == 0) return IDL_OK;
    if (!pts || !out) invalid("query and output buffers must not be NULL");
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    ensure_rank(*d);
    ensure_raster(*d, nullptr);
    const int32_t* q = upload_queries(*d, pts, n);
    d->qout.ensure((size_t)n * 4);
    k_locate<<<blocks(n), 256, 0, C.stream>>>(q, n, d->P, d->Wd, d->Hd, d->tgrid, d->qout.as<int32_t>());
    IDL_LAUNCH();
    IDL_CUDA(cudaMemcpyAsync(out, d->qout.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    IDL_API_END
}

int idl_delaunay_in_circumsphere(idl_delaunay* d, const int32_t* pts, const double* t, int64_t n, uint8_t* mask,
                                 int32_t* tids)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (n < 0) invalid("query count must not be negative");
    if (n == 0) return IDL_OK;
    if (!pts || !t || !mask || !tids) invalid("query and output buffers must not be NULL");
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    ensure_rank(*d);
    ensure_raster(*d, nullptr);
    ensure_topology(*d, nullptr);
    const int32_t* q = upload_queries(*d, pts, n);
    // one scratch block: t (8 B), tid (4 B), mask (1 B) per query
    d->qout.ensure((size_t)n * 13);
    double* dt = d->qout.as<double>();
    int32_t* dtid = reinterpret_cast<int32_t*>(dt + n);
    uint8_t* dm = reinterpret_cast<uint8_t*>(dtid + n);
    IDL_CUDA(cudaMemcpyAsync(dt, t, (size_t)n * 8, cudaMemcpyHostToDevice, C.stream));
    k_circumsphere<<<blocks(n), 256, 0, C.stream>>>(q, dt, n, d->P, d->Wd, d->Hd, d->tgrid, C.tris.as<int32_t>(),
                                                    d->sx, d->sy, dm, dtid);
    IDL_LAUNCH();
    IDL_CUDA(cudaMemcpyAsync(tids, dtid, (size_t)n * 4, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaMemcpyAsync(mask, dm, (size_t)n, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    IDL_API_END
}

int idl_delaunay_seeds(idl_delaunay* d, int32_t* xy_out, float* values_out, int64_t* n_values_out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (xy_out)
        for (int64_t i = 0; i < d->N; ++i) {
            xy_out[2 * i] = d->hx[i];
            xy_out[2 * i + 1] = d->hy[i];
        }
    if (values_out) std::copy(d->hvals.begin(), d->hvals.end(), values_out);
    if (n_values_out) *n_values_out = (int64_t)d->hvals.size();
    IDL_API_END
}

int idl_delaunay_sorted_rank(idl_delaunay* d, int32_t* out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (d->N == 0) return IDL_OK;
    if (!out) invalid("output must not be NULL");
    DeviceGuard g(d->device);
    ensure_rank(*d);
    IDL_CUDA(cudaMemcpyAsync(out, d->rank, (size_t)d->N * 4, cudaMemcpyDeviceToHost, d->stream));
    IDL_CUDA(cudaStreamSynchronize(d->stream));
    IDL_API_END
}

int idl_delaunay_voronoi(idl_delaunay* d, int32_t* out)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (!out) invalid("output must not be NULL");
    DeviceGuard g(d->device);
    Context& C = d->ctx();
    const size_t bytes = (size_t)d->W * d->H * 2 * 4;
    C.outgrid.ensure(bytes);
    if (d->N == 0) {
        IDL_CUDA(cudaMemsetAsync(C.outgrid.ptr, 0xFF, bytes, C.stream));
    } else {
        ensure_rank(*d);
        dim3 gr(blocks(d->W), d->H);
        k_out2<<<gr, 256, 0, C.stream>>>(d->planes, d->pitch, d->P, d->W, d->H, d->pos, d->rank,
                                        C.outgrid.as<int32_t>());
        IDL_LAUNCH();
    }
    IDL_CUDA(cudaMemcpyAsync(out, C.outgrid.ptr, bytes, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    IDL_API_END
}

int idl_delaunay_info(idl_delaunay* d, int64_t* info, int count)
{
    IDL_API_BEGIN
    check_handle(d);
    const Unbinder unbind_on_exit{d};
    if (!info) invalid("output must not be NULL");
    const int64_t device_bytes = (int64_t)(d->planes_bytes + d->tgrid_bytes + d->pix_bytes +
                                           (size_t)d->seed_cap * 32 + d->own.workspace_bytes()) +
                                 (int64_t)(d->stage.bytes + d->edge_keys.bytes + d->edge_tmp.bytes +
                                           d->sort_tmp.bytes + d->num_sel.bytes + d->scores.bytes +
                                           d->score_keys.bytes + d->score_sorted.bytes + d->qbuf.bytes +
                                           d->qout.bytes);
    const int64_t v[IDL_DI_COUNT] = {d->N, d->W, d->H, d->P, d->pending ? 1 : 0, (int64_t)d->generation,
                                     d->max_seeds, d->mode, d->have_values ? 1 : 0, device_bytes};
    for (int i = 0; i < count && i < IDL_DI_COUNT; ++i) info[i] = v[i];
    IDL_API_END
}

}  // extern "C"
