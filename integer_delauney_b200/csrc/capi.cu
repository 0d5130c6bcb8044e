// C ABI: context management and the batch entry points (Voronoi().compute,
// triangulate(), GridTriangulation.compute*), plus the output composition
// kernels.  The orchestration follows cuda_compute_triangulation
// (src/cuda/triangulation.cu:143-365) stage for stage, with every
// intermediate kept on the device and no host loops over pixels.
#include "context.cuh"

#include <algorithm>
#include <atomic>
#include <string>

namespace idl {

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
std::atomic<long long> g_allocs{0};
}

void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_alloc() { g_allocs.fetch_add(1, std::memory_order_relaxed); }

size_t Context::workspace_bytes() const
{
    size_t s = 0;
    const_cast<Context*>(this)->each_buf([&](DevBuf& b) { s += b.bytes; });
    return s;
}

void Context::fetch_scalars()
{
    IDL_CUDA(cudaMemcpyAsync(host_sc, scalars.ptr, sizeof(Scalars), cudaMemcpyDeviceToHost, stream));
    IDL_CUDA(cudaStreamSynchronize(stream));
}

Context::~Context()
{
    bool ordered = false;
    each_buf([&](DevBuf& b) { ordered |= b.async; });
    if (ordered) cudaDeviceSynchronize();   // stream-ordered buffers may still be in use
    each_buf([](DevBuf& b) { b.release(); });
    if (host_sc && !host_sc_borrowed) cudaFreeHost(host_sc);
    for (auto& e : timing.ev)
        if (e) cudaEventDestroy(e);
}

void ensure_scalars(Context& C)
{
    C.scalars.ensure(sizeof(Scalars));
    if (!C.host_sc) {
        count_alloc();
        IDL_CUDA(cudaMallocHost(reinterpret_cast<void**>(&C.host_sc), sizeof(Scalars)));
    }
}

namespace {

// ---- output composition ------------------------------------------------

// (H, W, 3): seed id and squared distance from the interior window of the
// detection canvas, triangle id from the assignment (triangulation.cu:391-412).
// A block composes 256 consecutive pixels of the flattened image in shared
// memory and stores their 3 KB as 16-byte vectors when the output is 16-byte
// aligned (each block's slice starts at a multiple of 3 KB), instead of
// three 4-byte stores 12 bytes apart per pixel.
constexpr int COMPOSE_PX = 256;

__global__ void __launch_bounds__(COMPOSE_PX)
k_compose3(const int32_t* __restrict__ lab, int pitch, int P, int W, int64_t n_px, const int32_t* __restrict__ xs,
           const int32_t* __restrict__ ys, const int32_t* __restrict__ tgrid, int32_t* __restrict__ out, bool vec)
{
    __shared__ __align__(16) int32_t stage[COMPOSE_PX * 3];
    const int64_t i0 = (int64_t)blockIdx.x * COMPOSE_PX;
    const int64_t i = i0 + threadIdx.x;
    if (i < n_px) {
        const int y = (int)(i / W), x = (int)(i - (int64_t)y * W);
        const int32_t l = lab[(size_t)(y + P) * pitch + x + P];
        int32_t d = -1;
        if (l >= 0) {
            const int32_t dx = x - __ldg(&xs[l]), dy = y - __ldg(&ys[l]);
            d = dx * dx + dy * dy;
        }
        stage[threadIdx.x * 3] = l;
        stage[threadIdx.x * 3 + 1] = d;
        stage[threadIdx.x * 3 + 2] = tgrid ? tgrid[i] : -1;
    }
    __syncthreads();
    const int64_t n_here = min((int64_t)COMPOSE_PX, n_px - i0) * 3;   // ints of this block's slice
    int32_t* dst = out + i0 * 3;
    if (vec && n_here == COMPOSE_PX * 3) {
        if (threadIdx.x < COMPOSE_PX * 3 / 4)
            reinterpret_cast<int4*>(dst)[threadIdx.x] = reinterpret_cast<const int4*>(stage)[threadIdx.x];
    } else {
        for (int k = threadIdx.x; k < n_here; k += COMPOSE_PX) dst[k] = stage[k];
    }
}

// k_compose3 four pixels of one row per thread, for W and P multiples of 4
// and a 16-byte aligned output: 16-byte loads of the labels and triangle ids,
// three 16-byte stores of the four (id, d2, triangle) triples.
__global__ void __launch_bounds__(256)
k_compose3x4(const int32_t* __restrict__ lab, int pitch, int P, int W, int64_t n_quads,
             const int32_t* __restrict__ xs, const int32_t* __restrict__ ys, const int32_t* __restrict__ tgrid,
             int32_t* __restrict__ out)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_quads) return;
    const int64_t i = q * 4;
    const int y = (int)(i / W), x = (int)(i - (int64_t)y * W);
    const int4 l4 = *reinterpret_cast<const int4*>(lab + (size_t)(y + P) * pitch + x + P);
    const int4 t4 = *reinterpret_cast<const int4*>(tgrid + i);
    const int32_t l[4] = {l4.x, l4.y, l4.z, l4.w};
    int32_t d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        d[k] = -1;
        if (l[k] >= 0) {
            const int32_t dx = x + k - __ldg(&xs[l[k]]), dy = y - __ldg(&ys[l[k]]);
            d[k] = dx * dx + dy * dy;
        }
    }
    int4* o = reinterpret_cast<int4*>(out + i * 3);
    o[0] = make_int4(l[0], d[0], t4.x, l[1]);
    o[1] = make_int4(d[1], t4.y, l[2], d[2]);
    o[2] = make_int4(t4.z, l[3], d[3], t4.w);
}

// (a, b, c) of each (x, y, a, b, c) triangle row.
__global__ void k_tri_vertices(const int32_t* __restrict__ tris, int64_t n, int32_t* __restrict__ verts)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * 3) return;
    const int64_t t = i / 3;
    verts[i] = tris[t * 5 + 2 + (i - t * 3)];
}

// GridTriangulation at P == 0 with the caller's grid: channels 0 and 1 are the
// caller's (triangulation.cu:406-411).
__global__ void k_compose3_from_grid(const int32_t* __restrict__ vgrid, int W, int H,
                                     const int32_t* __restrict__ tgrid, int32_t* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const size_t i = (size_t)y * W + x;
    out[i * 3] = vgrid[i * 2];
    out[i * 3 + 1] = vgrid[i * 2 + 1];
    out[i * 3 + 2] = tgrid[i];
}

// (H, W, 2) seed id + squared distance of a label plane (Voronoi().compute,
// and compute_debug's padded grid).  pos holds coordinates of the same canvas.
__global__ void k_compose2(const int32_t* __restrict__ lab, int pitch, int W, int H,
                           const uint32_t* __restrict__ pos, int32_t* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const int32_t l = lab[(size_t)y * pitch + x];
    const size_t i = (size_t)y * W + x;
    out[i * 2] = l;
    out[i * 2 + 1] = l >= 0 ? dist2(x, y, __ldg(&pos[l])) : -1;
}

// Label plane from a caller's (H, W, 2) grid, with the ids checked against
// the seed count (the reference indexes its seed arrays with them unchecked).
__global__ void k_labels_from_grid(const int32_t* __restrict__ vgrid, int W, int H, int pitch, int64_t n,
                                   int32_t* __restrict__ lab, Scalars* __restrict__ sc)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const int32_t l = vgrid[((size_t)y * W + x) * 2];
    if (l < -1 || l >= n) atomicOr(&sc->err_label, 1);
    lab[(size_t)y * pitch + x] = (l < -1 || l >= n) ? UNDEF : l;
}

int resolve_padding(int p)
{
    // binding_helpers.hpp:49-53: only the sentinel means "default".  Other
    // negatives are clamped to 0, as the NumPy reference does
    // (reference/triangulation.py:78); the reference CUDA path has no
    // defined behaviour for them.
    if (p == IDL_AUTO_BORDER_PADDING) return IDL_DEFAULT_BORDER_PADDING;
    return p < 0 ? 0 : p;
}

void check_mode(int mode)
{
    if (mode != IDL_MODE_REFERENCE && mode != IDL_MODE_NUMPY && mode != IDL_MODE_EXACT)
        invalid("mode must be one of IDL_MODE_REFERENCE, IDL_MODE_NUMPY, IDL_MODE_EXACT");
}

Canvas make_canvas(int Wd, int Hd)
{
    if (Wd > MAX_CANVAS_SIDE || Hd > MAX_CANVAS_SIDE)
        invalid("canvas side (including border padding) must not exceed " + std::to_string(MAX_CANVAS_SIDE));
    Canvas cv;
    cv.Wd = Wd;
    cv.Hd = Hd;
    cv.pitch = (Wd + 31) / 32 * 32;
    return cv;
}

void check_seed_count(int64_t n)
{
    if (n <= 0) invalid("seeds must not be empty");
    if (n > MAX_SEEDS) invalid("at most " + std::to_string(MAX_SEEDS) + " seeds are supported");
}

struct StageTimer {
    Context& C;
    bool on;
    StageTimer(Context& c, bool enable) : C(c), on(enable)
    {
        if (!on) return;
        for (auto& e : C.timing.ev)
            if (!e) IDL_CUDA(cudaEventCreate(&e));
    }
    void mark(int i)
    {
        if (on) IDL_CUDA(cudaEventRecord(C.timing.ev[i], C.stream));
    }
    float ms(int a, int b)
    {
        float t = 0.f;
        if (on) IDL_CUDA(cudaEventElapsedTime(&t, C.timing.ev[a], C.timing.ev[b]));
        return t;
    }
};

// Run stages (a) (b) (d) with seeds already in C.seeds_in.  Leaves labels in
// C.lab[0], triangles in C.tris, pixel ids in C.tgrid; returns triangle count.
int64_t run_triangulate(Context& C, int W, int H, int64_t n, const int32_t* vgrid_host_or_dev, bool vgrid_on_host,
                        int P, int mode, float* timings, int64_t* passes_out, Canvas& cv_out)
{
    const Canvas cv = make_canvas(W + 2 * P, H + 2 * P);
    cv_out = cv;
    C.prof.valid = false;
    for (bool& r : C.prof.recorded) r = false;
    C.prof.rounds = C.prof.tiles = C.prof.passes = 0;
    C.prof.prop_bytes = 0;
    C.mark(PM_START);
    sort_seeds_device(C, W, H, n, P);
    C.mark(PM_SEEDS);

    StageTimer T(C, timings != nullptr);
    int64_t passes = 0;
    if (P > 0 || !vgrid_host_or_dev) {
        if (mode == IDL_MODE_EXACT) {
            propagate_exact(C, cv, C.pos.as<uint32_t>(), n);
        } else {
            init_labels(C, cv, C.pos.as<uint32_t>(), n);
            passes = propagate(C, mode, cv, C.pos.as<uint32_t>(), n);
        }
    } else {
        const size_t gbytes = (size_t)W * H * 2 * sizeof(int32_t);
        C.vgrid.ensure(gbytes);
        IDL_CUDA(cudaMemcpyAsync(C.vgrid.ptr, vgrid_host_or_dev, gbytes,
                                 vgrid_on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, C.stream));
        C.lab[0].ensure((size_t)cv.pitch * cv.Hd * 4);
        IDL_CUDA(cudaMemsetAsync(&C.sc()->err_label, 0, sizeof(int32_t), C.stream));
        dim3 g(ceil_div(W, 256), H);
        k_labels_from_grid<<<g, 256, 0, C.stream>>>(C.vgrid.as<int32_t>(), W, H, cv.pitch, n, C.lab[0].as<int32_t>(),
                                                   C.sc());
        IDL_LAUNCH();
        C.fetch_scalars();
        if (C.host_sc->err_label) invalid("voronoi_grid seed ids must lie in [-1, number of seeds)");
    }
    if (passes_out) *passes_out = passes;
    C.mark(PM_PROPAGATE);

    T.mark(0);
    // detect_ms covers the fused detect + hash insert kernel, dedup_ms the
    // enumeration and canonical ranking (the reference's thrust sort/unique)
    detect_triangles(C, cv, C.lab[0].as<int32_t>(), C.pos.as<uint32_t>(), n, P,
                     T.on ? C.timing.ev[1] : nullptr);
    T.mark(2);
    C.mark(PM_DEDUP);
    // the triangle count came back with detection's own read-back (ranking
    // does not change it): no second host round trip here
    const int64_t nt = C.host_sc->n_triangles;
    T.mark(3);
    C.tgrid.ensure((size_t)W * H * sizeof(int32_t));
    assign_pixels(C, W, H, C.xs.as<int32_t>(), C.ys.as<int32_t>(), C.tgrid.as<int32_t>(), nt);
    C.mark(PM_ASSIGN);
    T.mark(4);
    if (timings) {
        IDL_CUDA(cudaEventSynchronize(C.timing.ev[4]));
        timings[IDL_T_DETECT_MS] = T.ms(0, 1);
        timings[IDL_T_DEDUP_MS] = T.ms(1, 2);
        timings[IDL_T_ASSIGN_MS] = T.ms(3, 4);
    }
    C.last_n_tri = nt;
    C.have_result = true;
    C.prof.canvas_px = (int64_t)cv.Wd * cv.Hd;
    C.prof.image_px = (int64_t)W * H;
    C.prof.n_triangles = nt;
    return nt;
}

void compose_triangulation(Context& C, const Canvas& cv, int W, int H, int P, bool from_grid, int32_t* d_out)
{
    dim3 g(ceil_div(W, 256), H);
    if (from_grid)
        k_compose3_from_grid<<<g, 256, 0, C.stream>>>(C.vgrid.as<int32_t>(), W, H, C.tgrid.as<int32_t>(), d_out);
    else if (W % 4 == 0 && P % 4 == 0 && cv.pitch % 4 == 0 && (reinterpret_cast<uintptr_t>(d_out) & 15) == 0) {
        const int64_t quads = (int64_t)W * H / 4;
        k_compose3x4<<<(unsigned)ceil_div(quads, (int64_t)256), 256, 0, C.stream>>>(
            C.lab[0].as<int32_t>(), cv.pitch, P, W, quads, C.xs.as<int32_t>(), C.ys.as<int32_t>(),
            C.tgrid.as<int32_t>(), d_out);
    } else
        k_compose3<<<(unsigned)ceil_div((int64_t)W * H, (int64_t)COMPOSE_PX), COMPOSE_PX, 0, C.stream>>>(
            C.lab[0].as<int32_t>(), cv.pitch, P, W, (int64_t)W * H, C.xs.as<int32_t>(), C.ys.as<int32_t>(),
            C.tgrid.as<int32_t>(), d_out, (reinterpret_cast<uintptr_t>(d_out) & 15) == 0);
    IDL_LAUNCH();
    C.mark(PM_COMPOSE);
    C.prof.valid = C.prof.enabled;
}

void upload_seeds(Context& C, const int32_t* xy, int64_t n, cudaMemcpyKind kind)
{
    C.seeds_in.ensure((size_t)n * 2 * sizeof(int32_t));
    IDL_CUDA(cudaMemcpyAsync(C.seeds_in.ptr, xy, (size_t)n * 2 * sizeof(int32_t), kind, C.stream));
}

void check_dims(int W, int H, int64_t n)
{
    if (W <= 0 || H <= 0) {
        if (n <= 0) invalid("seeds must not be empty");
        invalid("seed coordinate out of bounds");
    }
}

}  // namespace
}  // namespace idl

using namespace idl;


extern "C" {

const char* idl_last_error(void) { return g_last_error.c_str(); }

int idl_version(void) { return 100; }

long long idl_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

long long idl_alloc_count(void) { return g_allocs.load(std::memory_order_relaxed); }

int idl_selftest_grid_barrier(idl_context* ctx, int missing_arrivals, unsigned int spin_limit)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    DeviceGuard g(ctx->device);
    grid_barrier_selftest(*ctx, missing_arrivals, spin_limit);
    IDL_API_END
}

int idl_context_create(int device, idl_context** out)
{
    IDL_API_BEGIN
    if (!out) invalid("out must not be NULL");
    *out = nullptr;
    int dev = device;
    if (dev < 0) IDL_CUDA(cudaGetDevice(&dev));
    DeviceGuard g(dev);
    auto* c = new idl_context();
    c->device = dev;
    try {
        IDL_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev));
        ensure_scalars(*c);
    } catch (...) {
        delete c;
        throw;
    }
    *out = c;
    IDL_API_END
}

int idl_context_destroy(idl_context* ctx)
{
    IDL_API_BEGIN
    if (!ctx) return IDL_OK;
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
    IDL_API_END
}

int idl_context_set_stream(idl_context* ctx, void* stream)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    const cudaStream_t next = static_cast<cudaStream_t>(stream);
    // Workspace growth is freed in the order of the context's stream: finish
    // the old stream's work before later frees are ordered on the new one.
    if (next != ctx->stream) {
        DeviceGuard g(ctx->device);
        IDL_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    ctx->stream = next;
    IDL_API_END
}

int idl_context_set_schedule(idl_context* ctx, int dense_rounds)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    ctx->dense_rounds = dense_rounds;
    IDL_API_END
}

int idl_context_set_tile(idl_context* ctx, int shape, int* n_shapes_out)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    if (n_shapes_out) *n_shapes_out = key_tile_shapes();
    if (shape < 0 || shape >= key_tile_shapes()) invalid("tile shape index out of range");
    ctx->key_tile = shape;
    IDL_API_END
}

int idl_context_synchronize(idl_context* ctx)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    DeviceGuard g(ctx->device);
    IDL_CUDA(cudaStreamSynchronize(ctx->stream));
    IDL_API_END
}

int idl_context_workspace_bytes(idl_context* ctx, int64_t* bytes_out)
{
    IDL_API_BEGIN
    if (!ctx || !bytes_out) invalid("arguments must not be NULL");
    *bytes_out = (int64_t)ctx->workspace_bytes();
    IDL_API_END
}

int idl_context_set_profiling(idl_context* ctx, int enable)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    ctx->prof.enabled = enable != 0;
    ctx->prof.valid = false;
    IDL_API_END
}

int idl_context_pass_trace(idl_context* ctx, int64_t* ns_out, int32_t* tiles_out, int32_t* steps_out, int capacity,
                           int* n_out)
{
    IDL_API_BEGIN
    if (!ctx || !n_out) invalid("arguments must not be NULL");
    const Profile& P = ctx->prof;
    *n_out = (int)P.pass_ns.size();
    for (int i = 0; i < capacity && i < (int)P.pass_ns.size(); ++i) {
        if (ns_out) ns_out[i] = P.pass_ns[i];
        if (tiles_out) tiles_out[i] = P.pass_tiles[i];
        if (steps_out) steps_out[i] = i < (int)P.pass_steps.size() ? P.pass_steps[i] : 1;
    }
    IDL_API_END
}

int idl_context_set_tail_rounds(idl_context* ctx, int max_list)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    if (max_list < 0) invalid("max_list must not be negative");
    ctx->tail_rounds_below = max_list;
    IDL_API_END
}

int idl_context_last_profile(idl_context* ctx, double* out, int n)
{
    IDL_API_BEGIN
    if (!ctx || !out) invalid("arguments must not be NULL");
    if (!ctx->prof.valid) throw Error(IDL_ERR_STATE, "no profiled run on this context");
    DeviceGuard g(ctx->device);
    Profile& P = ctx->prof;
    double v[IDL_PROF_COUNT] = {};
    for (int m = PM_SEEDS; m < PM_COUNT; ++m) {
        int prev = m - 1;
        while (prev > PM_START && !P.recorded[prev]) --prev;
        if (P.recorded[m] && P.recorded[prev]) {
            IDL_CUDA(cudaEventSynchronize(P.ev[m]));
            float ms = 0.f;
            IDL_CUDA(cudaEventElapsedTime(&ms, P.ev[prev], P.ev[m]));
            v[m - 1] = ms;
        }
    }
    v[IDL_PROF_ROUNDS] = (double)P.rounds;
    v[IDL_PROF_TILES] = (double)P.tiles;
    v[IDL_PROF_PASSES] = (double)P.passes;
    v[IDL_PROF_TILE_W] = P.tile_w;
    v[IDL_PROF_TILE_H] = P.tile_h;
    v[IDL_PROF_STEPS] = P.steps_per_round;
    v[IDL_PROF_CANVAS_PX] = (double)P.canvas_px;
    v[IDL_PROF_IMAGE_PX] = (double)P.image_px;
    v[IDL_PROF_TRIANGLES] = (double)P.n_triangles;
    v[IDL_PROF_PROP_BYTES] = P.prop_bytes;
    for (int i = 0; i < n && i < IDL_PROF_COUNT; ++i) out[i] = v[i];
    IDL_API_END
}

int idl_voronoi(idl_context* ctx, int width, int height, const int32_t* seeds_xy, int64_t n_seeds, int mode,
                int32_t* grid_out, int64_t* passes_out)
{
    IDL_API_BEGIN
    if (!ctx || !grid_out) invalid("arguments must not be NULL");
    check_mode(mode);
    check_dims(width, height, n_seeds);
    check_seed_count(n_seeds);
    if (!seeds_xy) invalid("seeds must not be NULL");
    DeviceGuard g(ctx->device);
    Context& C = *ctx;
    const Canvas cv = make_canvas(width, height);
    upload_seeds(C, seeds_xy, n_seeds, cudaMemcpyHostToDevice);
    sort_seeds_device(C, width, height, n_seeds, 0);
    int64_t passes = 0;
    if (mode == IDL_MODE_EXACT) {
        propagate_exact(C, cv, C.pos.as<uint32_t>(), n_seeds);
    } else {
        init_labels(C, cv, C.pos.as<uint32_t>(), n_seeds);
        passes = propagate(C, mode, cv, C.pos.as<uint32_t>(), n_seeds);
    }
    const size_t bytes = (size_t)width * height * 2 * sizeof(int32_t);
    C.outgrid.ensure(bytes);
    dim3 gr(ceil_div(width, 256), height);
    k_compose2<<<gr, 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), cv.pitch, width, height, C.pos.as<uint32_t>(),
                                         C.outgrid.as<int32_t>());
    IDL_LAUNCH();
    IDL_CUDA(cudaMemcpyAsync(grid_out, C.outgrid.ptr, bytes, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    if (passes_out) *passes_out = passes;
    IDL_API_END
}

int idl_triangulate(idl_context* ctx, int width, int height, const int32_t* seeds_xy, int64_t n_seeds,
                    const int32_t* voronoi_grid, int border_padding, int mode, int32_t* grid_out,
                    int64_t* n_triangles_out, float* timings_out, int32_t* padded_grid_out)
{
    IDL_API_BEGIN
    if (!ctx || !grid_out) invalid("arguments must not be NULL");
    check_mode(mode);
    if (width <= 0 || height <= 0) invalid("width and height must be positive");
    check_seed_count(n_seeds);
    if (!seeds_xy) invalid("seeds must not be NULL");
    DeviceGuard g(ctx->device);
    Context& C = *ctx;
    C.have_result = false;
    const int P = resolve_padding(border_padding);
    upload_seeds(C, seeds_xy, n_seeds, cudaMemcpyHostToDevice);
    Canvas cv;
    const bool from_grid = (P == 0 && voronoi_grid != nullptr);
    const int64_t nt = run_triangulate(C, width, height, n_seeds, voronoi_grid, true, P, mode, timings_out,
                                       nullptr, cv);
    const size_t bytes = (size_t)width * height * 3 * sizeof(int32_t);
    C.outgrid.ensure(bytes);
    compose_triangulation(C, cv, width, height, P, from_grid, C.outgrid.as<int32_t>());
    IDL_CUDA(cudaMemcpyAsync(grid_out, C.outgrid.ptr, bytes, cudaMemcpyDeviceToHost, C.stream));
    if (padded_grid_out && P > 0) {
        const size_t pb = (size_t)cv.Wd * cv.Hd * 2 * sizeof(int32_t);
        C.padded.ensure(pb);
        dim3 gp(ceil_div(cv.Wd, 256), cv.Hd);
        k_compose2<<<gp, 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), cv.pitch, cv.Wd, cv.Hd, C.pos.as<uint32_t>(),
                                             C.padded.as<int32_t>());
        IDL_LAUNCH();
        IDL_CUDA(cudaMemcpyAsync(padded_grid_out, C.padded.ptr, pb, cudaMemcpyDeviceToHost, C.stream));
    }
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    if (n_triangles_out) *n_triangles_out = nt;
    IDL_API_END
}

int idl_get_triangle_vertices(idl_context* ctx, int32_t* verts_out, int64_t capacity)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    if (!ctx->have_result) throw Error(IDL_ERR_STATE, "no triangulation result on this context");
    if (capacity < ctx->last_n_tri) invalid("capacity is smaller than the triangle count");
    if (ctx->last_n_tri == 0) return IDL_OK;
    if (!verts_out) invalid("verts_out must not be NULL");
    DeviceGuard g(ctx->device);
    const int64_t n = ctx->last_n_tri;
    ctx->verts.ensure((size_t)n * 3 * sizeof(int32_t));
    k_tri_vertices<<<(unsigned)((n * 3 + 255) / 256), 256, 0, ctx->stream>>>(ctx->tris.as<int32_t>(), n,
                                                                          ctx->verts.as<int32_t>());
    IDL_LAUNCH();
    IDL_CUDA(cudaMemcpyAsync(verts_out, ctx->verts.ptr, (size_t)n * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             ctx->stream));
    IDL_CUDA(cudaStreamSynchronize(ctx->stream));
    IDL_API_END
}

int idl_get_triangles(idl_context* ctx, int32_t* tris_out, int64_t capacity)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    if (!ctx->have_result) throw Error(IDL_ERR_STATE, "no triangulation result on this context");
    if (capacity < ctx->last_n_tri) invalid("capacity is smaller than the triangle count");
    if (ctx->last_n_tri == 0) return IDL_OK;
    if (!tris_out) invalid("tris_out must not be NULL");
    DeviceGuard g(ctx->device);
    IDL_CUDA(cudaMemcpyAsync(tris_out, ctx->tris.ptr, (size_t)ctx->last_n_tri * 5 * sizeof(int32_t),
                             cudaMemcpyDeviceToHost, ctx->stream));
    IDL_CUDA(cudaStreamSynchronize(ctx->stream));
    IDL_API_END
}

int idl_triangulate_device(idl_context* ctx, int width, int height, const int32_t* d_seeds_xy, int64_t n_seeds,
                           int border_padding, int mode, int32_t* d_grid_out, int64_t* n_triangles_out)
{
    IDL_API_BEGIN
    if (!ctx || !d_grid_out || !d_seeds_xy) invalid("arguments must not be NULL");
    check_mode(mode);
    if (width <= 0 || height <= 0) invalid("width and height must be positive");
    check_seed_count(n_seeds);
    DeviceGuard g(ctx->device);
    Context& C = *ctx;
    C.have_result = false;
    const int P = resolve_padding(border_padding);
    upload_seeds(C, d_seeds_xy, n_seeds, cudaMemcpyDeviceToDevice);
    Canvas cv;
    const int64_t nt = run_triangulate(C, width, height, n_seeds, nullptr, false, P, mode, nullptr, nullptr, cv);
    compose_triangulation(C, cv, width, height, P, false, d_grid_out);
    if (n_triangles_out) {
        IDL_CUDA(cudaStreamSynchronize(C.stream));
        *n_triangles_out = nt;
    }
    IDL_API_END
}

int idl_triangles_device(idl_context* ctx, const int32_t** d_tris, const int64_t** d_count)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    if (!ctx->have_result) throw Error(IDL_ERR_STATE, "no triangulation result on this context");
    if (d_tris) *d_tris = ctx->tris.as<int32_t>();
    if (d_count) *d_count = &ctx->sc()->n_triangles;
    IDL_API_END
}

}  // extern "C"
