// idl_voronoi_noalloc: Voronoi().compute on device buffers with no memory
// allocation at all.
//
// Who needs it.  Some callers cannot call cudaMalloc: code on a latency budget
// where cudaMalloc/cudaFree would stall or synchronise the device, processes
// whose device memory is carved up in advance (a fixed per-tenant quota, a
// memory pool they must stay inside), and hosts embedding this library under
// an allocator they do not control.  For them every other entry point is off
// limits, because a context grows its workspace on demand.
//
// How.  All workspace of the stage-(a) pipeline (seed ordering bitmap and
// scans, sorted seed tables, both label planes, the propagation work lists,
// bitmaps, counters and barrier state) is carved out of one file-scope
// `static __device__` array of NA_SCRATCH_BYTES.  The caller passes the seeds
// and the output grid in device memory.  A GPU holds the array from the moment
// this file's module is loaded on it until the process exits.  Under CUDA's
// lazy module loading (the default since CUDA 12.2) that moment is the first
// call of this entry point on the device: its cudaGetSymbolAddress loads the
// module and commits the array, so that one call does take device memory and
// can fail if a quota is already used up.  Make it at set-up, outside any
// quota- or latency-critical section, or run with CUDA_MODULE_LOADING=EAGER
// to commit the array when the context is created.
//
// Set-up.  The array's name is only a host-side stand-in in host code, so the
// device address is fetched with cudaGetSymbolAddress, once per device, with
// that device current, the first time the entry point runs on it.  No call
// can be captured into a CUDA graph: each waits for its stream (seed
// validation, convergence).
//
// Sharing.  Every call uses the same array, which keeps whatever the previous
// call left there; the pipeline clears everything that must start at zero.
// Calls whose GPU work overlaps (two streams, two threads, or the same stream
// from two processes sharing a context) race on the array and must not be
// issued; the entry point itself serialises host-side set-up only.
#include "context.cuh"

#include <mutex>

namespace idl {
namespace {

// Limits of the fixed workspace.
constexpr int NA_MAX_SIDE = 1024;              // canvas width and height
constexpr int64_t NA_MAX_SEEDS = 65536;
constexpr size_t NA_PLANE = (size_t)NA_MAX_SIDE * NA_MAX_SIDE * 4;   // pitch <= 1024
constexpr size_t NA_SEEDS = (size_t)NA_MAX_SEEDS * 4;
constexpr size_t NA_BITS_WORDS = (size_t)NA_MAX_SIDE * NA_MAX_SIDE / 32;
constexpr size_t NA_TILES = 16384;             // work-list capacity (micro-tiles of the largest canvas)
constexpr size_t NA_COUNTS = 4 * (2 * NA_MAX_SIDE) + 64 + 2 + 64;   // per-pass list lengths
constexpr size_t NA_SCAN_ARENA = 4096;
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

constexpr size_t NA_SCRATCH_BYTES =
    3 * align256(NA_SEEDS) +                                  // xs, ys, pos
    3 * align256(NA_BITS_WORDS * 4 + 4) +                     // occupancy bitmap, popcounts, ranks
    align256(NA_SCAN_ARENA * 4) +                             // scan block sums
    2 * align256(NA_PLANE) +                                  // label planes
    2 * align256(NA_TILES * 4) +                              // work lists
    align256(NA_TILES / 32 * 2 * 4 + 8) +                     // work-list dedup bitmaps
    align256(NA_COUNTS * 4) +                                 // per-pass counts
    align256(NA_TILES * 4) +                                  // tile-round stamps
    align256(64) + align256(sizeof(Scalars));                 // barrier state, counters

}  // namespace
}  // namespace idl

// The workspace itself (about 9.8 MB); a device holds it once this module is loaded there.
static __device__ __align__(256) unsigned char g_noalloc_scratch[idl::NA_SCRATCH_BYTES];

namespace idl {
namespace {

constexpr int NA_MAX_DEVICES = 64;

struct NoAllocSlot {
    bool ready = false;
    Context ctx;              // workspace views into g_noalloc_scratch, never owning
    Scalars host_scalars{};   // host mirror of the counters (pageable, static)
};

NoAllocSlot g_slots[NA_MAX_DEVICES];
std::mutex g_setup_mutex;

// Carve the fixed workspace for `dev` (the current device).  Once per device.
Context& noalloc_context(int dev)
{
    if (dev < 0 || dev >= NA_MAX_DEVICES) invalid("device ordinal out of range for the no-allocation entry point");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    NoAllocSlot& s = g_slots[dev];
    if (s.ready) return s.ctx;
    void* base = nullptr;
    IDL_CUDA(cudaGetSymbolAddress(&base, g_noalloc_scratch));
    unsigned char* p = static_cast<unsigned char*>(base);
    auto take = [&p](DevBuf& b, size_t n) {
        b.borrow(p, n);
        p += align256(n);
    };
    Context& C = s.ctx;
    C.device = dev;
    C.dense_rounds = 0;   // the persistent kernel alone: its buffers are the ones carved below
    IDL_CUDA(cudaDeviceGetAttribute(&C.num_sms, cudaDevAttrMultiProcessorCount, dev));
    take(C.xs, NA_SEEDS);
    take(C.ys, NA_SEEDS);
    take(C.pos, NA_SEEDS);
    take(C.bitmap, NA_BITS_WORDS * 4 + 4);
    take(C.scan_b, NA_BITS_WORDS * 4 + 4);
    take(C.scan_c, NA_BITS_WORDS * 4 + 4);
    take(C.scan_a, NA_SCAN_ARENA * 4);
    take(C.lab[0], NA_PLANE);
    take(C.lab[1], NA_PLANE);
    take(C.tiles[0], NA_TILES * 4);
    take(C.tiles[1], NA_TILES * 4);
    take(C.bits, NA_TILES / 32 * 2 * 4 + 8);
    take(C.counts, NA_COUNTS * 4);
    take(C.stamps, NA_TILES * 4);
    take(C.gsync, 64);
    take(C.scalars, sizeof(Scalars));
    if ((size_t)(p - static_cast<unsigned char*>(base)) > NA_SCRATCH_BYTES)
        throw Error(IDL_ERR_INTERNAL, "no-allocation workspace layout exceeds its array");
    C.host_sc = &s.host_scalars;
    C.host_sc_borrowed = true;
    s.ready = true;
    return C;
}

__global__ void k_noalloc_compose2(const int32_t* __restrict__ lab, int pitch, int W, int H,
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

}  // namespace
}  // namespace idl

using namespace idl;

extern "C" {

int idl_voronoi_noalloc(int width, int height, const int32_t* d_seeds_xy, int64_t n_seeds, int mode,
                        int32_t* d_grid_out, void* stream, int64_t* passes_out)
{
    IDL_API_BEGIN
    if (!d_seeds_xy || !d_grid_out) invalid("arguments must not be NULL");
    if (mode != IDL_MODE_REFERENCE && mode != IDL_MODE_NUMPY)
        invalid("the no-allocation entry point supports IDL_MODE_REFERENCE and IDL_MODE_NUMPY");
    if (n_seeds <= 0) invalid("seeds must not be empty");
    if (width <= 0 || height <= 0) invalid("seed coordinate out of bounds");
    if (width > NA_MAX_SIDE || height > NA_MAX_SIDE)
        invalid("the no-allocation entry point handles canvases up to 1024 x 1024 pixels");
    if (n_seeds > NA_MAX_SEEDS) invalid("the no-allocation entry point handles up to 65536 seeds");
    int dev = 0;
    IDL_CUDA(cudaGetDevice(&dev));
    Context& C = noalloc_context(dev);
    C.stream = static_cast<cudaStream_t>(stream);
    C.prof.enabled = false;
    // the caller's seed buffer stands in for the uploaded copy
    C.seeds_in.borrow(const_cast<int32_t*>(d_seeds_xy), (size_t)n_seeds * 2 * sizeof(int32_t));

    Canvas cv;
    cv.Wd = width;
    cv.Hd = height;
    cv.pitch = (width + 31) / 32 * 32;
    sort_seeds_device(C, width, height, n_seeds, 0);
    init_labels(C, cv, C.pos.as<uint32_t>(), n_seeds);
    const int64_t passes = propagate(C, mode, cv, C.pos.as<uint32_t>(), n_seeds);
    dim3 g(ceil_div(width, 256), height);
    k_noalloc_compose2<<<g, 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), cv.pitch, width, height,
                                                C.pos.as<uint32_t>(), d_grid_out);
    IDL_LAUNCH();
    if (passes_out) *passes_out = passes;
    IDL_API_END
}

}  // extern "C"
