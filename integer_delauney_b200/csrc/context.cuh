// Per-device context: stream, grow-only device workspace and the small block
// of device-side counters one pipeline run uses.
//
// The reference allocates every intermediate per call and frees it on return
// (src/cuda/voronoi.cu:87-91, src/cuda/triangulation.cu:271-351); a cudaFree
// synchronises the device, so that design pays a full drain per buffer.  A
// context instead keeps each workspace buffer at its high-water mark and
// reuses it, so a steady stream of calls allocates nothing.
#pragma once

#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace idl {

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    bool fixed = false;   // borrowed memory of fixed size: never allocated or freed here
    bool async = false;   // ptr came from the stream-ordered allocator
    // When set, growth is stream-ordered on the owner's current stream
    // (cudaMallocAsync / cudaFreeAsync): it waits for nothing but the work
    // already queued there, instead of for the whole device as cudaFree does
    // -- which matters when many streams share a device (a server).
    const cudaStream_t* stream = nullptr;

    template <class T>
    T* as() const { return static_cast<T*>(ptr); }

    // Grow to at least `need` bytes (contents are not preserved).  A first
    // allocation is exact; a regrowth takes at least 1.5x the old size, so
    // buffers sized by a count that creeps up call after call (triangle rows
    // of a growing diagram, the scratch of requests of mixed sizes) are
    // reallocated O(log) times, not every call.
    void ensure(size_t need)
    {
        if (need <= bytes) return;
        if (fixed) invalid("request exceeds the fixed workspace of this entry point");
        size_t grow = need;
        if (bytes) grow = std::max(need, bytes + bytes / 2);
        grow = (grow + 255) / 256 * 256;
        drop();
        if (need == 0) return;
        count_alloc();
        if (stream) {
            IDL_CUDA(cudaMallocAsync(&ptr, grow, *stream));
            async = true;
        } else {
            IDL_CUDA(cudaMalloc(&ptr, grow));
        }
        bytes = grow;
    }
    void borrow(void* p, size_t n)
    {
        ptr = p;
        bytes = n;
        fixed = true;
        async = false;
    }
    // Free in stream order behind the work queued on the owner's stream.
    void drop() noexcept
    {
        if (ptr && !fixed) {
            if (async) cudaFreeAsync(ptr, *stream);
            else cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
        async = false;
    }
    // Free at teardown.  cudaFree does not wait for stream-ordered memory:
    // the owner synchronises first when any of its buffers is (see
    // Context::~Context).
    void release() noexcept
    {
        if (ptr && !fixed) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        async = false;
    }
};

// Device-side counters and flags of one pipeline run.  Lives in device memory;
// a pinned host mirror receives it when the host needs a count.
struct Scalars {
    int64_t n_triangles;      // unique triangles after dedup
    int64_t n_inserted;       // keys inserted into the hash table
    int64_t last_change;      // last propagation step (0-based) that changed a cell
    int32_t err_oob;          // a seed lay outside the canvas
    int32_t err_dup;          // two seeds share a pixel
    int32_t err_label;        // a caller-supplied label was outside [-1, n)
    int32_t overflow;         // hash table over its load limit or probe bound
    int32_t max_side;         // longest triangle side, float-truncated (triangulation.cu:355-368)
    int32_t n_big;            // tall triangles the raster hands to its block-per-triangle pass
    int32_t n_handoff;        // micro-tiles the last tile round hands to the persistent kernel
    int32_t tile_remaining;   // tiles listed for the tile round after the last one launched
};

struct Timing {
    cudaEvent_t ev[8] = {};
    bool on = false;
};

// Stage boundaries of the last pipeline run, recorded on the context's stream
// when profiling is enabled (idl_context_set_profiling).
enum ProfMark { PM_START = 0, PM_SEEDS, PM_PROPAGATE, PM_DETECT, PM_DEDUP, PM_ASSIGN, PM_COMPOSE, PM_COUNT };

struct Profile {
    bool enabled = false;
    bool valid = false;
    cudaEvent_t ev[PM_COUNT] = {};
    bool recorded[PM_COUNT] = {};
    int64_t rounds = 0;           // propagation rounds launched with work
    int64_t tiles = 0;            // tiles processed over all rounds
    int64_t passes = 0;           // propagation passes (reference semantics)
    double prop_bytes = 0;        // algorithmic HBM bytes of the propagation (8 B per cell update)
    int64_t canvas_px = 0;        // detection canvas pixels
    int64_t image_px = 0;         // output pixels
    int64_t n_triangles = 0;
    int tile_w = 0, tile_h = 0, steps_per_round = 0;
    // persistent sparse kernel: duration (ns) and work-list length of each pass
    std::vector<int64_t> pass_ns;
    std::vector<int32_t> pass_tiles;
    std::vector<int32_t> pass_steps;   // passes each entry advanced (1, 0 entering the round mode, or a round's)
};

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 148;

    // seeds
    DevBuf seeds_in;      // n x 2 int32 as the caller passed them
    DevBuf xs, ys;        // sorted seed coordinates (image space)
    DevBuf pos;           // sorted seed positions on the detection canvas, packed
    DevBuf bitmap;        // canvas occupancy bits, column major, for the (x, y) sort
    DevBuf scan_a, scan_b, scan_c;  // scan scratch

    // propagation
    DevBuf lab[2];        // label planes, pitch x Hd int32, ping-pong
    DevBuf tiles[2];      // active tile lists
    DevBuf stamps;        // per-tile "already listed for round r" marks
    DevBuf counts;        // per-round list lengths
    DevBuf gsync;         // grid barrier state of the persistent propagation kernel
    DevBuf trace;         // per-pass timestamps of the persistent kernel (profiling only)
    DevBuf rbig;          // raster: ids of tall triangles
    DevBuf bits;          // work-list dedup bitmaps of the persistent propagation kernel
    DevBuf big_tiles;     // tile rounds' last work list, handed to the persistent kernel
    DevBuf cellbits;      // cell-list tile rounds: three last-pass change bitmaps, in rotation
    DevBuf exact_dy;      // exact mode: row distance to each cell's column-nearest seed
    DevBuf exact_rmin;    // exact mode: per row, smallest squared row distance of each 32-column block
    int32_t stamp_epoch = 0;
    int dense_rounds = 3;  // propagation schedule from scratch (propagate.cu; idl_context_set_schedule)
    int key_tile = 9;      // tile shape of the owner-key tile round (propagate.cu; idl_context_set_tile)
    // The persistent kernel advances several passes per grid barrier once its
    // work list holds at most this many micro-tiles (sparse_jacobi.cu; 0:
    // never; idl_context_set_tail_rounds).
    int tail_rounds_below = 4096;
    // Whether the persistent tile shapes (key_tile >= 4) may run their rounds
    // as one device-filling cooperative launch (propagate.cu); off for
    // contexts whose work must overlap other streams' (a server's workers).
    bool persistent_rounds = true;

    // topology
    DevBuf hkeys;         // hash table of triangle keys -> first witness (key, value interleaved)
    DevBuf ukeys, uvals;  // compacted unique keys
    DevBuf cnt, off, fill, grp;  // group-by-smallest-vertex ranking
    DevBuf tris;          // n_tri x 5 int32 (x, y, a, b, c)
    DevBuf verts;         // n_tri x 3 int32 (a, b, c) staged for idl_get_triangle_vertices
    int64_t hash_cap = 0;

    // assignment / output
    DevBuf tgrid;         // W x H int32 triangle ids
    DevBuf vgrid;         // caller-supplied Voronoi grid (GridTriangulation at P = 0)
    DevBuf outgrid;       // H x W x 3 staging for host-pointer calls
    DevBuf padded;        // padded Voronoi grid for compute_debug

    // batched triangulation (batch.cu)
    DevBuf batch_img;       // per-image table
    DevBuf batch_seed_img;  // image of each input seed
    DevBuf batch_rows;      // image of each output row
    DevBuf batch_sid;       // image of each sorted seed
    DevBuf batch_stats;     // per-image triangle counts, longest sides, triangle offsets
    DevBuf batch_bad;       // first out-of-bounds / duplicate seed index
    DevBuf batch_ximg, batch_colimg, batch_rowimg;  // exact semantics: image table, column / row -> image

    DevBuf scalars;       // one Scalars
    Scalars* host_sc = nullptr;  // pinned mirror
    bool host_sc_borrowed = false;  // host_sc points at static storage, not cudaMallocHost memory

    const void* owner = nullptr; // object whose intermediates the buffers hold (shared workspaces)
    std::shared_ptr<void> batch_plan;  // layout of the last batch (batch.cu)
    int64_t last_n_tri = 0;      // triangles of the last triangulation (host copy)
    bool have_result = false;

    Timing timing;
    Profile prof;

    void mark(ProfMark m)
    {
        if (!prof.enabled) return;
        if (!prof.ev[m]) IDL_CUDA(cudaEventCreate(&prof.ev[m]));
        IDL_CUDA(cudaEventRecord(prof.ev[m], stream));
        prof.recorded[m] = true;
    }

    // Every workspace buffer, for set-up, sizing and teardown.
    template <class F>
    void each_buf(F&& f)
    {
        DevBuf* all[] = {&seeds_in, &xs, &ys, &pos, &bitmap, &scan_a, &scan_b, &scan_c, &lab[0], &lab[1],
                         &tiles[0], &tiles[1], &stamps, &counts, &gsync, &trace, &rbig, &bits, &big_tiles, &exact_dy, &exact_rmin, &hkeys,
                         &ukeys, &uvals, &cnt, &off, &fill, &grp, &tris, &tgrid, &vgrid, &outgrid, &padded,
                         &batch_img, &batch_seed_img, &batch_rows, &batch_sid, &batch_stats, &batch_bad,
                         &batch_ximg, &batch_colimg, &batch_rowimg, &scalars};
        for (DevBuf* b : all) f(*b);
    }
    Context()
    {
        each_buf([this](DevBuf& b) { b.stream = &stream; });
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;

    Scalars* sc() const { return scalars.as<Scalars>(); }
    size_t workspace_bytes() const;
    void fetch_scalars();        // D2H of the Scalars block + stream sync
    ~Context();
};

// RAII: make the context's device current for the duration of a call.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) IDL_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// ---- pipeline pieces (one .cu each) -----------------------------------

// Exclusive scan of n int32 values in place semantics: out[i] = sum(in[0..i)),
// and out[n] = total.  `out` must hold n + 1 values.  Uses ctx scan scratch.
void exclusive_scan(Context& C, const int32_t* in, int32_t* out, int64_t n);

// Validate and sort seeds on the device (seeds.cu).  Reads C.seeds_in (n x 2),
// writes C.xs / C.ys (sorted, image space) and C.pos (detection canvas, shifted
// by P).  Throws IDL_ERR_INVALID with the reference's messages.
void sort_seeds_device(Context& C, int W, int H, int64_t n, int P);

// (x asc, y asc) rank of n distinct, validated seeds given in insertion
// order (seeds.cu): rank[i], its inverse inv[rank[i]] = i, and the
// coordinates plus `off` scattered into sorted order.
void rank_seeds_device(Context& C, int W, int H, const int32_t* xs, const int32_t* ys, int64_t n, int off,
                       int32_t* rank, int32_t* inv, int32_t* xs_sorted, int32_t* ys_sorted);

// Stage (a) on the Wd x Hd detection canvas whose labels are in C.lab[0]
// (both planes must hold the same starting state); the result is left in
// C.lab[0].  Returns the pass count (propagate.cu).  From scratch (seed_pos ==
// nullptr) the n_seeds seeds of `pos` are the canvas's seeds in id order,
// which must be their (x, y) order (per image of a batch atlas); in reference
// semantics that propagation runs on owner keys (stencil.cuh), and
// C.lab[1] is scratch afterwards.  With seed_pos the state is a fixed point
// except at n_new freshly written seed cells, and ids may be in any order.
struct Canvas {
    int Wd, Hd, pitch;
};
int64_t propagate(Context& C, int mode, const Canvas& cv, const uint32_t* pos, int64_t n_seeds,
                  const uint32_t* seed_pos = nullptr, int64_t n_new = 0);
// Number of owner-key tile round shapes (Context::key_tile indexes them).
int key_tile_shapes();

// Reference-semantics propagation as one persistent kernel (sparse_jacobi.cu).
// `seed_pos` (may be nullptr): the state is a fixed point except at these
// n_new freshly written seed cells (packed canvas positions), so only the
// micro-tiles around them start active; otherwise every micro-tile does.
int64_t propagate_sparse(Context& C, const Canvas& cv, const uint32_t* pos, const uint32_t* seed_pos = nullptr,
                         int64_t n_new = 0, bool keys = false);

// As propagate_sparse from scratch, with the first work list built from a
// device list of n_big tiles of big_w x big_h cells (big_tiles_x per row;
// both multiples of the micro-tile side): all their micro-tiles.  Plane 0
// holds the starting state, and every micro-tile outside the list must hold
// the same state in both planes.
int64_t propagate_sparse_from_tiles(Context& C, const Canvas& cv, const uint32_t* pos, const int32_t* big_list,
                                    int n_big, int big_tiles_x, int big_w, int big_h, bool keys = false);
// As propagate_sparse from scratch, with the first work list given: `marked`
// holds n_marked distinct micro-tiles, and C.bits (sparse_bits_words(cv)
// words for each of the two passes' bitmaps) already has their bits set in
// the first bitmap and none in the second.  Plane 0 holds the starting state,
// the same in plane 1 outside the listed micro-tiles.  The list length is read
// on the device from C.sc()->n_handoff; n_marked is the host's copy of it (0:
// nothing to do) or negative when the host has not read it.  On return
// C.host_sc holds the scalars as the kernel left them.
int64_t propagate_sparse_from_marks(Context& C, const Canvas& cv, const uint32_t* pos, const int32_t* marked,
                                    int n_marked, bool keys);
int sparse_bits_words(const Canvas& cv);
struct SparseStart {
    const uint32_t* seed_pos = nullptr;   // new seeds: the micro-tiles around them
    int64_t n_new = 0;
    const int32_t* big_list = nullptr;    // tiles: all their micro-tiles
    int n_big = 0, big_tiles_x = 0, sub_x = 0, sub_y = 0;
    const int32_t* marked = nullptr;      // micro-tiles, bitmap already set
    int n_marked = 0;
};
int64_t propagate_sparse_impl(Context& C, const Canvas& cv, const uint32_t* pos, const SparseStart& start, bool keys);

// Held from launch to completion of a device-filling persistent kernel, one
// per device: such grids run one at a time, so each one's co-residency does
// not depend on other streams' grids (sparse_jacobi.cu).
std::mutex& persistent_grid_lock(int device);

// Run the persistent kernel's grid barrier alone (sparse_jacobi.cu) on one
// block per SM, waiting for `missing_arrivals` more blocks than the grid has,
// with at most `spin_limit` polls per wait.  Throws IDL_ERR_INTERNAL ("grid
// barrier timed out") when a wait ran out, exactly as propagation reports it.
void grid_barrier_selftest(Context& C, int missing_arrivals, unsigned spin_limit);

// Stage (a), exact semantics (exact.cu): nearest seed, ties to the higher id,
// for the n (x, y)-sorted seeds `pos` of the canvas; labels into C.lab[0]
// (C.lab[1] is scratch).
void propagate_exact(Context& C, const Canvas& cv, const uint32_t* pos, int64_t n);

// Reserve a range of per-item stamp values for `steps` steps (propagate.cu).
int32_t claim_stamps(Context& C, int n_items, int64_t steps);

// Seed the label planes: fill with UNDEF and write seed ids (propagate.cu).
void init_labels(Context& C, const Canvas& cv, const uint32_t* pos, int64_t n);

// Stage (b): detect + dedup + canonical numbering on the label plane
// (topology.cu).  Leaves the triangles in C.tris and their count in
// C.sc()->n_triangles; returns nothing to the host.
// `mid` (may be nullptr) is recorded between detection and deduplication.
// `rank` (may be nullptr): labels are raw ids (the block rule runs on them);
// keys, numbering and the recorded vertex ids use rank[label] instead.
void detect_triangles(Context& C, const Canvas& cv, const int32_t* labels, const uint32_t* pos, int64_t n,
                      int shift, cudaEvent_t mid = nullptr, const int32_t* rank = nullptr);

// Stage (d): per-pixel max triangle id over a W x H image (raster.cu).
void assign_pixels(Context& C, int W, int H, const int32_t* xs, const int32_t* ys, int32_t* tgrid,
                   int64_t max_tri);

void ensure_scalars(Context& C);

// One image of the last batch on a context (idl_voronoi_batch or a batched
// triangulation):
// its padded canvas sits at (ox, oy) of the atlas label planes C.lab[0/1]
// (row pitch `pitch`), its seeds are C.xs/C.ys[seed_off, seed_off + n) in
// (x, y) order with atlas labels seed_off + local id (batch.cu).
struct BatchImage {
    int W, H, ox, oy, P, pitch;
    int64_t seed_off, n;
};
bool batch_image(const Context& C, int k, BatchImage& out);

// The whole batched pipeline (idl_triangulate_batch) on host seeds, its
// result kept on the context: per-image triangle counts to tri_counts; the
// atlas labels for idl_delaunay_adopt and each image's grid and triangle
// rows for batch_fetch (batch.cu).
void triangulate_batch_keep(Context& C, int n_images, const int32_t* dims, const int64_t* counts,
                            const int32_t* seeds_xy, int P, int64_t* tri_counts);
// Queue on C.stream the copies of image k of the last triangulated batch:
// its grid (H x W x 3 int32) and its triangle rows (5 int32 each, image-local
// as idl_delaunay_triangles ids = 0 reports them) into host buffers.
void batch_fetch(Context& C, int k, int32_t* grid_out, int32_t* tris_out, int64_t capacity);

}  // namespace idl

// The C ABI's opaque context handle is a Context.
struct idl_context : public idl::Context {};
