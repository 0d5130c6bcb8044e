/*
 * idelaunay.h -- C ABI of the B200-native integer Delaunay library.
 *
 * This is the drop-in boundary for the hot path of timdahmen/integer_delauney:
 * every entry point below replaces one function of the reference's compiled
 * extension (the pybind11 module `_delauney_cuda`, src/cuda/bindings.cpp) or
 * of the C++ layer under it, cited per declaration as file:line relative to
 * the reference project root.  Plain C types only: pointers, sizes and status
 * codes; no PyTorch, pybind11 or C++ types cross this boundary.
 *
 * Conventions
 *   - Every function returns IDL_OK or an IDL_ERR_* status; the message of
 *     the last failure on the calling thread is idl_last_error().
 *     IDL_ERR_INVALID corresponds to the reference's std::invalid_argument
 *     (ValueError in Python), IDL_ERR_CUDA and IDL_ERR_STATE to its
 *     std::runtime_error / std::logic_error (RuntimeError).
 *   - Seeds are passed as n (x, y) int32 pairs in any order.  They are
 *     validated (bounds, non-empty, distinct) and numbered in (x asc, y asc)
 *     order, exactly as the reference's sort_seeds
 *     (src/cuda/bindings/binding_helpers.hpp:23-46) does.
 *   - Host-pointer entry points copy inputs in and results out and return
 *     after the results are in host memory.  *_device entry points take and
 *     produce device pointers on the context's device and are ordered on the
 *     context's stream; they synchronise only where a count must reach the
 *     host, as documented per function.
 *   - mode selects the Voronoi propagation semantics (see IDL_MODE_*).
 */
#ifndef IDELAUNAY_H
#define IDELAUNAY_H

#include <stdint.h>

#if defined(__GNUC__)
#define IDL_API __attribute__((visibility("default")))
#else
#define IDL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define IDL_OK 0
#define IDL_ERR_INVALID 1  /* invalid argument (ValueError) */
#define IDL_ERR_CUDA 2     /* CUDA runtime failure (RuntimeError) */
#define IDL_ERR_STATE 3    /* call not valid in the object's state (RuntimeError) */
#define IDL_ERR_INTERNAL 4 /* internal invariant broken (RuntimeError) */
#define IDL_ERR_BUDGET 5   /* server: request does not fit the memory budget (MemoryError) */
#define IDL_ERR_NOT_RESIDENT 6 /* server: the diagram is not resident (KeyError) */

/* ---- Voronoi propagation semantics --------------------------------- */
/* Synchronous Jacobi fixed point of src/cuda/voronoi.cu:32-53,100-113: the
 * reference CUDA path's own result, bit for bit.  Default. */
#define IDL_MODE_REFERENCE 0
/* Four-direction sweep of src/delauney/reference/voronoi.py:90-163: the
 * reference NumPy implementation's own result, bit for bit. */
#define IDL_MODE_NUMPY 1
/* Exact nearest seed, ties to the higher seed id: the contract both reference
 * implementations approximate (reference/voronoi.py:9-31).  History
 * independent, so an incremental state equals a full recompute. */
#define IDL_MODE_EXACT 2

/* src/cuda/triangulation.cuh:12 and src/delauney/__init__.py:16 */
#define IDL_DEFAULT_BORDER_PADDING 16
/* src/cuda/bindings/binding_helpers.hpp:20: the int spelling of "choose for me" */
#define IDL_AUTO_BORDER_PADDING (-1)

/* timings_out layout for triangulation calls (src/cuda/triangulation.cuh:30-34) */
#define IDL_T_DETECT_MS 0
#define IDL_T_DEDUP_MS 1
#define IDL_T_ASSIGN_MS 2
/* extra slots filled by the incremental calls (src/cuda/delaunay.cuh:8-14) */
#define IDL_T_BFS_MS 3
#define IDL_T_BFS_ITERS 4
#define IDL_T_COUNT 5

typedef struct idl_context idl_context;

/* Message of the last failure on this thread ("" if none). */
IDL_API const char* idl_last_error(void);
/* Library ABI version (major * 10000 + minor * 100 + patch). */
IDL_API int idl_version(void);
/* Number of CUDA kernels this library has launched in this process. */
IDL_API long long idl_launch_count(void);
/* Number of device and pinned host allocations (cudaMalloc, cudaMallocAsync,
 * cudaMallocHost) this library has made in this process. */
IDL_API long long idl_alloc_count(void);

/* Failure detection self-test.  No counterpart in the reference, whose BFS
 * loop has no device-side wait.  Runs the grid-wide barrier of the persistent
 * propagation kernel on its own (one block per SM, four barriers, on the
 * context's stream) with at most `spin_limit` polls per wait (1..2^24), waiting
 * for `missing_arrivals` (0..1024) blocks more than the grid holds.  With 0
 * every barrier completes: IDL_OK.  With more, the arrivals never come, every
 * block's wait runs out, the kernel raises its error flag and returns, and the
 * call reports IDL_ERR_INTERNAL "grid barrier timed out" -- the status the
 * propagation entry points return on a barrier timeout; the context stays
 * usable. */
IDL_API int idl_selftest_grid_barrier(idl_context* ctx, int missing_arrivals, unsigned int spin_limit);

/* ---- context: device, stream, persistent workspace ------------------ */
/* The reference allocates and frees device buffers on every call
 * (src/cuda/voronoi.cu:87-91, todo.txt); a context owns grow-only workspace
 * instead so repeated calls allocate nothing.  device < 0 = current device. */
IDL_API int idl_context_create(int device, idl_context** out);
IDL_API int idl_context_destroy(idl_context* ctx);
/* Order all following work on this cudaStream_t (NULL = legacy default stream). */
IDL_API int idl_context_set_stream(idl_context* ctx, void* stream);
IDL_API int idl_context_synchronize(idl_context* ctx);
/* Bytes of device workspace currently held by the context. */
IDL_API int idl_context_workspace_bytes(idl_context* ctx, int64_t* bytes_out);

/* Propagation schedule from scratch (reference semantics): the first
 * `dense_rounds` tile rounds (one HBM round trip per round of several passes,
 * over every tile that can change; see idl_context_set_tile), the rest in the persistent
 * sparse kernel; 0 = sparse kernel only, < 0 = tile rounds to convergence.
 * A continued propagation (an incremental object's insert using this context)
 * runs in the sparse kernel, or with dense_rounds < 0 as tile rounds starting
 * from the tiles around the new seeds.  Results do not depend on it, only the
 * time does.  Default 3 (the fastest at 4096 x 4096 with 200 000 uniform seeds;
 * integer_delauney_b200.autotune picks per input class).  No counterpart in
 * the reference (its schedule is one full pass per launch). */
IDL_API int idl_context_set_schedule(idl_context* ctx, int dense_rounds);

/* Tile shape of a from-scratch propagation's tile rounds (reference
 * semantics), as an index.  Register tile rounds, one launch per round:
 * 0 = 48 x 48 cells advanced 8 passes per round, 1 = 48 x 112 / 8 passes,
 * 2 = 56 x 56 / 4 passes, 3 = 40 x 104 / 12 passes; 4..7 = the same shapes
 * with all rounds in one cooperative launch separated by a bounded grid
 * barrier; 8..11 = cell-list tile rounds in shared memory, stepping only the
 * cells that can still change: 48 x 48 / 8, 56 x 56 / 4 (default),
 * 112 x 48 / 8, 96 x 96 / 16.  Results do not depend on it, only the time
 * does.  *n_shapes_out (may be NULL) receives the number of shapes; an index
 * outside [0, n) is IDL_ERR_INVALID.  No counterpart in the reference (fixed
 * 16 x 16 blocks, one pass per launch, src/cuda/voronoi.cu:97-98). */
IDL_API int idl_context_set_tile(idl_context* ctx, int shape, int* n_shapes_out);

/* Record per-stage CUDA events on the context's stream for every following
 * triangulation call (off by default; the reference's PhaseTimer,
 * src/cuda/phase_timer.cuh:17-62, plays the same role). */
IDL_API int idl_context_set_profiling(idl_context* ctx, int enable);
/* Stage times (ms, device clock) and work counters of the last profiled run;
 * waits for that run.  out[IDL_PROF_*], n = number of slots to fill. */
#define IDL_PROF_SEEDS_MS 0     /* seed validation + (x, y) ordering */
#define IDL_PROF_PROPAGATE_MS 1 /* stage (a) */
#define IDL_PROF_DETECT_MS 2    /* stage (b): 2x2 detection + hash insert */
#define IDL_PROF_DEDUP_MS 3     /* stage (b): enumeration + canonical ranking */
#define IDL_PROF_ASSIGN_MS 4    /* stage (d) */
#define IDL_PROF_COMPOSE_MS 5   /* (H, W, 3) output assembly */
#define IDL_PROF_ROUNDS 6       /* propagation rounds that had work */
#define IDL_PROF_TILES 7        /* tiles processed over all rounds */
#define IDL_PROF_PASSES 8       /* propagation passes, reference semantics */
#define IDL_PROF_TILE_W 9
#define IDL_PROF_TILE_H 10
#define IDL_PROF_STEPS 11       /* passes fused per tile round */
#define IDL_PROF_CANVAS_PX 12   /* detection canvas pixels */
#define IDL_PROF_IMAGE_PX 13    /* output pixels */
#define IDL_PROF_TRIANGLES 14
#define IDL_PROF_PROP_BYTES 15  /* algorithmic HBM bytes of stage (a): 8 per cell update */
#define IDL_PROF_COUNT 16
IDL_API int idl_context_last_profile(idl_context* ctx, double* out, int n);
/* Trace of the persistent propagation kernel in the last profiled run, one
 * entry per work-list generation: *n_out entries; up to `capacity` of them,
 * each one's duration in ns (GPU global timer) into ns_out, its work-list
 * length in 8 x 8 micro-tiles into tiles_out, and the Jacobi passes it
 * advanced into steps_out (1 for a single pass, a round's passes in the round
 * mode of idl_context_set_tail_rounds, 0 for entering that mode); any of the
 * three may be NULL.  Empty when the run did not use the kernel.  No
 * counterpart in the reference. */
IDL_API int idl_context_pass_trace(idl_context* ctx, int64_t* ns_out, int32_t* tiles_out, int32_t* steps_out,
                                   int capacity, int* n_out);

/* The persistent propagation kernel advances one pass per grid barrier while
 * its work list is long, and several (a round, each micro-tile with a halo
 * as wide as the round's passes) once the list holds at most `max_list`
 * micro-tiles; 0 = never.  Default 4096.  Results do not depend on it, only
 * the time does.  No counterpart in the reference. */
IDL_API int idl_context_set_tail_rounds(idl_context* ctx, int max_list);

/* ---- stage (a): Voronoi().compute ----------------------------------- */
/* Replaces cuda_compute_voronoi (src/cuda/voronoi.cuh:32-35,
 * src/cuda/voronoi.cu:60-117) behind PyVoronoi::compute
 * (src/cuda/bindings/py_voronoi.hpp:9-25).
 * grid_out: host, height*width*2 int32, (seed id, squared distance) per pixel.
 * passes_out (may be NULL): propagation passes including the final pass that
 * changed nothing (0 for IDL_MODE_EXACT). */
IDL_API int idl_voronoi(idl_context* ctx, int width, int height, const int32_t* seeds_xy, int64_t n_seeds,
                int mode, int32_t* grid_out, int64_t* passes_out);

/* ---- stages (a)+(b)+(d): triangulate() / GridTriangulation ----------- */
/* Replaces cuda_compute_triangulation (src/cuda/triangulation.cuh:47-56,
 * src/cuda/triangulation.cu:143-365) behind triangulate()
 * (src/cuda/bindings/triangulate.hpp:15-43) and PyGridTriangulation::compute,
 * compute_timed, compute_debug (src/cuda/bindings/py_grid_triangulation.hpp:10-73).
 *   voronoi_grid     host height*width*2 int32 or NULL; drives detection only
 *                    at border_padding == 0 (triangulation.cu:187-199) and then
 *                    also supplies output channels 0 and 1.
 *   border_padding   IDL_AUTO_BORDER_PADDING or >= 0 pixels.
 *   grid_out         host height*width*3 int32: seed id, squared distance,
 *                    triangle id or -1.
 *   n_triangles_out  number of triangles; fetch them with idl_get_triangles.
 *   timings_out      NULL or float[3] (IDL_T_DETECT_MS..IDL_T_ASSIGN_MS).
 *   padded_grid_out  NULL or host (height+2P)*(width+2P)*2 int32: the
 *                    detection canvas (compute_debug).  Filled only when P > 0,
 *                    as in the reference. */
IDL_API int idl_triangulate(idl_context* ctx, int width, int height, const int32_t* seeds_xy, int64_t n_seeds,
                    const int32_t* voronoi_grid, int border_padding, int mode, int32_t* grid_out,
                    int64_t* n_triangles_out, float* timings_out, int32_t* padded_grid_out);

/* Triangles of the last idl_triangulate / idl_triangulate_device call on this
 * context, 5 int32 each: (x, y, id_a, id_b, id_c), (x, y) the witnessing 2x2
 * block in image coordinates.  Row index = triangle id = rank of the sorted
 * vertex triple (src/cuda/triangulation.cu:254-256,326-327).  Of the blocks
 * witnessing a triangle, the first in row-major order supplies (x, y) and
 * the vertex order. */
IDL_API int idl_get_triangles(idl_context* ctx, int32_t* tris_out, int64_t capacity);

/* The vertex triples (id_a, id_b, id_c) of the same triangles, 3 int32 each
 * in triangle-id order: what triangulate(..., as_arrays=True) returns as its
 * vertex array (src/cuda/bindings/binding_helpers.hpp:61-87), packed on the
 * device so the host receives only these 12 bytes per triangle. */
IDL_API int idl_get_triangle_vertices(idl_context* ctx, int32_t* verts_out, int64_t capacity);

/* Device-resident triangulate: inputs, outputs and all intermediates stay on
 * the device.  d_seeds_xy: device n*2 int32.  d_grid_out: device
 * height*width*3 int32.  If n_triangles_out is non-NULL the call waits for the
 * stream and reports the count; otherwise it returns without synchronising
 * and the count stays on the device (idl_triangles_device). */
IDL_API int idl_triangulate_device(idl_context* ctx, int width, int height, const int32_t* d_seeds_xy, int64_t n_seeds,
                           int border_padding, int mode, int32_t* d_grid_out, int64_t* n_triangles_out);

/* Device view of the last triangulation's triangles (5 int32 each, as
 * idl_get_triangles) and of its triangle count (one int64 on the device).
 * Valid until the next triangulation call on this context. */
IDL_API int idl_triangles_device(idl_context* ctx, const int32_t** d_tris, const int64_t** d_count);

/* ---- Voronoi().compute without any memory allocation ---------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code with a latency budget that a cudaMalloc/cudaFree stall or device
 * synchronisation would break, processes whose device memory is fixed in
 * advance (a per-tenant quota, a pool they must stay inside), and hosts that
 * embed the library under an allocator of their own.  Same result as
 * idl_voronoi, but with device pointers, on `stream` (a cudaStream_t, NULL =
 * legacy default stream) and the current device, and all workspace taken
 * from one static device array of about 9.8 MB, which a GPU holds from the
 * first call on it (when lazy module loading, the CUDA default, loads the
 * array's module there; at context creation under CUDA_MODULE_LOADING=EAGER)
 * until the process exits.  That first call therefore does commit device
 * memory and can fail under an exhausted quota: make it at set-up.
 *   limits   width, height <= 1024 and n_seeds <= 65536 (larger is rejected
 *            with IDL_ERR_INVALID); modes IDL_MODE_REFERENCE, IDL_MODE_NUMPY.
 *   d_seeds_xy  device n_seeds * 2 int32, any order.
 *   d_grid_out  device height * width * 2 int32 (seed id, squared distance).
 * All calls share the one array: calls whose GPU work overlaps race and must
 * not be issued.  The call waits for its stream twice (seed validation,
 * convergence), so it cannot be captured into a CUDA graph, and returns with
 * the output grid written or in flight on `stream`. */
IDL_API int idl_voronoi_noalloc(int width, int height, const int32_t* d_seeds_xy, int64_t n_seeds, int mode,
                                int32_t* d_grid_out, void* stream, int64_t* passes_out);

/* ==== batched triangulation ==============================================
 * No counterpart in the reference, which triangulates one image per call
 * (src/cuda/bindings/triangulate.hpp:15-43).  n_images independent images of
 * any sizes and seed counts run through the pipeline together: one
 * propagation launch, one detection, one raster and one composition launch
 * for the whole batch, and a fixed number of host synchronisations.  Each
 * image's grid and triangles equal idl_triangulate on that image alone, bit
 * for bit.  In IDL_MODE_EXACT the propagation launch is replaced by the
 * separable exact search (three launches over all images, each image kept
 * within its own canvas).  Limits: modes IDL_MODE_REFERENCE and IDL_MODE_EXACT;
 * at most 2097151 seeds in total;
 * the padded canvases must shelf-pack into a 32767 x 32767 atlas (about
 * 10^9 padded pixels), otherwise IDL_ERR_INVALID asks for a smaller batch.
 *   dims         host n_images * 2 int32: (width, height) per image
 *   seed_counts  host n_images int64: seeds per image (each >= 1)
 *   seeds_xy     host (sum of seed_counts) * 2 int32, image after image
 *   grids_out    host (NULL allowed): the images' (height, width, 3) int32
 *                grids, concatenated in image order
 *   tri_counts_out  host n_images int64 (NULL allowed)
 * Validation errors name the image ("image k: ...").  The batch's triangles,
 * image after image with image-local seed ids and triangle ids, are then
 * available from idl_get_triangles (5 int32 each, as for one image). */
IDL_API int idl_triangulate_batch(idl_context* ctx, int n_images, const int32_t* dims, const int64_t* seed_counts,
                                  const int32_t* seeds_xy, int border_padding, int mode, int32_t* grids_out,
                                  int64_t* tri_counts_out, float* timings_out);

/* As idl_triangulate_batch with device seeds (d_seeds_xy) and device output
 * (d_grids_out, concatenated grids); ordered on the context's stream, waits
 * for it once for validation and once for the counts. */
IDL_API int idl_triangulate_batch_device(idl_context* ctx, int n_images, const int32_t* dims,
                                         const int64_t* seed_counts, const int32_t* d_seeds_xy, int border_padding,
                                         int mode, int32_t* d_grids_out, int64_t* tri_counts_out);

/* Stage (a) only for a batch, as idl_triangulate_batch lays it out: the
 * converged labels of every image stay in the context for idl_delaunay_adopt
 * (until the context's next triangulation or batch call).  No counterpart in
 * the reference; a server uses it to propagate many new diagrams in one
 * launch.  Arguments as idl_triangulate_batch; IDL_MODE_REFERENCE only.  Only
 * a batch in IDL_MODE_REFERENCE (this call's, or idl_triangulate_batch's) can
 * be adopted. */
IDL_API int idl_voronoi_batch(idl_context* ctx, int n_images, const int32_t* dims, const int64_t* seed_counts,
                              const int32_t* seeds_xy, int border_padding, int mode);

/* ==== incremental triangulation (stage (c)) ============================
 * An idl_delaunay holds one growing seed set on a padded canvas and keeps its
 * Voronoi diagram, triangles and pixel assignment on the device between
 * calls.  It replaces the reference's class Delaunay (src/cuda/delaunay.cuh,
 * bound as _delauney_cuda.Delaunay in src/cuda/bindings/py_delaunay.hpp).
 *
 * Seed ids.  Internally seeds are numbered in insertion order (0, 1, ...).
 * Outputs that the reference reports in batch numbering -- the triangle map
 * and grid of finalise, the Voronoi grid, finalise_device's views -- use the
 * (x asc, y asc) rank of each seed instead, exactly as the reference
 * translates through sorted_rank (src/cuda/delaunay_output.cu:39-110);
 * get_triangles / get_edges / get_seeds keep insertion ids, as there.
 *
 * Propagation.  IDL_MODE_REFERENCE continues the Jacobi iteration from the
 * previous fixed point after writing the new seeds, the reference's own
 * incremental trajectory (src/cuda/delaunay_voronoi.cu:12-108), ties going to
 * the higher insertion id.  IDL_MODE_EXACT recomputes the exact diagram of
 * the whole seed set (ties to the higher (x, y) rank) and detects on rank
 * labels, so after every insert the object equals idl_triangulate of all its
 * seeds in exact mode, bit for bit, whatever the insertion history.
 *
 * Triangles.  Detection runs on the insertion-id grid (the block rule's
 * lowest-id tie-break sees insertion ids, as in the reference) and triangles
 * are numbered canonically: triangle id = rank of the sorted triple of batch
 * ids, so ids are dense, deterministic and equal to the batch pipeline's.
 * (The reference numbers by registry slot order, src/cuda/delaunay_topology.cu:
 * 360-414, which depends on the insertion history.)  Pixels take the highest
 * id of the triangles containing them, over the whole triangle set. */
typedef struct idl_delaunay idl_delaunay;

/* Per-object info slots (idl_delaunay_info). */
#define IDL_DI_SEED_COUNT 0
#define IDL_DI_WIDTH 1
#define IDL_DI_HEIGHT 2
#define IDL_DI_BORDER_PADDING 3
#define IDL_DI_HAS_PENDING 4
#define IDL_DI_GENERATION 5
#define IDL_DI_MAX_SEEDS 6
#define IDL_DI_MODE 7
#define IDL_DI_HAS_VALUES 8
#define IDL_DI_DEVICE_BYTES 9 /* device memory the object holds, workspace included */
#define IDL_DI_COUNT 10

/* Delaunay::Delaunay (src/cuda/delaunay.cu:24-112).  Allocates every canvas-
 * sized buffer up front; border_padding < 0 selects IDL_DEFAULT_BORDER_PADDING.
 * Errors: width, height or max_seeds <= 0 -> IDL_ERR_INVALID ("dimensions and
 * max_seeds must be positive"); an allocation failure -> IDL_ERR_CUDA naming
 * cudaMalloc and this library's delaunay.cu. */
IDL_API int idl_delaunay_create(int device, int width, int height, int64_t max_seeds, int border_padding, int mode,
                                idl_delaunay** out);
IDL_API int idl_delaunay_destroy(idl_delaunay* d);
/* Empty the object and lay its existing allocations out for another canvas
 * (no allocation, no free).  No counterpart in the reference, whose objects
 * are sized once at construction: this lets a server recycle resident
 * diagrams.  IDL_ERR_INVALID if the canvas, padding or seed capacity needs
 * more memory than the object was created with. */
IDL_API int idl_delaunay_reset(idl_delaunay* d, int width, int height, int64_t max_seeds, int border_padding);
/* Order the object's work on `stream` (a cudaStream_t; NULL = legacy default). */
IDL_API int idl_delaunay_set_stream(idl_delaunay* d, void* stream);

/* Take scratch memory (hash table, work lists, triangle rows, ...) from the
 * context `ws` instead of the object's own, or go back to its own with NULL.
 * No counterpart in the reference.  Many resident objects can then share the
 * scratch of a few contexts -- one per stream a server runs -- so an object
 * holds only its persistent state.  Objects sharing a context must not run
 * at the same time.  ws must be on the object's device. */
IDL_API int idl_delaunay_set_workspace(idl_delaunay* d, idl_context* ws);

/* Delaunay::insert_deferred (src/cuda/delaunay.cu:276-323 with apply_batch_,
 * :184-268): validate and append k seeds (host int32 x, y pairs), write them
 * into the diagram and propagate.  values: NULL or k host floats, the scalar
 * field at the new seeds.  timings_out: NULL or IDL_T_COUNT floats; when
 * given, topology is also brought up to date inside the call so that
 * IDL_T_DETECT_MS / IDL_T_DEDUP_MS describe this insert.  k == 0 is a no-op.
 * Errors (nothing is changed): capacity, bounds and duplicate violations ->
 * IDL_ERR_INVALID with the reference's messages. */
IDL_API int idl_delaunay_insert(idl_delaunay* d, const int32_t* seeds_xy, int64_t k, const float* values,
                                float* timings_out);

/* As idl_delaunay_insert; with order = 1 the batch's seeds (and values) take
 * their ids in (x asc, y asc) order instead of the order given, which into an
 * empty object reproduces the batch pipeline's numbering (and so its result,
 * bit for bit) without a host-side sort.  No counterpart in the reference. */
IDL_API int idl_delaunay_insert_ordered(idl_delaunay* d, const int32_t* seeds_xy, int64_t k, const float* values,
                                        int order, float* timings_out);

/* Make an empty object (fresh or reset, same width, height and padding) hold
 * image `image` of the last idl_voronoi_batch or idl_triangulate_batch[_device]
 * on `src`: its converged labels
 * and its seeds, numbered in (x, y) order -- the state idl_delaunay_insert_
 * ordered(order = 1) of the same seeds would reach, bit for bit, without a
 * propagation of its own.  No counterpart in the reference.  Waits for the
 * copy; src may then run its next batch. */
IDL_API int idl_delaunay_adopt(idl_delaunay* d, idl_context* src, int image);

/* idl_delaunay_adopt for a group of n (1..16) distinct empty objects at once:
 * objs[k] adopts image images[k] of the last batch on `src`.  One launch
 * copies every image's labels and seeds, one host copy fills the host mirrors,
 * and the call waits for its stream once, instead of once per object.  All
 * objects must share one stream and device.  Each object ends in the state
 * idl_delaunay_adopt would leave it in.  No counterpart in the reference. */
IDL_API int idl_delaunay_adopt_group(idl_delaunay* const* objs, const int* images, int n, idl_context* src);

/* Delaunay::finalise (src/cuda/delaunay.cu:325-347): assign pixels for the
 * pending changes and write the (height, width, 3) int32 grid (batch seed id,
 * squared distance, triangle id) to host grid_out (may be NULL).  Reports the
 * triangle count; idl_delaunay_triangles returns the map.  timings_out: NULL or
 * IDL_T_COUNT floats (detect/dedup/assign of the work this call did). */
IDL_API int idl_delaunay_finalise(idl_delaunay* d, int32_t* grid_out, int64_t* n_triangles_out, float* timings_out);

/* Delaunay::finalise_device (src/cuda/delaunay.cu:349-361 and
 * crop_pixel_arrays_kernel, src/cuda/delaunay_output.cu:120-144): as finalise,
 * but the per-pixel results stay on the device, as three object-owned arrays
 * of width*height entries: triangle id (no triangle -> 0), batch seed id, and
 * a uint8 mask, 1 where no triangle contains the pixel.  They stay valid until
 * *generation_out changes (any insert, finalise or finalise_device call). */
IDL_API int idl_delaunay_finalise_device(idl_delaunay* d, int64_t* n_triangles_out, const int32_t** d_pixel_tids,
                                         const int32_t** d_pixel_seed_ids, const uint8_t** d_outside_mask,
                                         uint64_t* generation_out);

/* Triangles of the current topology, in triangle-id order.
 *   ids = 0: 5 int32 per triangle (x, y, a, b, c) in batch seed ids, (x, y)
 *            the witnessing block in image coordinates -- finalise's map
 *            (Delaunay::build_tri_map_, src/cuda/delaunay_output.cu:68-84);
 *   ids = 1: 3 int32 per triangle (a, b, c) in insertion ids --
 *            Delaunay::get_triangles (src/cuda/delaunay_output.cu:186-200);
 *   ids = 2: 3 int32 per triangle (a, b, c) in batch seed ids, the vertex
 *            columns of ids = 0 packed on the device: finalise's as_arrays
 *            vertex array without the rows' other columns crossing PCIe.
 * Valid between deferred inserts.  *n_out = triangle count; tris_out may be
 * NULL to query the count; otherwise capacity (int32 entries) must hold it. */
IDL_API int idl_delaunay_triangles(idl_delaunay* d, int ids, int32_t* tris_out, int64_t capacity, int64_t* n_out);

/* Delaunay::get_edges (src/cuda/delaunay_scalar_field.cu:293-312): distinct
 * undirected edges (a, b), a < b, insertion ids, ascending by (a, b). */
IDL_API int idl_delaunay_edges(idl_delaunay* d, int32_t* edges_out, int64_t capacity, int64_t* n_out);

/* Delaunay::edge_scores (src/cuda/delaunay_scalar_field.cu:206-224): per
 * edge of idl_delaunay_edges, |v[a] - v[b]| * |p[a] - p[b]| computed in
 * double and rounded to float, 0 for edges shorter than min_length.
 * IDL_ERR_STATE when no values were ever inserted (and edges exist). */
IDL_API int idl_delaunay_edge_scores(idl_delaunay* d, double min_length, float* scores_out, int64_t capacity,
                                     int64_t* n_out);

/* Delaunay::select_midpoints (src/cuda/delaunay_scalar_field.cu:226-291):
 * midpoints (x, y) of the `count` best edges under (score desc, edge index
 * asc) among those scoring above threshold, dropping midpoints on existing
 * seeds and collisions (lowest rank kept), ascending by padded pixel index. */
IDL_API int idl_delaunay_select_midpoints(idl_delaunay* d, double min_length, int count, float threshold,
                                          int32_t* xy_out, int64_t capacity, int64_t* n_out);

/* Delaunay::locate (src/cuda/delaunay_query.cu:187-227): triangle id
 * containing each of n query points (x, y int32 pairs, image coordinates), or
 * -1.  Valid before any finalise; agrees with the finalised grid. */
IDL_API int idl_delaunay_locate(idl_delaunay* d, const int32_t* pts_xy, int64_t n, int32_t* tids_out);

/* Delaunay::in_circumsphere (src/cuda/delaunay_query.cu:33-185): for each
 * query, whether (x, y, t) lies strictly inside the circumsphere of the
 * triangle containing (x, y) lifted to t = 0 (uint8 0/1), and that triangle. */
IDL_API int idl_delaunay_in_circumsphere(idl_delaunay* d, const int32_t* pts_xy, const double* t, int64_t n,
                                         uint8_t* mask_out, int32_t* tids_out);

/* Delaunay::get_seeds / get_values (src/cuda/delaunay_output.cu:202-224):
 * insertion-order seeds (seed_count x, y pairs) and the values inserted
 * with them (as many floats as were given; *n_values_out). */
IDL_API int idl_delaunay_seeds(idl_delaunay* d, int32_t* xy_out, float* values_out, int64_t* n_values_out);

/* Delaunay::sorted_rank (src/cuda/delaunay.cuh:245-247): insertion id ->
 * batch (x asc, y asc) id, seed_count int32. */
IDL_API int idl_delaunay_sorted_rank(idl_delaunay* d, int32_t* rank_out);

/* Delaunay::get_voronoi_grid (src/cuda/delaunay_output.cu:162-184): the
 * (height, width, 2) int32 grid (batch seed id, squared distance); -1, -1
 * where no seed has reached. */
IDL_API int idl_delaunay_voronoi(idl_delaunay* d, int32_t* grid_out);

/* Object properties (IDL_DI_* slots; src/cuda/delaunay.cuh:249-254). */
IDL_API int idl_delaunay_info(idl_delaunay* d, int64_t* info_out, int count);

/* ---- Serving: a native request loop over resident diagrams ----------
 * No counterpart in the reference (one caller, one image per call).  A server
 * keeps incremental objects resident on one device and runs two kinds of
 * request from any number of client threads:
 *   new    -- triangulate W x H (1..4096 each) from a seed set, in (x, y)
 *             order, and keep the diagram: its grid and triangles equal
 *             idl_triangulate of the same input bit for bit;
 *   insert -- add seeds to a resident diagram (idl_delaunay_insert order);
 * on `slots` worker threads, each with its own stream and scratch.  Queued
 * new diagrams are propagated together, several per launch
 * (idl_voronoi_batch + idl_delaunay_adopt).  Requests whose diagram is busy
 * or whose memory does not fit yet are passed over, not waited on.  Every
 * resident diagram, pooled object and slot workspace is charged to
 * budget_bytes; the least recently used idle diagram is retired into a reuse
 * pool (idl_delaunay_reset) when memory runs short.  A request whose
 * footprint can never fit fails with IDL_ERR_BUDGET.  A diagram's requests
 * run in submission order, one at a time, so results do not depend on the
 * mix.  Timestamps are nanoseconds of idl_server_clock_ns (CLOCK_MONOTONIC). */
typedef struct idl_server idl_server;

#define IDL_SR_STATUS 0      /* the request's status (also returned by idl_server_wait) */
#define IDL_SR_KIND 1        /* 0 new, 1 insert */
#define IDL_SR_DIAGRAM 2
#define IDL_SR_SEEDS 3       /* the diagram's seed count after the request */
#define IDL_SR_TRIANGLES 4
#define IDL_SR_ARRIVAL_NS 5
#define IDL_SR_START_NS 6
#define IDL_SR_DONE_NS 7
#define IDL_SR_COUNT 8

#define IDL_SI_USED_BYTES 0
#define IDL_SI_BUDGET_BYTES 1
#define IDL_SI_RESIDENT 2
#define IDL_SI_POOLED 3
#define IDL_SI_QUEUED 4
#define IDL_SI_GROUPS 5          /* grouped propagation launches */
#define IDL_SI_GROUPED 6         /* new diagrams they served */
#define IDL_SI_NEW_OBJECTS 7
#define IDL_SI_REUSED_OBJECTS 8
#define IDL_SI_EVICTED 9
#define IDL_SI_FREED_OBJECTS 10
#define IDL_SI_COUNT 11

IDL_API int64_t idl_server_clock_ns(void);
/* device < 0: the current device.  mode: IDL_MODE_REFERENCE (grouped
 * propagation) or IDL_MODE_EXACT.  Errors: slots outside [1, 64], budget <= 0,
 * another mode -> IDL_ERR_INVALID. */
IDL_API int idl_server_create(int device, int64_t budget_bytes, int slots, int border_padding, int mode,
                              idl_server** out);
/* Propagation schedules (idl_context_set_schedule) of every slot: of the
 * grouped new diagrams (group_rounds, default 1) and of inserts (insert_rounds,
 * default -1: tile rounds from the new seeds' tiles, plain launches that
 * overlap other slots' work; 0 or more: the device-wide persistent kernel).
 * Before the first request; IDL_ERR_STATE after it. */
IDL_API int idl_server_set_schedule(idl_server* s, int group_rounds, int insert_rounds);
/* Tile shape (idl_context_set_tile) of every slot's grouped propagation of new
 * diagrams; shapes that run as one cooperative launch run as separate
 * launches here, so that workers overlap.  Set before the first request. */
IDL_API int idl_server_set_tile(idl_server* s, int shape);
/* Runs what is queued, stops the workers and frees every object. */
IDL_API int idl_server_destroy(idl_server* s);
/* Queue a new diagram (seeds copied; n <= 200000).  fetch != 0: grid_out
 * (H x W x 3 int32, host) receives the finalised grid and the triangles are
 * kept for idl_server_wait; it must stay valid until then.  arrival_ns <= 0:
 * now.  *diagram_out can take inserts at once. */
IDL_API int idl_server_submit_new(idl_server* s, int width, int height, const int32_t* seeds_xy, int64_t n,
                                  int fetch, int32_t* grid_out, int64_t arrival_ns, int64_t* request_out,
                                  int64_t* diagram_out);
/* Queue an insert; IDL_ERR_NOT_RESIDENT if the diagram is not resident. */
IDL_API int idl_server_submit_insert(idl_server* s, int64_t diagram, const int32_t* seeds_xy, int64_t n, int fetch,
                                     int32_t* grid_out, int64_t arrival_ns, int64_t* request_out);
/* Wait for a request (timeout_s < 0: without limit) and collect it: its
 * result row (IDL_SR_COUNT int64) and, for a fetched request, its triangles
 * (5 int32 each, as idl_delaunay_triangles ids = 0) if tris_out is given --
 * capacity too small -> IDL_ERR_INVALID and the request stays uncollected.
 * Returns the request's own status; collecting twice -> IDL_ERR_INVALID. */
IDL_API int idl_server_wait(idl_server* s, int64_t request, double timeout_s, int64_t* result_out,
                            int32_t* tris_out, int64_t capacity);
/* Wait until every queued request has run. */
IDL_API int idl_server_drain(idl_server* s);
/* Retire an idle diagram now, keeping its object for reuse. */
IDL_API int idl_server_recycle(idl_server* s, int64_t diagram, int* recycled_out);
IDL_API int idl_server_info(idl_server* s, int64_t* info_out, int count);
/* Ids of resident diagrams (and of those whose creation is queued). */
IDL_API int idl_server_resident(idl_server* s, int64_t* ids_out, int64_t capacity, int64_t* n_out);

#ifdef __cplusplus
}
#endif

#endif /* IDELAUNAY_H */
