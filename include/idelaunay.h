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
#define IDL_PROF_COUNT 15
IDL_API int idl_context_last_profile(idl_context* ctx, double* out, int n);

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
 * from one static device array of about 9.8 MB that every GPU loading the
 * library reserves until the process exits.
 *   limits   width, height <= 1024 and n_seeds <= 65536 (larger is rejected
 *            with IDL_ERR_INVALID); modes IDL_MODE_REFERENCE, IDL_MODE_NUMPY.
 *   d_seeds_xy  device n_seeds * 2 int32, any order.
 *   d_grid_out  device height * width * 2 int32 (seed id, squared distance).
 * The first call on a device looks up the array's device address and should
 * therefore come before any stream capture starts.  All calls share the one
 * array: calls whose GPU work overlaps race and must not be issued.  The call
 * waits for its stream twice (seed validation, convergence) and returns with
 * the output grid written or in flight on `stream`. */
IDL_API int idl_voronoi_noalloc(int width, int height, const int32_t* d_seeds_xy, int64_t n_seeds, int mode,
                                int32_t* d_grid_out, void* stream, int64_t* passes_out);

#ifdef __cplusplus
}
#endif

#endif /* IDELAUNAY_H */
