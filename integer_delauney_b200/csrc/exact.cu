// Stage (a), exact semantics (IDL_MODE_EXACT): every cell takes the nearest
// seed in squared L2 distance, ties to the higher seed id -- the contract the
// reference's two implementations approximate (src/delauney/reference/
// voronoi.py:9-31; its NumPy sweep meets it on every probe, its CUDA Jacobi
// iteration misses a few "orphan" cells).  The result depends only on the
// seed set, not on any propagation history.
//
// Separable and exact, in two data-parallel phases over the canvas:
//   1. column phase: each cell finds the nearest seed in its own column
//      (a walk down the column's run of the (x, y)-sorted seeds; a tie
//      between the seed above and the one below goes to the lower one, whose
//      y -- and so id -- is larger);
//   2. row phase: each cell takes the best (distance, id) over its row's
//      column candidates.  Canvases up to HULL_MAX_W columns wide use the
//      lower-hull pass of row_hull.cuh, O(W) per row whatever the seed
//      layout; wider ones scan the columns outward, k = 0, 1, 2, ..., until
//      k^2 exceeds the best distance (no column further out can beat or tie
//      it), jumping over 32-column blocks whose nearest candidate is too far.
// Completeness: the nearest seed s* of a cell lies in some column x*, whose
// column candidate is at least as near (and, if as near, is the higher-id
// one of the two equidistant seeds in that column); two candidates from
// different columns at equal distance are ordered by column, i.e. by id.
// Seed ids are (x asc, y asc) ranks, so "higher id" is a comparison of ids.
#include "context.cuh"
#include "row_hull.cuh"

#include <atomic>

namespace idl {
namespace {

// cs[c] = first sorted seed with canvas x >= c, for c in [0, Wd].
__global__ void k_col_start(const uint32_t* __restrict__ pos, int64_t n, int Wd, int32_t* __restrict__ cs)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > Wd) return;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int)pos_x(__ldg(&pos[mid])) < c) lo = mid + 1;
        else hi = mid;
    }
    cs[c] = (int32_t)lo;
}

// Phase 1: nearest seed of each cell within its column (or UNDEF), and its
// row distance |dy| (so the row phase reads distances instead of gathering
// seed positions).  One thread walks one column through a band of CHUNK rows,
// advancing through the column's seeds as the row advances (one binary search
// per band), so a warp of adjacent columns writes each row coalesced.  The
// warp also reduces, per row, the smallest dy^2 over its 32 columns into
// rmin[y][x / 32] (INT_MAX where none of them has a seed) for the row phase.
constexpr int CHUNK = 64;
constexpr int RB = 32;   // columns per row block of the row phase

__global__ void k_col_nearest(const uint32_t* __restrict__ pos, const int32_t* __restrict__ cs, int Wd, int Hd,
                              int pitch, int32_t* __restrict__ col, int32_t* __restrict__ coldy,
                              int32_t* __restrict__ rmin, int nb)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int y0 = blockIdx.y * CHUNK, y1 = min(Hd, y0 + CHUNK);
    const bool in = x < Wd;
    const int32_t lo = in ? __ldg(&cs[x]) : 0, hi = in ? __ldg(&cs[x + 1]) : 0;
    int32_t a = lo, b = hi;   // first seed of the column with y >= y0
    while (a < b) {
        const int32_t m = (a + b) >> 1;
        if ((int)pos_y(__ldg(&pos[m])) < y0) a = m + 1;
        else b = m;
    }
    int next_y = a < hi ? (int)pos_y(__ldg(&pos[a])) : 0x7FFFFFFF;     // seed at or below
    int prev_y = a > lo ? (int)pos_y(__ldg(&pos[a - 1])) : -0x3FFFFFFF; // seed above
    for (int y = y0; y < y1; ++y) {
        int32_t v = 0x7FFFFFFF;
        if (in) {
            if (lo == hi) {
                col[(size_t)y * pitch + x] = UNDEF;
                coldy[(size_t)y * pitch + x] = 0;
            } else {
                while (next_y < y) {   // the seed below was passed: it becomes the one above
                    prev_y = next_y;
                    ++a;
                    next_y = a < hi ? (int)pos_y(__ldg(&pos[a])) : 0x7FFFFFFF;
                }
                const int below = next_y - y, above = y - prev_y;   // tie: the larger y, the higher id
                const bool take_below = a < hi && (a == lo || below <= above);
                const int dy = take_below ? below : above;
                col[(size_t)y * pitch + x] = take_below ? a : a - 1;
                coldy[(size_t)y * pitch + x] = dy;
                v = dy * dy;
            }
        }
        if (rmin) {   // uniform: only the outward-scan row phase reads it
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
            if (lane == 0 && x < Wd) rmin[(size_t)y * nb + x / RB] = v;
        }
    }
}

// Phase 2: best column candidate of the row, scanning outward from each cell.
// When the scan reaches a block's nearest column at distance k, every
// candidate of the block costs at least k^2 + rmin[y][block]; if that exceeds
// the best distance so far, nothing in the block can beat or tie it and the
// scan jumps over it.  Cells far from every seed (clustered inputs) thus test
// blocks instead of columns; the scan still stops once k^2 exceeds the best
// distance.
__device__ __forceinline__ void scan_side(const int32_t* __restrict__ row, const int32_t* __restrict__ rdy,
                                          const int32_t* __restrict__ bmin, int x, int Wd, int dir, int32_t& bl,
                                          long long& bd)
{
    int k = 1;
    for (;;) {
        const int xx = x + dir * k;
        if (xx < 0 || xx >= Wd) return;
        const long long kk = (long long)k * k;
        if (kk > bd) return;
        const bool entering = dir > 0 ? (xx % RB) == 0 : (xx % RB) == RB - 1;
        if (entering && kk + __ldg(&bmin[xx / RB]) > bd) {
            k += RB;
            continue;
        }
        const int32_t l = row[xx];
        if (l >= 0) {
            const long long dy = rdy[xx];
            const long long d = kk + dy * dy;
            if (d < bd || (d == bd && l > bl)) {
                bd = d;
                bl = l;
            }
        }
        ++k;
    }
}

__global__ void k_row_nearest(const int32_t* __restrict__ col, const int32_t* __restrict__ coldy,
                              const int32_t* __restrict__ rmin, int nb, int Wd, int pitch, int32_t* __restrict__ lab)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= Wd) return;
    const int32_t* row = col + (size_t)y * pitch;
    const int32_t* rdy = coldy + (size_t)y * pitch;
    const int32_t* bmin = rmin + (size_t)y * nb;
    int32_t bl = row[x];
    long long bd = 0x7FFFFFFFFFFFFFFFll;
    if (bl >= 0) {
        const long long dy = rdy[x];
        bd = dy * dy;
    }
    scan_side(row, rdy, bmin, x, Wd, -1, bl, bd);
    scan_side(row, rdy, bmin, x, Wd, +1, bl, bd);
    lab[(size_t)y * pitch + x] = bl;
}

// Phase 2: the lower-hull row pass (row_hull.cuh), one block per row.
__global__ void __launch_bounds__(HULL_THREADS)
k_row_hull(const int32_t* __restrict__ col, const int32_t* __restrict__ coldy, int Wd, int pitch,
           int32_t* __restrict__ lab)
{
    const size_t o = (size_t)blockIdx.x * pitch;
    row_hull(col + o, coldy + o, Wd, lab + o);
}

}  // namespace

void propagate_exact(Context& C, const Canvas& cv, const uint32_t* pos, int64_t n)
{
    const size_t plane = (size_t)cv.pitch * cv.Hd * 4;
    C.lab[0].ensure(plane);
    C.lab[1].ensure(plane);
    C.counts.ensure(((size_t)cv.Wd + 1) * 4);
    int32_t* cs = C.counts.as<int32_t>();
    k_col_start<<<(unsigned)((cv.Wd + 1 + 255) / 256), 256, 0, C.stream>>>(pos, n, cv.Wd, cs);
    IDL_LAUNCH();
    C.exact_dy.ensure(plane);
    const dim3 gc((unsigned)ceil_div(cv.Wd, 128), (unsigned)ceil_div(cv.Hd, CHUNK));
    const bool hull = cv.Wd <= HULL_MAX_W;
    const int nb = ceil_div(cv.Wd, RB);
    int32_t* rmin = nullptr;
    if (!hull) {
        C.exact_rmin.ensure((size_t)nb * cv.Hd * 4);
        rmin = C.exact_rmin.as<int32_t>();
    }
    k_col_nearest<<<gc, 128, 0, C.stream>>>(pos, cs, cv.Wd, cv.Hd, cv.pitch, C.lab[1].as<int32_t>(),
                                            C.exact_dy.as<int32_t>(), rmin, nb);
    IDL_LAUNCH();
    if (hull) {
        // lower-hull row pass: O(W) per row
        const size_t smem = row_hull_smem(cv.Wd);
        static std::atomic<uint64_t> opted{0};   // the shared-memory opt-in is per device
        const uint64_t bit = 1ull << (C.device & 63);
        if (!(opted.load(std::memory_order_acquire) & bit)) {
            IDL_CUDA(cudaFuncSetAttribute((const void*)k_row_hull, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)row_hull_smem(HULL_MAX_W)));
            opted.fetch_or(bit, std::memory_order_acq_rel);
        }
        k_row_hull<<<(unsigned)cv.Hd, HULL_THREADS, smem, C.stream>>>(
            C.lab[1].as<int32_t>(), C.exact_dy.as<int32_t>(), cv.Wd, cv.pitch, C.lab[0].as<int32_t>());
    } else {
        // wider canvases: the outward scan
        const dim3 g((unsigned)ceil_div(cv.Wd, 256), (unsigned)cv.Hd);
        k_row_nearest<<<g, 256, 0, C.stream>>>(C.lab[1].as<int32_t>(), C.exact_dy.as<int32_t>(), rmin, nb, cv.Wd,
                                               cv.pitch, C.lab[0].as<int32_t>());
    }
    IDL_LAUNCH();
    if (C.prof.enabled) {
        C.prof.passes = 0;
        C.prof.rounds = 2;
        C.prof.tiles = 0;
        C.prof.prop_bytes = (double)cv.Wd * cv.Hd * 20.0;   // column labels and distances out and in, labels out
        C.prof.tile_w = C.prof.tile_h = 0;
        C.prof.steps_per_round = 0;
    }
}

}  // namespace idl
