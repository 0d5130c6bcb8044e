// Stage (a), exact semantics (IDL_MODE_EXACT): every cell takes the nearest
// seed in squared L2 distance, ties to the higher seed id -- the contract the
// reference's two implementations approximate (src/delauney/reference/
// voronoi.py:9-31; its NumPy sweep meets it on every probe, its CUDA Jacobi
// iteration misses a few "orphan" cells).  The result depends only on the
// seed set, not on any propagation history.
//
// Separable and exact, in two data-parallel phases over the canvas:
//   1. column phase: each cell finds the nearest seed in its own column
//      (binary search in the column's run of the (x, y)-sorted seeds; a tie
//      between the seed above and the one below goes to the lower one, whose
//      y -- and so id -- is larger);
//   2. row phase: each cell scans the columns outward, k = 0, 1, 2, ..., taking
//      the best (distance, id) over the column candidates, and stops once k^2
//      exceeds its best distance: no column further out can beat or tie it.
// Completeness: the nearest seed s* of a cell lies in some column x*, whose
// column candidate is at least as near (and, if as near, is the higher-id
// one of the two equidistant seeds in that column); two candidates from
// different columns at equal distance are ordered by column, i.e. by id.
// Seed ids are (x asc, y asc) ranks, so "higher id" is a comparison of ids.
//
// Work is O(cells x distance to the nearest seed / 1 px) in the row phase:
// dense seed sets (a few px apart) finish in a handful of column reads per
// cell; cells in large empty regions scan further.
#include "context.cuh"

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

// Phase 1: nearest seed of each cell within its column (or UNDEF).
__global__ void k_col_nearest(const uint32_t* __restrict__ pos, const int32_t* __restrict__ cs, int Wd, int Hd,
                              int pitch, int32_t* __restrict__ col)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= Wd) return;
    const int32_t lo = __ldg(&cs[x]), hi = __ldg(&cs[x + 1]);
    int32_t best = UNDEF;
    if (lo < hi) {
        int32_t a = lo, b = hi;   // first seed of the column with y >= this row
        while (a < b) {
            const int32_t m = (a + b) >> 1;
            if ((int)pos_y(__ldg(&pos[m])) < y) a = m + 1;
            else b = m;
        }
        if (a == hi) best = hi - 1;
        else if (a == lo) best = lo;
        else {
            const int below = (int)pos_y(__ldg(&pos[a])) - y, above = y - (int)pos_y(__ldg(&pos[a - 1]));
            best = below <= above ? a : a - 1;   // tie: the larger y, the higher id
        }
    }
    col[(size_t)y * pitch + x] = best;
}

// Phase 2: best column candidate of the row, scanning outward.
__global__ void k_row_nearest(const int32_t* __restrict__ col, const uint32_t* __restrict__ pos, int Wd, int Hd,
                              int pitch, int32_t* __restrict__ lab)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= Wd) return;
    const int32_t* row = col + (size_t)y * pitch;
    int32_t bl = row[x];
    long long bd = 0x7FFFFFFFFFFFFFFFll;
    if (bl >= 0) {
        const int dy = y - (int)pos_y(__ldg(&pos[bl]));
        bd = (long long)dy * dy;
    }
    for (int k = 1;; ++k) {
        const long long kk = (long long)k * k;
        if (kk > bd || (x - k < 0 && x + k >= Wd)) break;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int xx = side ? x + k : x - k;
            if (xx < 0 || xx >= Wd) continue;
            const int32_t l = row[xx];
            if (l < 0) continue;
            const int dy = y - (int)pos_y(__ldg(&pos[l]));
            const long long d = kk + (long long)dy * dy;
            if (d < bd || (d == bd && l > bl)) {
                bd = d;
                bl = l;
            }
        }
    }
    lab[(size_t)y * pitch + x] = bl;
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
    const dim3 g((unsigned)ceil_div(cv.Wd, 256), (unsigned)cv.Hd);
    k_col_nearest<<<g, 256, 0, C.stream>>>(pos, cs, cv.Wd, cv.Hd, cv.pitch, C.lab[1].as<int32_t>());
    IDL_LAUNCH();
    k_row_nearest<<<g, 256, 0, C.stream>>>(C.lab[1].as<int32_t>(), pos, cv.Wd, cv.Hd, cv.pitch,
                                           C.lab[0].as<int32_t>());
    IDL_LAUNCH();
    if (C.prof.enabled) {
        C.prof.passes = 0;
        C.prof.rounds = 2;
        C.prof.tiles = 0;
        C.prof.prop_bytes = (double)cv.Wd * cv.Hd * 12.0;   // column labels out, in, final labels out
        C.prof.tile_w = C.prof.tile_h = 0;
        C.prof.steps_per_round = 0;
    }
}

}  // namespace idl
