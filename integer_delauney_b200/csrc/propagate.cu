// Stage (a): Voronoi propagation on the detection canvas.
//
// Two update rules, each reproducing one reference implementation bit for bit:
//
//   IDL_MODE_REFERENCE  one synchronous Jacobi step per pass: every cell takes
//                       the best (d, id) among itself and its 4 neighbours'
//                       owners, lower squared distance first, higher id on a
//                       tie, distance recomputed from the owner seed
//                       (src/cuda/voronoi.cu:32-53, geometry_device.cuh:22-66).
//   IDL_MODE_NUMPY      one iteration = four directional sub-steps (left,
//                       right, up, down neighbour), each synchronous, adopting
//                       the neighbour's owner where the cell is undefined,
//                       strictly closer, or tied with a higher id
//                       (src/delauney/reference/voronoi.py:90-163).
//
// Both run until a pass (iteration) changes nothing.  The reference does one
// kernel launch, one flag round trip and one full-canvas HBM pass per step
// (voronoi.cu:100-113).  Here the canvas is cut into TW x TH tiles; a CTA
// loads one tile plus a K-cell halo into shared memory and advances it K
// steps there.  A cell's value after K steps depends only on cells within K of
// it (the light cone of a 5-point / directional stencil), so the inner tile is
// exact after K steps and one HBM round trip carries K passes.
//
// Only tiles that can still change are processed: keys only ever improve, so
// a cell whose closed neighbourhood did not change in a step cannot change in
// the next.  A tile is therefore re-run in round r+1 only if it or one of its
// 8 neighbours changed in round r (the halo of radius K <= tile size reaches
// no further).  Active tiles form a device-side work list built by the round
// kernel itself; the host only checks, every few rounds, whether it emptied.
//
// Both label planes hold the same state at the start; a round reads plane
// r%2 and writes plane (r+1)%2.  A tile processed in round r and unchanged
// wrote its unchanged state to the other plane; a tile that changed is
// processed again in round r+1.  By induction every tile not being processed
// holds the same state in both planes, so reads of the frozen neighbours of an
// active tile are always current, and at convergence the planes agree.
#include "context.cuh"
#include "gridsync.cuh"
#include "stencil.cuh"

#include <atomic>
#include <vector>

namespace idl {
namespace {

// CTA geometry: a 64 x 64 region = the 48 x 48 tile plus an 8-cell halo.
// 8 warps own 8 rows each; lane l owns columns 2l and 2l+1 of its warp's rows,
// so each thread keeps 16 cells (label and squared distance) in registers.
// Horizontal neighbours come from the adjacent lane by shuffle, vertical ones
// from the thread's own registers, and only each warp's top and bottom rows go
// through shared memory to the warps above and below.
constexpr int RW = 64, RH = 64, KSTEPS = 8;
constexpr int TW = RW - 2 * KSTEPS, TH = RH - 2 * KSTEPS;   // 48 x 48 inner tile
constexpr int WARPS = 8, ROWS = RH / WARPS;
constexpr int THREADS = WARPS * 32;
static_assert(ROWS * 2 <= 32, "cell mask must fit 32 bits");

struct Edges {
    int32_t lab[2][WARPS][2][RW];   // [parity][warp][0 = top row, 1 = bottom row][column]
    uint32_t chg[2][WARPS][2][2];   // [parity][warp][top/bottom][column 0/1 of each lane]: lane ballots
};

__device__ __forceinline__ void publish(Edges& E, int par, int warp, int lane, const int32_t (&L)[ROWS][2],
                                        uint32_t chg)
{
    E.lab[par][warp][0][2 * lane] = L[0][0];
    E.lab[par][warp][0][2 * lane + 1] = L[0][1];
    E.lab[par][warp][1][2 * lane] = L[ROWS - 1][0];
    E.lab[par][warp][1][2 * lane + 1] = L[ROWS - 1][1];
    const uint32_t t0 = __ballot_sync(FULL, chg & 1u), t1 = __ballot_sync(FULL, chg & 2u);
    const uint32_t b0 = __ballot_sync(FULL, chg & (1u << (2 * ROWS - 2)));
    const uint32_t b1 = __ballot_sync(FULL, chg & (1u << (2 * ROWS - 1)));
    if (lane == 0) {
        E.chg[par][warp][0][0] = t0;
        E.chg[par][warp][0][1] = t1;
        E.chg[par][warp][1][0] = b0;
        E.chg[par][warp][1][1] = b1;
    }
}

template <int MODE>
__global__ void __launch_bounds__(THREADS, 3)
k_round(const int32_t* __restrict__ src, int32_t* __restrict__ dst, int pitch, int Wd, int Hd,
        const uint32_t* __restrict__ pos, const int32_t* __restrict__ list_in, const int32_t* __restrict__ count_in,
        int32_t* __restrict__ list_out, int32_t* __restrict__ count_out, int32_t* __restrict__ stamp,
        int32_t stamp_next, int tiles_x, int tiles_y, long long step_base, long long* __restrict__ last_change)
{
    __shared__ Edges E;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cx0 = 2 * lane, cy0 = warp * ROWS;

    // cells of this thread that lie in the inner tile: bit 2r + c
    uint32_t inner = 0;
#pragma unroll
    for (int r = 0; r < ROWS; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (cx0 + c >= KSTEPS && cx0 + c < KSTEPS + TW && cy0 + r >= KSTEPS && cy0 + r < KSTEPS + TH)
                inner |= 1u << (2 * r + c);

    const int n_items = *count_in;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const int t = list_in[item];
        const int tx = t % tiles_x, ty = t / tiles_x;
        const int gx = tx * TW - KSTEPS + cx0;   // canvas column of this thread's column 0
        const int gyb = ty * TH - KSTEPS + cy0;  // canvas row of this thread's row 0

        int32_t L[ROWS][2], D[ROWS][2];
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            const int gy = gyb + r;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const bool in = gx + c >= 0 && gx + c < Wd && gy >= 0 && gy < Hd;
                const int32_t l = in ? src[(size_t)gy * pitch + gx + c] : OUTSIDE;
                L[r][c] = l;
                D[r][c] = l >= 0 ? dist2(gx + c, gy, __ldg(&pos[l])) : FAR;
            }
        }
        publish(E, 1, warp, lane, L, 0xFFFFFFFFu);
        __syncthreads();

        uint32_t chg = 0;
        int last_step = -1;
        int par = 1;   // parity of the last publication
#pragma unroll 1
        for (int s = 0; s < KSTEPS; ++s) {
            uint32_t new_chg = 0;
            if (MODE == IDL_MODE_REFERENCE) {
                // ---- one Jacobi step (voronoi.cu:32-53) ----
                const int pp = par;
                int32_t up0 = warp > 0 ? E.lab[pp][warp - 1][1][cx0] : OUTSIDE;
                int32_t up1 = warp > 0 ? E.lab[pp][warp - 1][1][cx0 + 1] : OUTSIDE;
                const int32_t dn0 = warp < WARPS - 1 ? E.lab[pp][warp + 1][0][cx0] : OUTSIDE;
                const int32_t dn1 = warp < WARPS - 1 ? E.lab[pp][warp + 1][0][cx0 + 1] : OUTSIDE;
                // a cell can change only if a cell of its closed neighbourhood changed in the previous step
                uint32_t dirty;
                if (s == 0) {
                    dirty = (1u << (2 * ROWS)) - 1u;
                } else {
                    dirty = chg | (chg << 2) | (chg >> 2) | ((chg & 0x55555555u) << 1) | ((chg & 0xAAAAAAAAu) >> 1);
                    const uint32_t lc = __shfl_up_sync(FULL, chg, 1), rc = __shfl_down_sync(FULL, chg, 1);
                    if (lane > 0) dirty |= (lc & 0xAAAAAAAAu) >> 1;
                    if (lane < 31) dirty |= (rc & 0x55555555u) << 1;
                    if (warp > 0) {
                        dirty |= (E.chg[pp][warp - 1][1][0] >> lane) & 1u;
                        dirty |= ((E.chg[pp][warp - 1][1][1] >> lane) & 1u) << 1;
                    }
                    if (warp < WARPS - 1) {
                        dirty |= ((E.chg[pp][warp + 1][0][0] >> lane) & 1u) << (2 * ROWS - 2);
                        dirty |= ((E.chg[pp][warp + 1][0][1] >> lane) & 1u) << (2 * ROWS - 1);
                    }
                    dirty &= (1u << (2 * ROWS)) - 1u;
                }
                if (__any_sync(FULL, dirty != 0)) {
#pragma unroll
                    for (int r = 0; r < ROWS; ++r) {
                        const int32_t o0 = L[r][0], o1 = L[r][1];
                        int32_t left = __shfl_up_sync(FULL, o1, 1);
                        int32_t right = __shfl_down_sync(FULL, o0, 1);
                        if (lane == 0) left = OUTSIDE;
                        if (lane == 31) right = OUTSIDE;
                        const int32_t b0 = r + 1 < ROWS ? L[r + 1][0] : dn0;
                        const int32_t b1 = r + 1 < ROWS ? L[r + 1][1] : dn1;
                        const int gy = gyb + r;
                        if (((dirty >> (2 * r)) & 1u) && o0 >= UNDEF) {
                            int32_t bl = o0, bd = D[r][0];
                            relax(bl, bd, left, gx, gy, pos);
                            relax(bl, bd, o1, gx, gy, pos);
                            relax(bl, bd, up0, gx, gy, pos);
                            relax(bl, bd, b0, gx, gy, pos);
                            if (bl != o0) {
                                L[r][0] = bl;
                                D[r][0] = bd;
                                new_chg |= 1u << (2 * r);
                            }
                        }
                        if (((dirty >> (2 * r + 1)) & 1u) && o1 >= UNDEF) {
                            int32_t bl = o1, bd = D[r][1];
                            relax(bl, bd, o0, gx + 1, gy, pos);
                            relax(bl, bd, right, gx + 1, gy, pos);
                            relax(bl, bd, up1, gx + 1, gy, pos);
                            relax(bl, bd, b1, gx + 1, gy, pos);
                            if (bl != o1) {
                                L[r][1] = bl;
                                D[r][1] = bd;
                                new_chg |= 1u << (2 * r + 1);
                            }
                        }
                        up0 = o0;
                        up1 = o1;
                    }
                }
                par ^= 1;
                publish(E, par, warp, lane, L, new_chg);
            } else {
                // ---- one NumPy iteration (voronoi.py:113-157): left, right, up, down ----
#pragma unroll
                for (int r = 0; r < ROWS; ++r) {   // neighbour on the left
                    const int32_t o0 = L[r][0], o1 = L[r][1];
                    int32_t left = __shfl_up_sync(FULL, o1, 1);
                    if (lane == 0) left = OUTSIDE;
                    const int gy = gyb + r;
                    if (o0 >= UNDEF) relax(L[r][0], D[r][0], left, gx, gy, pos);
                    if (o1 >= UNDEF) relax(L[r][1], D[r][1], o0, gx + 1, gy, pos);
                    new_chg |= (uint32_t(L[r][0] != o0) << (2 * r)) | (uint32_t(L[r][1] != o1) << (2 * r + 1));
                }
#pragma unroll
                for (int r = 0; r < ROWS; ++r) {   // neighbour on the right
                    const int32_t o0 = L[r][0], o1 = L[r][1];
                    int32_t right = __shfl_down_sync(FULL, o0, 1);
                    if (lane == 31) right = OUTSIDE;
                    const int gy = gyb + r;
                    if (o0 >= UNDEF) relax(L[r][0], D[r][0], o1, gx, gy, pos);
                    if (o1 >= UNDEF) relax(L[r][1], D[r][1], right, gx + 1, gy, pos);
                    new_chg |= (uint32_t(L[r][0] != o0) << (2 * r)) | (uint32_t(L[r][1] != o1) << (2 * r + 1));
                }
                par ^= 1;
                publish(E, par, warp, lane, L, 0u);
                __syncthreads();
                {   // neighbour above: rows bottom-up read not-yet-updated rows
                    const int32_t up0 = warp > 0 ? E.lab[par][warp - 1][1][cx0] : OUTSIDE;
                    const int32_t up1 = warp > 0 ? E.lab[par][warp - 1][1][cx0 + 1] : OUTSIDE;
#pragma unroll
                    for (int r = ROWS - 1; r >= 0; --r) {
                        const int32_t o0 = L[r][0], o1 = L[r][1];
                        const int32_t n0 = r > 0 ? L[r - 1][0] : up0, n1 = r > 0 ? L[r - 1][1] : up1;
                        const int gy = gyb + r;
                        if (o0 >= UNDEF) relax(L[r][0], D[r][0], n0, gx, gy, pos);
                        if (o1 >= UNDEF) relax(L[r][1], D[r][1], n1, gx + 1, gy, pos);
                        new_chg |= (uint32_t(L[r][0] != o0) << (2 * r)) | (uint32_t(L[r][1] != o1) << (2 * r + 1));
                    }
                }
                par ^= 1;
                publish(E, par, warp, lane, L, 0u);
                __syncthreads();
                {   // neighbour below: rows top-down read not-yet-updated rows
                    const int32_t dn0 = warp < WARPS - 1 ? E.lab[par][warp + 1][0][cx0] : OUTSIDE;
                    const int32_t dn1 = warp < WARPS - 1 ? E.lab[par][warp + 1][0][cx0 + 1] : OUTSIDE;
#pragma unroll
                    for (int r = 0; r < ROWS; ++r) {
                        const int32_t o0 = L[r][0], o1 = L[r][1];
                        const int32_t n0 = r + 1 < ROWS ? L[r + 1][0] : dn0, n1 = r + 1 < ROWS ? L[r + 1][1] : dn1;
                        const int gy = gyb + r;
                        if (o0 >= UNDEF) relax(L[r][0], D[r][0], n0, gx, gy, pos);
                        if (o1 >= UNDEF) relax(L[r][1], D[r][1], n1, gx + 1, gy, pos);
                        new_chg |= (uint32_t(L[r][0] != o0) << (2 * r)) | (uint32_t(L[r][1] != o1) << (2 * r + 1));
                    }
                }
                par ^= 1;
                publish(E, par, warp, lane, L, 0u);
            }
            chg = new_chg;
            if (__syncthreads_or((new_chg & inner) != 0u)) last_step = s;
        }

#pragma unroll
        for (int r = 0; r < ROWS; ++r)
#pragma unroll
            for (int c = 0; c < 2; ++c)
                if ((inner >> (2 * r + c)) & 1u) {
                    const int gy = gyb + r;
                    if (gx + c < Wd && gy < Hd) dst[(size_t)gy * pitch + gx + c] = L[r][c];
                }

        if (last_step >= 0) {
            if (threadIdx.x == 0) atomicMax(last_change, step_base + last_step);
            if (threadIdx.x < 9) {
                const int nx = tx + int(threadIdx.x % 3) - 1, ny = ty + int(threadIdx.x / 3) - 1;
                if (nx >= 0 && nx < tiles_x && ny >= 0 && ny < tiles_y) {
                    const int nt = ny * tiles_x + nx;
                    if (atomicExch(&stamp[nt], stamp_next) != stamp_next) {
                        const int slot = atomicAdd(count_out, 1);
                        list_out[slot] = nt;
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Reference semantics on owner keys (stencil.cuh): the tile round of k_round
// with the label planes holding packed owner positions, so a candidate's
// distance is pure arithmetic on its key and every cell update is branch-free.
// Geometry is a template: NW warps of 8 rows each, 2 columns per lane, so the
// region is 64 x 8NW cells; KS Jacobi steps per HBM round trip leave an inner
// tile of (64 - 2KS) x (8NW - 2KS).
// ---------------------------------------------------------------------------
template <int NW, int KS>
struct KeyTile {
    static constexpr int RW = 64, ROWS = 8, RH = NW * ROWS;
    static constexpr int TW = RW - 2 * KS, TH = RH - 2 * KS;
    static constexpr int THREADS = NW * 32;
    static_assert(KS >= 1 && KS <= TW && KS <= TH, "a round's light cone must stay within the neighbour tiles");
    static_assert(TW % 8 == 0 && TH % 8 == 0, "tiles must be whole 8 x 8 micro-tiles for the sparse hand-off");
    static_assert(KS % 2 == 0, "a lane's two columns must start on an even column for paired loads");
};

template <int NW>
struct KeyEdges {
    int32_t lab[2][NW][2][64];   // [parity][warp][0 = top row, 1 = bottom row][column]
    uint32_t chg[2][NW][2][2];   // [parity][warp][top/bottom][column 0/1 of each lane]: lane ballots
};

template <int NW>
__device__ __forceinline__ void key_publish(KeyEdges<NW>& E, int par, int warp, int lane, const int32_t (&L)[8][2],
                                            uint32_t chg)
{
    E.lab[par][warp][0][2 * lane] = L[0][0];
    E.lab[par][warp][0][2 * lane + 1] = L[0][1];
    E.lab[par][warp][1][2 * lane] = L[7][0];
    E.lab[par][warp][1][2 * lane + 1] = L[7][1];
    const uint32_t t0 = __ballot_sync(FULL, chg & 1u), t1 = __ballot_sync(FULL, chg & 2u);
    const uint32_t b0 = __ballot_sync(FULL, chg & (1u << 14)), b1 = __ballot_sync(FULL, chg & (1u << 15));
    if (lane == 0) {
        E.chg[par][warp][0][0] = t0;
        E.chg[par][warp][0][1] = t1;
        E.chg[par][warp][1][0] = b0;
        E.chg[par][warp][1][1] = b1;
    }
}

// One cell's Jacobi step on keys: the best of its own owner (k, d) and four
// candidate keys; cells below UNDEF (outside the canvas, batch walls) never change.
__device__ __forceinline__ void key_cell(int32_t& k, int32_t& d, int32_t a, int32_t b, int32_t c, int32_t e, int x,
                                         int y)
{
    int32_t bk = k, bd = d;
    relax_key(bk, bd, a, x, y);
    relax_key(bk, bd, b, x, y);
    relax_key(bk, bd, c, x, y);
    relax_key(bk, bd, e, x, y);
    const bool fixed = k < UNDEF;
    k = fixed ? k : bk;
    d = fixed ? d : bd;
}

// The inner-cell mask of a thread (bit 2r + c: row r, column c of its cells).
template <int NW, int KS>
__device__ __forceinline__ uint32_t key_inner_mask(int cx0, int cy0)
{
    using T = KeyTile<NW, KS>;
    uint32_t inner = 0;
#pragma unroll
    for (int r = 0; r < T::ROWS; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (cx0 + c >= KS && cx0 + c < KS + T::TW && cy0 + r >= KS && cy0 + r < KS + T::TH)
                inner |= 1u << (2 * r + c);
    return inner;
}

// Advance tile t by KS Jacobi steps (src -> dst, inner cells written) and, if
// an inner cell changed, list the tile and its 8 neighbours for the next round.
// L2: load the plane through L2 only (ld.global.cg), for a persistent kernel
// whose other blocks rewrite the planes between rounds.
template <int NW, int KS, bool L2>
__device__ __forceinline__ void key_tile(KeyEdges<NW>& E, const int32_t* src, int32_t* dst, int pitch, int Wd, int Hd,
                                         int t, int tiles_x, int tiles_y, int32_t* list_out, int32_t* count_out,
                                         int32_t* stamp, int32_t stamp_next, long long step_base,
                                         long long* last_change, uint32_t inner)
{
    using T = KeyTile<NW, KS>;
    constexpr int ROWS = T::ROWS;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cx0 = 2 * lane;
    const int tx = t % tiles_x, ty = t / tiles_x;
    const int gx = tx * T::TW - KS + cx0;
    const int gyb = ty * T::TH - KS + warp * ROWS;

    int32_t L[ROWS][2], D[ROWS][2];
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        const int gy = gyb + r;
        const bool row_in = gy >= 0 && gy < Hd;
        int32_t l0 = OUTSIDE, l1 = OUTSIDE;
        if (row_in) {
            const int32_t* row = src + (size_t)gy * pitch;
            if (gx >= 0 && gx + 1 < Wd) {
                const int2 v = L2 ? __ldcg(reinterpret_cast<const int2*>(row + gx))
                                  : *reinterpret_cast<const int2*>(row + gx);
                l0 = v.x;
                l1 = v.y;
            } else {
                if (gx >= 0 && gx < Wd) l0 = L2 ? __ldcg(row + gx) : row[gx];
                if (gx + 1 >= 0 && gx + 1 < Wd) l1 = L2 ? __ldcg(row + gx + 1) : row[gx + 1];
            }
        }
        L[r][0] = l0;
        L[r][1] = l1;
        D[r][0] = l0 >= 0 ? key_dist2(gx, gy, l0) : FAR;
        D[r][1] = l1 >= 0 ? key_dist2(gx + 1, gy, l1) : FAR;
    }
    key_publish<NW>(E, 1, warp, lane, L, 0xFFFFFFFFu);
    __syncthreads();

    uint32_t chg = 0;
    int last_step = -1;
    int par = 1;
#pragma unroll 1
    for (int s = 0; s < KS; ++s) {
        uint32_t new_chg = 0;
        const int pp = par;
        int32_t up0 = warp > 0 ? E.lab[pp][warp - 1][1][cx0] : OUTSIDE;
        int32_t up1 = warp > 0 ? E.lab[pp][warp - 1][1][cx0 + 1] : OUTSIDE;
        const int32_t dn0 = warp < NW - 1 ? E.lab[pp][warp + 1][0][cx0] : OUTSIDE;
        const int32_t dn1 = warp < NW - 1 ? E.lab[pp][warp + 1][0][cx0 + 1] : OUTSIDE;
        uint32_t dirty;
        if (s == 0) {
            dirty = 0xFFFFu;
        } else {
            dirty = chg | (chg << 2) | (chg >> 2) | ((chg & 0x5555u) << 1) | ((chg & 0xAAAAu) >> 1);
            const uint32_t lc = __shfl_up_sync(FULL, chg, 1), rc = __shfl_down_sync(FULL, chg, 1);
            if (lane > 0) dirty |= (lc & 0xAAAAu) >> 1;
            if (lane < 31) dirty |= (rc & 0x5555u) << 1;
            if (warp > 0) {
                dirty |= (E.chg[pp][warp - 1][1][0] >> lane) & 1u;
                dirty |= ((E.chg[pp][warp - 1][1][1] >> lane) & 1u) << 1;
            }
            if (warp < NW - 1) {
                dirty |= ((E.chg[pp][warp + 1][0][0] >> lane) & 1u) << 14;
                dirty |= ((E.chg[pp][warp + 1][0][1] >> lane) & 1u) << 15;
            }
            dirty &= 0xFFFFu;
        }
        if (__any_sync(FULL, dirty != 0)) {
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
                const int32_t o0 = L[r][0], o1 = L[r][1];
                int32_t left = __shfl_up_sync(FULL, o1, 1);
                int32_t right = __shfl_down_sync(FULL, o0, 1);
                if (lane == 0) left = OUTSIDE;
                if (lane == 31) right = OUTSIDE;
                const int32_t b0 = r + 1 < ROWS ? L[r + 1][0] : dn0;
                const int32_t b1 = r + 1 < ROWS ? L[r + 1][1] : dn1;
                // a cell can change only if its neighbourhood changed in the
                // last step (dirty) and a neighbour has another owner; the warp
                // skips a row none of whose cells can
                const bool need0 = ((dirty >> (2 * r)) & 1u) && (left != o0 || o1 != o0 || up0 != o0 || b0 != o0);
                const bool need1 = ((dirty >> (2 * r + 1)) & 1u) && (o0 != o1 || right != o1 || up1 != o1 || b1 != o1);
                if (__any_sync(FULL, need0 || need1)) {
                    const int gy = gyb + r;
                    key_cell(L[r][0], D[r][0], left, o1, up0, b0, gx, gy);
                    key_cell(L[r][1], D[r][1], o0, right, up1, b1, gx + 1, gy);
                    new_chg |= (uint32_t(L[r][0] != o0) << (2 * r)) | (uint32_t(L[r][1] != o1) << (2 * r + 1));
                }
                up0 = o0;
                up1 = o1;
            }
        }
        par ^= 1;
        key_publish<NW>(E, par, warp, lane, L, new_chg);
        chg = new_chg;
        if (__syncthreads_or((new_chg & inner) != 0u)) last_step = s;
    }

    // inner cells only: a lane's two columns are both inner or both not
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        const int gy = gyb + r;
        if (!((inner >> (2 * r)) & 1u) || gy >= Hd) continue;
        int32_t* row = dst + (size_t)gy * pitch;
        if (gx + 1 < Wd) {
            *reinterpret_cast<int2*>(row + gx) = make_int2(L[r][0], L[r][1]);
        } else if (gx < Wd) {
            row[gx] = L[r][0];
        }
    }

    if (last_step >= 0) {
        if (threadIdx.x == 0) atomicMax(last_change, step_base + last_step);
        if (threadIdx.x < 9) {
            const int nx = tx + int(threadIdx.x % 3) - 1, ny = ty + int(threadIdx.x / 3) - 1;
            if (nx >= 0 && nx < tiles_x && ny >= 0 && ny < tiles_y) {
                const int nt = ny * tiles_x + nx;
                if (atomicExch(&stamp[nt], stamp_next) != stamp_next) {
                    const int slot = atomicAdd(count_out, 1);
                    list_out[slot] = nt;
                }
            }
        }
    }
    __syncthreads();
}

// One tile round: every tile of list_in advanced KS steps.
template <int NW, int KS>
__global__ void __launch_bounds__(NW * 32, (NW <= 8 ? 3 : 2))
k_round_keys(const int32_t* __restrict__ src, int32_t* __restrict__ dst, int pitch, int Wd, int Hd,
             const int32_t* __restrict__ list_in, const int32_t* __restrict__ count_in,
             int32_t* __restrict__ list_out, int32_t* __restrict__ count_out, int32_t* __restrict__ stamp,
             int32_t stamp_next, int tiles_x, int tiles_y, long long step_base, long long* __restrict__ last_change)
{
    __shared__ KeyEdges<NW> E;
    const uint32_t inner = key_inner_mask<NW, KS>(2 * (threadIdx.x & 31), (threadIdx.x >> 5) * 8);
    const int n_items = *count_in;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x)
        key_tile<NW, KS, false>(E, src, dst, pitch, Wd, Hd, list_in[item], tiles_x, tiles_y, list_out, count_out,
                                stamp, stamp_next, step_base, last_change, inner);
}

// Up to max_rounds tile rounds in one cooperative launch, separated by the
// bounded grid barrier: round r runs list r%2 from plane r%2 into plane
// (r+1)%2 and builds list (r+1)%2, exactly as successive k_round_keys
// launches would.  Stops when a round's list is empty; gs->passes receives
// the rounds run.
template <int NW, int KS>
__global__ void __launch_bounds__(NW * 32, (NW <= 8 ? 3 : 2))
k_rounds_keys(int32_t* plane0, int32_t* plane1, int pitch, int Wd, int Hd, int32_t* list0, int32_t* list1,
              int32_t* counts, int32_t* stamp, int32_t epoch, int tiles_x, int tiles_y, int max_rounds,
              long long* last_change, GridSync* gs)
{
    __shared__ KeyEdges<NW> E;
    const uint32_t inner = key_inner_mask<NW, KS>(2 * (threadIdx.x & 31), (threadIdx.x >> 5) * 8);
    unsigned gen_local = 0;
    int r = 0;
    for (; r < max_rounds; ++r) {
        const int n = __ldcg(&counts[r]);
        if (n == 0) break;
        const int32_t* src = (r & 1) ? plane1 : plane0;
        int32_t* dst = (r & 1) ? plane0 : plane1;
        const int32_t* lin = (r & 1) ? list1 : list0;
        int32_t* lout = (r & 1) ? list0 : list1;
        for (int item = blockIdx.x; item < n; item += gridDim.x)
            key_tile<NW, KS, true>(E, src, dst, pitch, Wd, Hd, __ldcg(&lin[item]), tiles_x, tiles_y, lout,
                                   counts + r + 1, stamp, epoch + r + 1, (long long)r * KS, last_change, inner);
        if (!grid_sync(gs, gridDim.x, gen_local)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) gs->passes = r;
}

// ---------------------------------------------------------------------------
// Owner-key tile round on cell lists.  The RW x RH region (inner tile plus a
// KS-cell halo on every side) lives in shared memory in two buffers, A (the
// state after the last step) and B (the one before), and each step
// evaluates only the cells of its list: the 4-neighbours of the cells that
// changed in the step before (a cell none of whose neighbours changed keeps
// its owner).  The round's first list comes from the previous round's
// last-pass changes (CellBits; from scratch, the seed cells), or, with no
// such record, is every cell with a neighbour owned by another seed -- a
// superset of the cells that can change.  A listed cell writes its new value
// to B; a cell that changed but is not listed for the next step is copied
// into that step's output buffer, so that every cell a step does not write
// holds the same value in both buffers; the buffers then swap.  Work per step
// is proportional to the active cells, not to the region, which is what thin
// fronts and the settling tail need.
// ---------------------------------------------------------------------------
template <int RW, int RH, int KS>
struct CellTile {
    static constexpr int TW = RW - 2 * KS, TH = RH - 2 * KS;
    static constexpr int N = RW * RH;
    static constexpr int WORDS = N / 32;
    static constexpr int THREADS = 256;
    static constexpr int WPT = (WORDS + THREADS - 1) / THREADS;   // bitmap words per thread in a compaction
    static_assert(RW % 32 == 0 && N % 32 == 0, "rows of whole words");
    static_assert(KS >= 1 && KS <= TW && KS <= TH, "a round's light cone must stay within the neighbour tiles");
    static_assert(TW % 8 == 0 && TH % 8 == 0, "tiles must be whole 8 x 8 micro-tiles for the sparse hand-off");
    static_assert(N <= 65536, "cell indices are 16 bits");
    static_assert(WPT <= 2, "a compaction handles at most two bitmap words per thread");
    static_assert(N % THREADS == 0, "every warp covers whole bitmap words in the first-list pass");
    // dynamic shared memory: two label buffers, two lists, the mark bitmap, scan scratch and counters
    static constexpr size_t SMEM = 2 * N * 4 + 2 * N * 2 + WORDS * 4 + 32 * 4 + 16;
};

// The cells of `bits` (one bit per cell, rows of RW / 32 words) into `list`
// in ascending order; the bitmap is cleared on the way.  With DILATE, `bits`
// holds the cells that changed in the step just run and the list takes their
// four neighbours within the region (the cells that can change in the next
// step: a cell none of whose neighbours changed keeps its value, since the
// best of its owner and unchanged neighbours is already its owner), built
// word by word instead of one shared atomic per mark.  With COPY, the changed
// cells outside that list follow it (*n_copy of them): the next step only
// copies their new value into its output buffer, so that every cell it does
// not write holds the same value in both buffers.  Returns the length of the
// list proper (every thread); *inner_changed tells whether a changed cell lies
// in the inner tile [KS, KS + TW) x [KS, KS + TH).
template <int RW, int RH, int KS, int TW, int TH, int WPT, bool DILATE, bool COPY>
__device__ __forceinline__ int cell_compact(uint32_t* bits, uint16_t* list, int* warp_sums, bool* inner_changed,
                                            int* n_copy)
{
    constexpr int WR = RW / 32, WORDS = RW * RH / 32;
    static_assert(RW * RH < 65536, "two list lengths share one 32-bit scan");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    uint32_t w[WPT], wc[WPT];
    int cnt = 0;   // list cells, plus copy cells << 16
    bool inner = false;
#pragma unroll
    for (int j = 0; j < WPT; ++j) {
        const int i = tid * WPT + j;
        uint32_t m = 0u, mc = 0u;
        if (i < WORDS) {
            const uint32_t c = bits[i];
            if (DILATE) {
                const int row = i / WR, wi = i % WR;
                m = (c << 1) | (c >> 1);
                if (wi > 0) m |= bits[i - 1] >> 31;
                if (wi < WR - 1) m |= bits[i + 1] << 31;
                if (row > 0) m |= bits[i - WR];
                if (row < RH - 1) m |= bits[i + WR];
                if (COPY) mc = c & ~m;
                if (row >= KS && row < KS + TH) {
                    const int lo = max(KS - wi * 32, 0), hi = min(KS + TW - wi * 32, 32);
                    if (hi > lo) {
                        const uint32_t span = hi - lo == 32 ? 0xFFFFFFFFu : ((1u << (hi - lo)) - 1u) << lo;
                        inner = inner || (c & span) != 0u;
                    }
                }
            } else {
                m = c;
            }
        }
        w[j] = m;
        wc[j] = mc;
        cnt += __popc(m) + (COPY ? __popc(mc) << 16 : 0);
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sums[warp] = incl;
    *inner_changed = __syncthreads_or(inner) != 0;   // also: every word was read before any is cleared
    // every warp adds up the few warp counts itself (no second barrier)
    int before = 0, total = 0;
    for (int k = 0; k < nwarps; ++k) {
        const int v = warp_sums[k];
        before += k < warp ? v : 0;
        total += v;
    }
    const int start = before + incl - cnt;
    const int n_list = total & 0xFFFF;
    int pos = start & 0xFFFF, pos_c = n_list + (start >> 16);
#pragma unroll
    for (int j = 0; j < WPT; ++j) {
        const int i = tid * WPT + j;
        uint32_t m = w[j];
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            list[pos++] = (uint16_t)(i * 32 + b);
        }
        if (COPY) {
            uint32_t mc = wc[j];
            while (mc) {
                const int b = __ffs(mc) - 1;
                mc &= mc - 1;
                list[pos_c++] = (uint16_t)(i * 32 + b);
            }
        }
        if (i < WORDS) bits[i] = 0u;
    }
    __syncthreads();   // the list is read, the bitmap and warp_sums rewritten, by the next use
    if (COPY) *n_copy = total >> 16;
    return n_list;
}

// What the last tile round before the persistent kernel leaves it (bits null:
// not the last round): the 8 x 8 micro-tiles that can change in the next
// pass, as that kernel's first work list with its dedup bitmap set.
struct Handoff {
    uint32_t* bits;
    int32_t* list;
    int32_t* count;
    int mt_x;
};

// Last-pass changes passed from one tile round to the next: one bit per
// canvas cell, rows of `stride` words (bit x of row y: word y * stride + x / 32).
// A round writes into `out` the inner cells that changed in its last pass; the
// next round reads them as `in`, and its first list is those cells and their
// neighbours -- exactly the cells that can change in its first pass, where the
// neighbour test (in null) also lists every settled boundary.  `clear`, a
// bitmap no round of this launch or the previous one touches, is zeroed for
// the round after next.
struct CellBits {
    const uint32_t* in;
    uint32_t* out;
    uint32_t* clear;
    int stride;   // words per row
    int words;    // words per bitmap
};

// Bits g .. g + 31 of a row of `stride` words (g may be negative); zeros
// outside the row.
__device__ __forceinline__ uint32_t row_bits32(const uint32_t* row, int stride, int g)
{
    const int w = g >> 5, sh = g & 31;
    const uint32_t lo = (w >= 0 && w < stride) ? row[w] : 0u;
    const uint32_t hi = (w + 1 >= 0 && w + 1 < stride) ? row[w + 1] : 0u;
    return __funnelshift_r(lo, hi, sh);
}

// The inner cells marked in the region bitmap `bits` into cb.out (region
// origin ox, oy on the canvas; inner cells start at ox + KS = tx * TW >= 0).
template <int RW, int RH, int KS, int TW, int TH>
__device__ __forceinline__ void cell_bits_out(const uint32_t* bits, const CellBits& cb, int ox, int oy, int Hd)
{
    constexpr int WR = RW / 32;
    const int gx0 = ox + KS;
    const int w0 = gx0 >> 5, nw = ((gx0 + TW - 1) >> 5) - w0 + 1;
    for (int task = threadIdx.x; task < TH * nw; task += blockDim.x) {
        const int iy = task / nw, gw = w0 + task % nw;
        const int gy = oy + KS + iy;
        if (gy >= Hd) continue;
        const int rb = gw * 32 - ox;   // region column of the word's bit 0
        const int lo = max(KS - rb, 0), hi = min(KS + TW - rb, 32);
        const uint32_t span = hi - lo >= 32 ? 0xFFFFFFFFu : ((1u << (hi - lo)) - 1u) << lo;
        const uint32_t v = row_bits32(bits + (KS + iy) * WR, WR, rb) & span;
        if (v) atomicOr(&cb.out[(size_t)gy * cb.stride + gw], v);
    }
}

// Both region buffers take the labels of the RW x RH region at (ox, oy)
// (OUTSIDE beyond the canvas).
template <int RW, int RH, bool L2>
__device__ __forceinline__ void load_region(int32_t* bufA, int32_t* bufB, const int32_t* src, int pitch, int Wd,
                                            int Hd, int ox, int oy)
{
    for (int i = threadIdx.x; i < RW * RH; i += blockDim.x) {
        const int cx = i % RW, cy = i / RW;
        const int gx = ox + cx, gy = oy + cy;
        int32_t v = OUTSIDE;
        if (gx >= 0 && gx < Wd && gy >= 0 && gy < Hd) {
            const int32_t* p = src + (size_t)gy * pitch + gx;
            v = L2 ? __ldcg(p) : *p;
        }
        bufA[i] = v;
        bufB[i] = v;
    }
}

template <int RW, int RH, int KS, bool L2>
__device__ __forceinline__ void cell_tile(unsigned char* smem, const int32_t* src, int32_t* dst, int pitch, int Wd,
                                          int Hd, int t, int tiles_x, int tiles_y, int32_t* list_out,
                                          int32_t* count_out, int32_t* stamp, int32_t stamp_next, long long step_base,
                                          long long* last_change, Handoff ho, const CellBits& cb)
{
    using T = CellTile<RW, RH, KS>;
    constexpr int N = T::N;
    int32_t* bufA = reinterpret_cast<int32_t*>(smem);
    int32_t* bufB = bufA + N;
    uint16_t* listA = reinterpret_cast<uint16_t*>(bufB + N);
    uint16_t* listB = listA + N;
    uint32_t* bits = reinterpret_cast<uint32_t*>(listB + N);
    int* warp_sums = reinterpret_cast<int*>(bits + T::WORDS);   // 32 entries
    const int tid = threadIdx.x;
    const int tx = t % tiles_x, ty = t / tiles_x;
    const int ox = tx * T::TW - KS, oy = ty * T::TH - KS;

    bool inner_changed = false;
    int n, n_copy = 0;
    if (cb.in) {
        // first list: the previous round's last-pass changes and their
        // neighbours.  A region with none only brings the output plane up to
        // date: its inner cells are copied, nothing is evaluated.
        constexpr int WR = RW / 32;
        bool any = false;
        for (int i = tid; i < T::WORDS; i += blockDim.x) {
            const int gy = oy + i / WR;
            const uint32_t w = (gy >= 0 && gy < Hd)
                                   ? row_bits32(cb.in + (size_t)gy * cb.stride, cb.stride, ox + 32 * (i % WR))
                                   : 0u;
            bits[i] = w;
            any = any || w != 0u;
        }
        if (!__syncthreads_or(any)) {
            for (int i = tid; i < T::TW * T::TH; i += blockDim.x) {
                const int gx = ox + KS + i % T::TW, gy = oy + KS + i / T::TW;
                if (gx < Wd && gy < Hd) {
                    const int32_t* p = src + (size_t)gy * pitch + gx;
                    dst[(size_t)gy * pitch + gx] = L2 ? __ldcg(p) : *p;
                }
            }
            return;
        }
        load_region<RW, RH, L2>(bufA, bufB, src, pitch, Wd, Hd, ox, oy);
        __syncthreads();
        // (both buffers start equal: nothing to copy)
        n = cell_compact<RW, RH, KS, T::TW, T::TH, T::WPT, true, false>(bits, listA, warp_sums, &inner_changed,
                                                                        &n_copy);
    } else {
        load_region<RW, RH, L2>(bufA, bufB, src, pitch, Wd, Hd, ox, oy);
        __syncthreads();
        // first list: cells with a neighbour owned by another seed; the block's
        // 32-cell strides are warp-aligned, so each warp's ballot is one word
        for (int i = tid; i < N; i += blockDim.x) {
            const int32_t o = bufA[i];
            const int cx = i % RW, cy = i / RW;
            const bool diff = o >= UNDEF && ((cx > 0 && bufA[i - 1] != o) || (cx < RW - 1 && bufA[i + 1] != o) ||
                                             (cy > 0 && bufA[i - RW] != o) || (cy < RH - 1 && bufA[i + RW] != o));
            const uint32_t word = __ballot_sync(0xFFFFFFFFu, diff);
            if ((tid & 31) == 0) bits[i >> 5] = word;
        }
        __syncthreads();
        n = cell_compact<RW, RH, KS, T::TW, T::TH, T::WPT, false, false>(bits, listA, warp_sums, &inner_changed,
                                                                         &n_copy);
    }

    int32_t* cur = bufA;
    int32_t* nxt = bufB;
    uint16_t* lc = listA;
    uint16_t* ln = listB;
    int last_step = -1;
#pragma unroll 1
    for (int s = 0; s < KS && n > 0; ++s) {
        for (int i = tid; i < n; i += blockDim.x) {
            const int c = lc[i];
            const int32_t own = cur[c];
            if (own < UNDEF) continue;
            const int cx = c % RW, cy = c / RW;
            const int32_t l = cx > 0 ? cur[c - 1] : OUTSIDE;
            const int32_t r = cx < RW - 1 ? cur[c + 1] : OUTSIDE;
            const int32_t u = cy > 0 ? cur[c - RW] : OUTSIDE;
            const int32_t d = cy < RH - 1 ? cur[c + RW] : OUTSIDE;
            const int gx = ox + cx, gy = oy + cy;
            int32_t k = own;
            int32_t dd = own >= 0 ? key_dist2(gx, gy, own) : FAR;
            relax_key(k, dd, l, gx, gy);
            relax_key(k, dd, r, gx, gy);
            relax_key(k, dd, u, gx, gy);
            relax_key(k, dd, d, gx, gy);
            nxt[c] = k;
            if (k != own) atomicOr(&bits[c >> 5], 1u << (c & 31));
        }
        // cells that changed in the step before but cannot change now
        for (int i = tid; i < n_copy; i += blockDim.x) {
            const int c = lc[n + i];
            nxt[c] = cur[c];
        }
        __syncthreads();
        if (cb.out && s == KS - 1) cell_bits_out<RW, RH, KS, T::TW, T::TH>(bits, cb, ox, oy, Hd);
        // the next list: changed cells and their neighbours
        n = cell_compact<RW, RH, KS, T::TW, T::TH, T::WPT, true, true>(bits, ln, warp_sums, &inner_changed,
                                                                       &n_copy);
        if (inner_changed) last_step = s;
        int32_t* tb = cur; cur = nxt; nxt = tb;
        uint16_t* tl = lc; lc = ln; ln = tl;
    }

    if (ho.bits) {
        // The cells marked by the last step's changes are those that can
        // change in the next pass.  Kept: inner cells and the ring just
        // outside them.  A ring cell's mark here may come from a stale halo
        // value, which only adds a micro-tile; its true marks come from the
        // tile whose inner cells it borders.  The compactions left `bits`
        // clear, so it holds the tile's micro-tiles here, ring included.
        constexpr int MX = T::TW / MICRO_TILE + 2, MY = T::TH / MICRO_TILE + 2;
        static_assert(MX * MY <= T::WORDS * 32, "micro-tile marks fit the cell bitmap");
        const int mx0 = tx * (T::TW / MICRO_TILE) - 1, my0 = ty * (T::TH / MICRO_TILE) - 1;
        for (int i = tid; i < n; i += blockDim.x) {
            const int c = lc[i];
            const int cx = c % RW, cy = c / RW;
            if (cx < KS - 1 || cx > KS + T::TW || cy < KS - 1 || cy > KS + T::TH) continue;
            const int gx = ox + cx, gy = oy + cy;
            if (gx < 0 || gy < 0 || gx >= Wd || gy >= Hd) continue;
            const int j = (gy / MICRO_TILE - my0) * MX + gx / MICRO_TILE - mx0;
            atomicOr(&bits[j >> 5], 1u << (j & 31));
        }
        __syncthreads();
        for (int j = tid; j < MX * MY; j += blockDim.x) {
            if (!((bits[j >> 5] >> (j & 31)) & 1u)) continue;
            const int mx = mx0 + j % MX, my = my0 + j / MX;
            const int mt = my * ho.mt_x + mx;
            const uint32_t bit = 1u << (mt & 31);
            if (!(atomicOr(&ho.bits[mt >> 5], bit) & bit)) ho.list[atomicAdd(ho.count, 1)] = pack_mt(mx, my);
        }
        __syncthreads();   // the next tile clears `bits` before its first use
    }

    // inner cells of the latest state
    for (int i = tid; i < T::TW * T::TH; i += blockDim.x) {
        const int cx = KS + i % T::TW, cy = KS + i / T::TW;
        const int gx = ox + cx, gy = oy + cy;
        if (gx < Wd && gy < Hd) dst[(size_t)gy * pitch + gx] = cur[cy * RW + cx];
    }

    if (last_step >= 0) {
        if (tid == 0) atomicMax(last_change, step_base + last_step);
        // The next round's changes spread from this round's last-pass changes
        // alone: only those list the neighbourhood.  Any change lists the tile
        // itself, whose next run copies its inner cells to the other plane
        // (a tile no round runs must hold the same state in both).
        if ((last_step == KS - 1 && tid < 9) || tid == 4) {
            const int nx = tx + int(tid % 3) - 1, ny = ty + int(tid / 3) - 1;
            if (nx >= 0 && nx < tiles_x && ny >= 0 && ny < tiles_y) {
                const int nt = ny * tiles_x + nx;
                if (atomicExch(&stamp[nt], stamp_next) != stamp_next) {
                    const int slot = atomicAdd(count_out, 1);
                    list_out[slot] = nt;
                }
            }
        }
    }
    __syncthreads();
}

template <int RW, int RH, int KS>
__global__ void __launch_bounds__(256)
k_round_cells(const int32_t* __restrict__ src, int32_t* __restrict__ dst, int pitch, int Wd, int Hd,
              const int32_t* __restrict__ list_in, const int32_t* __restrict__ count_in,
              int32_t* __restrict__ list_out, int32_t* __restrict__ count_out, int32_t* __restrict__ stamp,
              int32_t stamp_next, int tiles_x, int tiles_y, long long step_base, long long* __restrict__ last_change,
              Handoff ho, CellBits cb)
{
    extern __shared__ __align__(16) unsigned char cell_smem[];
    if (cb.clear)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cb.words; i += gridDim.x * blockDim.x) cb.clear[i] = 0u;
    const int n_items = *count_in;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x)
        cell_tile<RW, RH, KS, false>(cell_smem, src, dst, pitch, Wd, Hd, list_in[item], tiles_x, tiles_y, list_out,
                                     count_out, stamp, stamp_next, step_base, last_change, ho, cb);
}

// Plane `dst` takes plane `src`'s inner cells of the listed tiles: after it,
// the planes agree everywhere once they agreed outside those tiles.
__global__ void k_copy_tiles(const int32_t* __restrict__ src, int32_t* __restrict__ dst, int pitch, int Wd, int Hd,
                             const int32_t* __restrict__ list, const int32_t* __restrict__ count, int tiles_x, int tw,
                             int th)
{
    // tiles start at multiples of tw (a multiple of 8) on 32-aligned rows, so
    // whole 4-cell groups are 16-byte aligned; the canvas edge goes cell by cell
    const int n_items = *count;
    const int groups = tw / 4;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const int t = list[item];
        const int x0 = (t % tiles_x) * tw, y0 = (t / tiles_x) * th;
        for (int i = threadIdx.x; i < groups * th; i += blockDim.x) {
            const int gy = y0 + i / groups, gx = x0 + (i % groups) * 4;
            if (gy >= Hd) continue;
            const size_t o = (size_t)gy * pitch + gx;
            if (gx + 4 <= Wd) {
                *reinterpret_cast<int4*>(dst + o) = *reinterpret_cast<const int4*>(src + o);
            } else {
                for (int k = 0; k < 4 && gx + k < Wd; ++k) dst[o + k] = src[o + k];
            }
        }
    }
}

// Seed cells of both planes take their seeds' keys (the rest of the planes
// already holds UNDEF, or walls for a batch atlas).
__global__ void k_seed_keys(int32_t* __restrict__ a, int32_t* __restrict__ b, int pitch,
                            const uint32_t* __restrict__ pos, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = pos[i];
    const size_t o = (size_t)pos_y(p) * pitch + pos_x(p);
    const int32_t k = key_from_pos(p);
    a[o] = k;
    b[o] = k;
}

// One bit per seed cell in a change bitmap of rows of `stride` words: from
// scratch, the seeds are the change the first pass reacts to.
__global__ void k_mark_cells(const uint32_t* __restrict__ pos, int64_t n, uint32_t* __restrict__ bits, int stride)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = pos[i];
    atomicOr(&bits[(size_t)pos_y(p) * stride + (pos_x(p) >> 5)], 1u << (pos_x(p) & 31));
}

// Keys back to ids: `ids` (the other plane, free once both planes agree)
// takes at each seed cell that seed's id; every owned cell of `lab` then
// looks its owner's id up at the owner's own cell.  Only seed cells of `ids`
// are read, and `lab` is the only plane written.
__global__ void k_seed_ids(int32_t* __restrict__ ids, int pitch, const uint32_t* __restrict__ pos, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = pos[i];
    ids[(size_t)pos_y(p) * pitch + pos_x(p)] = (int32_t)i;
}

__global__ void k_keys_to_ids(int32_t* __restrict__ lab, const int32_t* __restrict__ ids, int pitch, int Wd)
{
    int32_t* row = lab + (size_t)blockIdx.y * pitch;
    for (int x = (blockIdx.x * blockDim.x + threadIdx.x) * 4; x < Wd; x += gridDim.x * blockDim.x * 4) {
        if (x + 3 < Wd) {
            int4 v = *reinterpret_cast<const int4*>(row + x);
            if (v.x >= 0) v.x = __ldg(&ids[(size_t)key_y(v.x) * pitch + key_x(v.x)]);
            if (v.y >= 0) v.y = __ldg(&ids[(size_t)key_y(v.y) * pitch + key_x(v.y)]);
            if (v.z >= 0) v.z = __ldg(&ids[(size_t)key_y(v.z) * pitch + key_x(v.z)]);
            if (v.w >= 0) v.w = __ldg(&ids[(size_t)key_y(v.w) * pitch + key_x(v.w)]);
            *reinterpret_cast<int4*>(row + x) = v;
        } else {
            for (int c = x; c < Wd; ++c) {
                const int32_t k = row[c];
                if (k >= 0) row[c] = __ldg(&ids[(size_t)key_y(k) * pitch + key_x(k)]);
            }
        }
    }
}

__global__ void k_iota(int32_t* __restrict__ a, int n, int32_t* __restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
    if (i == 0) *count = n;
}

__global__ void k_set_i64(long long* p, long long v) { *p = v; }

// First work list of a continued propagation: the tiles holding the n new
// seeds and their 8 neighbours (a wave from a seed reaches at most KSTEPS <=
// TW cells into the next tile in one round), each listed once.
__global__ void k_seed_round_tiles(const uint32_t* __restrict__ seed_pos, int64_t n, int tiles_x, int tiles_y,
                                   int32_t* __restrict__ stamp, int32_t stamp_val, int32_t* __restrict__ list,
                                   int32_t* __restrict__ count)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * 9) return;
    const uint32_t p = seed_pos[i / 9];
    const int k = (int)(i % 9);
    const int nx = (int)pos_x(p) / TW + k % 3 - 1, ny = (int)pos_y(p) / TH + k / 3 - 1;
    if (nx < 0 || nx >= tiles_x || ny < 0 || ny >= tiles_y) return;
    const int t = ny * tiles_x + nx;
    if (atomicExch(&stamp[t], stamp_val) != stamp_val) list[atomicAdd(count, 1)] = t;
}

__global__ void k_write_seeds(int32_t* __restrict__ a, int32_t* __restrict__ b, int pitch,
                              const uint32_t* __restrict__ pos, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = pos[i];
    const size_t o = (size_t)pos_y(p) * pitch + pos_x(p);
    a[o] = (int32_t)i;
    b[o] = (int32_t)i;
}

}  // namespace

void init_labels(Context& C, const Canvas& cv, const uint32_t* pos, int64_t n)
{
    const size_t bytes = (size_t)cv.pitch * cv.Hd * sizeof(int32_t);
    for (int b = 0; b < 2; ++b) {
        C.lab[b].ensure(bytes);
        IDL_CUDA(cudaMemsetAsync(C.lab[b].ptr, 0xFF, bytes, C.stream));
    }
    if (n > 0) {
        k_write_seeds<<<(unsigned)((n + 255) / 256), 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), C.lab[1].as<int32_t>(),
                                                                        cv.pitch, pos, n);
        IDL_LAUNCH();
    }
}

// Reserve a fresh range of stamp values for a run of `steps` steps over
// `n_items` work items (stamps never need clearing between runs).
int32_t claim_stamps(Context& C, int n_items, int64_t steps)
{
    if (C.stamps.bytes < (size_t)n_items * 4) {
        C.stamps.ensure((size_t)n_items * 4);
        IDL_CUDA(cudaMemsetAsync(C.stamps.ptr, 0, C.stamps.bytes, C.stream));
        C.stamp_epoch = 0;
    }
    if (C.stamp_epoch > (1 << 30) - steps - 8) {
        IDL_CUDA(cudaMemsetAsync(C.stamps.ptr, 0, C.stamps.bytes, C.stream));
        C.stamp_epoch = 0;
    }
    const int32_t epoch = C.stamp_epoch;
    C.stamp_epoch += int32_t(steps + 4);
    return epoch;
}

namespace {

// Owner-key tile round shapes (C.key_tile): warps per CTA x steps per round.
struct KeyShape {
    int nw, ks, tw, th;
};
constexpr KeyShape KEY_SHAPES[] = {
    {8, 8, KeyTile<8, 8>::TW, KeyTile<8, 8>::TH},        // 48 x 48 inner tile, 8 passes per round trip
    {16, 8, KeyTile<16, 8>::TW, KeyTile<16, 8>::TH},     // 48 x 112, 8 passes
    {8, 4, KeyTile<8, 4>::TW, KeyTile<8, 4>::TH},        // 56 x 56, 4 passes
    {16, 12, KeyTile<16, 12>::TW, KeyTile<16, 12>::TH},  // 40 x 104, 12 passes
};
constexpr int N_KEY_SHAPES = int(sizeof(KEY_SHAPES) / sizeof(KEY_SHAPES[0]));

// Cell-list tile round shapes (k_round_cells): region width x height and steps.
struct CellShape {
    int rw, rh, ks, tw, th;
};
constexpr CellShape CELL_SHAPES[] = {
    {64, 64, 8, CellTile<64, 64, 8>::TW, CellTile<64, 64, 8>::TH},          // 48 x 48, 8 passes
    {64, 64, 4, CellTile<64, 64, 4>::TW, CellTile<64, 64, 4>::TH},          // 56 x 56, 4 passes
    {128, 64, 8, CellTile<128, 64, 8>::TW, CellTile<128, 64, 8>::TH},       // 112 x 48, 8 passes
    {128, 128, 16, CellTile<128, 128, 16>::TW, CellTile<128, 128, 16>::TH},  // 96 x 96, 16 passes
};
constexpr int N_CELL_SHAPES = int(sizeof(CELL_SHAPES) / sizeof(CELL_SHAPES[0]));

template <int RW, int RH, int KS>
void launch_round_cells(Context& C, const int32_t* src, int32_t* dst, const Canvas& cv, const int32_t* lin,
                        const int32_t* cin, int32_t* lout, int32_t* cout, int32_t* stamp, int32_t stamp_next,
                        int tiles_x, int tiles_y, long long base, long long* last, Handoff ho, const CellBits& cb)
{
    using T = CellTile<RW, RH, KS>;
    // the shared-memory opt-in belongs to each device's context: set once per device
    static std::atomic<uint64_t> opted{0};
    const uint64_t bit = 1ull << (C.device & 63);
    if (!(opted.load(std::memory_order_acquire) & bit)) {
        IDL_CUDA(cudaFuncSetAttribute((const void*)k_round_cells<RW, RH, KS>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM));
        opted.fetch_or(bit, std::memory_order_acq_rel);
    }
    int per_sm = 0;
    IDL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_round_cells<RW, RH, KS>, T::THREADS, T::SMEM));
    const int grid = std::max(1, std::min(tiles_x * tiles_y, std::max(per_sm, 1) * C.num_sms));
    k_round_cells<RW, RH, KS><<<grid, T::THREADS, T::SMEM, C.stream>>>(src, dst, cv.pitch, cv.Wd, cv.Hd, lin, cin,
                                                                      lout, cout, stamp, stamp_next, tiles_x,
                                                                      tiles_y, base, last, ho, cb);
}

template <int NW, int KS>
void launch_round_keys(Context& C, int per_sm, const int32_t* src, int32_t* dst, const Canvas& cv, const int32_t* lin,
                       const int32_t* cin, int32_t* lout, int32_t* cout, int32_t* stamp, int32_t stamp_next,
                       int tiles_x, int tiles_y, long long base, long long* last)
{
    const int grid = std::min(tiles_x * tiles_y, C.num_sms * per_sm);
    k_round_keys<NW, KS><<<grid, NW * 32, 0, C.stream>>>(src, dst, cv.pitch, cv.Wd, cv.Hd, lin, cin, lout, cout, stamp,
                                                         stamp_next, tiles_x, tiles_y, base, last);
}

int64_t propagate_rounds(Context& C, int mode, const Canvas& cv, const uint32_t* pos, const uint32_t* seed_pos,
                         int64_t n_new, bool keys, const uint32_t* start_pos = nullptr, int64_t n_start = 0);

// Up to `rounds_cap` owner-key tile rounds in one cooperative launch (the
// first work list already in C.tiles[0] and counts[0]); returns the rounds run.
template <int NW, int KS>
int64_t run_rounds_keys(Context& C, const Canvas& cv, int32_t* counts, int32_t epoch, int tiles_x, int tiles_y,
                        int64_t rounds_cap, long long* last)
{
    int per_sm = 0;
    IDL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rounds_keys<NW, KS>, NW * 32, 0));
    if (per_sm < 1) throw Error(IDL_ERR_INTERNAL, "tile round kernel cannot be resident");
    const int grid = std::max(1, std::min(tiles_x * tiles_y, per_sm * C.num_sms));
    C.gsync.ensure(sizeof(GridSync));
    IDL_CUDA(cudaMemsetAsync(C.gsync.ptr, 0, sizeof(GridSync), C.stream));
    int32_t* p0 = C.lab[0].as<int32_t>();
    int32_t* p1 = C.lab[1].as<int32_t>();
    int32_t* l0 = C.tiles[0].as<int32_t>();
    int32_t* l1 = C.tiles[1].as<int32_t>();
    int32_t* stamp = C.stamps.as<int32_t>();
    GridSync* gs = C.gsync.as<GridSync>();
    int pitch = cv.pitch, Wd = cv.Wd, Hd = cv.Hd, tx = tiles_x, ty = tiles_y;
    int cap = (int)std::min<int64_t>(rounds_cap, 1 << 30);
    void* args[] = {&p0, &p1, &pitch, &Wd, &Hd, &l0, &l1, &counts, &stamp, &epoch, &tx, &ty, &cap, &last, &gs};
    GridSync h{};
    {
        std::lock_guard<std::mutex> lock(persistent_grid_lock(C.device));
        IDL_CUDA(cudaLaunchCooperativeKernel((const void*)k_rounds_keys<NW, KS>, dim3(grid), dim3(NW * 32), args, 0,
                                             C.stream));
        count_launch();
        IDL_CUDA(cudaMemcpyAsync(&h, gs, sizeof(GridSync), cudaMemcpyDeviceToHost, C.stream));
        IDL_CUDA(cudaStreamSynchronize(C.stream));
    }
    if (h.error) throw Error(IDL_ERR_INTERNAL, "Voronoi propagation: grid barrier timed out");
    return h.passes;
}

}  // namespace

// Indices N_KEY_SHAPES .. 2 N_KEY_SHAPES - 1 are the same shapes with the
// rounds run as one cooperative launch (run_rounds_keys); the next
// N_CELL_SHAPES are the cell-list tile rounds (k_round_cells).
int key_tile_shapes() { return 2 * N_KEY_SHAPES + N_CELL_SHAPES; }

int64_t propagate(Context& C, int mode, const Canvas& cv, const uint32_t* pos, int64_t n_seeds,
                  const uint32_t* seed_pos, int64_t n_new)
{
    C.prof.tiles = C.prof.rounds = C.prof.passes = 0;
    C.prof.prop_bytes = 0.0;
    C.prof.pass_ns.clear();
    C.prof.pass_tiles.clear();
    if (mode != IDL_MODE_REFERENCE || seed_pos) return propagate_rounds(C, mode, cv, pos, seed_pos, n_new, false);
    // From scratch in reference semantics: run on owner keys, then map every
    // owned cell back to its owner's id.
    if (n_seeds > 0) {
        k_seed_keys<<<(unsigned)((n_seeds + 255) / 256), 256, 0, C.stream>>>(
            C.lab[0].as<int32_t>(), C.lab[1].as<int32_t>(), cv.pitch, pos, n_seeds);
        IDL_LAUNCH();
    }
    const int64_t passes = propagate_rounds(C, mode, cv, pos, nullptr, 0, true, pos, n_seeds);
    // the result is in plane 0 (both planes agree); plane 1 takes the ids at the seed cells
    if (n_seeds > 0) {
        k_seed_ids<<<(unsigned)((n_seeds + 255) / 256), 256, 0, C.stream>>>(C.lab[1].as<int32_t>(), cv.pitch, pos,
                                                                           n_seeds);
        IDL_LAUNCH();
        const int gx = std::max(1, std::min(ceil_div(cv.Wd, 4 * 256), 4));
        k_keys_to_ids<<<dim3(gx, cv.Hd), 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), C.lab[1].as<int32_t>(),
                                                              cv.pitch, cv.Wd);
        IDL_LAUNCH();
    }
    return passes;
}

namespace {

int64_t propagate_rounds(Context& C, int mode, const Canvas& cv, const uint32_t* pos, const uint32_t* seed_pos,
                         int64_t n_new, bool keys, const uint32_t* start_pos, int64_t n_start)
{
    // Reference semantics.  A continued propagation (seed_pos) is local from
    // its first pass: the sparse kernel alone, or with C.dense_rounds < 0 tile
    // rounds starting from the tiles around the new seeds (plain launches, no
    // device-wide persistent grid, so streams of other work overlap them).
    // From scratch, the first passes change most of the canvas, which the
    // tile rounds (several passes per HBM round trip, no per-pass bookkeeping)
    // do best; once the changes thin out, the sparse kernel takes over the
    // tail, whose single passes touch few cells.  C.dense_rounds sets the
    // switch (0: sparse only, < 0: tile rounds to convergence).
    const bool seeded_rounds = mode == IDL_MODE_REFERENCE && seed_pos && C.dense_rounds < 0;
    const bool hybrid = mode == IDL_MODE_REFERENCE && !seed_pos && C.dense_rounds != 0;
    if (mode == IDL_MODE_REFERENCE && !hybrid && !seeded_rounds)
        return propagate_sparse(C, cv, pos, seed_pos, n_new, keys);
    if (seed_pos && n_new == 0) return 0;
    const int64_t round_limit = hybrid && C.dense_rounds > 0 ? C.dense_rounds : -1;
    const int tile = std::min(std::max(C.key_tile, 0), key_tile_shapes() - 1);
    const bool cells = keys && tile >= 2 * N_KEY_SHAPES;
    const int base_shape = cells ? 0 : tile % N_KEY_SHAPES;
    const bool persistent = keys && C.persistent_rounds && !cells && tile >= N_KEY_SHAPES;
    const KeyShape shape = KEY_SHAPES[base_shape];
    const CellShape cshape = CELL_SHAPES[cells ? tile - 2 * N_KEY_SHAPES : 0];
    const int tw = cells ? cshape.tw : keys ? shape.tw : TW;
    const int th = cells ? cshape.th : keys ? shape.th : TH;
    const int steps = cells ? cshape.ks : keys ? shape.ks : KSTEPS;
    const int tiles_x = ceil_div(cv.Wd, tw), tiles_y = ceil_div(cv.Hd, th);
    const int n_tiles = tiles_x * tiles_y;
    // Bound on rounds: far above any real run (a pass count beyond the canvas
    // area cannot occur since every change strictly improves one of Wd*Hd keys
    // drawn from a finite set, but the bound only has to stop a runaway loop).
    const int64_t max_rounds = (int64_t)4 * (cv.Wd + cv.Hd) + 64;

    C.tiles[0].ensure((size_t)n_tiles * 4);
    C.tiles[1].ensure((size_t)n_tiles * 4);
    const int32_t epoch = claim_stamps(C, n_tiles, max_rounds);

    const size_t count_len = (size_t)max_rounds + 2;
    C.counts.ensure(count_len * 4);
    IDL_CUDA(cudaMemsetAsync(C.counts.ptr, 0, count_len * 4, C.stream));
    int32_t* counts = C.counts.as<int32_t>();

    if (seeded_rounds) {
        k_seed_round_tiles<<<(unsigned)((n_new * 9 + 255) / 256), 256, 0, C.stream>>>(
            seed_pos, n_new, tiles_x, tiles_y, C.stamps.as<int32_t>(), epoch + int32_t(max_rounds) + 2,
            C.tiles[0].as<int32_t>(), counts);   // a stamp value of the claimed range no round uses
    } else {
        k_iota<<<(unsigned)((n_tiles + 255) / 256), 256, 0, C.stream>>>(C.tiles[0].as<int32_t>(), n_tiles, counts);
    }
    IDL_LAUNCH();
    long long* last = reinterpret_cast<long long*>(&C.sc()->last_change);
    k_set_i64<<<1, 1, 0, C.stream>>>(last, -1);
    IDL_LAUNCH();

    // Cell-list rounds before the persistent kernel: the last one lists the
    // micro-tiles that can still change, so the kernel's first pass runs only
    // those, not every micro-tile of the tiles left active.
    const bool handoff = cells && round_limit > 0;
    Handoff ho_last{nullptr, nullptr, nullptr, 0};
    if (handoff) {
        const int mt_x = ceil_div(cv.Wd, MICRO_TILE), mt_y = ceil_div(cv.Hd, MICRO_TILE);
        C.bits.ensure((size_t)sparse_bits_words(cv) * 2 * 4);
        C.big_tiles.ensure((size_t)mt_x * mt_y * 4);
        ho_last = Handoff{C.bits.as<uint32_t>(), C.big_tiles.as<int32_t>(), &C.sc()->n_handoff, mt_x};
    }

    // cell-list rounds: round r reads the change bits of round r - 1 from
    // bitmap r % 3, writes its own to (r + 1) % 3 and clears (r + 2) % 3.
    // From scratch (start_pos: the seeds), round 0 reads the seed cells from
    // bitmap 0: their neighbours are the cells the first pass can change.
    int cb_stride = 0, cb_words = 0;
    const bool start_bits = cells && start_pos && n_start > 0;
    if (cells) {
        cb_stride = ceil_div(tiles_x * tw, 32) + 1;
        cb_words = cb_stride * cv.Hd;
        C.cellbits.ensure((size_t)cb_words * 3 * 4);
        IDL_CUDA(cudaMemsetAsync(C.cellbits.ptr, 0, (size_t)cb_words * 3 * 4, C.stream));
        if (start_bits) {
            k_mark_cells<<<(unsigned)((n_start + 255) / 256), 256, 0, C.stream>>>(start_pos, n_start,
                                                                                C.cellbits.as<uint32_t>(), cb_stride);
            IDL_LAUNCH();
        }
    }
    auto cell_bits = [&](int64_t rr) {
        uint32_t* b = C.cellbits.as<uint32_t>();
        return CellBits{rr > 0 || start_bits ? b + (size_t)(rr % 3) * cb_words : nullptr,
                        b + (size_t)((rr + 1) % 3) * cb_words,
                        rr > 0 ? b + (size_t)((rr + 2) % 3) * cb_words : nullptr, cb_stride, cb_words};
    };

    const int grid = std::min(n_tiles, C.num_sms * 3);
    int64_t r = 0;
    // a fixed number of rounds goes out in one group (one host round trip);
    // to convergence, groups double from 2
    int group = round_limit > 0 ? (int)std::min<int64_t>(round_limit, 64) : 2;
    int32_t remaining = 0;
    if (persistent) {
        // every round in one cooperative launch, rounds separated by the grid barrier
        const int64_t cap = round_limit >= 0 ? round_limit : max_rounds;
        switch (base_shape) {
        case 1: r = run_rounds_keys<16, 8>(C, cv, counts, epoch, tiles_x, tiles_y, cap, last); break;
        case 2: r = run_rounds_keys<8, 4>(C, cv, counts, epoch, tiles_x, tiles_y, cap, last); break;
        case 3: r = run_rounds_keys<16, 12>(C, cv, counts, epoch, tiles_x, tiles_y, cap, last); break;
        default: r = run_rounds_keys<8, 8>(C, cv, counts, epoch, tiles_x, tiles_y, cap, last);
        }
        IDL_CUDA(cudaMemcpy(&remaining, counts + r, 4, cudaMemcpyDeviceToHost));
        if (round_limit < 0 && remaining != 0) throw Error(IDL_ERR_INTERNAL, "Voronoi propagation did not converge");
    }
    for (; !persistent;) {
        for (int g = 0; g < group && r < max_rounds && (round_limit < 0 || r < round_limit); ++g, ++r) {
            const int32_t* srcp = C.lab[r & 1].as<int32_t>();
            int32_t* dstp = C.lab[(r + 1) & 1].as<int32_t>();
            const int32_t* lin = C.tiles[r & 1].as<int32_t>();
            int32_t* lout = C.tiles[(r + 1) & 1].as<int32_t>();
            const long long base = (long long)r * steps;
            const int32_t stamp_next = epoch + int32_t(r) + 1;
            int32_t* stamp = C.stamps.as<int32_t>();
            if (cells) {
                Handoff ho{nullptr, nullptr, nullptr, 0};
                if (handoff && r + 1 == round_limit) {
                    ho = ho_last;
                    IDL_CUDA(cudaMemsetAsync(ho.bits, 0, (size_t)sparse_bits_words(cv) * 2 * 4, C.stream));
                    IDL_CUDA(cudaMemsetAsync(ho.count, 0, 4, C.stream));
                }
                const CellBits cb = cell_bits(r);
                switch (tile - 2 * N_KEY_SHAPES) {
                case 1:
                    launch_round_cells<64, 64, 4>(C, srcp, dstp, cv, lin, counts + r, lout, counts + r + 1, stamp,
                                                  stamp_next, tiles_x, tiles_y, base, last, ho, cb);
                    break;
                case 2:
                    launch_round_cells<128, 64, 8>(C, srcp, dstp, cv, lin, counts + r, lout, counts + r + 1, stamp,
                                                   stamp_next, tiles_x, tiles_y, base, last, ho, cb);
                    break;
                case 3:
                    launch_round_cells<128, 128, 16>(C, srcp, dstp, cv, lin, counts + r, lout, counts + r + 1, stamp,
                                                     stamp_next, tiles_x, tiles_y, base, last, ho, cb);
                    break;
                default:
                    launch_round_cells<64, 64, 8>(C, srcp, dstp, cv, lin, counts + r, lout, counts + r + 1, stamp,
                                                  stamp_next, tiles_x, tiles_y, base, last, ho, cb);
                }
            } else if (keys) {
                switch (base_shape) {
                case 1:
                    launch_round_keys<16, 8>(C, 2, srcp, dstp, cv, lin, counts + r, lout, counts + r + 1, stamp,
                                             stamp_next, tiles_x, tiles_y, base, last);
                    break;
                case 2:
                    launch_round_keys<8, 4>(C, 3, srcp, dstp, cv, lin, counts + r, lout, counts + r + 1, stamp,
                                            stamp_next, tiles_x, tiles_y, base, last);
                    break;
                case 3:
                    launch_round_keys<16, 12>(C, 2, srcp, dstp, cv, lin, counts + r, lout, counts + r + 1, stamp,
                                              stamp_next, tiles_x, tiles_y, base, last);
                    break;
                default:
                    launch_round_keys<8, 8>(C, 3, srcp, dstp, cv, lin, counts + r, lout, counts + r + 1, stamp,
                                            stamp_next, tiles_x, tiles_y, base, last);
                }
            } else if (mode == IDL_MODE_NUMPY) {
                k_round<IDL_MODE_NUMPY><<<grid, THREADS, 0, C.stream>>>(
                    srcp, dstp, cv.pitch, cv.Wd, cv.Hd, pos, lin, counts + r, lout, counts + r + 1, stamp,
                    stamp_next, tiles_x, tiles_y, base, last);
            } else {
                k_round<IDL_MODE_REFERENCE><<<grid, THREADS, 0, C.stream>>>(
                    srcp, dstp, cv.pitch, cv.Wd, cv.Hd, pos, lin, counts + r, lout, counts + r + 1, stamp,
                    stamp_next, tiles_x, tiles_y, base, last);
            }
            IDL_LAUNCH();
        }
        // With the hand-off, the rounds, the plane copy and the persistent
        // kernel all take their list lengths from the device: no read-back
        // here (the kernel's own brings the scalars; an empty list ends it).
        if (handoff && r == round_limit) {
            remaining = -1;
            break;
        }
        // the list length and the scalars (last change, hand-off count) in one read-back
        IDL_CUDA(cudaMemcpyAsync(&C.sc()->tile_remaining, counts + r, 4, cudaMemcpyDeviceToDevice, C.stream));
        C.fetch_scalars();
        remaining = C.host_sc->tile_remaining;
        if (remaining == 0) break;
        if (round_limit >= 0 && r >= round_limit) break;
        if (r >= max_rounds) throw Error(IDL_ERR_INTERNAL, "Voronoi propagation did not converge");
        group = std::min(group * 2, 8);
    }
    if (persistent) C.fetch_scalars();   // the loop above read them with its last list length
    // after a hand-off (remaining < 0: not read) these are refreshed below
    int64_t lc = C.host_sc->last_change;
    int64_t passes = lc < 0 ? 1 : lc + 2;
    if (C.prof.enabled) {
        // tile rounds: 8 B per inner cell (label in, label out) per processed
        // tile and round, in micro-tile-pass equivalents for the tile count
        std::vector<int32_t> h((size_t)r + 1);
        IDL_CUDA(cudaMemcpy(h.data(), counts, h.size() * 4, cudaMemcpyDeviceToHost));
        int64_t tiles = 0, rounds = 0;
        for (int64_t i = 0; i < r; ++i) {
            tiles += h[i];
            rounds += h[i] > 0;
        }
        C.prof.tiles = tiles * (tw / 8) * (th / 8) * steps;
        C.prof.rounds = rounds;
        C.prof.prop_bytes = (double)tiles * tw * th * 8.0;
        C.prof.passes = passes;
        C.prof.tile_w = tw;
        C.prof.tile_h = th;
        C.prof.steps_per_round = steps;
    }
    if (remaining != 0) {
        // Hand the tail to the sparse kernel: the latest state goes to plane 0.
        if (r & 1) std::swap(C.lab[0], C.lab[1]);
        int64_t sparse = 0;
        if (handoff && r == round_limit) {
            // Its first work list is the last round's: the micro-tiles that can
            // change.  The planes differ only on tiles the last round changed,
            // all of which are on the next round's list: make them agree.
            const int copy_grid = std::min(n_tiles, C.num_sms * 8);
            k_copy_tiles<<<copy_grid, 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), C.lab[1].as<int32_t>(), cv.pitch,
                                                         cv.Wd, cv.Hd, C.tiles[r & 1].as<int32_t>(), counts + r,
                                                         tiles_x, tw, th);
            IDL_LAUNCH();
            sparse = propagate_sparse_from_marks(C, cv, pos, C.big_tiles.as<int32_t>(), -1, keys);
            lc = C.host_sc->last_change;   // read back with the persistent kernel's state
            passes = lc < 0 ? 1 : lc + 2;
        } else {
            // Its first work list is every micro-tile of the tiles the next
            // round would have run (a superset of those that can change).
            C.big_tiles.ensure((size_t)remaining * 4);
            IDL_CUDA(cudaMemcpyAsync(C.big_tiles.ptr, C.tiles[r & 1].ptr, (size_t)remaining * 4,
                                     cudaMemcpyDeviceToDevice, C.stream));
            sparse = propagate_sparse_from_tiles(C, cv, pos, C.big_tiles.as<int32_t>(), remaining, tiles_x, tw, th,
                                                 keys);
        }
        passes = sparse >= 2 ? r * steps + sparse : passes;
        if (C.prof.enabled) C.prof.passes = passes;
    }
    return passes;
}

}  // namespace

}  // namespace idl
