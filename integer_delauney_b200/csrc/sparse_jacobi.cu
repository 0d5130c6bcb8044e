// Stage (a), reference semantics: the synchronous Jacobi fixed point of
// src/cuda/voronoi.cu:32-53,100-113, computed by one persistent cooperative
// kernel that steps only the parts of the canvas that can still change.
//
// Why sparse.  At 4096 x 4096 with 200 000 uniform seeds the reference runs
// 51 full-canvas passes (51 x 17 M cell updates) but only 18 M labels ever
// change and only 68 M cell evaluations have a changed neighbour; the
// clustered case runs 1 100 passes with a thin moving front.  A cell can only
// change in pass t+1 if a cell of its closed 4-neighbourhood changed in pass t
// (keys only improve, and a pass is a pure function of the neighbourhood), so
// per pass only the 8 x 8 micro-tiles holding or bordering a change need work.
//
// How.  Pass t reads label plane t%2 and writes plane (t+1)%2.  The
// micro-tiles to run in pass t form work list t%2.  A micro-tile whose cells
// change lists itself, and the neighbour across any edge whose row or column
// changed, for pass t+1; bitmap (t+1)%2 deduplicates them (each task clears
// its own bit of bitmap t%2, which is then pass t+1's target).  A processed
// micro-tile always writes all its cells, so any micro-tile not being
// processed holds the same state in both planes (by induction), and the
// 1-cell border reads of an active micro-tile are always current.  Passes are
// separated by a grid-wide barrier with a bounded wait; no host round trip
// happens until the list runs empty.  Each warp advances GROUP micro-tiles at
// once, with all loads issued before any compute, and next-pass list entries
// are staged per block so the list counter sees one atomic per block per pass.
//
// Coherence: planes, lists and bitmaps are rewritten by other blocks between
// passes, so they are read with ld.global.cg (L2), never through L1 or the
// read-only path; barrier arrival and departure are release/acquire.
#include "context.cuh"
#include "gridsync.cuh"
#include "stencil.cuh"

#include <cuda/atomic>
#include <mutex>
#include <vector>

namespace idl {
namespace {

constexpr int MT = MICRO_TILE;              // micro-tile side
constexpr int SJ_THREADS = 1024;
constexpr int SJ_WARPS = SJ_THREADS / 32;
constexpr int GROUP = 2;                    // micro-tiles a warp advances together
constexpr int STAGE = 6144;                 // per-block staging of next-pass list entries

// The Jacobi update of one cell owned by `b` from its four neighbours' owners
// (geometry_device.cuh:40-66).  The owner's and the candidates' distances are
// gathered together so the seed-table loads overlap; the choice is then pure
// arithmetic.
__device__ __forceinline__ void best_of4(int32_t& b, int32_t n0, int32_t n1, int32_t n2, int32_t n3, int x, int y,
                                         const uint32_t* __restrict__ pos)
{
    const int32_t own = b;
    const int32_t n[4] = {n0, n1, n2, n3};
    int32_t d[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) d[j] = (n[j] >= 0 && n[j] != own) ? dist2(x, y, __ldg(&pos[n[j]])) : FAR;
    int32_t bd = own >= 0 ? dist2(x, y, __ldg(&pos[own])) : FAR;
    int32_t bl = own;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (n[j] < 0 || n[j] == own) continue;
        if (d[j] < bd || (d[j] == bd && n[j] > bl)) {
            bl = n[j];
            bd = d[j];
        }
    }
    b = bl;
}

// best_of4 on owner keys (stencil.cuh): no seed-table loads.
__device__ __forceinline__ void best_of4_keys(int32_t& b, int32_t n0, int32_t n1, int32_t n2, int32_t n3, int x,
                                              int y)
{
    int32_t bd = b >= 0 ? key_dist2(x, y, b) : FAR;
    relax_key(b, bd, n0, x, y);
    relax_key(b, bd, n1, x, y);
    relax_key(b, bd, n2, x, y);
    relax_key(b, bd, n3, x, y);
}

// Per-block staging of next-pass list entries.  Groups reserve slots with
// atomicAdd on *n; a group whose slots would run past STAGE goes to the global
// list instead and lowers *cut to its first slot, so that only the prefix
// s_list[0, min(*n, *cut)) -- which every earlier group filled -- is flushed.
struct Stage {
    int32_t* list;
    int* n;
    int* cut;
};

// Advance `cnt` (<= GROUP, warp-uniform) micro-tiles by one Jacobi pass and
// list the micro-tiles pass t+1 must run.  KEYS: labels are owner keys.
template <bool KEYS>
__device__ __forceinline__ void advance(const int (&ids)[GROUP], int cnt, const int32_t* cur, int32_t* nxt,
                                        int pitch, int Wd, int Hd, int mt_x, int mt_y,
                                        const uint32_t* __restrict__ pos, uint32_t* bin, uint32_t* bout,
                                        int32_t* lout, int32_t* count_out, Stage st, int lane)
{
    const int r = lane >> 2, c0 = (lane & 3) * 2;
    int32_t a0[GROUP], a1[GROUP], u0[GROUP], u1[GROUP], d0[GROUP], d1[GROUP], lf[GROUP], rt[GROUP];
    int gx[GROUP], gy[GROUP];
    bool in0[GROUP], in1[GROUP];
    // loads: own two cells and, on the micro-tile's edges, the cells across
#pragma unroll
    for (int k = 0; k < GROUP; ++k) {
        a0[k] = a1[k] = u0[k] = u1[k] = d0[k] = d1[k] = lf[k] = rt[k] = OUTSIDE;
        in0[k] = in1[k] = false;
        gx[k] = gy[k] = 0;
        if (k < cnt) {
            const int mx = ids[k] & 0xFFFF, my = ids[k] >> 16;
            const int lin = my * mt_x + mx;
            if (lane == 0) atomicAnd(&bin[lin >> 5], ~(1u << (lin & 31)));
            gx[k] = mx * MT + c0;
            gy[k] = my * MT + r;
            const bool row_in = gy[k] < Hd;
            in0[k] = row_in && gx[k] < Wd;
            in1[k] = row_in && gx[k] + 1 < Wd;
            const size_t o = (size_t)gy[k] * pitch + gx[k];
            if (in1[k]) {
                const int2 v = __ldcg(reinterpret_cast<const int2*>(cur + o));
                a0[k] = v.x;
                a1[k] = v.y;
            } else if (in0[k]) {
                a0[k] = __ldcg(&cur[o]);
            }
            if (r == 0 && gy[k] > 0) {
                if (in0[k]) u0[k] = __ldcg(&cur[o - pitch]);
                if (in1[k]) u1[k] = __ldcg(&cur[o - pitch + 1]);
            }
            if (r == MT - 1 && gy[k] + 1 < Hd) {
                if (in0[k]) d0[k] = __ldcg(&cur[o + pitch]);
                if (in1[k]) d1[k] = __ldcg(&cur[o + pitch + 1]);
            }
            if ((lane & 3) == 0 && in0[k] && gx[k] > 0) lf[k] = __ldcg(&cur[o - 1]);
            if ((lane & 3) == 3 && in1[k] && gx[k] + 2 < Wd) rt[k] = __ldcg(&cur[o + 2]);
        }
    }
#pragma unroll
    for (int k = 0; k < GROUP; ++k) {
        if (k >= cnt) break;
        // neighbours inside the micro-tile come from the lanes that own them
        const int32_t su0 = __shfl_up_sync(FULL, a0[k], 4), su1 = __shfl_up_sync(FULL, a1[k], 4);
        const int32_t sd0 = __shfl_down_sync(FULL, a0[k], 4), sd1 = __shfl_down_sync(FULL, a1[k], 4);
        const int32_t sl = __shfl_up_sync(FULL, a1[k], 1), sr = __shfl_down_sync(FULL, a0[k], 1);
        if (r != 0) { u0[k] = su0; u1[k] = su1; }
        if (r != MT - 1) { d0[k] = sd0; d1[k] = sd1; }
        if ((lane & 3) != 0) lf[k] = sl;
        if ((lane & 3) != 3) rt[k] = sr;

        // cells below UNDEF are walls between packed images: never updated
        int32_t b0 = a0[k], b1 = a1[k];
        if (KEYS) {
            int32_t c0 = b0, c1 = b1;
            best_of4_keys(c0, lf[k], a1[k], u0[k], d0[k], gx[k], gy[k]);
            best_of4_keys(c1, a0[k], rt[k], u1[k], d1[k], gx[k] + 1, gy[k]);
            b0 = (in0[k] && b0 >= UNDEF) ? c0 : b0;
            b1 = (in1[k] && b1 >= UNDEF) ? c1 : b1;
        } else {
            if (in0[k] && b0 >= UNDEF && (lf[k] != b0 || a1[k] != b0 || u0[k] != b0 || d0[k] != b0))
                best_of4(b0, lf[k], a1[k], u0[k], d0[k], gx[k], gy[k], pos);
            if (in1[k] && b1 >= UNDEF && (a0[k] != b1 || rt[k] != b1 || u1[k] != b1 || d1[k] != b1))
                best_of4(b1, a0[k], rt[k], u1[k], d1[k], gx[k] + 1, gy[k], pos);
        }
        const size_t o = (size_t)gy[k] * pitch + gx[k];
        if (in1[k]) *reinterpret_cast<int2*>(nxt + o) = make_int2(b0, b1);
        else if (in0[k]) nxt[o] = b0;

        const bool ch0 = b0 != a0[k], ch1 = b1 != a1[k];
        const unsigned any = __ballot_sync(FULL, ch0 || ch1);
        if (any) {
            const unsigned left = __ballot_sync(FULL, ch0 && (lane & 3) == 0);
            const unsigned right = __ballot_sync(FULL, ch1 && (lane & 3) == 3);
            // list entries are packed (mx | my << 16); the dedup bitmaps use
            // the linear index my * mt_x + mx
            const int mx = ids[k] & 0xFFFF, my = ids[k] >> 16;
            const int mt = my * mt_x + mx;
            int target = -1, packed = 0;
            if (lane == 0) { target = mt; packed = ids[k]; }
            if (lane == 1 && (any & 0xFu) && my > 0) { target = mt - mt_x; packed = ids[k] - 0x10000; }
            if (lane == 2 && (any & 0xF0000000u) && my + 1 < mt_y) { target = mt + mt_x; packed = ids[k] + 0x10000; }
            if (lane == 3 && left && mx > 0) { target = mt - 1; packed = ids[k] - 1; }
            if (lane == 4 && right && mx + 1 < mt_x) { target = mt + 1; packed = ids[k] + 1; }
            bool fresh = false;
            if (target >= 0) {
                const uint32_t bit = 1u << (target & 31);
                fresh = !(atomicOr(&bout[target >> 5], bit) & bit);
            }
            const unsigned fb = __ballot_sync(FULL, fresh);
            if (fb) {
                const int m = __popc(fb);
                int base = 0;
                if (lane == 0) base = atomicAdd(st.n, m);
                base = __shfl_sync(FULL, base, 0);
                const int rank = __popc(fb & ((1u << lane) - 1u));
                if (base + m <= STAGE) {
                    if (fresh) st.list[base + rank] = packed;
                } else {
                    int gbase = 0;
                    if (lane == 0) {
                        atomicMin(st.cut, base);
                        gbase = atomicAdd(count_out, m);
                    }
                    gbase = __shfl_sync(FULL, gbase, 0);
                    if (fresh) lout[gbase + rank] = packed;
                }
            }
        }
    }
}

// Appends `packed` (micro-tile index `target`) to the next work list when
// `want` and its bit in `bout` was clear.  Warp-wide; staging as in advance.
__device__ __forceinline__ void append_fresh(bool want, int target, int32_t packed, uint32_t* bout, int32_t* lout,
                                             int32_t* count_out, Stage st, int lane)
{
    bool fresh = false;
    if (want) {
        const uint32_t bit = 1u << (target & 31);
        fresh = !(atomicOr(&bout[target >> 5], bit) & bit);
    }
    const unsigned fb = __ballot_sync(FULL, fresh);
    if (!fb) return;
    const int m = __popc(fb);
    int base = 0;
    if (lane == 0) base = atomicAdd(st.n, m);
    base = __shfl_sync(FULL, base, 0);
    const int rank = __popc(fb & ((1u << lane) - 1u));
    if (base + m <= STAGE) {
        if (fresh) st.list[base + rank] = packed;
    } else {
        int gbase = 0;
        if (lane == 0) {
            atomicMin(st.cut, base);
            gbase = atomicAdd(count_out, m);
        }
        gbase = __shfl_sync(FULL, gbase, 0);
        if (fresh) lout[gbase + rank] = packed;
    }
}

// Round mode.  Once the work list is short, the kernel advances RK passes per
// grid barrier: a warp takes one micro-tile with an RK-cell halo (a 16 x 16
// region; lane l holds region row l / 2, columns 8 (l % 2) .. + 7, in
// registers) and runs RK Jacobi passes on it, neighbours by shuffles and
// region cells beyond the canvas OUTSIDE.  Errors from the region's frozen
// edge travel one cell per pass, so after RK passes the inner 8 x 8 cells are
// exact (the light cone of the tile rounds); they go to the other plane.
// Next list: the micro-tile itself if any inner cell changed in the round
// (so that, rewritten next round, its planes agree again), and each
// neighbour that an inner cell changed in the round's last pass can reach in
// RK passes (the state one pass back is otherwise stable around it, so the
// next RK passes cannot change it).  With RK = MT / 2 the reach of a cell is
// its quadrant's side and corner neighbours.
constexpr int RK = 4;
constexpr int RR = MT + 2 * RK;
static_assert(RR == 16 && MT == 8 && RK == MT / 2, "lane layout: 16 rows of two 8-cell halves");

template <bool KEYS>
__device__ __forceinline__ void round_mt(int32_t id, const int32_t* cur, int32_t* nxt, int pitch, int Wd, int Hd,
                                         int mt_x, int mt_y, const uint32_t* __restrict__ pos, uint32_t* bin,
                                         uint32_t* bout, int32_t* lout, int32_t* count_out, Stage st, int lane,
                                         int pass0, int& last_pass)
{
    const int mx = id & 0xFFFF, my = id >> 16;
    const int mt = my * mt_x + mx;
    if (lane == 0) atomicAnd(&bin[mt >> 5], ~(1u << (mt & 31)));
    const int r = lane >> 1, h = lane & 1;
    const int gy = my * MT - RK + r;
    const int gx0 = mx * MT - RK + 8 * h;
    const bool row_in = gy >= 0 && gy < Hd;
    int32_t c[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int gx = gx0 + j;
        c[j] = (row_in && gx >= 0 && gx < Wd) ? __ldcg(cur + (size_t)gy * pitch + gx) : OUTSIDE;
    }
    // this lane's inner cells: region rows RK .. RK + MT - 1, columns RK .. RK + MT - 1
    const bool inner_row = r >= RK && r < RK + MT;
    // (registers are indexed statically: h picks c[0..3] or c[4..7])
    int32_t c0[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) c0[q] = h ? c[q] : c[4 + q];
    int last = -1;
    bool ch = false;   // an inner cell of this lane changed in the latest pass
#pragma unroll 1
    for (int p = 0; p < RK; ++p) {
        const int32_t lft = __shfl_up_sync(FULL, c[7], 1), rgt = __shfl_down_sync(FULL, c[0], 1);
        int32_t nv[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int32_t up = __shfl_up_sync(FULL, c[j], 2), dn = __shfl_down_sync(FULL, c[j], 2);
            const int32_t L = j > 0 ? c[j - 1] : (h ? lft : OUTSIDE);
            const int32_t R = j < 7 ? c[j + 1] : (h ? OUTSIDE : rgt);
            const int32_t U = r > 0 ? up : OUTSIDE;
            const int32_t D = r < RR - 1 ? dn : OUTSIDE;
            int32_t b = c[j];
            if (KEYS) {
                int32_t k = b;
                best_of4_keys(k, L, R, U, D, gx0 + j, gy);
                b = b >= UNDEF ? k : b;
            } else if (b >= UNDEF && (L != b || R != b || U != b || D != b)) {
                best_of4(b, L, R, U, D, gx0 + j, gy, pos);
            }
            nv[j] = b;
        }
        ch = false;
#pragma unroll
        for (int q = 0; q < 4; ++q) ch = ch || (h ? nv[q] != c[q] : nv[4 + q] != c[4 + q]);
        ch = ch && inner_row;
        if (__any_sync(FULL, ch)) last = p;
#pragma unroll
        for (int j = 0; j < 8; ++j) c[j] = nv[j];
    }
    if (inner_row && gy < Hd) {
        const int gxi = mx * MT + 4 * h;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (gxi + q < Wd) nxt[(size_t)gy * pitch + gxi + q] = h ? c[q] : c[4 + q];
    }
    bool moved = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) moved = moved || (h ? c[q] : c[4 + q]) != c0[q];
    if (!__any_sync(FULL, moved && inner_row)) return;
    last_pass = max(last_pass, pass0 + last);
    // quadrants of the inner tile with a change in the last pass: lanes 8..15
    // hold its top half, 16..23 the bottom; even lanes the left half
    const unsigned lb = __ballot_sync(FULL, ch);   // ch: changes of the last pass
    const bool tl = lb & 0x00005500u, tr = lb & 0x0000AA00u, bl = lb & 0x00550000u, br = lb & 0x00AA0000u;
    int dx = 0, dy = 0;
    bool want = false;
    switch (lane) {
    case 0: want = true; break;
    case 1: dx = -1; want = tl || bl; break;
    case 2: dx = 1; want = tr || br; break;
    case 3: dy = -1; want = tl || tr; break;
    case 4: dy = 1; want = bl || br; break;
    case 5: dx = -1; dy = -1; want = tl; break;
    case 6: dx = 1; dy = -1; want = tr; break;
    case 7: dx = -1; dy = 1; want = bl; break;
    case 8: dx = 1; dy = 1; want = br; break;
    default: break;
    }
    const int nx = mx + dx, ny = my + dy;
    want = want && nx >= 0 && nx < mt_x && ny >= 0 && ny < mt_y;
    append_fresh(want, ny * mt_x + nx, pack_mt(nx, ny), bout, lout, count_out, st, lane);
}

// Entering the round mode: the list holds the micro-tiles that can change in
// the next pass; a round needs those that can change in the next RK passes,
// which lie within one micro-tile of them (RK <= MT).  Warp-wide per entry.
__device__ __forceinline__ void dilate_mt(int32_t id, int mt_x, int mt_y, uint32_t* bin, uint32_t* bout,
                                          int32_t* lout, int32_t* count_out, Stage st, int lane)
{
    const int mx = id & 0xFFFF, my = id >> 16;
    const int mt = my * mt_x + mx;
    if (lane == 0) atomicAnd(&bin[mt >> 5], ~(1u << (mt & 31)));
    const int nx = mx + (lane % 3) - 1, ny = my + (lane / 3) - 1;
    const bool want = lane < 9 && nx >= 0 && nx < mt_x && ny >= 0 && ny < mt_y;
    append_fresh(want, ny * mt_x + nx, pack_mt(nx, ny), bout, lout, count_out, st, lane);
}

// counts[g]: micro-tiles listed for work-list generation g, which runs list
// g%2 and appends generation g+1's micro-tiles to list (g+1)%2.  A generation
// is one pass while the list is longer than rounds_below, then (once) the
// dilation into the round mode, then rounds of RK passes.  The mode is the
// same in every block: it depends only on the list lengths all of them read.
template <bool KEYS>
__global__ void __launch_bounds__(SJ_THREADS, 1)
k_sparse_jacobi(int32_t* plane0, int32_t* plane1, int pitch, int Wd, int Hd, const uint32_t* __restrict__ pos,
                uint32_t* bits0, uint32_t* bits1, int32_t* list0, int32_t* list1, int32_t* counts, int max_steps,
                int mt_x, int mt_y, int rounds_below, GridSync* gs, unsigned long long* trace)
{
    // trace (profiling only): the global timer at the start and after each
    // generation, and from trace[max_steps + 2] on the passes each advanced
    if (trace && blockIdx.x == 0 && threadIdx.x == 0) trace[0] = global_timer_ns();
    __shared__ int32_t s_list[STAGE];
    __shared__ int s_n, s_cut, s_base, s_m, s_last;
    const int lane = threadIdx.x & 31;
    // warp slots numbered across the blocks first, so that a short list
    // spreads over every SM instead of filling the first blocks' warps
    const int gwarp = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    const int nwarps = gridDim.x * SJ_WARPS;
    unsigned gen_local = 0;
    int t = 0;              // passes done
    int g = 0;              // generation
    int par = 0;            // plane holding the current state
    bool rounds = false;
    bool converged = false;
    for (; t < max_steps; ++g) {
        const int n = *reinterpret_cast<volatile int32_t*>(&counts[g]);
        if (n == 0) {
            converged = true;
            break;
        }
        int kind = 0;   // 0: one pass, 1: dilation into the round mode, 2: a round of RK passes
        if (rounds) {
            kind = 2;
        } else if (n <= rounds_below) {
            kind = 1;
            rounds = true;
        }
        if (threadIdx.x == 0) {
            s_n = 0;
            s_cut = STAGE;
            s_last = -1;
        }
        __syncthreads();
        const int32_t* cur = par ? plane1 : plane0;
        int32_t* nxt = par ? plane0 : plane1;
        uint32_t* bin = (g & 1) ? bits1 : bits0;
        uint32_t* bout = (g & 1) ? bits0 : bits1;
        const int32_t* lin = (g & 1) ? list1 : list0;
        int32_t* lout = (g & 1) ? list0 : list1;
        const Stage stg{s_list, &s_n, &s_cut};
        if (kind == 0) {
            for (int i0 = gwarp * GROUP; i0 < n; i0 += nwarps * GROUP) {
                int ids[GROUP];
                const int cnt = min(GROUP, n - i0);
#pragma unroll
                for (int k = 0; k < GROUP; ++k) ids[k] = k < cnt ? __ldcg(&lin[i0 + k]) : 0;
                advance<KEYS>(ids, cnt, cur, nxt, pitch, Wd, Hd, mt_x, mt_y, pos, bin, bout, lout, counts + g + 1,
                              stg, lane);
            }
        } else if (kind == 1) {
            // the list was made by changes of pass t - 1 (none if t == 0)
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(&gs->last1, t);
            for (int i = gwarp; i < n; i += nwarps)
                dilate_mt(__ldcg(&lin[i]), mt_x, mt_y, bin, bout, lout, counts + g + 1, stg, lane);
        } else {
            int last = -1;
            for (int i = gwarp; i < n; i += nwarps)
                round_mt<KEYS>(__ldcg(&lin[i]), cur, nxt, pitch, Wd, Hd, mt_x, mt_y, pos, bin, bout, lout,
                               counts + g + 1, stg, lane, t, last);
            if (lane == 0 && last >= 0) atomicMax(&s_last, last);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int m = min(s_n, s_cut);
            s_m = m;
            s_base = m ? atomicAdd(&counts[g + 1], m) : 0;
            if (s_last >= 0) atomicMax(&gs->last1, s_last + 1);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < s_m; i += blockDim.x) lout[s_base + i] = s_list[i];
        const int advanced = kind == 0 ? 1 : (kind == 2 ? RK : 0);
        t += advanced;
        if (advanced) par ^= 1;
        if (!grid_sync(gs, gridDim.x, gen_local)) return;
        if (trace && blockIdx.x == 0 && threadIdx.x == 0) {
            trace[g + 1] = global_timer_ns();
            trace[max_steps + 2 + g] = (unsigned long long)advanced;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // the pass count of the one-pass schedule: the first pass whose list
        // would be empty (last change + 2, or 1 if nothing ever changed)
        gs->passes = !converged ? max_steps : (rounds ? atomicAdd(&gs->last1, 0) + 1 : t);
        gs->gens = g;
    }
}

// The barrier above on its own: `rounds` barriers of a grid that waits for
// `expected` arrivals.  With expected > gridDim.x some arrivals never come, so
// every block's wait runs out after spin_limit polls and the error flag is set.
__global__ void k_barrier_selftest(GridSync* gs, unsigned expected, unsigned spin_limit, int rounds)
{
    unsigned gen_local = 0;
    int r = 0;
    for (; r < rounds; ++r)
        if (!grid_sync(gs, expected, gen_local, spin_limit)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) gs->passes = r;
}

__global__ void k_iota_list(int32_t* __restrict__ list, int n, int mt_x, int32_t* __restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) list[i] = pack_mt(i % mt_x, i / mt_x);
    if (i == 0) *count = n;
}

// Initial work list of a continued propagation: the micro-tiles holding a new
// seed cell or one of its 4 neighbours (the only cells pass 0 can change).
__global__ void k_seed_tiles(const uint32_t* __restrict__ seed_pos, int n_new, int Wd, int Hd, int mt_x,
                             uint32_t* __restrict__ bits, int32_t* __restrict__ list, int32_t* __restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_new) return;
    const uint32_t p = seed_pos[i];
    const int x = pos_x(p), y = pos_y(p);
    const int dx[5] = {0, -1, 1, 0, 0}, dy[5] = {0, 0, 0, -1, 1};
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        const int cx = x + dx[j], cy = y + dy[j];
        if (cx < 0 || cy < 0 || cx >= Wd || cy >= Hd) continue;
        const int mt = (cy / MT) * mt_x + cx / MT;
        const uint32_t bit = 1u << (mt & 31);
        if (!(atomicOr(&bits[mt >> 5], bit) & bit)) list[atomicAdd(count, 1)] = pack_mt(cx / MT, cy / MT);
    }
}

__global__ void k_fill_bits(uint32_t* __restrict__ bits, int n_words, int n_items)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_words) return;
    const int k = n_items - w * 32;
    bits[w] = k >= 32 ? 0xFFFFFFFFu : (k <= 0 ? 0u : ((1u << k) - 1u));
}

}  // namespace

namespace {

// First work list from a list of big tiles: all their micro-tiles.  Big
// tiles are distinct, so their micro-tiles are too.
__global__ void k_expand_tiles(const int32_t* __restrict__ big, int big_tiles_x, int sub_x, int sub_y, int mt_x,
                               int mt_y, uint32_t* __restrict__ bits, int32_t* __restrict__ list,
                               int32_t* __restrict__ count)
{
    const int32_t b = big[blockIdx.x];
    const int bx = b % big_tiles_x, by = b / big_tiles_x;
    for (int j = threadIdx.x; j < sub_x * sub_y; j += blockDim.x) {
        const int mx = bx * sub_x + j % sub_x, my = by * sub_y + j / sub_x;
        if (mx >= mt_x || my >= mt_y) continue;
        const int mt = my * mt_x + mx;
        atomicOr(&bits[mt >> 5], 1u << (mt & 31));
        list[atomicAdd(count, 1)] = pack_mt(mx, my);
    }
}

}  // namespace

std::mutex& persistent_grid_lock(int device)
{
    static std::mutex locks[64];
    return locks[device & 63];
}

void grid_barrier_selftest(Context& C, int missing_arrivals, unsigned spin_limit)
{
    if (missing_arrivals < 0 || missing_arrivals > 1024) invalid("missing_arrivals must be in [0, 1024]");
    if (spin_limit < 1 || spin_limit > SPIN_LIMIT) invalid("spin_limit must be in [1, 2^24]");
    constexpr int rounds = 4;
    C.gsync.ensure(sizeof(GridSync));
    GridSync* gs = C.gsync.as<GridSync>();
    IDL_CUDA(cudaMemsetAsync(gs, 0, sizeof(GridSync), C.stream));
    unsigned expected = (unsigned)C.num_sms + (unsigned)missing_arrivals;
    int r = rounds;
    void* args[] = {&gs, &expected, &spin_limit, &r};
    IDL_CUDA(cudaLaunchCooperativeKernel((const void*)k_barrier_selftest, dim3(C.num_sms), dim3(128), args, 0,
                                         C.stream));
    count_launch();
    GridSync h{};
    IDL_CUDA(cudaMemcpyAsync(&h, gs, sizeof(GridSync), cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    if (h.error) throw Error(IDL_ERR_INTERNAL, "grid barrier timed out");
    if (h.passes != rounds) throw Error(IDL_ERR_INTERNAL, "grid barrier self-test did not complete its rounds");
}

int sparse_bits_words(const Canvas& cv) { return ceil_div(ceil_div(cv.Wd, MT) * ceil_div(cv.Hd, MT), 32); }

int64_t propagate_sparse_from_tiles(Context& C, const Canvas& cv, const uint32_t* pos, const int32_t* big_list,
                                    int n_big, int big_tiles_x, int big_w, int big_h, bool keys)
{
    if (big_w % MT != 0 || big_h % MT != 0) throw Error(IDL_ERR_INTERNAL, "tile sides must be micro-tile multiples");
    SparseStart st;
    st.big_list = big_list;
    st.n_big = n_big;
    st.big_tiles_x = big_tiles_x;
    st.sub_x = big_w / MT;
    st.sub_y = big_h / MT;
    return propagate_sparse_impl(C, cv, pos, st, keys);
}

int64_t propagate_sparse_from_marks(Context& C, const Canvas& cv, const uint32_t* pos, const int32_t* marked,
                                    int n_marked, bool keys)
{
    SparseStart st;
    st.marked = marked;
    st.n_marked = n_marked;
    return propagate_sparse_impl(C, cv, pos, st, keys);
}

int64_t propagate_sparse(Context& C, const Canvas& cv, const uint32_t* pos, const uint32_t* seed_pos,
                         int64_t n_new, bool keys)
{
    SparseStart st;
    st.seed_pos = seed_pos;
    st.n_new = n_new;
    return propagate_sparse_impl(C, cv, pos, st, keys);
}

int64_t propagate_sparse_impl(Context& C, const Canvas& cv, const uint32_t* pos, const SparseStart& st, bool keys)
{
    const int mt_x = ceil_div(cv.Wd, MT), mt_y = ceil_div(cv.Hd, MT);
    const int n_mt = mt_x * mt_y;
    const int n_words = ceil_div(n_mt, 32);
    // bound on passes: far above any real run; only stops a runaway loop
    const int max_steps = (int)std::min<int64_t>((int64_t)4 * (cv.Wd + cv.Hd) + 64, (1 << 29));
    C.tiles[0].ensure((size_t)n_mt * 4);
    C.tiles[1].ensure((size_t)n_mt * 4);
    if (st.marked && C.bits.bytes < (size_t)n_words * 2 * 4)
        throw Error(IDL_ERR_INTERNAL, "hand-off bitmap was not sized for this canvas");
    C.bits.ensure((size_t)n_words * 2 * 4);
    uint32_t* b0 = C.bits.as<uint32_t>();
    uint32_t* b1 = b0 + n_words;
    C.counts.ensure(((size_t)max_steps + 2) * 4);
    IDL_CUDA(cudaMemsetAsync(C.counts.ptr, 0, ((size_t)max_steps + 2) * 4, C.stream));
    int32_t* counts = C.counts.as<int32_t>();
    int32_t* l0 = C.tiles[0].as<int32_t>();
    int32_t* l1 = C.tiles[1].as<int32_t>();
    if (st.marked) {
        // the hand-off list (capacity n_mt) serves as the first list itself;
        // its length comes from the device (an empty one ends the kernel at
        // once); n_marked < 0: the host has not read it
        if (st.n_marked == 0) return 0;
        if (st.n_marked > n_mt) throw Error(IDL_ERR_INTERNAL, "hand-off list longer than the canvas");
        l0 = const_cast<int32_t*>(st.marked);
        IDL_CUDA(cudaMemcpyAsync(counts, &C.sc()->n_handoff, 4, cudaMemcpyDeviceToDevice, C.stream));
    } else if (st.big_list) {
        if (st.n_big == 0) return 0;
        IDL_CUDA(cudaMemsetAsync(b0, 0, (size_t)n_words * 2 * 4, C.stream));
        k_expand_tiles<<<(unsigned)st.n_big, 64, 0, C.stream>>>(st.big_list, st.big_tiles_x, st.sub_x, st.sub_y, mt_x,
                                                                mt_y, b0, l0, counts);
        IDL_LAUNCH();
    } else if (st.seed_pos) {
        if (st.n_new == 0) return 0;
        IDL_CUDA(cudaMemsetAsync(b0, 0, (size_t)n_words * 2 * 4, C.stream));
        k_seed_tiles<<<(unsigned)((st.n_new + 255) / 256), 256, 0, C.stream>>>(st.seed_pos, (int)st.n_new, cv.Wd,
                                                                               cv.Hd, mt_x, b0, l0, counts);
        IDL_LAUNCH();
    } else {
        k_fill_bits<<<(unsigned)((n_words + 255) / 256), 256, 0, C.stream>>>(b0, n_words, n_mt);
        IDL_LAUNCH();
        IDL_CUDA(cudaMemsetAsync(b1, 0, (size_t)n_words * 4, C.stream));
        k_iota_list<<<(unsigned)((n_mt + 255) / 256), 256, 0, C.stream>>>(l0, n_mt, mt_x, counts);
        IDL_LAUNCH();
    }
    C.gsync.ensure(sizeof(GridSync));
    IDL_CUDA(cudaMemsetAsync(C.gsync.ptr, 0, sizeof(GridSync), C.stream));

    int per_sm = 0;
    const void* kernel = keys ? (const void*)k_sparse_jacobi<true> : (const void*)k_sparse_jacobi<false>;
    IDL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SJ_THREADS, 0));
    if (per_sm < 1) throw Error(IDL_ERR_INTERNAL, "propagation kernel cannot be resident");
    const int grid = per_sm * C.num_sms;
    int32_t* p0 = C.lab[0].as<int32_t>();
    int32_t* p1 = C.lab[1].as<int32_t>();
    GridSync* gs = C.gsync.as<GridSync>();
    int pitch = cv.pitch, Wd = cv.Wd, Hd = cv.Hd, ms = max_steps, mx = mt_x, my = mt_y;
    int rb = std::max(C.tail_rounds_below, 0);
    unsigned long long* trace = nullptr;
    if (C.prof.enabled) {
        C.trace.ensure(((size_t)max_steps + 2) * 2 * 8);   // timestamps, then passes per generation
        trace = C.trace.as<unsigned long long>();
    }
    void* args[] = {&p0, &p1, &pitch, &Wd, &Hd, (void*)&pos, &b0, &b1, &l0, &l1, &counts, &ms, &mx, &my, &rb, &gs,
                    &trace};
    GridSync h{};
    {
        // One persistent grid per device at a time: the kernel fills every SM,
        // so two contexts' launches on different streams could not run side by
        // side anyway, and holding the device lock from launch to completion
        // keeps each grid's co-residency independent of the other streams.
        std::lock_guard<std::mutex> lock(persistent_grid_lock(C.device));
        IDL_CUDA(cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(SJ_THREADS), args, 0, C.stream));
        count_launch();
        IDL_CUDA(cudaMemcpyAsync(&h, gs, sizeof(GridSync), cudaMemcpyDeviceToHost, C.stream));
        // the scalars ride along: a caller that launched its tile rounds
        // without a read-back takes their last change from here
        IDL_CUDA(cudaMemcpyAsync(C.host_sc, C.scalars.ptr, sizeof(Scalars), cudaMemcpyDeviceToHost, C.stream));
        IDL_CUDA(cudaStreamSynchronize(C.stream));
    }
    if (h.error) throw Error(IDL_ERR_INTERNAL, "Voronoi propagation: grid barrier timed out");
    const int64_t passes = h.passes;
    if (passes >= max_steps) throw Error(IDL_ERR_INTERNAL, "Voronoi propagation did not converge");
    if (C.prof.enabled) {
        const int gens = h.gens;
        std::vector<int32_t> hc((size_t)gens + 1);
        IDL_CUDA(cudaMemcpy(hc.data(), counts, hc.size() * 4, cudaMemcpyDeviceToHost));
        std::vector<unsigned long long> ht((size_t)gens + 1), hs((size_t)std::max(gens, 1));
        IDL_CUDA(cudaMemcpy(ht.data(), trace, ht.size() * 8, cudaMemcpyDeviceToHost));
        if (gens > 0)
            IDL_CUDA(cudaMemcpy(hs.data(), trace + max_steps + 2, (size_t)gens * 8, cudaMemcpyDeviceToHost));
        C.prof.pass_ns.clear();
        C.prof.pass_tiles.clear();
        C.prof.pass_steps.clear();
        int64_t tiles = 0;
        double bytes = 0;
        for (int i = 0; i < gens; ++i) {
            C.prof.pass_ns.push_back((int64_t)(ht[i + 1] - ht[i]));
            C.prof.pass_tiles.push_back(hc[i]);
            C.prof.pass_steps.push_back((int32_t)hs[i]);
            tiles += (int64_t)hc[i] * (int64_t)hs[i];
            bytes += (double)hc[i] * (double)hs[i] * MT * MT * 8.0;   // label in, label out per cell-pass
        }
        // accumulated: a hybrid run has counted its tile rounds already
        C.prof.tiles += tiles;
        C.prof.rounds += gens;
        C.prof.passes = passes;
        C.prof.prop_bytes += bytes;
        C.prof.tile_w = MT;
        C.prof.tile_h = MT;
        C.prof.steps_per_round = 1;
    }
    return passes;
}

}  // namespace idl
