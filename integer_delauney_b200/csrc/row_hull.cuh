// Exact-semantics row pass shared by the single-image and batched pipelines:
// each cell of a row takes the best of its row's column candidates (the
// nearest seed of each column, from the column pass) in O(W) per row.
#pragma once

#include "common.cuh"

namespace idl {

// One block per row, O(W) whatever the seed layout.  With F_x =
// dy_x^2 + x^2 for each column x that has a candidate, the cell at column t
// takes the column minimising F_x - 2 t x (its squared distance minus t^2),
// ties to the larger x -- the higher id, since ids ascend with x across
// columns.  The minimisers over t are the vertices of the lower convex hull of
// the points (x, F_x) (the lower envelope of the columns' parabolas), in x
// order; a point on a hull edge's interior never wins alone and, where it
// ties, the edge's right end wins too, so the hull is kept strictly convex.
// Vertex k (k >= 1) wins from t = ceil((F_k - F_{k-1}) / (2 (x_k - x_{k-1})))
// on, a tie at that t included; the test "vertex k wins at t" is
// F_k - F_{k-1} <= t * 2 (x_k - x_{k-1}), exact in 64-bit integers.
//
// Each of the HULL_THREADS threads builds the hull of a chunk of columns
// (monotone chain, exact integer cross products); the chunk hulls are merged
// pairwise in log2(HULL_THREADS) levels, each merge finding the lower common
// tangent of two x-separated hulls by the standard two-sided walk.  A merged hull is a
// prefix of the left one and a suffix of the right one, so it is kept as
// linked chunk ranges, not copied.  The final hull is flattened; each thread
// finds the vertex of the first cell of its chunk by binary search and walks
// the hull across the chunk, so the whole row costs O(W + H).  Convex hull merging: Preparata & Hong (1977).
constexpr int HULL_THREADS = 128;              // threads (= chunks) per row
constexpr int32_t HULL_ABSENT = 0x7FFFFFFF;    // a column with no seed (real F < 2^31 - 1)
constexpr int HULL_MAX_W = 28000;              // F and two int16 index rows fit shared memory

// Dynamic shared memory of row_hull for rows of W columns.
inline size_t row_hull_smem(int W) { return (size_t)W * 4 + (size_t)((W + 1) & ~1) * 2 * 2; }

__device__ __forceinline__ long long hull_cross(int xa, int32_t fa, int xb, int32_t fb, int xc, int32_t fc)
{
    return (long long)(xb - xa) * (long long)(fc - fb) - (long long)(fb - fa) * (long long)(xc - xb);
}

// Exclusive prefix over the block's threads in thread order: the sum of the
// values of the threads before this one, or (max_op) their maximum (-1 for
// the first).  tmp: shared scratch of T / 32 + 1 ints.  Ends with a barrier.
template <int T>
__device__ __forceinline__ int block_excl_scan(int v, bool max_op, int* tmp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc = max_op ? max(inc, u) : inc + u;
    }
    if (lane == 31) tmp[warp] = inc;
    __syncthreads();
    int pre = max_op ? -1 : 0;
    for (int w = 0; w < warp; ++w) pre = max_op ? max(pre, tmp[w]) : pre + tmp[w];
    int excl = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
    if (lane == 0) excl = max_op ? -1 : 0;
    __syncthreads();   // tmp may be reused by the next scan
    return max_op ? max(pre, excl) : pre + excl;
}

// One row of Wd columns: lrow / drow hold each column's candidate label
// (negative: none) and its |dy|; out receives the row's labels.  Called by a
// block of HULL_THREADS threads with row_hull_smem(Wd) bytes of dynamic
// shared memory.
__device__ __forceinline__ void row_hull(const int32_t* __restrict__ lrow, const int32_t* __restrict__ drow, int Wd,
                                         int32_t* __restrict__ out)
{
    extern __shared__ __align__(16) int32_t hull_smem[];
    int32_t* F = hull_smem;                                          // Wd
    int16_t* hx = reinterpret_cast<int16_t*>(F + Wd);                // chunk hulls, each in its chunk's slots
    int16_t* flat = hx + ((Wd + 1) & ~1);                            // the final hull, in x order
    constexpr int T = HULL_THREADS;
    __shared__ int cb[T], ce[T], cprev[T], cnext[T], gfirst[T], glast[T];
    __shared__ int n_hull, scan_tmp[T / 32 + 1];
    const int tid = threadIdx.x;
    for (int x = tid; x < Wd; x += T) {
        const int32_t l = lrow[x];
        const uint32_t dy = (uint32_t)drow[x];
        F[x] = l >= 0 ? (int32_t)(dy * dy + (uint32_t)x * (uint32_t)x) : HULL_ABSENT;
    }
    __syncthreads();

    // chunk hulls; an odd chunk length keeps the threads' F reads on distinct banks
    const int C = ((Wd + T - 1) / T) | 1;
    const int x0 = tid * C, x1 = min(Wd, x0 + C);
    int h = x0;   // the chunk's hull occupies hx[x0, h); its top two points also in registers
    int x1t = 0, x2t = 0;
    int32_t f1t = 0, f2t = 0;
    for (int x = x0; x < x1; ++x) {
        const int32_t f = F[x];
        if (f == HULL_ABSENT) continue;
        while (h - x0 >= 2 && hull_cross(x2t, f2t, x1t, f1t, x, f) <= 0) {
            --h;
            x1t = x2t;
            f1t = f2t;
            if (h - x0 >= 2) {
                x2t = hx[h - 2];
                f2t = F[x2t];
            }
        }
        hx[h++] = (int16_t)x;
        x2t = x1t;
        f2t = f1t;
        x1t = x;
        f1t = f;
    }
    cb[tid] = x0;
    ce[tid] = h;
    cprev[tid] = cnext[tid] = -1;
    gfirst[tid] = glast[tid] = h > x0 ? tid : -1;
    __syncthreads();

    // merge groups of s chunks pairwise; a group's state lives at its first chunk
    for (int s = 1; s < T; s <<= 1) {
        if ((tid & (2 * s - 1)) == 0) {
            const int L = tid, R = tid + s;
            const int lf = gfirst[L], ll = glast[L], rf = gfirst[R], rl = glast[R];
            if (lf < 0) {
                gfirst[L] = rf;
                glast[L] = rl;
            } else if (rf >= 0) {
                int pc = ll, pi = ce[ll] - 1;   // p: the left hull's last point
                int qc = rf, qi = cb[rf];       // q: the right hull's first point
                int xp = hx[pi], xq = hx[qi];   // and their points, kept in registers
                int32_t fp = F[xp], fq = F[xq];
                for (;;) {
                    bool moved = false;
                    for (;;) {   // p leftwards while its predecessor does not turn left onto q
                        int ac, ai;
                        if (pi > cb[pc]) {
                            ac = pc;
                            ai = pi - 1;
                        } else if (pc != lf) {
                            ac = cprev[pc];
                            ai = ce[ac] - 1;
                        } else {
                            break;
                        }
                        const int xa = hx[ai];
                        const int32_t fa = F[xa];
                        if (hull_cross(xa, fa, xp, fp, xq, fq) > 0) break;
                        pc = ac;
                        pi = ai;
                        xp = xa;
                        fp = fa;
                        moved = true;
                    }
                    for (;;) {   // q rightwards while p, q and its successor do not turn left
                        int bc, bi;
                        if (qi + 1 < ce[qc]) {
                            bc = qc;
                            bi = qi + 1;
                        } else if (qc != rl) {
                            bc = cnext[qc];
                            bi = cb[bc];
                        } else {
                            break;
                        }
                        const int xb = hx[bi];
                        const int32_t fb = F[xb];
                        if (hull_cross(xp, fp, xq, fq, xb, fb) > 0) break;
                        qc = bc;
                        qi = bi;
                        xq = xb;
                        fq = fb;
                        moved = true;
                    }
                    if (!moved) break;
                }
                ce[pc] = pi + 1;
                cb[qc] = qi;
                cnext[pc] = qc;
                cprev[qc] = pc;
                glast[L] = rl;
                // chunks the bridge passes over leave the hull: empty them, so
                // that the final hull is every non-empty chunk in index order
                for (int c = pc + 1; c < R; ++c) ce[c] = cb[c];
                for (int c = R; c < qc; ++c) ce[c] = cb[c];
            }
        }
        __syncthreads();
    }

    // flatten: offsets of the non-empty chunks by a block-wide scan
    const int kept = ce[tid] - cb[tid];
    const int off = block_excl_scan<T>(kept, false, scan_tmp);
    if (tid == T - 1) n_hull = off + kept;
    for (int i = cb[tid]; i < ce[tid]; ++i) flat[off + i - cb[tid]] = hx[i];
    __syncthreads();
    const int H = n_hull;
    if (H == 0) {
        for (int t = tid; t < Wd; t += T) out[t] = UNDEF;
        return;
    }
    // Vertex k owns the cells [S_k, S_k+1): S_0 = 0, S_H = Wd, and for k >= 1
    // S_k = ceil((F_k - F_{k-1}) / (2 (x_k - x_{k-1}))) clamped to [0, Wd],
    // non-decreasing along the hull.  Each vertex with a non-empty range marks
    // its first cell (hx, free now, holds the marks), and a max-scan over the
    // row carries the mark forward: cell t's winner is the last mark at or
    // before t.
    auto start = [&](int k) {
        if (k <= 0) return 0;
        if (k >= H) return Wd;
        const int xa = flat[k - 1], xb = flat[k];
        const int32_t num = F[xb] - F[xa];
        if (num <= 0) return 0;
        const uint32_t den = 2u * (uint32_t)(xb - xa);
        const uint32_t q = ((uint32_t)num + den - 1u) / den;
        return q >= (uint32_t)Wd ? Wd : (int)q;
    };
    for (int t = tid; t < Wd; t += T) hx[t] = -1;
    __syncthreads();
    for (int k = tid; k < H; k += T) {
        const int s0 = start(k);
        if (s0 < Wd && start(k + 1) > s0) hx[s0] = (int16_t)k;
    }
    __syncthreads();
    int last = -1;
    for (int t = x0; t < x1; ++t)
        if (hx[t] >= 0) last = hx[t];
    const int carry = block_excl_scan<T>(last, true, scan_tmp);
    int run = carry;
    for (int t = x0; t < x1; ++t) {
        if (hx[t] >= 0) run = hx[t];
        else hx[t] = (int16_t)run;
    }
    __syncthreads();
#pragma unroll 4
    for (int t = tid; t < Wd; t += T) out[t] = lrow[flat[hx[t]]];
}

}  // namespace idl
