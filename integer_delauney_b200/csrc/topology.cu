// Stage (b): Delaunay triangles from 2x2 label blocks, deduplicated and
// numbered canonically, entirely on the device.
//
// The rule (src/cuda/triangle_detect.cuh:75-166): a block whose four labels
// hold three distinct seeds witnesses one triangle, emitted in first-seen
// order; four distinct seeds are a degree-4 Voronoi vertex, cut along the
// shorter diagonal of the quad ordered cyclically around its centroid, ties
// going to the diagonal that avoids the lowest seed id; any UNDEF label skips
// the block.  The reference orders the quad with double-precision atan2; here
// the order is exact integer arithmetic that sorts the same way atan2's
// values do (see angle_less), so no transcendental is needed.
//
// Dedup and numbering.  The reference appends 32-byte records through one
// global atomic counter, sorts them with thrust::sort, uniques them and copies
// them to the host (triangulation.cu:229-271); which duplicate survives is up
// to the unstable sort.  Here each emitted triangle goes straight into an
// open-addressing hash table keyed by its sorted vertex triple packed in 63
// bits (21 bits per id, as delaunay.cuh:372-374 packs it); the value kept per
// key is an atomicMin over (row-major block index, vertex order), so the
// witness is the first block in scan order, deterministically.  Canonical ids
// (rank of the sorted triple, what thrust::sort(RawLess) yields,
// triangulation.cu:254) come from grouping keys by their smallest vertex: a
// count per seed, an exclusive scan, and a rank within each (tiny) group.
#include "context.cuh"

namespace idl {
namespace {

constexpr unsigned long long EMPTY_KEY = ~0ull;
constexpr int MAX_PROBES = 1 << 14;

__device__ __forceinline__ unsigned long long mix64(unsigned long long k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

// atan2(v.y, v.x) < atan2(u'.y, u'.x) decided exactly for integer vectors.
// atan2 maps to (-pi, pi]: y < 0 gives (-pi, 0), (x >= 0, y == 0) gives 0
// (the zero vector included, atan2(+0, +0) = +0), y > 0 gives (0, pi) and
// (x < 0, y == 0) gives pi.  Within the two open half planes the order is
// the sign of the cross product.
__device__ __forceinline__ int angle_class(long long x, long long y)
{
    if (y < 0) return 0;
    if (y == 0) return x >= 0 ? 1 : 3;
    return 2;
}

__device__ __forceinline__ bool angle_less(long long ax, long long ay, long long bx, long long by)
{
    const int ca = angle_class(ax, ay), cb = angle_class(bx, by);
    if (ca != cb) return ca < cb;
    if (ca == 1 || ca == 3) return false;
    return ax * by - ay * bx > 0;
}

struct Emit {
    int32_t o[2][3];
    int n;
};

// The block rule of triangle_detect.cuh:75-166 on labels (a, b, c, d) =
// (top-left, top-right, bottom-left, bottom-right).
__device__ __forceinline__ void block_rule(int32_t a, int32_t b, int32_t c, int32_t d,
                                           const uint32_t* __restrict__ pos, Emit& e)
{
    e.n = 0;
    const int32_t q[4] = {a, b, c, d};
    int32_t s[4];
    int n = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (q[i] < 0) return;
        bool dup = false;
        for (int j = 0; j < n; ++j) dup |= (s[j] == q[i]);
        if (!dup) s[n++] = q[i];
    }
    if (n == 3) {
        e.o[0][0] = s[0]; e.o[0][1] = s[1]; e.o[0][2] = s[2];
        e.n = 1;
        return;
    }
    if (n != 4) return;

    long long px[4], py[4];
    long long sxs = 0, sys = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t p = __ldg(&pos[q[i]]);
        px[i] = pos_x(p);
        py[i] = pos_y(p);
        sxs += px[i];
        sys += py[i];
    }
    // 4 * (p - centroid), exact in integers
    long long vx[4], vy[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) { vx[i] = 4 * px[i] - sxs; vy[i] = 4 * py[i] - sys; }
    int ord[4] = {0, 1, 2, 3};
    for (int i = 1; i < 4; ++i) {   // stable insertion sort by angle
        const int k = ord[i];
        int j = i - 1;
        while (j >= 0 && angle_less(vx[k], vy[k], vx[ord[j]], vy[ord[j]])) { ord[j + 1] = ord[j]; --j; }
        ord[j + 1] = k;
    }
    auto len2 = [&](int i, int j) {
        const long long dx = px[i] - px[j], dy = py[i] - py[j];
        return dx * dx + dy * dy;
    };
    const int d0a = ord[0], d0b = ord[2], d1a = ord[1], d1b = ord[3];
    const long long l0 = len2(d0a, d0b), l1 = len2(d1a, d1b);
    int pa, pb;
    if (l0 < l1) { pa = d0a; pb = d0b; }
    else if (l1 < l0) { pa = d1a; pb = d1b; }
    else {
        int lowest = 0;
        for (int i = 1; i < 4; ++i) if (q[i] < q[lowest]) lowest = i;
        if (lowest == d0a || lowest == d0b) { pa = d1a; pb = d1b; }
        else { pa = d0a; pb = d0b; }
    }
    int ra = -1, rb = -1;
    for (int i = 0; i < 4; ++i) {
        if (i == pa || i == pb) continue;
        if (ra < 0) ra = i; else rb = i;
    }
    e.o[0][0] = q[pa]; e.o[0][1] = q[pb]; e.o[0][2] = q[ra];
    e.o[1][0] = q[pa]; e.o[1][1] = q[pb]; e.o[1][2] = q[rb];
    e.n = 2;
}

// Sorted key plus a 4-bit code of the order the block saw the vertices in.
// With a rank map the key and the recorded ids are ranks (the numbering the
// outputs use) while the rule itself ran on the raw labels.
__device__ __forceinline__ void make_key(const int32_t in[3], const int32_t* __restrict__ rank, unsigned long long& key,
                                         unsigned& code)
{
    const int32_t o[3] = {rank ? __ldg(&rank[in[0]]) : in[0], rank ? __ldg(&rank[in[1]]) : in[1],
                          rank ? __ldg(&rank[in[2]]) : in[2]};
    int32_t a = o[0], b = o[1], c = o[2], t;
    if (a > b) { t = a; a = b; b = t; }
    if (b > c) { t = b; b = c; c = t; }
    if (a > b) { t = a; a = b; b = t; }
    key = ((unsigned long long)a << 42) | ((unsigned long long)b << 21) | (unsigned long long)c;
    const unsigned i0 = o[0] == a ? 0u : (o[0] == b ? 1u : 2u);
    const unsigned i1 = o[1] == a ? 0u : (o[1] == b ? 1u : 2u);
    code = i0 * 3u + i1;
}

// The table interleaves each slot's key and value (table[2s], table[2s + 1]),
// so an insert touches one 16-byte pair in one memory sector.
__device__ __forceinline__ void hash_insert(unsigned long long key, unsigned long long val,
                                            unsigned long long* __restrict__ table, unsigned long long mask,
                                            Scalars* __restrict__ sc)
{
    unsigned long long slot = mix64(key) & mask;
    for (int probe = 0; probe < MAX_PROBES; ++probe) {
        const unsigned long long prev = atomicCAS(&table[2 * slot], EMPTY_KEY, key);
        if (prev == EMPTY_KEY || prev == key) {
            atomicMin(&table[2 * slot + 1], val);
            return;
        }
        slot = (slot + 1) & mask;
    }
    atomicOr(&sc->overflow, 1);
}

// One thread per 2 x 2 block; a warp covers 32 adjacent blocks of a row.  A
// key the block one column left (the previous lane) emitted as well is not
// inserted again: that block's row-major index is smaller, so its atomicMin
// already keeps a smaller witness than this one would.
__global__ void __launch_bounds__(256)
k_detect(const int32_t* __restrict__ lab, int pitch, int Wd, int Hd, const uint32_t* __restrict__ pos,
         const int32_t* __restrict__ rank, unsigned long long* __restrict__ table, unsigned long long mask,
         Scalars* __restrict__ sc)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (y >= Hd - 1) return;   // uniform over the warp (blockDim.x = 32)
    unsigned long long k0 = EMPTY_KEY, k1 = EMPTY_KEY;
    unsigned code0 = 0, code1 = 0;
    if (x < Wd - 1) {
        const int32_t a = lab[(size_t)y * pitch + x], b = lab[(size_t)y * pitch + x + 1];
        const int32_t c = lab[(size_t)(y + 1) * pitch + x], d = lab[(size_t)(y + 1) * pitch + x + 1];
        if (!(a == b && a == c && a == d) && !((a == b && c == d) || (a == c && b == d))) {
            Emit e;
            block_rule(a, b, c, d, pos, e);
            if (e.n > 0) make_key(e.o[0], rank, k0, code0);
            if (e.n > 1) make_key(e.o[1], rank, k1, code1);
        }
    }
    const unsigned long long l0 = __shfl_up_sync(0xffffffffu, k0, 1), l1 = __shfl_up_sync(0xffffffffu, k1, 1);
    const bool first = threadIdx.x == 0;
    const unsigned long long blk = (unsigned long long)y * Wd + x;
    if (k0 != EMPTY_KEY && (first || (k0 != l0 && k0 != l1))) hash_insert(k0, (blk << 4) | code0, table, mask, sc);
    if (k1 != EMPTY_KEY && (first || (k1 != l0 && k1 != l1))) hash_insert(k1, (blk << 4) | code1, table, mask, sc);
}


// Compaction of the occupied slots with one atomic per block on the row
// counter (one per warp, 65 k of them on a 2 M-slot table, serialised on that
// one address): a block counts the occupied slots of its contiguous span,
// reserves that many rows, and writes them in slot order, the second read of
// the span coming from L2.  Row order is free: k_rank numbers the triangles
// canonically.
constexpr int ENUM_THREADS = 256;

__global__ void __launch_bounds__(ENUM_THREADS)
k_enumerate(const unsigned long long* __restrict__ table, long long cap, unsigned long long* __restrict__ ukeys,
            unsigned long long* __restrict__ uvals, int32_t* __restrict__ cnt, Scalars* __restrict__ sc)
{
    constexpr int NW = ENUM_THREADS / 32;
    __shared__ int warp_cnt[NW];
    __shared__ unsigned long long s_base;
    const long long span = ((cap + gridDim.x - 1) / gridDim.x + ENUM_THREADS - 1) / ENUM_THREADS * ENUM_THREADS;
    const long long b0 = (long long)blockIdx.x * span, b1 = min(cap, b0 + span);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned mine = 0;
    for (long long s = b0 + threadIdx.x; s < b1; s += ENUM_THREADS) mine += table[2 * s] != EMPTY_KEY;
    mine = __reduce_add_sync(0xffffffffu, mine);
    if (lane == 0) warp_cnt[warp] = (int)mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long total = 0;
        for (int w = 0; w < NW; ++w) total += (unsigned)warp_cnt[w];
        s_base = total ? atomicAdd(reinterpret_cast<unsigned long long*>(&sc->n_triangles), total) : 0ull;
    }
    __syncthreads();
    unsigned long long base = s_base;
    for (long long s0 = b0; s0 < b1; s0 += ENUM_THREADS) {
        const long long s = s0 + threadIdx.x;
        const unsigned long long k = s < b1 ? table[2 * s] : EMPTY_KEY;
        const bool occ = k != EMPTY_KEY;
        const unsigned ballot = __ballot_sync(0xffffffffu, occ);
        if (lane == 0) warp_cnt[warp] = __popc(ballot);
        __syncthreads();
        int before = 0, all = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const int c = warp_cnt[w];
            before += w < warp ? c : 0;
            all += c;
        }
        if (occ) {
            const unsigned long long u = base + before + __popc(ballot & ((1u << lane) - 1u));
            ukeys[u] = k;
            uvals[u] = table[2 * s + 1];
            atomicAdd(&cnt[(int)(k >> 42)], 1);
        }
        base += all;
        __syncthreads();   // warp_cnt is rewritten next iteration
    }
}

__global__ void k_group(const unsigned long long* __restrict__ ukeys, const Scalars* __restrict__ sc,
                        const int32_t* __restrict__ off, int32_t* __restrict__ fill, int32_t* __restrict__ grp)
{
    const long long nu = sc->n_triangles;
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < nu;
         u += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(ukeys[u] >> 42);
        const int slot = atomicAdd(&fill[a], 1);
        grp[off[a] + slot] = (int32_t)u;
    }
}

__global__ void k_rank(const unsigned long long* __restrict__ ukeys, const unsigned long long* __restrict__ uvals,
                       const Scalars* __restrict__ sc, const int32_t* __restrict__ off,
                       const int32_t* __restrict__ grp, int Wd, int shift, int32_t* __restrict__ tris)
{
    const long long nu = sc->n_triangles;
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < nu;
         u += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = ukeys[u];
        const int a = (int)(k >> 42);
        const int lo = off[a], hi = off[a + 1];
        int r = 0;
        for (int j = lo; j < hi; ++j) r += ukeys[grp[j]] < k;
        const long long tid = lo + r;
        const int32_t id[3] = {(int32_t)(k >> 42), (int32_t)((k >> 21) & 0x1FFFFF), (int32_t)(k & 0x1FFFFF)};
        const unsigned long long v = uvals[u];
        const unsigned code = (unsigned)(v & 15u);
        const unsigned long long blk = v >> 4;
        const unsigned i0 = code / 3u, i1 = code % 3u, i2 = 3u - i0 - i1;
        int32_t* o = tris + tid * 5;
        o[0] = (int32_t)(blk % (unsigned long long)Wd) - shift;
        o[1] = (int32_t)(blk / (unsigned long long)Wd) - shift;
        o[2] = id[i0];
        o[3] = id[i1];
        o[4] = id[i2];
    }
}

}  // namespace

void detect_triangles(Context& C, const Canvas& cv, const int32_t* labels, const uint32_t* pos, int64_t n,
                      int shift, cudaEvent_t mid, const int32_t* rank)
{
    // Unique triangles of a planar triangulation number under 2n; the table
    // starts at four times that, and on the rare probe overflow it grows and
    // the detection is redone.  The occupied slots are counted while they are
    // compacted (one atomic per block), not while they are inserted, where a
    // single counter would serialise every new key.
    int64_t cap = std::max<int64_t>(next_pow2(8 * n + 1024), C.hash_cap);
    C.cnt.ensure((size_t)(n + 1) * 4);
    C.off.ensure((size_t)(n + 2) * 4);
    C.fill.ensure((size_t)(n + 1) * 4);
    for (int attempt = 0;; ++attempt) {
        C.hkeys.ensure((size_t)cap * 16);
        C.ukeys.ensure((size_t)cap * 8);
        C.uvals.ensure((size_t)cap * 8);
        // grouping and ranking follow with no read-back between: their
        // buffers hold as many triangles as the table has slots, and their
        // count comes from the device
        C.grp.ensure((size_t)cap * 4);
        C.tris.ensure((size_t)cap * 5 * 4);
        IDL_CUDA(cudaMemsetAsync(C.hkeys.ptr, 0xFF, (size_t)cap * 16, C.stream));
        IDL_CUDA(cudaMemsetAsync(&C.sc()->overflow, 0, sizeof(int32_t), C.stream));
        IDL_CUDA(cudaMemsetAsync(&C.sc()->n_triangles, 0, sizeof(int64_t), C.stream));
        IDL_CUDA(cudaMemsetAsync(C.cnt.ptr, 0, (size_t)(n + 1) * 4, C.stream));

        dim3 blk(32, 8);
        dim3 grd(ceil_div(std::max(cv.Wd - 1, 1), 32), ceil_div(std::max(cv.Hd - 1, 1), 8));
        k_detect<<<grd, blk, 0, C.stream>>>(labels, cv.pitch, cv.Wd, cv.Hd, pos, rank, C.hkeys.as<unsigned long long>(),
                                            (unsigned long long)(cap - 1), C.sc());
        IDL_LAUNCH();
        if (mid) IDL_CUDA(cudaEventRecord(mid, C.stream));
        C.mark(PM_DETECT);
        const int g1 = (int)std::min<int64_t>(ceil_div(cap, 256), C.num_sms * 16);
        k_enumerate<<<g1, ENUM_THREADS, 0, C.stream>>>(C.hkeys.as<unsigned long long>(), cap,
                                              C.ukeys.as<unsigned long long>(),
                                              C.uvals.as<unsigned long long>(), C.cnt.as<int32_t>(), C.sc());
        IDL_LAUNCH();
        IDL_CUDA(cudaMemsetAsync(C.fill.ptr, 0, (size_t)(n + 1) * 4, C.stream));
        exclusive_scan(C, C.cnt.as<int32_t>(), C.off.as<int32_t>(), n);
        const int g2 = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(2 * n + 2, 256), C.num_sms * 16));
        k_group<<<g2, 256, 0, C.stream>>>(C.ukeys.as<unsigned long long>(), C.sc(), C.off.as<int32_t>(),
                                          C.fill.as<int32_t>(), C.grp.as<int32_t>());
        IDL_LAUNCH();
        k_rank<<<g2, 256, 0, C.stream>>>(C.ukeys.as<unsigned long long>(), C.uvals.as<unsigned long long>(), C.sc(),
                                         C.off.as<int32_t>(), C.grp.as<int32_t>(), cv.Wd, shift, C.tris.as<int32_t>());
        IDL_LAUNCH();
        // one read-back: overflow (then all of it again, with a larger table) and the count
        C.fetch_scalars();
        if (!C.host_sc->overflow) break;
        if (attempt >= 6) throw Error(IDL_ERR_INTERNAL, "triangle hash table overflow");
        cap *= 4;
    }
    const int64_t nu = C.host_sc->n_triangles;
    if (nu > cap / 2) cap *= 4;          // keep the next run's table at most half full
    C.hash_cap = cap;
}

}  // namespace idl
