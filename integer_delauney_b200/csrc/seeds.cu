// Seed validation and (x, y) ordering on the device, plus the exclusive scan
// the rest of the library shares.
//
// The reference sorts seeds on the host with std::sort after a Python-object
// loop (src/cuda/bindings/binding_helpers.hpp:23-46).  Seeds are distinct
// pixels, so their (x asc, y asc) order is the order of their pixels in a
// column-major walk of the canvas: set one bit per seed in a column-major
// occupancy bitmap (a repeat hit is a duplicate), prefix-popcount the bitmap,
// and each seed's rank is the number of set bits before its own.  O(n + W*H/32)
// work, no comparison sort, and the duplicate check falls out of the atomicOr.
#include "context.cuh"

#include <vector>

namespace idl {

// ---------------------------------------------------------------------------
// exclusive scan (int32), 3-phase: per-block scan, scan of block totals,
// add-back.  4096 items per block.
// ---------------------------------------------------------------------------
namespace {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_block(const int32_t* __restrict__ in, int32_t* __restrict__ out, int64_t n,
             int32_t* __restrict__ block_sums)
{
    __shared__ int32_t warp_tot[SCAN_THREADS / 32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int32_t v[SCAN_ITEMS];
    int32_t run = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        const int64_t j = base + i;
        v[i] = j < n ? in[j] : 0;
        const int32_t t = v[i];
        v[i] = run;          // exclusive within the thread
        run += t;
    }
    // inclusive warp scan of thread totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int32_t w = lane < SCAN_THREADS / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_THREADS / 32) warp_tot[lane] = w;   // inclusive
    }
    __syncthreads();
    const int32_t warp_excl = warp > 0 ? warp_tot[warp - 1] : 0;
    const int32_t thread_excl = warp_excl + x - run;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        const int64_t j = base + i;
        if (j < n) out[j] = thread_excl + v[i];
    }
    if (threadIdx.x == SCAN_THREADS - 1) block_sums[blockIdx.x] = thread_excl + run;
}

__global__ void k_scan_add(int32_t* __restrict__ out, int64_t n, const int32_t* __restrict__ offs)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) out[j] += offs[j / SCAN_TILE];
}

__global__ void k_set_total(int32_t* __restrict__ out, int64_t n, const int32_t* __restrict__ total)
{
    out[n] = *total;
}

}  // namespace

void exclusive_scan(Context& C, const int32_t* in, int32_t* out, int64_t n)
{
    // level sizes (fixed-size bookkeeping: no host allocation on this path;
    // 4096^8 items is far beyond any int32 count)
    constexpr int MAX_LEVELS = 8;
    int64_t lens[MAX_LEVELS];
    int nlev = 0;
    int64_t m = n;
    for (;;) {
        const int64_t nb = (m + SCAN_TILE - 1) / SCAN_TILE;
        if (nlev == MAX_LEVELS) throw Error(IDL_ERR_INTERNAL, "scan too large");
        lens[nlev++] = nb > 0 ? nb : 1;
        if (nb <= 1) break;
        m = nb;
    }
    // scratch: per level, block sums (nb) and their scan (nb + 1)
    size_t need = 0;
    for (int l = 0; l < nlev; ++l) need += size_t(2 * lens[l] + 1);
    C.scan_a.ensure(need * sizeof(int32_t));
    int32_t* arena = C.scan_a.as<int32_t>();

    int32_t* sums[MAX_LEVELS];
    int32_t* scans[MAX_LEVELS];
    size_t at = 0;
    for (int l = 0; l < nlev; ++l) {
        sums[l] = arena + at;  at += lens[l];
        scans[l] = arena + at; at += lens[l] + 1;
    }
    // down: scan each level's input into its output
    const int32_t* lin = in;
    int32_t* lout = out;
    int64_t len = n;
    for (int l = 0; l < nlev; ++l) {
        const int64_t nb = lens[l];
        k_scan_block<<<(unsigned)nb, SCAN_THREADS, 0, C.stream>>>(lin, lout, len, sums[l]);
        IDL_LAUNCH();
        if (nb <= 1) {
            k_set_total<<<1, 1, 0, C.stream>>>(lout, len, sums[l]);
            IDL_LAUNCH();
            break;
        }
        lin = sums[l];
        lout = scans[l];
        len = nb;
    }
    // up: add scanned block offsets back, deepest first
    for (int l = nlev - 2; l >= 0; --l) {
        int32_t* target = (l == 0) ? out : scans[l - 1];
        const int64_t tlen = (l == 0) ? n : lens[l - 1];
        k_scan_add<<<(unsigned)((tlen + 255) / 256), 256, 0, C.stream>>>(target, tlen, scans[l]);
        IDL_LAUNCH();
        // total of this level = last entry of scans[l]
        k_set_total<<<1, 1, 0, C.stream>>>(target, tlen, scans[l] + lens[l]);
        IDL_LAUNCH();
    }
}

// ---------------------------------------------------------------------------
// seeds
// ---------------------------------------------------------------------------
namespace {

__global__ void k_seed_mark(const int32_t* __restrict__ xy, int64_t n, int W, int H,
                            uint32_t* __restrict__ bitmap, Scalars* __restrict__ sc)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = xy[2 * i], y = xy[2 * i + 1];
    if (x < 0 || x >= W || y < 0 || y >= H) {
        atomicOr(&sc->err_oob, 1);
        return;
    }
    const int64_t bit = (int64_t)x * H + y;
    const uint32_t m = 1u << (bit & 31);
    const uint32_t old = atomicOr(&bitmap[bit >> 5], m);
    if (old & m) atomicOr(&sc->err_dup, 1);
}

__global__ void k_popc(const uint32_t* __restrict__ bitmap, int64_t nwords, int32_t* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nwords) out[i] = __popc(bitmap[i]);
}

__global__ void k_seed_rank(const int32_t* __restrict__ xy, int64_t n, int W, int H, int P,
                            const uint32_t* __restrict__ bitmap, const int32_t* __restrict__ word_rank,
                            int32_t* __restrict__ xs, int32_t* __restrict__ ys, uint32_t* __restrict__ pos)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = xy[2 * i], y = xy[2 * i + 1];
    if (x < 0 || x >= W || y < 0 || y >= H) return;
    const int64_t bit = (int64_t)x * H + y;
    const uint32_t below = bitmap[bit >> 5] & ((1u << (bit & 31)) - 1u);
    const int32_t r = word_rank[bit >> 5] + __popc(below);
    xs[r] = x;
    ys[r] = y;
    pos[r] = pack_pos(x + P, y + P);
}

__global__ void k_mark_xy(const int32_t* __restrict__ xs, const int32_t* __restrict__ ys, int64_t n, int H,
                          uint32_t* __restrict__ bitmap)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t bit = (int64_t)xs[i] * H + ys[i];
    atomicOr(&bitmap[bit >> 5], 1u << (bit & 31));
}

__global__ void k_rank_xy(const int32_t* __restrict__ xs, const int32_t* __restrict__ ys, int64_t n, int H,
                          const uint32_t* __restrict__ bitmap, const int32_t* __restrict__ word_rank, int off,
                          int32_t* __restrict__ rank, int32_t* __restrict__ inv, int32_t* __restrict__ xs_sorted,
                          int32_t* __restrict__ ys_sorted)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t bit = (int64_t)xs[i] * H + ys[i];
    const uint32_t below = bitmap[bit >> 5] & ((1u << (bit & 31)) - 1u);
    const int32_t r = word_rank[bit >> 5] + __popc(below);
    rank[i] = r;
    inv[r] = (int32_t)i;
    xs_sorted[r] = xs[i] + off;
    ys_sorted[r] = ys[i] + off;
}

}  // namespace

void rank_seeds_device(Context& C, int W, int H, const int32_t* xs, const int32_t* ys, int64_t n, int off,
                       int32_t* rank, int32_t* inv, int32_t* xs_sorted, int32_t* ys_sorted)
{
    if (n <= 0) return;
    const int64_t nwords = ((int64_t)W * H + 31) / 32;
    C.bitmap.ensure(size_t(nwords) * 4);
    C.scan_b.ensure(size_t(nwords) * 4);
    C.scan_c.ensure(size_t(nwords + 1) * 4);
    IDL_CUDA(cudaMemsetAsync(C.bitmap.ptr, 0, size_t(nwords) * 4, C.stream));
    const unsigned gs = (unsigned)((n + 255) / 256);
    k_mark_xy<<<gs, 256, 0, C.stream>>>(xs, ys, n, H, C.bitmap.as<uint32_t>());
    IDL_LAUNCH();
    k_popc<<<(unsigned)((nwords + 255) / 256), 256, 0, C.stream>>>(C.bitmap.as<uint32_t>(), nwords,
                                                                  C.scan_b.as<int32_t>());
    IDL_LAUNCH();
    exclusive_scan(C, C.scan_b.as<int32_t>(), C.scan_c.as<int32_t>(), nwords);
    k_rank_xy<<<gs, 256, 0, C.stream>>>(xs, ys, n, H, C.bitmap.as<uint32_t>(), C.scan_c.as<int32_t>(), off, rank,
                                        inv, xs_sorted, ys_sorted);
    IDL_LAUNCH();
}

void sort_seeds_device(Context& C, int W, int H, int64_t n, int P)
{
    const int64_t bits = (int64_t)W * H;
    const int64_t nwords = (bits + 31) / 32;
    C.bitmap.ensure(size_t(nwords) * 4);
    C.scan_b.ensure(size_t(nwords) * 4);
    C.scan_c.ensure(size_t(nwords + 1) * 4);
    C.xs.ensure(size_t(n) * 4);
    C.ys.ensure(size_t(n) * 4);
    C.pos.ensure(size_t(n) * 4);

    IDL_CUDA(cudaMemsetAsync(C.bitmap.ptr, 0, size_t(nwords) * 4, C.stream));
    IDL_CUDA(cudaMemsetAsync(&C.sc()->err_oob, 0, 2 * sizeof(int32_t), C.stream));
    const unsigned gs = (unsigned)((n + 255) / 256);
    k_seed_mark<<<gs, 256, 0, C.stream>>>(C.seeds_in.as<int32_t>(), n, W, H, C.bitmap.as<uint32_t>(), C.sc());
    IDL_LAUNCH();
    C.fetch_scalars();
    if (C.host_sc->err_oob) invalid("seed coordinate out of bounds");
    if (C.host_sc->err_dup) invalid("duplicate seed positions are not allowed");

    k_popc<<<(unsigned)((nwords + 255) / 256), 256, 0, C.stream>>>(C.bitmap.as<uint32_t>(), nwords,
                                                                  C.scan_b.as<int32_t>());
    IDL_LAUNCH();
    exclusive_scan(C, C.scan_b.as<int32_t>(), C.scan_c.as<int32_t>(), nwords);
    k_seed_rank<<<gs, 256, 0, C.stream>>>(C.seeds_in.as<int32_t>(), n, W, H, P, C.bitmap.as<uint32_t>(),
                                          C.scan_c.as<int32_t>(), C.xs.as<int32_t>(), C.ys.as<int32_t>(),
                                          C.pos.as<uint32_t>());
    IDL_LAUNCH();
}

}  // namespace idl
