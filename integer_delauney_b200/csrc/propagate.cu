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

#include <vector>

namespace idl {
namespace {

constexpr int32_t OUTSIDE = -2;   // halo cell beyond the canvas edge

template <int TW, int TH, int K>
struct TileShape {
    static constexpr int RW = TW + 2 * K;
    static constexpr int RH = TH + 2 * K;
    static constexpr int RN = RW * RH;
};

// One Jacobi step for the cell at region index i (rules of geometry_device.cuh:40-66).
__device__ __forceinline__ int32_t jacobi_cell(const int32_t* __restrict__ B, int i, int cx, int cy, int RW,
                                               int RH, int gx, int gy, const uint32_t* __restrict__ pos)
{
    const int32_t c = B[i];
    if (c == OUTSIDE) return c;
    const int32_t nb[4] = {cx > 0 ? B[i - 1] : OUTSIDE, cx < RW - 1 ? B[i + 1] : OUTSIDE,
                           cy > 0 ? B[i - RW] : OUTSIDE, cy < RH - 1 ? B[i + RW] : OUTSIDE};
    int32_t best = c;
    int32_t bd = -1;   // distance of `best`, computed on demand
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int32_t n = nb[k];
        if (n < 0 || n == c || n == best) continue;
        const int32_t nd = dist2(gx, gy, __ldg(&pos[n]));
        if (best < 0) { best = n; bd = nd; continue; }
        if (bd < 0) bd = dist2(gx, gy, __ldg(&pos[best]));
        if (nd < bd || (nd == bd && n > best)) { best = n; bd = nd; }
    }
    return best;
}

// One directional sub-step of the NumPy sweep (voronoi.py:136-154).
__device__ __forceinline__ int32_t sweep_cell(int32_t c, int32_t n, int gx, int gy, const uint32_t* __restrict__ pos)
{
    if (c == OUTSIDE || n < 0 || n == c) return c;
    if (c == UNDEF) return n;
    const int32_t cd = dist2(gx, gy, __ldg(&pos[n]));
    const int32_t dc = dist2(gx, gy, __ldg(&pos[c]));
    return (cd < dc || (cd == dc && n > c)) ? n : c;
}

template <int TW, int TH, int K, int MODE>
__global__ void __launch_bounds__(256)
k_round(const int32_t* __restrict__ src, int32_t* __restrict__ dst, int pitch, int Wd, int Hd,
        const uint32_t* __restrict__ pos, const int32_t* __restrict__ list_in, const int32_t* __restrict__ count_in,
        int32_t* __restrict__ list_out, int32_t* __restrict__ count_out, int32_t* __restrict__ stamp,
        int32_t stamp_next, int tiles_x, int tiles_y, long long step_base, long long* __restrict__ last_change)
{
    using S = TileShape<TW, TH, K>;
    constexpr int RW = S::RW, RH = S::RH, RN = S::RN;
    __shared__ int32_t buf[2][RN];

    const int n_items = *count_in;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const int t = list_in[item];
        const int tx = t % tiles_x, ty = t / tiles_x;
        const int gx0 = tx * TW - K, gy0 = ty * TH - K;

        for (int i = threadIdx.x; i < RN; i += blockDim.x) {
            const int cx = i % RW, cy = i / RW;
            const int gx = gx0 + cx, gy = gy0 + cy;
            buf[0][i] = (gx >= 0 && gx < Wd && gy >= 0 && gy < Hd) ? src[(size_t)gy * pitch + gx] : OUTSIDE;
        }
        __syncthreads();

        int cur = 0;
        int last_step = -1;
        for (int s = 0; s < K; ++s) {
            bool inner_changed = false;
            if (MODE == IDL_MODE_REFERENCE) {
                for (int i = threadIdx.x; i < RN; i += blockDim.x) {
                    const int cx = i % RW, cy = i / RW;
                    const int32_t v = jacobi_cell(buf[cur], i, cx, cy, RW, RH, gx0 + cx, gy0 + cy, pos);
                    buf[cur ^ 1][i] = v;
                    if (v != buf[cur][i] && cx >= K && cx < K + TW && cy >= K && cy < K + TH) inner_changed = true;
                }
                cur ^= 1;
                if (__syncthreads_or(inner_changed)) last_step = s;
            } else {
                // left, right, up, down neighbour, each a synchronous sub-step
#pragma unroll 1
                for (int dir = 0; dir < 4; ++dir) {
                    const int32_t* B = buf[cur];
                    for (int i = threadIdx.x; i < RN; i += blockDim.x) {
                        const int cx = i % RW, cy = i / RW;
                        int32_t n;
                        if (dir == 0) n = cx > 0 ? B[i - 1] : OUTSIDE;
                        else if (dir == 1) n = cx < RW - 1 ? B[i + 1] : OUTSIDE;
                        else if (dir == 2) n = cy > 0 ? B[i - RW] : OUTSIDE;
                        else n = cy < RH - 1 ? B[i + RW] : OUTSIDE;
                        const int32_t c = B[i];
                        const int32_t v = sweep_cell(c, n, gx0 + cx, gy0 + cy, pos);
                        buf[cur ^ 1][i] = v;
                        if (v != c && cx >= K && cx < K + TW && cy >= K && cy < K + TH) inner_changed = true;
                    }
                    cur ^= 1;
                    __syncthreads();
                }
                if (__syncthreads_or(inner_changed)) last_step = s;
            }
        }

        for (int i = threadIdx.x; i < TW * TH; i += blockDim.x) {
            const int ix = i % TW, iy = i / TW;
            const int gx = tx * TW + ix, gy = ty * TH + iy;
            if (gx < Wd && gy < Hd) dst[(size_t)gy * pitch + gx] = buf[cur][(iy + K) * RW + ix + K];
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

__global__ void k_iota(int32_t* __restrict__ a, int n, int32_t* __restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
    if (i == 0) *count = n;
}

__global__ void k_set_i64(long long* p, long long v) { *p = v; }

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

constexpr int TW = 32, TH = 32, KSTEPS = 8;

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

int64_t propagate(Context& C, int mode, const Canvas& cv, const uint32_t* pos)
{
    const int tiles_x = ceil_div(cv.Wd, TW), tiles_y = ceil_div(cv.Hd, TH);
    const int n_tiles = tiles_x * tiles_y;
    // Bound on rounds: far above any real run (a pass count beyond the canvas
    // area cannot occur since every change strictly improves one of Wd*Hd keys
    // drawn from a finite set, but the bound only has to stop a runaway loop).
    const int64_t max_rounds = (int64_t)4 * (cv.Wd + cv.Hd) + 64;

    C.tiles[0].ensure((size_t)n_tiles * 4);
    C.tiles[1].ensure((size_t)n_tiles * 4);
    if (C.stamps.bytes < (size_t)n_tiles * 4) {
        C.stamps.ensure((size_t)n_tiles * 4);
        IDL_CUDA(cudaMemsetAsync(C.stamps.ptr, 0, (size_t)n_tiles * 4, C.stream));
        C.stamp_epoch = 0;
    }
    if (C.stamp_epoch > (1 << 30) - max_rounds - 8) {
        IDL_CUDA(cudaMemsetAsync(C.stamps.ptr, 0, C.stamps.bytes, C.stream));
        C.stamp_epoch = 0;
    }
    const int32_t epoch = C.stamp_epoch;
    C.stamp_epoch += int32_t(max_rounds + 4);

    const size_t count_len = (size_t)max_rounds + 2;
    C.counts.ensure(count_len * 4);
    IDL_CUDA(cudaMemsetAsync(C.counts.ptr, 0, count_len * 4, C.stream));
    int32_t* counts = C.counts.as<int32_t>();

    k_iota<<<(unsigned)((n_tiles + 255) / 256), 256, 0, C.stream>>>(C.tiles[0].as<int32_t>(), n_tiles, counts);
    IDL_LAUNCH();
    long long* last = reinterpret_cast<long long*>(&C.sc()->last_change);
    k_set_i64<<<1, 1, 0, C.stream>>>(last, -1);
    IDL_LAUNCH();

    const int grid = std::min(n_tiles, C.num_sms * 8);
    int64_t r = 0;
    int group = 2;
    for (;;) {
        for (int g = 0; g < group && r < max_rounds; ++g, ++r) {
            const int32_t* srcp = C.lab[r & 1].as<int32_t>();
            int32_t* dstp = C.lab[(r + 1) & 1].as<int32_t>();
            const int32_t* lin = C.tiles[r & 1].as<int32_t>();
            int32_t* lout = C.tiles[(r + 1) & 1].as<int32_t>();
            const long long base = (long long)r * KSTEPS;
            const int32_t stamp_next = epoch + int32_t(r) + 1;
            if (mode == IDL_MODE_NUMPY)
                k_round<TW, TH, KSTEPS, IDL_MODE_NUMPY><<<grid, 256, 0, C.stream>>>(
                    srcp, dstp, cv.pitch, cv.Wd, cv.Hd, pos, lin, counts + r, lout, counts + r + 1,
                    C.stamps.as<int32_t>(), stamp_next, tiles_x, tiles_y, base, last);
            else
                k_round<TW, TH, KSTEPS, IDL_MODE_REFERENCE><<<grid, 256, 0, C.stream>>>(
                    srcp, dstp, cv.pitch, cv.Wd, cv.Hd, pos, lin, counts + r, lout, counts + r + 1,
                    C.stamps.as<int32_t>(), stamp_next, tiles_x, tiles_y, base, last);
            IDL_LAUNCH();
        }
        int32_t remaining = 0;
        IDL_CUDA(cudaMemcpyAsync(&remaining, counts + r, 4, cudaMemcpyDeviceToHost, C.stream));
        IDL_CUDA(cudaStreamSynchronize(C.stream));
        if (remaining == 0) break;
        if (r >= max_rounds) throw Error(IDL_ERR_INTERNAL, "Voronoi propagation did not converge");
        group = std::min(group * 2, 8);
    }
    C.fetch_scalars();
    const int64_t lc = C.host_sc->last_change;
    const int64_t passes = lc < 0 ? 1 : lc + 2;
    if (C.prof.enabled) {
        std::vector<int32_t> h((size_t)r + 1);
        IDL_CUDA(cudaMemcpy(h.data(), counts, h.size() * 4, cudaMemcpyDeviceToHost));
        int64_t tiles = 0, rounds = 0;
        for (int32_t c : h) {
            tiles += c;
            rounds += c > 0;
        }
        C.prof.tiles = tiles;
        C.prof.rounds = rounds;
        C.prof.passes = passes;
        C.prof.tile_w = TW;
        C.prof.tile_h = TH;
        C.prof.steps_per_round = KSTEPS;
    }
    return passes;
}

}  // namespace idl
