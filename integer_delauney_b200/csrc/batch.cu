// Batched triangulation: many independent images of uneven size and seed
// count through one pass of the pipeline.  Each image's result equals
// idl_triangulate on that image alone, bit for bit.
//
// The images' padded detection canvases are shelf-packed into one atlas with
// a one-cell wall between neighbours.  Wall cells hold a label below UNDEF,
// which the propagation never updates and never takes as a candidate, and
// which makes the block rule skip every 2x2 block touching it, so no image
// sees another.  Seeds get global ids image after image, each image's in its
// own (x asc, y asc) order, so within an image the id order -- the Jacobi tie
// rule, the block rule's lowest-id tie-break and the canonical triangle rank --
// is the single-image order shifted by a constant.  Then:
//   * one persistent launch propagates every image (the micro-tile work list
//     of the sparse kernel is the packed tile queue: images that converge
//     early drop out of it, images that need many passes keep only their
//     own active micro-tiles in it);
//   * one detection + dedup + numbering over the atlas; canonical global
//     ranks group by image (ids are contiguous per image), so an image's
//     triangle ids are the global ranks minus the count of earlier images';
//   * one raster launch over all triangles, each clipped to its own image with
//     its own image's degenerate-case window (per-image longest side);
//   * one composition launch writing every image's (H, W, 3) grid.
// The number of launches and host synchronisations is independent of the
// number of images.
#include "raster.cuh"
#include "row_hull.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

namespace idl {
namespace {

constexpr int32_t WALL = (int32_t)0xFEFEFEFE;   // memset pattern 0xFE: below UNDEF

struct BImg {
    int W, H;          // image size
    int ox, oy;        // atlas origin of the padded canvas
    long long seed_off;  // first global seed id
    long long px_off;    // first output pixel (prefix of W*H); also the bitmap base
    long long row_off;   // first output row (prefix of H)
};

__global__ void k_b_mark(const int32_t* __restrict__ xy, int64_t n, const int32_t* __restrict__ seed_img,
                         const BImg* __restrict__ imgs, uint32_t* __restrict__ bitmap,
                         unsigned long long* __restrict__ first_bad)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BImg m = imgs[seed_img[i]];
    const int32_t x = xy[2 * i], y = xy[2 * i + 1];
    if (x < 0 || y < 0 || x >= m.W || y >= m.H) {
        atomicMin(&first_bad[0], (unsigned long long)i);
        return;
    }
    const long long bit = m.px_off + (long long)x * m.H + y;
    const uint32_t b = 1u << (bit & 31);
    if (atomicOr(&bitmap[bit >> 5], b) & b) atomicMin(&first_bad[1], (unsigned long long)i);
}

__global__ void k_b_popc(const uint32_t* __restrict__ bitmap, int64_t nwords, int32_t* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nwords) out[i] = __popc(bitmap[i]);
}

__global__ void k_b_rank(const int32_t* __restrict__ xy, int64_t n, const int32_t* __restrict__ seed_img,
                         const BImg* __restrict__ imgs, int P, const uint32_t* __restrict__ bitmap,
                         const int32_t* __restrict__ word_rank, int32_t* __restrict__ xs, int32_t* __restrict__ ys,
                         uint32_t* __restrict__ pos, int32_t* __restrict__ sid_img)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int im = seed_img[i];
    const BImg m = imgs[im];
    const int32_t x = xy[2 * i], y = xy[2 * i + 1];
    const long long bit = m.px_off + (long long)x * m.H + y;
    const int32_t r = word_rank[bit >> 5] + __popc(bitmap[bit >> 5] & ((1u << (bit & 31)) - 1u));
    xs[r] = x;
    ys[r] = y;
    pos[r] = pack_pos(m.ox + P + x, m.oy + P + y);
    sid_img[r] = im;
}

// Each image's padded canvas starts UNDEF (the rest of the atlas is WALL).
__global__ void k_b_open(int32_t* __restrict__ a, int32_t* __restrict__ b, int pitch, const BImg* __restrict__ imgs,
                         int P)
{
    const BImg m = imgs[blockIdx.y];
    const int Wp = m.W + 2 * P, Hp = m.H + 2 * P;
    for (int r = blockIdx.x; r < Hp; r += gridDim.x) {
        const size_t o = (size_t)(m.oy + r) * pitch + m.ox;
        for (int c = threadIdx.x; c < Wp; c += blockDim.x) {
            a[o + c] = UNDEF;
            b[o + c] = UNDEF;
        }
    }
}

__global__ void k_b_seeds(int32_t* __restrict__ a, int32_t* __restrict__ b, int pitch, const uint32_t* __restrict__ pos,
                          int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = pos[i];
    const size_t o = (size_t)pos_y(p) * pitch + pos_x(p);
    a[o] = (int32_t)i;
    b[o] = (int32_t)i;
}

// ---- exact semantics over the atlas -------------------------------------
// The separable nearest-seed search of the single-image exact mode (exact.cu),
// run for every image of the atlas at once and kept inside each image: a
// column walk uses only its image's seeds, a row scan only its image's
// columns, so no label crosses a wall.  Labels are global seed ids, as the
// Jacobi path leaves them.
struct XImg {
    int ox, oy, Wp, Hp;    // padded canvas origin and size in the atlas
    int col_off, row_off;  // first entry of this image in the column / row tables
    long long s0, s1;      // its seeds: global ids [s0, s1), (x, y)-sorted
};
constexpr int XCHUNK = 64;

// cs[col_off + c] = first seed of the image with atlas x >= ox + c, c in [0, Wp].
__global__ void k_bx_col_start(const uint32_t* __restrict__ pos, const XImg* __restrict__ xi,
                               const int32_t* __restrict__ colimg, int64_t n_cols, int32_t* __restrict__ cs)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_cols) return;
    const XImg m = xi[colimg[g]];
    const int c = m.ox + (int)(g - m.col_off);
    long long lo = m.s0, hi = m.s1;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if ((int)pos_x(__ldg(&pos[mid])) < c) lo = mid + 1;
        else hi = mid;
    }
    cs[g] = (int32_t)lo;
}

// Nearest seed of each cell within its image column (a tie between the seed
// above and the one below goes to the lower one, the higher id), and its row
// distance; one thread walks one column through a band of XCHUNK rows.
__global__ void k_bx_col_nearest(const uint32_t* __restrict__ pos, const XImg* __restrict__ xi,
                                 const int32_t* __restrict__ colimg, const int32_t* __restrict__ cs, int64_t n_cols,
                                 int pitch, int32_t* __restrict__ col, int32_t* __restrict__ coldy)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_cols) return;
    const XImg m = xi[colimg[g]];
    const int c = (int)(g - m.col_off);
    const int y0 = blockIdx.y * XCHUNK;
    if (c >= m.Wp || y0 >= m.Hp) return;   // the image's extra start entry, or past its rows
    const int y1 = min(m.Hp, y0 + XCHUNK);
    const int x = m.ox + c;
    const int32_t lo = cs[g], hi = cs[g + 1];
    if (lo == hi) {
        for (int y = y0; y < y1; ++y) {
            col[(size_t)(m.oy + y) * pitch + x] = UNDEF;
            coldy[(size_t)(m.oy + y) * pitch + x] = 0;
        }
        return;
    }
    int32_t a = lo, b = hi;   // first seed of the column at or below the band
    while (a < b) {
        const int32_t mid = (a + b) >> 1;
        if ((int)pos_y(__ldg(&pos[mid])) < m.oy + y0) a = mid + 1;
        else b = mid;
    }
    int next_y = a < hi ? (int)pos_y(__ldg(&pos[a])) : 0x7FFFFFFF;
    int prev_y = a > lo ? (int)pos_y(__ldg(&pos[a - 1])) : -0x3FFFFFFF;
    for (int y = y0; y < y1; ++y) {
        const int ya = m.oy + y;
        while (next_y < ya) {
            prev_y = next_y;
            ++a;
            next_y = a < hi ? (int)pos_y(__ldg(&pos[a])) : 0x7FFFFFFF;
        }
        const int below = next_y - ya, above = ya - prev_y;
        const bool take_below = a < hi && (a == lo || below <= above);
        col[(size_t)ya * pitch + x] = take_below ? a : a - 1;
        coldy[(size_t)ya * pitch + x] = take_below ? below : above;
    }
}

// Best column candidate of each cell of an image row, scanning outward until
// no column further away can beat or tie it.
__global__ void k_bx_row_nearest(const int32_t* __restrict__ col, const int32_t* __restrict__ coldy,
                                 const XImg* __restrict__ xi, const int32_t* __restrict__ rowimg, int pitch,
                                 int32_t* __restrict__ lab)
{
    const int64_t r = blockIdx.x;
    const XImg m = xi[rowimg[r]];
    const int x = blockIdx.y * blockDim.x + threadIdx.x;
    if (x >= m.Wp) return;
    const int y = m.oy + (int)(r - m.row_off);
    const int32_t* row = col + (size_t)y * pitch + m.ox;
    const int32_t* rdy = coldy + (size_t)y * pitch + m.ox;
    int32_t bl = row[x];
    long long bd = 0x7FFFFFFFFFFFFFFFll;
    if (bl >= 0) {
        const long long dy = rdy[x];
        bd = dy * dy;
    }
    for (int k = 1;; ++k) {
        const long long kk = (long long)k * k;
        if (kk > bd || (x - k < 0 && x + k >= m.Wp)) break;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int xx = side ? x + k : x - k;
            if (xx < 0 || xx >= m.Wp) continue;
            const int32_t l = row[xx];
            if (l < 0) continue;
            const long long dy = rdy[xx];
            const long long d = kk + dy * dy;
            if (d < bd || (d == bd && l > bl)) {
                bd = d;
                bl = l;
            }
        }
    }
    lab[(size_t)y * pitch + m.ox + x] = bl;
}

// The lower-hull row pass (row_hull.cuh) on one image row of the atlas per
// block: O(Wp) whatever the image's seed layout.
__global__ void __launch_bounds__(HULL_THREADS)
k_bx_row_hull(const int32_t* __restrict__ col, const int32_t* __restrict__ coldy, const XImg* __restrict__ xi,
              const int32_t* __restrict__ rowimg, int pitch, int32_t* __restrict__ lab)
{
    const int64_t r = blockIdx.x;
    const XImg m = xi[rowimg[r]];
    const size_t o = (size_t)(m.oy + (int)(r - m.row_off)) * pitch + m.ox;
    row_hull(col + o, coldy + o, m.Wp, lab + o);
}

__device__ __forceinline__ int tri_image(const int32_t* row, const int32_t* __restrict__ sid_img)
{
    return sid_img[min(row[2], min(row[3], row[4]))];
}

// Per-image triangle count and per-image longest side.
__global__ void k_b_tri_stats(const int32_t* __restrict__ tris, const Scalars* __restrict__ sc,
                              const int32_t* __restrict__ sid_img, const int32_t* __restrict__ xs,
                              const int32_t* __restrict__ ys, int32_t* __restrict__ count, int32_t* __restrict__ side)
{
    const long long nt = sc->n_triangles;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nt;
         t += (long long)gridDim.x * blockDim.x) {
        const int32_t* row = tris + t * 5;
        const int im = tri_image(row, sid_img);
        atomicAdd(&count[im], 1);
        const int s = tri_max_side(row + 2, xs, ys);
        if (s > 0) atomicMax(&side[im], s);
    }
}

// One warp per triangle, into its own image's grid, with its image's window.
__global__ void __launch_bounds__(256)
k_b_raster(const int32_t* __restrict__ tris, const Scalars* __restrict__ sc, const int32_t* __restrict__ sid_img,
           const BImg* __restrict__ imgs, const int32_t* __restrict__ xs, const int32_t* __restrict__ ys,
           const int32_t* __restrict__ side, const int32_t* __restrict__ tri_off, int32_t* __restrict__ tgrid)
{
    const long long nt = sc->n_triangles;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nt; t += warps) {
        const int32_t* row = tris + t * 5;
        const int im = tri_image(row, sid_img);
        const BImg m = imgs[im];
        raster_one(row + 2, (int32_t)(t - tri_off[im]), xs, ys, m.W, m.H, max(20, side[im] + 3),
                   tgrid + m.px_off, lane);
    }
}

// Block per output row: (local seed id, squared distance, triangle id).
__global__ void k_b_compose(const int32_t* __restrict__ lab, int pitch, int P, const BImg* __restrict__ imgs,
                            const int32_t* __restrict__ row_img, const int32_t* __restrict__ xs,
                            const int32_t* __restrict__ ys, const int32_t* __restrict__ tgrid,
                            int32_t* __restrict__ out)
{
    const long long r = blockIdx.x;
    const int im = row_img[r];
    const BImg m = imgs[im];
    const int y = (int)(r - m.row_off);
    const int32_t* src = lab + (size_t)(m.oy + P + y) * pitch + m.ox + P;
    const size_t base = (size_t)m.px_off + (size_t)y * m.W;
    for (int x = threadIdx.x; x < m.W; x += blockDim.x) {
        const int32_t l = src[x];
        int32_t d = -1, id = l;
        if (l >= 0) {
            const int32_t dx = x - __ldg(&xs[l]), dy = y - __ldg(&ys[l]);
            d = dx * dx + dy * dy;
            id = (int32_t)(l - m.seed_off);
        }
        int32_t* o = out + (base + x) * 3;
        o[0] = id;
        o[1] = d;
        o[2] = tgrid[base + x];
    }
}

// Triangle rows to image-local form: witness relative to the image (shifted
// by -P as the single-image path reports it), vertex ids local.
__global__ void k_b_localise(int32_t* __restrict__ tris, const Scalars* __restrict__ sc,
                             const int32_t* __restrict__ sid_img, const BImg* __restrict__ imgs, int P)
{
    const long long nt = sc->n_triangles;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nt;
         t += (long long)gridDim.x * blockDim.x) {
        int32_t* row = tris + t * 5;
        const BImg m = imgs[tri_image(row, sid_img)];
        row[0] -= m.ox + P;
        row[1] -= m.oy + P;
        row[2] = (int32_t)(row[2] - m.seed_off);
        row[3] = (int32_t)(row[3] - m.seed_off);
        row[4] = (int32_t)(row[4] - m.seed_off);
    }
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

struct Plan {
    std::vector<BImg> imgs;
    std::vector<int32_t> seed_img, row_img;
    int AW = 0, AH = 0;
    int64_t n_seeds = 0, n_px = 0, n_rows = 0;
};

// Shelf packing of the padded canvases, tallest first, one wall cell apart.
Plan make_plan(int n_images, const int32_t* dims, const int64_t* counts, int P)
{
    if (n_images <= 0) invalid("a batch needs at least one image");
    if (n_images > 65535) invalid("at most 65535 images per batch are supported");
    Plan pl;
    pl.imgs.resize(n_images);
    double area = 0;
    int max_wp = 0;
    for (int i = 0; i < n_images; ++i) {
        const int W = dims[2 * i], H = dims[2 * i + 1];
        const int64_t n = counts[i];
        if (W <= 0 || H <= 0) {
            if (n <= 0) invalid("image " + std::to_string(i) + ": seeds must not be empty");
            invalid("image " + std::to_string(i) + ": seed coordinate out of bounds");
        }
        if (n <= 0) invalid("image " + std::to_string(i) + ": seeds must not be empty");
        if ((int64_t)W + 2 * P + 1 > MAX_CANVAS_SIDE || (int64_t)H + 2 * P + 1 > MAX_CANVAS_SIDE)
            invalid("image " + std::to_string(i) + ": canvas side (including border padding) must not exceed " +
                    std::to_string(MAX_CANVAS_SIDE - 1));
        BImg& m = pl.imgs[i];
        m.W = W;
        m.H = H;
        m.seed_off = pl.n_seeds;
        m.px_off = pl.n_px;
        m.row_off = pl.n_rows;
        pl.n_seeds += n;
        pl.n_px += (int64_t)W * H;
        pl.n_rows += H;
        area += (double)(W + 2 * P + 1) * (H + 2 * P + 1);
        max_wp = std::max(max_wp, W + 2 * P + 1);
    }
    if (pl.n_seeds > MAX_SEEDS) invalid("at most " + std::to_string(MAX_SEEDS) + " seeds per batch are supported");
    std::vector<int> order(n_images);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return pl.imgs[a].H > pl.imgs[b].H; });
    int AW = std::max(max_wp, (int)std::ceil(std::sqrt(area) * 1.05));
    AW = std::min(MAX_CANVAS_SIDE, (AW + 31) / 32 * 32);
    int x = 0, y = 0, shelf = 0;
    for (int i : order) {
        BImg& m = pl.imgs[i];
        const int wp = m.W + 2 * P + 1, hp = m.H + 2 * P + 1;
        if (x + wp > AW) {
            y += shelf;
            x = 0;
            shelf = 0;
        }
        m.ox = x;
        m.oy = y;
        x += wp;
        shelf = std::max(shelf, hp);
    }
    const int64_t AH = (int64_t)y + shelf;
    if (AH > MAX_CANVAS_SIDE) invalid("batch too large for one atlas: split it into smaller batches");
    pl.AW = AW;
    pl.AH = (int)AH;
    pl.seed_img.resize(pl.n_seeds);
    pl.row_img.resize(pl.n_rows);
    for (int i = 0; i < n_images; ++i) {
        std::fill(pl.seed_img.begin() + pl.imgs[i].seed_off, pl.seed_img.begin() + pl.imgs[i].seed_off + counts[i], i);
        std::fill(pl.row_img.begin() + pl.imgs[i].row_off, pl.row_img.begin() + pl.imgs[i].row_off + pl.imgs[i].H, i);
    }
    return pl;
}

// The pipeline; seeds already in C.seeds_in.  Leaves per-image grids in
// d_out (or C.outgrid) and image-local triangle rows in C.tris.
// What idl_delaunay_adopt (and batch_fetch) need of the last batch on a
// context: the atlas layout, and after the whole pipeline, where each
// image's grid and triangle rows are.
struct BatchPlan {
    std::vector<BImg> imgs;
    int P = 0, pitch = 0;
    int64_t n_seeds = 0;
    bool full = false;               // grids in `grids`, image-local rows in C.tris
    bool exact = false;              // labels of the exact semantics (not adoptable)
    const int32_t* grids = nullptr;  // device, n_px x 3 int32
    std::vector<int64_t> tri_off;    // n_images + 1 row offsets
};

// Exact-semantics labels of every image into C.lab[0] (the atlas's walls
// stay); C.lab[1] and C.exact_dy are scratch.
void exact_atlas(Context& C, const Plan& pl, int P, const Canvas& cv)
{
    const int n_images = (int)pl.imgs.size();
    std::vector<XImg> xi(n_images);
    std::vector<int32_t> colimg, rowimg;
    int max_wp = 0, max_hp = 0;
    for (int i = 0; i < n_images; ++i) {
        const BImg& b = pl.imgs[i];
        XImg& m = xi[i];
        m.ox = b.ox;
        m.oy = b.oy;
        m.Wp = b.W + 2 * P;
        m.Hp = b.H + 2 * P;
        m.col_off = (int)colimg.size();
        m.row_off = (int)rowimg.size();
        m.s0 = b.seed_off;
        m.s1 = i + 1 < n_images ? pl.imgs[i + 1].seed_off : pl.n_seeds;
        colimg.insert(colimg.end(), (size_t)m.Wp + 1, i);
        rowimg.insert(rowimg.end(), (size_t)m.Hp, i);
        max_wp = std::max(max_wp, m.Wp);
        max_hp = std::max(max_hp, m.Hp);
    }
    const int64_t n_cols = (int64_t)colimg.size(), n_rows = (int64_t)rowimg.size();
    C.batch_ximg.ensure(xi.size() * sizeof(XImg));
    C.batch_colimg.ensure((size_t)n_cols * 4);
    C.batch_rowimg.ensure((size_t)n_rows * 4);
    C.counts.ensure((size_t)n_cols * 4);
    C.exact_dy.ensure((size_t)cv.pitch * cv.Hd * 4);
    IDL_CUDA(cudaMemcpyAsync(C.batch_ximg.ptr, xi.data(), xi.size() * sizeof(XImg), cudaMemcpyHostToDevice,
                             C.stream));
    IDL_CUDA(cudaMemcpyAsync(C.batch_colimg.ptr, colimg.data(), (size_t)n_cols * 4, cudaMemcpyHostToDevice,
                             C.stream));
    IDL_CUDA(cudaMemcpyAsync(C.batch_rowimg.ptr, rowimg.data(), (size_t)n_rows * 4, cudaMemcpyHostToDevice,
                             C.stream));
    const XImg* d_xi = C.batch_ximg.as<XImg>();
    const int32_t* d_colimg = C.batch_colimg.as<int32_t>();
    int32_t* cs = C.counts.as<int32_t>();
    const uint32_t* pos = C.pos.as<uint32_t>();
    k_bx_col_start<<<nblk(n_cols), 256, 0, C.stream>>>(pos, d_xi, d_colimg, n_cols, cs);
    IDL_LAUNCH();
    k_bx_col_nearest<<<dim3(nblk(n_cols, 128), (unsigned)((max_hp + XCHUNK - 1) / XCHUNK)), 128, 0, C.stream>>>(
        pos, d_xi, d_colimg, cs, n_cols, cv.pitch, C.lab[1].as<int32_t>(), C.exact_dy.as<int32_t>());
    IDL_LAUNCH();
    if (max_wp <= HULL_MAX_W) {
        static std::atomic<uint64_t> opted{0};   // the shared-memory opt-in is per device
        const uint64_t bit = 1ull << (C.device & 63);
        if (!(opted.load(std::memory_order_acquire) & bit)) {
            IDL_CUDA(cudaFuncSetAttribute((const void*)k_bx_row_hull, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)row_hull_smem(HULL_MAX_W)));
            opted.fetch_or(bit, std::memory_order_acq_rel);
        }
        k_bx_row_hull<<<(unsigned)n_rows, HULL_THREADS, row_hull_smem(max_wp), C.stream>>>(
            C.lab[1].as<int32_t>(), C.exact_dy.as<int32_t>(), d_xi, C.batch_rowimg.as<int32_t>(), cv.pitch,
            C.lab[0].as<int32_t>());
    } else {
        k_bx_row_nearest<<<dim3((unsigned)n_rows, (unsigned)((max_wp + 255) / 256)), 256, 0, C.stream>>>(
            C.lab[1].as<int32_t>(), C.exact_dy.as<int32_t>(), d_xi, C.batch_rowimg.as<int32_t>(), cv.pitch,
            C.lab[0].as<int32_t>());
    }
    IDL_LAUNCH();
}

void run_batch(Context& C, const Plan& pl, int P, int n_images, int32_t* d_out, int64_t* tri_counts,
               float* timings, bool labels_only = false, int mode = IDL_MODE_REFERENCE)
{
    C.batch_plan.reset();
    const int64_t n = pl.n_seeds;
    C.batch_img.ensure(pl.imgs.size() * sizeof(BImg));
    C.batch_seed_img.ensure((size_t)n * 4);
    C.batch_rows.ensure((size_t)pl.n_rows * 4);
    C.batch_sid.ensure((size_t)n * 4);
    C.batch_stats.ensure(((size_t)n_images * 3 + 1) * 4);
    BImg* d_imgs = C.batch_img.as<BImg>();
    IDL_CUDA(cudaMemcpyAsync(d_imgs, pl.imgs.data(), pl.imgs.size() * sizeof(BImg), cudaMemcpyHostToDevice,
                             C.stream));
    IDL_CUDA(cudaMemcpyAsync(C.batch_seed_img.ptr, pl.seed_img.data(), (size_t)n * 4, cudaMemcpyHostToDevice,
                             C.stream));
    IDL_CUDA(cudaMemcpyAsync(C.batch_rows.ptr, pl.row_img.data(), (size_t)pl.n_rows * 4, cudaMemcpyHostToDevice,
                             C.stream));
    cudaEvent_t ev[5] = {};
    if (timings)
        for (auto& e : ev) IDL_CUDA(cudaEventCreate(&e));
    struct Ev {
        cudaEvent_t* e;
        ~Ev()
        {
            for (int i = 0; i < 5; ++i)
                if (e[i]) cudaEventDestroy(e[i]);
        }
    } ev_guard{ev};
    auto mark = [&](int i) {
        if (timings) IDL_CUDA(cudaEventRecord(ev[i], C.stream));
    };

    // validate + rank
    const int64_t nwords = (pl.n_px + 31) / 32;
    C.bitmap.ensure((size_t)nwords * 4);
    C.scan_b.ensure((size_t)nwords * 4);
    C.scan_c.ensure((size_t)(nwords + 1) * 4);
    C.xs.ensure((size_t)n * 4);
    C.ys.ensure((size_t)n * 4);
    C.pos.ensure((size_t)n * 4);
    C.batch_bad.ensure(16);
    unsigned long long* bad = C.batch_bad.as<unsigned long long>();
    IDL_CUDA(cudaMemsetAsync(C.bitmap.ptr, 0, (size_t)nwords * 4, C.stream));
    IDL_CUDA(cudaMemsetAsync(bad, 0xFF, 16, C.stream));
    mark(0);
    k_b_mark<<<nblk(n), 256, 0, C.stream>>>(C.seeds_in.as<int32_t>(), n, C.batch_seed_img.as<int32_t>(), d_imgs,
                                           C.bitmap.as<uint32_t>(), bad);
    IDL_LAUNCH();
    unsigned long long hb[2] = {0, 0};
    IDL_CUDA(cudaMemcpyAsync(hb, bad, 16, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    auto image_of = [&](unsigned long long i) { return (int)pl.seed_img[(size_t)i]; };
    if (hb[0] != ~0ull) invalid("image " + std::to_string(image_of(hb[0])) + ": seed coordinate out of bounds");
    if (hb[1] != ~0ull)
        invalid("image " + std::to_string(image_of(hb[1])) + ": duplicate seed positions are not allowed");
    k_b_popc<<<nblk(nwords), 256, 0, C.stream>>>(C.bitmap.as<uint32_t>(), nwords, C.scan_b.as<int32_t>());
    IDL_LAUNCH();
    exclusive_scan(C, C.scan_b.as<int32_t>(), C.scan_c.as<int32_t>(), nwords);
    k_b_rank<<<nblk(n), 256, 0, C.stream>>>(C.seeds_in.as<int32_t>(), n, C.batch_seed_img.as<int32_t>(), d_imgs, P,
                                           C.bitmap.as<uint32_t>(), C.scan_c.as<int32_t>(), C.xs.as<int32_t>(),
                                           C.ys.as<int32_t>(), C.pos.as<uint32_t>(), C.batch_sid.as<int32_t>());
    IDL_LAUNCH();

    // atlas planes: walls everywhere, each image's padded canvas open, seeds in
    const Canvas cv{pl.AW, pl.AH, (pl.AW + 31) / 32 * 32};
    const size_t plane = (size_t)cv.pitch * cv.Hd * 4;
    C.lab[0].ensure(plane);
    C.lab[1].ensure(plane);
    IDL_CUDA(cudaMemsetAsync(C.lab[0].ptr, 0xFE, plane, C.stream));
    IDL_CUDA(cudaMemsetAsync(C.lab[1].ptr, 0xFE, plane, C.stream));
    k_b_open<<<dim3(64, n_images), 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), C.lab[1].as<int32_t>(), cv.pitch,
                                                       d_imgs, P);
    IDL_LAUNCH();
    mark(1);
    if (mode == IDL_MODE_EXACT) {
        exact_atlas(C, pl, P, cv);
    } else {
        k_b_seeds<<<nblk(n), 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), C.lab[1].as<int32_t>(), cv.pitch,
                                                C.pos.as<uint32_t>(), n);
        IDL_LAUNCH();
        propagate(C, IDL_MODE_REFERENCE, cv, C.pos.as<uint32_t>(), n);
    }
    mark(2);
    auto bp = std::make_shared<BatchPlan>();
    bp->imgs = pl.imgs;
    bp->P = P;
    bp->pitch = cv.pitch;
    bp->n_seeds = n;
    bp->exact = mode == IDL_MODE_EXACT;
    C.batch_plan = bp;
    if (labels_only) return;
    detect_triangles(C, cv, C.lab[0].as<int32_t>(), C.pos.as<uint32_t>(), n, 0, timings ? ev[3] : nullptr);

    // per-image counts, offsets and windows; raster; compose
    int32_t* cnt = C.batch_stats.as<int32_t>();
    int32_t* side = cnt + n_images;
    int32_t* off = side + n_images;   // n_images + 1
    IDL_CUDA(cudaMemsetAsync(cnt, 0, (size_t)n_images * 2 * 4, C.stream));
    k_b_tri_stats<<<C.num_sms * 8, 256, 0, C.stream>>>(C.tris.as<int32_t>(), C.sc(), C.batch_sid.as<int32_t>(),
                                                       C.xs.as<int32_t>(), C.ys.as<int32_t>(), cnt, side);
    IDL_LAUNCH();
    exclusive_scan(C, cnt, off, n_images);
    C.tgrid.ensure((size_t)pl.n_px * 4);
    IDL_CUDA(cudaMemsetAsync(C.tgrid.ptr, 0xFF, (size_t)pl.n_px * 4, C.stream));
    k_b_raster<<<C.num_sms * 16, 256, 0, C.stream>>>(C.tris.as<int32_t>(), C.sc(), C.batch_sid.as<int32_t>(), d_imgs,
                                                     C.xs.as<int32_t>(), C.ys.as<int32_t>(), side, off,
                                                     C.tgrid.as<int32_t>());
    IDL_LAUNCH();
    int32_t* out = d_out;
    if (!out) {
        C.outgrid.ensure((size_t)pl.n_px * 12);
        out = C.outgrid.as<int32_t>();
    }
    k_b_compose<<<(unsigned)pl.n_rows, 256, 0, C.stream>>>(C.lab[0].as<int32_t>(), cv.pitch, P, d_imgs,
                                                          C.batch_rows.as<int32_t>(), C.xs.as<int32_t>(),
                                                          C.ys.as<int32_t>(), C.tgrid.as<int32_t>(), out);
    IDL_LAUNCH();
    k_b_localise<<<C.num_sms * 8, 256, 0, C.stream>>>(C.tris.as<int32_t>(), C.sc(), C.batch_sid.as<int32_t>(),
                                                      d_imgs, P);
    IDL_LAUNCH();
    mark(4);
    std::vector<int32_t> hc(n_images);
    IDL_CUDA(cudaMemcpyAsync(hc.data(), cnt, (size_t)n_images * 4, cudaMemcpyDeviceToHost, C.stream));
    C.fetch_scalars();
    C.last_n_tri = C.host_sc->n_triangles;
    C.have_result = true;
    if (tri_counts)
        for (int i = 0; i < n_images; ++i) tri_counts[i] = hc[i];
    bp->tri_off.assign((size_t)n_images + 1, 0);
    for (int i = 0; i < n_images; ++i) bp->tri_off[i + 1] = bp->tri_off[i] + hc[i];
    bp->grids = out;
    bp->full = true;
    if (timings) {
        float a = 0, b = 0, c = 0, d = 0;
        IDL_CUDA(cudaEventElapsedTime(&a, ev[1], ev[2]));
        IDL_CUDA(cudaEventElapsedTime(&b, ev[2], ev[3]));
        IDL_CUDA(cudaEventElapsedTime(&c, ev[3], ev[4]));
        IDL_CUDA(cudaEventElapsedTime(&d, ev[0], ev[1]));
        timings[IDL_T_BFS_MS] = a;
        timings[IDL_T_DETECT_MS] = b;
        timings[IDL_T_DEDUP_MS] = 0.f;
        timings[IDL_T_ASSIGN_MS] = c;
        timings[IDL_T_BFS_ITERS] = 0.f;
        (void)d;
    }
}

}  // namespace

void triangulate_batch_keep(Context& C, int n_images, const int32_t* dims, const int64_t* counts,
                            const int32_t* seeds_xy, int P, int64_t* tri_counts)
{
    if (!dims || !counts) invalid("dims and seed_counts must not be NULL");
    const Plan pl = make_plan(n_images, dims, counts, P);
    if (!seeds_xy) invalid("seeds must not be NULL");
    DeviceGuard g(C.device);
    C.have_result = false;
    C.batch_plan.reset();
    C.seeds_in.ensure((size_t)pl.n_seeds * 8);
    IDL_CUDA(cudaMemcpyAsync(C.seeds_in.ptr, seeds_xy, (size_t)pl.n_seeds * 8, cudaMemcpyHostToDevice, C.stream));
    run_batch(C, pl, P, n_images, nullptr, tri_counts, nullptr);
}

void batch_fetch(Context& C, int k, int32_t* grid_out, int32_t* tris_out, int64_t capacity)
{
    const auto* bp = static_cast<const BatchPlan*>(C.batch_plan.get());
    if (!bp || !bp->full || k < 0 || k >= (int)bp->imgs.size())
        throw Error(IDL_ERR_STATE, "no triangulated batch image " + std::to_string(k) + " on this context");
    const BImg& m = bp->imgs[k];
    if (grid_out)
        IDL_CUDA(cudaMemcpyAsync(grid_out, bp->grids + (size_t)m.px_off * 3, (size_t)m.W * m.H * 12,
                                 cudaMemcpyDeviceToHost, C.stream));
    const int64_t rows = bp->tri_off[k + 1] - bp->tri_off[k];
    if (tris_out && rows) {
        if (capacity < rows * 5) invalid("triangle buffer too small");
        IDL_CUDA(cudaMemcpyAsync(tris_out, C.tris.as<int32_t>() + bp->tri_off[k] * 5, (size_t)rows * 20,
                                 cudaMemcpyDeviceToHost, C.stream));
    }
}

bool batch_image(const Context& C, int k, BatchImage& out)
{
    const auto* lo = static_cast<const BatchPlan*>(C.batch_plan.get());
    if (!lo || lo->exact || k < 0 || k >= (int)lo->imgs.size()) return false;
    const BImg& m = lo->imgs[k];
    out.W = m.W;
    out.H = m.H;
    out.ox = m.ox;
    out.oy = m.oy;
    out.P = lo->P;
    out.pitch = lo->pitch;
    out.seed_off = m.seed_off;
    out.n = (k + 1 < (int)lo->imgs.size() ? lo->imgs[k + 1].seed_off : lo->n_seeds) - m.seed_off;
    return true;
}

}  // namespace idl

using namespace idl;

extern "C" {

int idl_voronoi_batch(idl_context* ctx, int n_images, const int32_t* dims, const int64_t* seed_counts,
                      const int32_t* seeds_xy, int border_padding, int mode)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    if (!dims || !seed_counts) invalid("dims and seed_counts must not be NULL");
    if (mode != IDL_MODE_REFERENCE) invalid("batched propagation supports voronoi_mode 'reference' only");
    const int P = border_padding == IDL_AUTO_BORDER_PADDING ? IDL_DEFAULT_BORDER_PADDING
                                                            : std::max(0, border_padding);
    const Plan pl = make_plan(n_images, dims, seed_counts, P);
    if (!seeds_xy) invalid("seeds must not be NULL");
    DeviceGuard g(ctx->device);
    Context& C = *ctx;
    C.have_result = false;
    C.batch_plan.reset();
    C.seeds_in.ensure((size_t)pl.n_seeds * 8);
    IDL_CUDA(cudaMemcpyAsync(C.seeds_in.ptr, seeds_xy, (size_t)pl.n_seeds * 8, cudaMemcpyHostToDevice, C.stream));
    run_batch(C, pl, P, n_images, nullptr, nullptr, nullptr, true);
    IDL_API_END
}

int idl_triangulate_batch(idl_context* ctx, int n_images, const int32_t* dims, const int64_t* seed_counts,
                          const int32_t* seeds_xy, int border_padding, int mode, int32_t* grids_out,
                          int64_t* tri_counts_out, float* timings_out)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    if (!dims || !seed_counts) invalid("dims and seed_counts must not be NULL");
    if (mode != IDL_MODE_REFERENCE && mode != IDL_MODE_EXACT)
        invalid("batched triangulation supports voronoi_mode 'reference' and 'exact'");
    const int P = border_padding == IDL_AUTO_BORDER_PADDING ? IDL_DEFAULT_BORDER_PADDING
                                                            : std::max(0, border_padding);
    const Plan pl = make_plan(n_images, dims, seed_counts, P);
    if (!seeds_xy) invalid("seeds must not be NULL");
    DeviceGuard g(ctx->device);
    Context& C = *ctx;
    C.have_result = false;
    C.seeds_in.ensure((size_t)pl.n_seeds * 8);
    IDL_CUDA(cudaMemcpyAsync(C.seeds_in.ptr, seeds_xy, (size_t)pl.n_seeds * 8, cudaMemcpyHostToDevice, C.stream));
    run_batch(C, pl, P, n_images, nullptr, tri_counts_out, timings_out, false, mode);
    if (grids_out)
        IDL_CUDA(cudaMemcpyAsync(grids_out, C.outgrid.ptr, (size_t)pl.n_px * 12, cudaMemcpyDeviceToHost, C.stream));
    IDL_CUDA(cudaStreamSynchronize(C.stream));
    IDL_API_END
}

int idl_triangulate_batch_device(idl_context* ctx, int n_images, const int32_t* dims, const int64_t* seed_counts,
                                 const int32_t* d_seeds_xy, int border_padding, int mode, int32_t* d_grids_out,
                                 int64_t* tri_counts_out)
{
    IDL_API_BEGIN
    if (!ctx) invalid("context must not be NULL");
    if (!dims || !seed_counts) invalid("dims and seed_counts must not be NULL");
    if (mode != IDL_MODE_REFERENCE && mode != IDL_MODE_EXACT)
        invalid("batched triangulation supports voronoi_mode 'reference' and 'exact'");
    const int P = border_padding == IDL_AUTO_BORDER_PADDING ? IDL_DEFAULT_BORDER_PADDING
                                                            : std::max(0, border_padding);
    const Plan pl = make_plan(n_images, dims, seed_counts, P);
    if (!d_seeds_xy || !d_grids_out) invalid("device buffers must not be NULL");
    DeviceGuard g(ctx->device);
    Context& C = *ctx;
    C.have_result = false;
    C.seeds_in.ensure((size_t)pl.n_seeds * 8);
    IDL_CUDA(cudaMemcpyAsync(C.seeds_in.ptr, d_seeds_xy, (size_t)pl.n_seeds * 8, cudaMemcpyDeviceToDevice,
                             C.stream));
    run_batch(C, pl, P, n_images, d_grids_out, tri_counts_out, nullptr, false, mode);
    IDL_API_END
}

}  // extern "C"
