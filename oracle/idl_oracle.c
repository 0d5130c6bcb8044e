/*
 * CPU oracle for the integer Delaunay hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Nothing in the product links or calls this file.  It is loaded by tests/,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, always as
 * the checker or the timed CPU baseline, never as the thing measured.
 *
 * Every function restates one piece of the reference algorithm in plain C,
 * citing the reference file:line it follows (paths relative to the
 * timdahmen/integer_delauney project root):
 *
 *   or_voronoi_jacobi      src/cuda/voronoi.cu:32-53,100-113 and
 *                          src/cuda/geometry_device.cuh:22-66
 *   or_voronoi_sweep       src/delauney/reference/voronoi.py:90-163
 *   or_voronoi_nearest     the contract stated in
 *                          src/delauney/reference/voronoi.py:9-31
 *                          (nearest seed, ties to the higher seed id)
 *   or_detect              src/cuda/triangle_detect.cuh:75-182
 *   or_dedup               src/cuda/triangulation.cu:254-256 (tid = rank of
 *                          the sorted triple); the surviving witness is made
 *                          deterministic (smallest row-major block index)
 *   or_assign              src/cuda/triangulation.cu:79-137,355-368 and
 *                          src/cuda/geometry_device.cuh:68-86
 *   or_assign_bbox_rows    the same rule per triangle over its bounding box
 *   or_triangulate         src/cuda/triangulation.cu:143-365
 *
 * Parity is pinned in tests/ against golden vectors generated from the
 * reference's own NumPy implementation (tests/golden/) and, on a B200, the
 * reference's own CUDA batch path built into oracle/_ref.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define UNDEF (-1)

static inline int32_t d2(int x, int y, int32_t sx, int32_t sy)
{
    int32_t dx = x - sx, dy = y - sy;
    return dx * dx + dy * dy;
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------
 * Stage (a), reference CUDA semantics: synchronous Jacobi to a fixed point.
 *
 * voronoi.cu:100-113 runs one voronoi_step_kernel per pass until no pixel
 * changes; each pixel takes the best (d, id) among itself and its 4
 * neighbours' owners (geometry_device.cuh:40-66), lower d first, higher id on
 * a tie (geometry_device.cuh:22-28).  d is recomputed from the owner seed,
 * never accumulated.  `lab` holds the starting state (seed pixels set, the
 * rest UNDEF for a batch run; a previous fixed point plus newly written seeds
 * for the incremental path, delaunay_voronoi.cu:12-25,66-108) and receives the
 * fixed point.  Returns the number of passes run, including the last pass
 * that changed nothing, as the reference's loop does.
 * ---------------------------------------------------------------------- */
int64_t or_voronoi_jacobi(int W, int H, const int32_t* sx, const int32_t* sy,
                          int32_t* lab, int64_t max_passes)
{
    const size_t N = (size_t)W * H;
    int32_t* tmp = (int32_t*)malloc(N * sizeof(int32_t));
    int32_t* src = lab;
    int32_t* dst = tmp;
    int64_t passes = 0;
    for (;;) {
        int changed = 0;
#pragma omp parallel for schedule(static) reduction(| : changed)
        for (int y = 0; y < H; ++y) {
            for (int x = 0; x < W; ++x) {
                const int32_t cur = src[(size_t)y * W + x];
                int32_t best = cur;
                int32_t bd = cur >= 0 ? d2(x, y, sx[cur], sy[cur]) : -1;
                const int nx[4] = {x - 1, x + 1, x, x};
                const int ny[4] = {y, y, y - 1, y + 1};
                for (int k = 0; k < 4; ++k) {
                    if (nx[k] < 0 || nx[k] >= W || ny[k] < 0 || ny[k] >= H) continue;
                    const int32_t n = src[(size_t)ny[k] * W + nx[k]];
                    if (n == UNDEF) continue;
                    const int32_t nd = d2(x, y, sx[n], sy[n]);
                    if (best == UNDEF || nd < bd || (nd == bd && n > best)) {
                        best = n;
                        bd = nd;
                    }
                }
                dst[(size_t)y * W + x] = best;
                if (best != cur) changed = 1;
            }
        }
        int32_t* t = src; src = dst; dst = t;
        ++passes;
        if (!changed || (max_passes > 0 && passes >= max_passes)) break;
    }
    if (src != lab) memcpy(lab, src, N * sizeof(int32_t));
    free(tmp);
    return passes;
}

/* ------------------------------------------------------------------------
 * Stage (a), NumPy reference semantics (reference/voronoi.py:90-163).
 *
 * One iteration is four directional sub-steps applied in sequence: take the
 * owner of the left, right, upper, lower neighbour (voronoi.py:115-134) and
 * adopt it where the cell is undefined, strictly closer, or equally close
 * with a higher id (voronoi.py:136-154).  Each sub-step is synchronous over
 * the whole grid (NumPy evaluates the shifted copy before assigning); doing
 * it in place in the scan order that reads only not-yet-updated cells is the
 * same thing.  Loops until an iteration changes nothing.  Returns iterations.
 * ---------------------------------------------------------------------- */
static inline int sweep_try(int x, int y, int32_t* cell, int32_t n,
                            const int32_t* sx, const int32_t* sy)
{
    if (n == UNDEF) return 0;
    const int32_t cur = *cell;
    const int32_t cd = d2(x, y, sx[n], sy[n]);
    if (cur == UNDEF) { *cell = n; return 1; }
    const int32_t dcur = d2(x, y, sx[cur], sy[cur]);
    if (cd < dcur || (cd == dcur && n > cur)) { *cell = n; return 1; }
    return 0;
}

int64_t or_voronoi_sweep(int W, int H, const int32_t* sx, const int32_t* sy,
                         int32_t* lab, int64_t max_iters)
{
    int64_t iters = 0;
    for (;;) {
        int changed = 0;
        /* neighbour on the left: n[x] = s[x-1]; descending x reads old values */
#pragma omp parallel for schedule(static) reduction(| : changed)
        for (int y = 0; y < H; ++y) {
            int32_t* row = lab + (size_t)y * W;
            for (int x = W - 1; x >= 1; --x) changed |= sweep_try(x, y, &row[x], row[x - 1], sx, sy);
        }
        /* neighbour on the right: n[x] = s[x+1]; ascending x */
#pragma omp parallel for schedule(static) reduction(| : changed)
        for (int y = 0; y < H; ++y) {
            int32_t* row = lab + (size_t)y * W;
            for (int x = 0; x + 1 < W; ++x) changed |= sweep_try(x, y, &row[x], row[x + 1], sx, sy);
        }
        /* neighbour above: n[y] = s[y-1]; descending y */
#pragma omp parallel for schedule(static) reduction(| : changed)
        for (int x = 0; x < W; ++x) {
            for (int y = H - 1; y >= 1; --y)
                changed |= sweep_try(x, y, &lab[(size_t)y * W + x], lab[(size_t)(y - 1) * W + x], sx, sy);
        }
        /* neighbour below: n[y] = s[y+1]; ascending y */
#pragma omp parallel for schedule(static) reduction(| : changed)
        for (int x = 0; x < W; ++x) {
            for (int y = 0; y + 1 < H; ++y)
                changed |= sweep_try(x, y, &lab[(size_t)y * W + x], lab[(size_t)(y + 1) * W + x], sx, sy);
        }
        ++iters;
        if (!changed || (max_iters > 0 && iters >= max_iters)) break;
    }
    return iters;
}

/* ------------------------------------------------------------------------
 * Stage (a), exact nearest seed with ties to the higher id: the contract
 * reference/voronoi.py:9-31 describes.  Seeds are bucketed on a coarse grid
 * and searched ring by ring until no unvisited bucket can hold a seed at a
 * distance <= the best found (<= because an equally near seed with a higher
 * id would still win).
 * ---------------------------------------------------------------------- */
void or_voronoi_nearest(int W, int H, const int32_t* sx, const int32_t* sy,
                        int n, int32_t* lab)
{
    const int B = 16;
    const int BX = (W + B - 1) / B, BY = (H + B - 1) / B;
    int* cnt = (int*)calloc((size_t)BX * BY + 1, sizeof(int));
    int* idx = (int*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    for (int i = 0; i < n; ++i) cnt[(sy[i] / B) * BX + sx[i] / B + 1]++;
    for (int b = 0; b < BX * BY; ++b) cnt[b + 1] += cnt[b];
    int* fill = (int*)calloc((size_t)BX * BY, sizeof(int));
    for (int i = 0; i < n; ++i) {
        const int b = (sy[i] / B) * BX + sx[i] / B;
        idx[cnt[b] + fill[b]++] = i;
    }
    const int maxr = (BX > BY ? BX : BY);
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            int32_t best = UNDEF;
            int64_t bd = -1;
            const int bx = x / B, by = y / B;
            for (int r = 0; r <= maxr; ++r) {
                /* every bucket at Chebyshev ring r is at least (r-1)*B+1 px away */
                if (best != UNDEF && r >= 1) {
                    const int64_t gap = (int64_t)(r - 1) * B + 1;
                    if (gap * gap > bd) break;
                }
                for (int cy = by - r; cy <= by + r; ++cy) {
                    if (cy < 0 || cy >= BY) continue;
                    for (int cx = bx - r; cx <= bx + r; ++cx) {
                        if (cx < 0 || cx >= BX) continue;
                        if (cx != bx - r && cx != bx + r && cy != by - r && cy != by + r) continue;
                        const int b = cy * BX + cx;
                        for (int k = cnt[b]; k < cnt[b + 1]; ++k) {
                            const int s = idx[k];
                            const int64_t dx = x - sx[s], dy = y - sy[s];
                            const int64_t d = dx * dx + dy * dy;
                            if (best == UNDEF || d < bd || (d == bd && s > best)) { best = s; bd = d; }
                        }
                    }
                }
            }
            lab[(size_t)y * W + x] = best;
        }
    }
    free(cnt); free(idx); free(fill);
}

/* ------------------------------------------------------------------------
 * Stage (b): the 2x2 block rule, triangle_detect.cuh:75-166, restated with
 * the reference's own double-precision atan2 and stable insertion sort.
 * ---------------------------------------------------------------------- */
typedef struct {
    int32_t a, b, c;            /* sorted key */
    int32_t oa, ob, oc;         /* order the block saw */
    int64_t block;              /* row-major index of the block's top-left */
} or_raw_t;

typedef struct {
    or_raw_t* v;
    size_t n, cap;
} raw_vec;

static void raw_push(raw_vec* r, int32_t oa, int32_t ob, int32_t oc, int64_t block)
{
    if (r->n == r->cap) {
        r->cap = r->cap ? r->cap * 2 : 1024;
        r->v = (or_raw_t*)realloc(r->v, r->cap * sizeof(or_raw_t));
    }
    int32_t s0 = oa, s1 = ob, s2 = oc, t;
    if (s0 > s1) { t = s0; s0 = s1; s1 = t; }
    if (s1 > s2) { t = s1; s1 = s2; s2 = t; }
    if (s0 > s1) { t = s0; s0 = s1; s1 = t; }
    or_raw_t e = {s0, s1, s2, oa, ob, oc, block};
    r->v[r->n++] = e;
}

/* emits 0, 1 or 2 triangles; returns count, writes orig triples to out[k][3] */
int or_block_rule(int32_t a, int32_t b, int32_t c, int32_t d,
                  const int32_t* sx, const int32_t* sy, int32_t out[2][3])
{
    const int32_t quad[4] = {a, b, c, d};
    int32_t s[4];
    int n = 0;
    for (int i = 0; i < 4; ++i) {
        if (quad[i] == UNDEF) return 0;
        int dup = 0;
        for (int j = 0; j < n; ++j) if (s[j] == quad[i]) { dup = 1; break; }
        if (!dup) s[n++] = quad[i];
    }
    if (n == 3) { out[0][0] = s[0]; out[0][1] = s[1]; out[0][2] = s[2]; return 1; }
    if (n != 4) return 0;

    double cx = 0.0, cy = 0.0;
    for (int i = 0; i < 4; ++i) { cx += sx[quad[i]]; cy += sy[quad[i]]; }
    cx *= 0.25; cy *= 0.25;
    double ang[4];
    for (int i = 0; i < 4; ++i)
        ang[i] = atan2((double)sy[quad[i]] - cy, (double)sx[quad[i]] - cx);
    int ord[4] = {0, 1, 2, 3};
    for (int i = 1; i < 4; ++i) {
        int k = ord[i], j = i - 1;
        while (j >= 0 && ang[ord[j]] > ang[k]) { ord[j + 1] = ord[j]; --j; }
        ord[j + 1] = k;
    }
#define LEN2(i, j) (((int64_t)sx[quad[i]] - sx[quad[j]]) * ((int64_t)sx[quad[i]] - sx[quad[j]]) + \
                    ((int64_t)sy[quad[i]] - sy[quad[j]]) * ((int64_t)sy[quad[i]] - sy[quad[j]]))
    const int d0a = ord[0], d0b = ord[2], d1a = ord[1], d1b = ord[3];
    const int64_t l0 = LEN2(d0a, d0b), l1 = LEN2(d1a, d1b);
#undef LEN2
    int pa, pb;
    if (l0 < l1) { pa = d0a; pb = d0b; }
    else if (l1 < l0) { pa = d1a; pb = d1b; }
    else {
        int lowest = 0;
        for (int i = 1; i < 4; ++i) if (quad[i] < quad[lowest]) lowest = i;
        if (lowest == d0a || lowest == d0b) { pa = d1a; pb = d1b; }
        else { pa = d0a; pb = d0b; }
    }
    int ra = -1, rb = -1;
    for (int i = 0; i < 4; ++i) {
        if (i == pa || i == pb) continue;
        if (ra < 0) ra = i; else rb = i;
    }
    out[0][0] = quad[pa]; out[0][1] = quad[pb]; out[0][2] = quad[ra];
    out[1][0] = quad[pa]; out[1][1] = quad[pb]; out[1][2] = quad[rb];
    return 2;
}

static int raw_cmp(const void* p, const void* q)
{
    const or_raw_t* a = (const or_raw_t*)p;
    const or_raw_t* b = (const or_raw_t*)q;
    if (a->a != b->a) return a->a < b->a ? -1 : 1;
    if (a->b != b->b) return a->b < b->b ? -1 : 1;
    if (a->c != b->c) return a->c < b->c ? -1 : 1;
    if (a->block != b->block) return a->block < b->block ? -1 : 1;
    return 0;
}

/*
 * Detect over a W x H label grid and deduplicate.  Writes up to `cap`
 * triangles as 5 int32 each: (x, y, orig_a, orig_b, orig_c) with (x, y) the
 * witnessing block's top-left corner shifted by (-shift, -shift)
 * (triangulation.cu:270-271,326-327).  Triangles are numbered by the rank of
 * their sorted triple (thrust::sort(RawLess) + unique, triangulation.cu:254);
 * among duplicates the one from the smallest row-major block index is kept.
 * Returns the number of triangles, or -(needed) if cap is too small.
 */
int64_t or_detect(int W, int H, const int32_t* lab, const int32_t* sx, const int32_t* sy,
                  int shift, int32_t* tri_out, int64_t cap)
{
    raw_vec r = {0, 0, 0};
    for (int y = 0; y + 1 < H; ++y) {
        for (int x = 0; x + 1 < W; ++x) {
            int32_t out[2][3];
            const int k = or_block_rule(lab[(size_t)y * W + x], lab[(size_t)y * W + x + 1],
                                        lab[(size_t)(y + 1) * W + x], lab[(size_t)(y + 1) * W + x + 1],
                                        sx, sy, out);
            for (int e = 0; e < k; ++e)
                raw_push(&r, out[e][0], out[e][1], out[e][2], (int64_t)y * W + x);
        }
    }
    qsort(r.v, r.n, sizeof(or_raw_t), raw_cmp);
    int64_t nt = 0;
    for (size_t i = 0; i < r.n; ++i) {
        if (i > 0 && r.v[i].a == r.v[i - 1].a && r.v[i].b == r.v[i - 1].b && r.v[i].c == r.v[i - 1].c)
            continue;
        if (nt < cap) {
            int32_t* o = tri_out + nt * 5;
            o[0] = (int32_t)(r.v[i].block % W) - shift;
            o[1] = (int32_t)(r.v[i].block / W) - shift;
            o[2] = r.v[i].oa; o[3] = r.v[i].ob; o[4] = r.v[i].oc;
        }
        ++nt;
    }
    free(r.v);
    return nt <= cap ? nt : -nt;
}

/* ------------------------------------------------------------------------
 * Stage (d): pixel assignment exactly as triangulation.cu:101-137 computes it.
 *
 * window_cap = max(20, max_side + 3) with max_side the longest side over all
 * triangles, as truncated float sqrt of float squared length
 * (triangulation.cu:355-368).  Per pixel: every seed within Chebyshev
 * window_cap, every triangle of that seed (seed -> triangle CSR,
 * triangle_csr.cuh:13-39), closed float point-in-triangle
 * (geometry_device.cuh:68-86), highest tid wins, -1 if none.
 * Compile with -ffp-contract=off so float expressions round like the
 * reference's separate multiplies and adds.
 * ---------------------------------------------------------------------- */
static float cross2f(float ox, float oy, float ax, float ay, float bx, float by)
{
    float t1 = (ax - ox) * (by - oy);
    float t2 = (ay - oy) * (bx - ox);
    return t1 - t2;
}

static int pit_f(float px, float py, float ax, float ay, float bx, float by, float cx, float cy)
{
    float d1 = cross2f(px, py, ax, ay, bx, by);
    float d2_ = cross2f(px, py, bx, by, cx, cy);
    float d3 = cross2f(px, py, cx, cy, ax, ay);
    int has_neg = (d1 < 0.f) || (d2_ < 0.f) || (d3 < 0.f);
    int has_pos = (d1 > 0.f) || (d2_ > 0.f) || (d3 > 0.f);
    return !(has_neg && has_pos);
}

int or_window_cap(const int32_t* tris, int64_t ntri, const int32_t* sx, const int32_t* sy)
{
    int max_side = 0;
    for (int64_t t = 0; t < ntri; ++t) {
        const int32_t* v = tris + t * 5 + 2;
        const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        for (int k = 0; k < 3; ++k) {
            float dx = (float)(sx[v[pairs[k][0]]] - sx[v[pairs[k][1]]]);
            float dy = (float)(sy[v[pairs[k][0]]] - sy[v[pairs[k][1]]]);
            float sq = dx * dx;
            float sq2 = dy * dy;
            float s = sq + sq2;
            int l = (int)sqrtf(s);
            if (l > max_side) max_side = l;
        }
    }
    int wc = max_side + 3;
    return wc > 20 ? wc : 20;
}

void or_assign(int W, int H, const int32_t* sx, const int32_t* sy, int n,
               const int32_t* tris, int64_t ntri, int32_t* tgrid)
{
    if (ntri == 0) {
        for (size_t i = 0; i < (size_t)W * H; ++i) tgrid[i] = -1;
        return;
    }
    const int wc = or_window_cap(tris, ntri, sx, sy);
    int32_t* ptr = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    for (int64_t t = 0; t < ntri; ++t)
        for (int k = 0; k < 3; ++k) ptr[tris[t * 5 + 2 + k] + 1]++;
    for (int s = 0; s < n; ++s) ptr[s + 1] += ptr[s];
    int32_t* idx = (int32_t*)malloc((size_t)(ptr[n] > 0 ? ptr[n] : 1) * sizeof(int32_t));
    int32_t* fill = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    for (int64_t t = 0; t < ntri; ++t)
        for (int k = 0; k < 3; ++k) {
            const int32_t s = tris[t * 5 + 2 + k];
            idx[ptr[s] + fill[s]++] = (int32_t)t;
        }
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const float px = (float)x, py = (float)y;
            int32_t best = -1;
            for (int s = 0; s < n; ++s) {
                if (abs(sx[s] - x) > wc) continue;
                if (abs(sy[s] - y) > wc) continue;
                for (int j = ptr[s]; j < ptr[s + 1]; ++j) {
                    const int32_t t = idx[j];
                    const int32_t* v = tris + (int64_t)t * 5 + 2;
                    if (pit_f(px, py, (float)sx[v[0]], (float)sy[v[0]], (float)sx[v[1]], (float)sy[v[1]],
                              (float)sx[v[2]], (float)sy[v[2]]))
                        if (best == -1 || t > best) best = t;
                }
            }
            tgrid[(size_t)y * W + x] = best;
        }
    }
    free(ptr); free(idx); free(fill);
}

/* The same assignment as or_assign (src/cuda/triangulation.cu:101-137: the
 * highest triangle index whose closed float test contains the pixel, -1 if
 * none), evaluated per triangle instead of per pixel over the seed window.
 * A proper triangle containing a pixel has the pixel inside its bounding box,
 * within its longest side of every vertex and so inside the window or_assign
 * searches; its bounding box is scanned.  A degenerate (collinear) triangle
 * passes the closed test at every pixel of its supporting line, and or_assign
 * finds it wherever one of its vertices lies within the window cap
 * (Chebyshev distance); the union of those windows is scanned with that
 * condition.  Both loops thus test the same (pixel, triangle) pairs that can
 * succeed, with the same test; this one costs the triangles' box areas
 * instead of pixels x seeds, which makes full-size checks feasible.  Rows
 * [y0, y1) of the W x H grid into tgrid_rows. */
void or_assign_bbox_rows(int W, int H, const int32_t* sx, const int32_t* sy, const int32_t* tris, int64_t ntri,
                         int y0, int y1, int32_t* tgrid_rows)
{
    (void)H;
    const size_t n_px = (size_t)(y1 - y0) * W;
    for (size_t i = 0; i < n_px; ++i) tgrid_rows[i] = -1;
    if (ntri == 0) return;
    const int wc = or_window_cap(tris, ntri, sx, sy);
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    const int rows = y1 - y0;
    const int chunk = (rows + nthreads - 1) / nthreads;
#pragma omp parallel for schedule(static, 1)
    for (int c = 0; c < nthreads; ++c) {
        const int r0 = y0 + c * chunk, r1 = r0 + chunk < y1 ? r0 + chunk : y1;
        if (r0 >= r1) continue;
        for (int64_t t = 0; t < ntri; ++t) {     /* ascending: a later containing triangle wins */
            const int32_t* v = tris + t * 5 + 2;
            const int ax = sx[v[0]], ay = sy[v[0]], bx = sx[v[1]], by = sy[v[1]], cx = sx[v[2]], cy = sy[v[2]];
            const int64_t area2 = (int64_t)(bx - ax) * (cy - ay) - (int64_t)(by - ay) * (cx - ax);
            const int pad = area2 == 0 ? wc : 0;
            int lo_y = ay < by ? ay : by;
            lo_y = (lo_y < cy ? lo_y : cy) - pad;
            int hi_y = ay > by ? ay : by;
            hi_y = (hi_y > cy ? hi_y : cy) + pad;
            if (hi_y < r0 || lo_y >= r1) continue;
            int lo_x = ax < bx ? ax : bx;
            lo_x = (lo_x < cx ? lo_x : cx) - pad;
            int hi_x = ax > bx ? ax : bx;
            hi_x = (hi_x > cx ? hi_x : cx) + pad;
            if (lo_x < 0) lo_x = 0;
            if (hi_x > W - 1) hi_x = W - 1;
            if (lo_y < r0) lo_y = r0;
            if (hi_y > r1 - 1) hi_y = r1 - 1;
            for (int y = lo_y; y <= hi_y; ++y)
                for (int x = lo_x; x <= hi_x; ++x) {
                    if (pad && !((abs(ax - x) <= wc && abs(ay - y) <= wc) || (abs(bx - x) <= wc && abs(by - y) <= wc) ||
                                 (abs(cx - x) <= wc && abs(cy - y) <= wc)))
                        continue;
                    if (pit_f((float)x, (float)y, (float)ax, (float)ay, (float)bx, (float)by, (float)cx, (float)cy))
                        tgrid_rows[(size_t)(y - y0) * W + x] = (int32_t)t;
                }
        }
    }
}

/* assignment restricted to rows [y0, y1), for bounded CPU-baseline samples */
void or_assign_rows(int W, int H, const int32_t* sx, const int32_t* sy, int n,
                    const int32_t* tris, int64_t ntri, int y0, int y1, int32_t* tgrid_rows)
{
    (void)H;
    const int wc = or_window_cap(tris, ntri, sx, sy);
    int32_t* ptr = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    for (int64_t t = 0; t < ntri; ++t)
        for (int k = 0; k < 3; ++k) ptr[tris[t * 5 + 2 + k] + 1]++;
    for (int s = 0; s < n; ++s) ptr[s + 1] += ptr[s];
    int32_t* idx = (int32_t*)malloc((size_t)(ptr[n] > 0 ? ptr[n] : 1) * sizeof(int32_t));
    int32_t* fill = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    for (int64_t t = 0; t < ntri; ++t)
        for (int k = 0; k < 3; ++k) {
            const int32_t s = tris[t * 5 + 2 + k];
            idx[ptr[s] + fill[s]++] = (int32_t)t;
        }
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = y0; y < y1; ++y) {
        for (int x = 0; x < W; ++x) {
            const float px = (float)x, py = (float)y;
            int32_t best = -1;
            for (int s = 0; s < n; ++s) {
                if (abs(sx[s] - x) > wc) continue;
                if (abs(sy[s] - y) > wc) continue;
                for (int j = ptr[s]; j < ptr[s + 1]; ++j) {
                    const int32_t t = idx[j];
                    const int32_t* v = tris + (int64_t)t * 5 + 2;
                    if (pit_f(px, py, (float)sx[v[0]], (float)sy[v[0]], (float)sx[v[1]], (float)sy[v[1]],
                              (float)sx[v[2]], (float)sy[v[2]]))
                        if (best == -1 || t > best) best = t;
                }
            }
            tgrid_rows[(size_t)(y - y0) * W + x] = best;
        }
    }
    free(ptr); free(idx); free(fill);
}

/* ------------------------------------------------------------------------
 * The whole batch pipeline, triangulation.cu:143-365.
 *
 * mode: 0 = reference CUDA Jacobi, 1 = NumPy sweep, 2 = exact nearest.
 * Seeds must already be sorted by (x, y) and distinct (the binding's
 * sort_seeds, binding_helpers.hpp:23-46).  vgrid_in (H*W*2, may be NULL)
 * drives detection only at P == 0, as in the reference.
 * out_grid receives H*W*3 int32 (seed id, squared distance, triangle id).
 * tri_out receives up to cap triangles (5 int32 each); returns the count or
 * -(needed) when cap is too small.  passes_out (may be NULL) receives the
 * propagation pass count.
 * ---------------------------------------------------------------------- */
static int64_t run_mode(int mode, int W, int H, const int32_t* sx, const int32_t* sy, int n, int32_t* lab)
{
    if (mode == 2) { or_voronoi_nearest(W, H, sx, sy, n, lab); return 0; }
    for (size_t i = 0; i < (size_t)W * H; ++i) lab[i] = UNDEF;
    for (int i = 0; i < n; ++i) lab[(size_t)sy[i] * W + sx[i]] = i;
    if (mode == 1) return or_voronoi_sweep(W, H, sx, sy, lab, 0);
    return or_voronoi_jacobi(W, H, sx, sy, lab, 0);
}

int64_t or_voronoi(int mode, int W, int H, const int32_t* sx, const int32_t* sy, int n, int32_t* out_grid2)
{
    int32_t* lab = (int32_t*)malloc((size_t)W * H * sizeof(int32_t));
    const int64_t passes = run_mode(mode, W, H, sx, sy, n, lab);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int32_t l = lab[(size_t)y * W + x];
            out_grid2[((size_t)y * W + x) * 2] = l;
            out_grid2[((size_t)y * W + x) * 2 + 1] = l >= 0 ? d2(x, y, sx[l], sy[l]) : -1;
        }
    free(lab);
    return passes;
}

int64_t or_triangulate(int W, int H, const int32_t* sx, const int32_t* sy, int n, int P, int mode,
                       const int32_t* vgrid_in, int32_t* out_grid, int32_t* tri_out, int64_t cap,
                       int64_t* passes_out)
{
    const int Wd = W + 2 * P, Hd = H + 2 * P;
    int32_t* lab = (int32_t*)malloc((size_t)Wd * Hd * sizeof(int32_t));
    int64_t passes = 0;
    if (P > 0) {
        int32_t* px = (int32_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
        int32_t* py = (int32_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
        for (int i = 0; i < n; ++i) { px[i] = sx[i] + P; py[i] = sy[i] + P; }
        passes = run_mode(mode, Wd, Hd, px, py, n, lab);
        free(px); free(py);
    } else if (vgrid_in) {
        for (size_t i = 0; i < (size_t)W * H; ++i) lab[i] = vgrid_in[i * 2];
    } else {
        passes = run_mode(mode, W, H, sx, sy, n, lab);
    }
    if (passes_out) *passes_out = passes;

    /* detection runs on the padded canvas with padded seed coordinates */
    int32_t* dx = (int32_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    int32_t* dy = (int32_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    for (int i = 0; i < n; ++i) { dx[i] = sx[i] + P; dy[i] = sy[i] + P; }
    int64_t nt = or_detect(Wd, Hd, lab, dx, dy, P, tri_out, cap);
    free(dx); free(dy);
    if (nt < 0) { free(lab); return nt; }

    int32_t* tg = (int32_t*)malloc((size_t)W * H * sizeof(int32_t));
    or_assign(W, H, sx, sy, n, tri_out, nt, tg);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t o = ((size_t)y * W + x) * 3;
            if (P > 0 || !vgrid_in) {
                const int32_t l = lab[(size_t)(y + P) * Wd + (x + P)];
                out_grid[o] = l;
                out_grid[o + 1] = l >= 0 ? d2(x, y, sx[l], sy[l]) : -1;
            } else {
                out_grid[o] = vgrid_in[((size_t)y * W + x) * 2];
                out_grid[o + 1] = vgrid_in[((size_t)y * W + x) * 2 + 1];
            }
            out_grid[o + 2] = tg[(size_t)y * W + x];
        }
    free(tg);
    free(lab);
    return nt;
}
