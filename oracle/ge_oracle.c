/*
 * ge_oracle.c -- CPU restatement of Galaxy Engine's gravity path.
 * TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline); see ge_oracle.h
 * for the reference line map and the deliberate conventions.
 *
 * Built twice by oracle/Makefile:
 *   liboracle.so      -ffp-contract=off : every float operation rounds on its
 *                     own, as written.  This is the strict parity oracle.
 *   liboracle_fma.so  GCC's default for gnu modes (-ffp-contract=fast) with
 *                     -mavx2 -mfma, i.e. the reference's shipped flags
 *                     (CMakeLists.txt:57,61,68).  Used to measure how much
 *                     FMA contraction alone moves the results.
 */
#include "ge_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <immintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EMPTY UINT32_MAX

static double now_ms(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

/* ------------------------------------------------------------------ */
/* bounding box: globalLogic.cpp:1083-1099 / :1460-1477                */
/* glm::min/max per component, then a square (cube) of side equal to   */
/* the largest extent, centred on the extents.                          */
/* ------------------------------------------------------------------ */
static inline float fmin_ref(float a, float b) { return (b < a) ? b : a; }
static inline float fmax_ref(float a, float b) { return (a < b) ? b : a; }

void or_bbox2d(int64_t n, const float *x, const float *y, float out[3]) {
    float lox = FLT_MAX, loy = FLT_MAX, hix = -FLT_MAX, hiy = -FLT_MAX;
    for (int64_t i = 0; i < n; i++) {
        lox = fmin_ref(lox, x[i]); loy = fmin_ref(loy, y[i]);
        hix = fmax_ref(hix, x[i]); hiy = fmax_ref(hiy, y[i]);
    }
    float ex = hix - lox, ey = hiy - loy;
    float size = fmax_ref(ex, ey);
    float cx = (lox + hix) * 0.5f, cy = (loy + hiy) * 0.5f;
    out[0] = cx - size * 0.5f;
    out[1] = cy - size * 0.5f;
    out[2] = size;
}

void or_bbox3d(int64_t n, const float *x, const float *y, const float *z, float out[4]) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = 0; i < n; i++) {
        lo[0] = fmin_ref(lo[0], x[i]); hi[0] = fmax_ref(hi[0], x[i]);
        lo[1] = fmin_ref(lo[1], y[i]); hi[1] = fmax_ref(hi[1], y[i]);
        lo[2] = fmin_ref(lo[2], z[i]); hi[2] = fmax_ref(hi[2], z[i]);
    }
    float size = fmax_ref(fmax_ref(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
    for (int a = 0; a < 3; a++) out[a] = (lo[a] + hi[a]) * 0.5f - size * 0.5f;
    out[3] = size;
}

/* ------------------------------------------------------------------ */
/* Morton keys: morton.cpp:3-38 (2D, 18 bits/axis, scale 2^18)          */
/*              morton.cpp:67-112 (3D, 21 bits/axis, scale 2^21-1)      */
/* ------------------------------------------------------------------ */
static inline float clampf_ref(float v, float lo, float hi) {
    /* std::clamp(v, lo, hi): v < lo ? lo : (hi < v ? hi : v) */
    return (v < lo) ? lo : ((hi < v) ? hi : v);
}

uint64_t or_scale_to_grid2d(float p, float lo, float hi) {
    if (hi <= lo) return 0;
    float c = clampf_ref(p, lo, hi);
    float u = (c - lo) / (hi - lo);
    uint64_t q = (uint64_t)(u * 262144.0f);
    return q < 262143u ? q : 262143u;
}

uint64_t or_scale_to_grid3d(float p, float lo, float hi) {
    if (hi <= lo) return 0;
    float c = clampf_ref(p, lo, hi);
    float u = (c - lo) / (hi - lo);
    uint64_t q = (uint64_t)(u * 2097151.0f);
    return q < 2097151u ? q : 2097151u;
}

/* interleave: bit b of v goes to bit stride*b */
static inline uint64_t spread(uint64_t v, int bits, int stride) {
    uint64_t r = 0;
    for (int b = 0; b < bits; b++) r |= ((v >> b) & 1ull) << (stride * b);
    return r;
}

void or_keys2d(int64_t n, const float *x, const float *y, const float bb[3], uint64_t *keys) {
    float ext = bb[2] > 1e-6f ? bb[2] : 1e-6f;   /* std::max(posSize.z, 1e-6f) */
    float hx = bb[0] + ext, hy = bb[1] + ext;
    for (int64_t i = 0; i < n; i++) {
        uint64_t ix = or_scale_to_grid2d(x[i], bb[0], hx);
        uint64_t iy = or_scale_to_grid2d(y[i], bb[1], hy);
        keys[i] = spread(ix & 0x3FFFFu, 18, 2) | (spread(iy & 0x3FFFFu, 18, 2) << 1);
    }
}

void or_keys3d(int64_t n, const float *x, const float *y, const float *z, const float bb[4],
               uint64_t *keys) {
    float hx = bb[0] + bb[3], hy = bb[1] + bb[3], hz = bb[2] + bb[3];
    for (int64_t i = 0; i < n; i++) {
        uint64_t ix = or_scale_to_grid3d(x[i], bb[0], hx);
        uint64_t iy = or_scale_to_grid3d(y[i], bb[1], hy);
        uint64_t iz = or_scale_to_grid3d(z[i], bb[2], hz);
        keys[i] = spread(ix, 21, 3) | (spread(iy, 21, 3) << 1) | (spread(iz, 21, 3) << 2);
    }
}

/* stable LSD radix sort of (key, index), 16-bit digits */
void or_sort_perm(int64_t n, const uint64_t *keys, uint32_t *perm) {
    uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    uint32_t *cnt = (uint32_t *)malloc(sizeof(uint32_t) * 65537);
    for (int64_t i = 0; i < n; i++) perm[i] = (uint32_t)i;
    uint64_t allor = 0;
    for (int64_t i = 0; i < n; i++) allor |= keys[i];
    uint32_t *src = perm, *dst = tmp;
    for (int shift = 0; shift < 64; shift += 16) {
        if ((allor >> shift) == 0) break;
        memset(cnt, 0, sizeof(uint32_t) * 65537);
        for (int64_t i = 0; i < n; i++) cnt[((keys[src[i]] >> shift) & 0xFFFF) + 1]++;
        for (int d = 0; d < 65536; d++) cnt[d + 1] += cnt[d];
        for (int64_t i = 0; i < n; i++) dst[cnt[(keys[src[i]] >> shift) & 0xFFFF]++] = src[i];
        uint32_t *s = src; src = dst; dst = s;
    }
    if (src != perm) memcpy(perm, src, sizeof(uint32_t) * (size_t)n);
    free(tmp);
    free(cnt);
}

/* ------------------------------------------------------------------ */
/* tree build                                                          */
/* ------------------------------------------------------------------ */
int or_tree_alloc(or_tree *t, int dims, int64_t cap) {
    memset(t, 0, sizeof(*t));
    t->cap = cap;
    t->dims = dims;
    t->pos = (float *)malloc(sizeof(float) * cap * dims);
    t->size = (float *)malloc(sizeof(float) * cap);
    t->com = (float *)malloc(sizeof(float) * cap * dims);
    t->mass = (float *)malloc(sizeof(float) * cap);
    t->temp = (float *)malloc(sizeof(float) * cap);
    t->start = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    t->end = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    t->next = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    t->child = (uint32_t *)malloc(sizeof(uint32_t) * cap * (1 << dims));
    if (!t->pos || !t->size || !t->com || !t->mass || !t->temp || !t->start || !t->end ||
        !t->next || !t->child) {
        or_tree_free(t);
        return -1;
    }
    return 0;
}

void or_tree_free(or_tree *t) {
    free(t->pos); free(t->size); free(t->com); free(t->mass); free(t->temp);
    free(t->start); free(t->end); free(t->next); free(t->child);
    memset(t, 0, sizeof(*t));
}

/* std::partition_point(first, last, [](v){ return v < mid; }) with the
 * halving probe sequence of the GNU C++ library (the reference calls
 * std::partition_point, quadtree.cpp:42-65).  The probe sequence matters:
 * when float midpoint compares disagree with the Morton order the range is
 * not partitioned, and the result is wherever this search lands. */
static uint32_t part_point(const float *v, uint32_t first, uint32_t last, float mid) {
    uint32_t len = last - first;
    while (len > 0) {
        uint32_t half = len >> 1;
        uint32_t probe = first + half;
        if (v[probe] < mid) {
            first = probe + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    return first;
}

typedef struct {
    or_tree *t;
    const float *p[3];
    const float *m, *temp;
    uint32_t leaf_cap;
    float size_gate, min_size;
} build_ctx;

static int is_leaf(const build_ctx *c, uint32_t cnt, float size) {
    /* quadtree.cpp:16 / :120 with the leaf capacity (4) and the size gate
     * (2.0f) parameterised; min_size is the 1e-6f floor */
    return ((cnt <= c->leaf_cap && size <= c->size_gate) || cnt == 1) || size <= c->min_size;
}

/* computeLeafMass / computeLeafMass3D (quadtree.h:53-67, :159-174) */
static void leaf_mass(build_ctx *c, uint32_t self, int dims) {
    or_tree *t = c->t;
    float gm = 0.0f, gt = 0.0f, com[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t i = t->start[self]; i < t->end[self]; i++) {
        float mi = c->m[i];
        gm += mi;
        if (c->temp) gt += c->temp[i];
        for (int a = 0; a < dims; a++) com[a] += c->p[a][i] * mi;
    }
    if (gm > 0) for (int a = 0; a < dims; a++) com[a] /= gm;
    t->mass[self] = gm;
    t->temp[self] = gt;
    for (int a = 0; a < dims; a++) t->com[(int64_t)self * dims + a] = com[a];
}

/* one node of the recursive build.  Children are numbered in emission
 * order, each child index taken just before the child's own subtree is
 * built, so the node array is in DFS pre-order (quadtree.cpp:67-87). */
static void build_node(build_ctx *c, uint32_t self, const float *pos, float size,
                       uint32_t s, uint32_t e, int depth) {
    or_tree *t = c->t;
    const int dims = t->dims, nq = 1 << dims;
    if (depth > t->max_depth) t->max_depth = depth;
    for (int a = 0; a < dims; a++) t->pos[(int64_t)self * dims + a] = pos[a];
    t->size[self] = size;
    t->start[self] = s;
    t->end[self] = e;
    t->next[self] = 0;
    for (int q = 0; q < nq; q++) t->child[(int64_t)self * nq + q] = EMPTY;

    if (is_leaf(c, e - s, size)) {
        leaf_mass(c, self, dims);
        return;
    }
    float half = size * 0.5f;
    float mid[3];
    for (int a = 0; a < dims; a++) mid[a] = pos[a] + half;
    uint32_t b[9];
    if (dims == 2) {
        /* quadtree.cpp:30-65: split on y, then x in each half */
        b[0] = s; b[4] = e;
        b[2] = part_point(c->p[1], b[0], b[4], mid[1]);
        b[1] = part_point(c->p[0], b[0], b[2], mid[0]);
        b[3] = part_point(c->p[0], b[2], b[4], mid[0]);
    } else {
        /* quadtree.cpp:148-198: split on z, then y, then x */
        b[0] = s; b[8] = e;
        b[4] = part_point(c->p[2], b[0], b[8], mid[2]);
        b[2] = part_point(c->p[1], b[0], b[4], mid[1]);
        b[6] = part_point(c->p[1], b[4], b[8], mid[1]);
        b[1] = part_point(c->p[0], b[0], b[2], mid[0]);
        b[3] = part_point(c->p[0], b[2], b[4], mid[0]);
        b[5] = part_point(c->p[0], b[4], b[6], mid[0]);
        b[7] = part_point(c->p[0], b[6], b[8], mid[0]);
    }
    for (int q = 0; q < nq; q++) {
        if (b[q + 1] > b[q]) {
            float cp[3];
            for (int a = 0; a < dims; a++) cp[a] = pos[a] + (((q >> a) & 1) ? half : 0.0f);
            if (t->count >= t->cap) { t->overflow = 1; return; }
            uint32_t ci = (uint32_t)t->count++;
            build_node(c, ci, cp, half, b[q], b[q + 1], depth + 1);
            t->child[(int64_t)self * nq + q] = ci;
        }
    }
    /* computeInternalMass (quadtree.h:69-92) / computeInternalMass3D
     * (quadtree.cpp:227-252): subGrids[x][y]([z]) loops with x outermost,
     * so the accumulation order over q is x-major. */
    float gm = 0.0f, gt = 0.0f, com[3] = {0.0f, 0.0f, 0.0f};
    uint32_t nx = 0;
    for (int k = 0; k < nq; k++) {
        int q;
        if (dims == 2) q = ((k >> 1) & 1) | ((k & 1) << 1);           /* k = x*2 + y */
        else q = ((k >> 2) & 1) | (((k >> 1) & 1) << 1) | ((k & 1) << 2); /* k = x*4+y*2+z */
        uint32_t ci = t->child[(int64_t)self * nq + q];
        if (ci == EMPTY) continue;
        float cm = t->mass[ci];
        gm += cm;
        gt += t->temp[ci];
        for (int a = 0; a < dims; a++) com[a] += t->com[(int64_t)ci * dims + a] * cm;
        /* calculateNextNeighbor: next = sum over children of (1 + child.next) */
        nx += 1 + t->next[ci];
    }
    if (gm > 0) for (int a = 0; a < dims; a++) com[a] /= gm;
    t->mass[self] = gm;
    t->temp[self] = gt;
    for (int a = 0; a < dims; a++) t->com[(int64_t)self * dims + a] = com[a];
    t->next[self] = nx;
}

static int build_tree(or_tree *t, int dims, int64_t n, const float *x, const float *y,
                      const float *z, const float *m, const float *temp, const float *bb,
                      uint32_t leaf_cap, float size_gate, float min_size) {
    build_ctx c;
    c.t = t; c.p[0] = x; c.p[1] = y; c.p[2] = z; c.m = m; c.temp = temp;
    c.leaf_cap = leaf_cap; c.size_gate = size_gate; c.min_size = min_size;
    t->count = 0; t->overflow = 0; t->max_depth = 0; t->dims = dims;
    if (n <= 0) return 0;
    if (t->cap < 1) { t->overflow = 1; return -1; }
    t->count = 1;
    build_node(&c, 0, bb, bb[dims], 0, (uint32_t)n, 0);
    return t->overflow ? -1 : 0;
}

int or_build_quadtree(or_tree *t, int64_t n, const float *x, const float *y, const float *m,
                      const float *temp, const float bb[3], uint32_t leaf_cap,
                      float size_gate, float min_size) {
    return build_tree(t, 2, n, x, y, NULL, m, temp, bb, leaf_cap, size_gate, min_size);
}

int or_build_octree(or_tree *t, int64_t n, const float *x, const float *y, const float *z,
                    const float *m, const float *temp, const float bb[4], uint32_t leaf_cap,
                    float size_gate, float min_size) {
    return build_tree(t, 3, n, x, y, z, m, temp, bb, leaf_cap, size_gate, min_size);
}

/* ------------------------------------------------------------------ */
/* force: scalar tree walk, physics.cpp:91-205 / physics3D.cpp:131-253 */
/* ------------------------------------------------------------------ */
static inline float wrap_d(float d, float dom, float halfd) {
    /* d -= domain * ((d > half) - (d < -half))  (physics.cpp:118-121) */
    return d - dom * (float)((d > halfd) - (d < -halfd));
}

static inline int node_is_leaf(const or_tree *t, uint32_t k) {
    const int nq = 1 << t->dims;
    for (int q = 0; q < nq; q++)
        if (t->child[(int64_t)k * nq + q] != EMPTY) return 0;
    return 1;
}

void or_walk2d(int64_t n, const float *x, const float *y, const float *m, float *temp,
               const or_tree *t, const or_params *p, float *ax, float *ay,
               uint32_t *inter, float *cond, int nthreads) {
    const uint32_t ncount = (uint32_t)t->count;
    const float thetaSq = p->theta * p->theta;
    const float eps2 = p->eps2;
    const float Gf = p->G;
    const int per = p->periodic;
    const float dx_dom = p->domain[0], dy_dom = p->domain[1];
    const float hx = dx_dom * 0.5f, hy = dy_dom * 0.5f;
    const int use_temp = p->temp_enabled && temp;
    /* other particles' temperatures (and the nodes' sums, taken at build
       time) are read as they were before the walk; each particle accumulates
       its own in walk order (see the header) */
    float *told = use_temp ? (float *)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1)) : NULL;
    if (told) memcpy(told, temp, sizeof(float) * (size_t)n);
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        float fx = 0.0f, fy = 0.0f;
        double absf = 0.0;
        float ti = told ? told[i] : 0.0f;
        uint32_t cnt = 0;
        const float pm = m[i], xi = x[i], yi = y[i];
        uint32_t k = 0;
        while (k < ncount) {
            float gmass = t->mass[k];
            if (gmass <= 0.0f) { k += t->next[k] + 1; continue; }
            float dx = t->com[2 * (int64_t)k] - xi;
            float dy = t->com[2 * (int64_t)k + 1] - yi;
            if (per) { dx = wrap_d(dx, dx_dom, hx); dy = wrap_d(dy, dy_dom, hy); }
            float r2 = dx * dx + dy * dy + eps2;
            float sz = t->size[k];
            if (sz * sz < thetaSq * r2) {
                float inv = 1.0f / sqrtf(r2);
                float inv3 = inv * inv * inv;
                float fm = Gf * pm * gmass * inv3;
                fx += dx * fm;
                fy += dy * fm;
                absf += sqrt((double)(dx * fm) * (dx * fm) + (double)(dy * fm) * (dy * fm));
                cnt++;
                if (use_temp) {
                    uint32_t c = t->end[k] - t->start[k];
                    if (c > 0) {
                        float avg = t->temp[k] / (float)c;
                        float diff = avg - ti;
                        float dist = 0.0f;
                        if (r2 > 1e-16f) dist = 1.0f / inv;
                        if (dist > 1e-8f) ti += p->heat_cond * diff / dist * p->dt;
                    }
                }
                k += t->next[k] + 1;
            } else if (node_is_leaf(t, k)) {
                for (uint32_t j = t->start[k]; j < t->end[k]; j++) {
                    if ((int64_t)j == i) continue;
                    float ddx = x[j] - xi, ddy = y[j] - yi;
                    if (per) { ddx = wrap_d(ddx, dx_dom, hx); ddy = wrap_d(ddy, dy_dom, hy); }
                    float rr = ddx * ddx + ddy * ddy + eps2;
                    float inv = 1.0f / sqrtf(rr);
                    float inv3 = inv * inv * inv;
                    float fm = Gf * pm * m[j] * inv3;
                    fx += ddx * fm;
                    fy += ddy * fm;
                    absf += sqrt((double)(ddx * fm) * (ddx * fm) + (double)(ddy * fm) * (ddy * fm));
                    cnt++;
                    if (use_temp) {
                        float diff = told[j] - ti;
                        float dist = 0.0f;
                        if (rr > 1e-16f) dist = 1.0f / inv;
                        if (dist > 1e-8f) ti += p->heat_cond * diff / dist * p->dt;
                    }
                }
                k += t->next[k] + 1;
            } else {
                ++k;
            }
        }
        ax[i] = fx / m[i];
        ay[i] = fy / m[i];
        if (told) temp[i] = ti;
        if (inter) inter[i] = cnt;
        if (cond) {
            double net = sqrt((double)fx * fx + (double)fy * fy);
            cond[i] = net > 0 ? (float)(absf / net) : INFINITY;
        }
    }
    free(told);
}

void or_walk3d(int64_t n, const float *x, const float *y, const float *z, const float *m,
               float *temp, const or_tree *t, const or_params *p,
               float *ax, float *ay, float *az, uint32_t *inter, float *cond, int nthreads) {
    const uint32_t ncount = (uint32_t)t->count;
    const float thetaSq = p->theta * p->theta;
    const float eps2 = p->eps2;
    const float Gf = p->G;
    const int per = p->periodic;
    const float hx = p->domain[0] * 0.5f, hy = p->domain[1] * 0.5f, hz = p->domain[2] * 0.5f;
    const int use_temp = p->temp_enabled && temp;
    float *told = use_temp ? (float *)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1)) : NULL;
    if (told) memcpy(told, temp, sizeof(float) * (size_t)n);
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        double absf = 0.0;
        float ti = told ? told[i] : 0.0f;
        uint32_t cnt = 0;
        const float pm = m[i], xi = x[i], yi = y[i], zi = z[i];
        uint32_t k = 0;
        while (k < ncount) {
            float gmass = t->mass[k];
            if (gmass <= 0.0f) { k += t->next[k] + 1; continue; }
            float dx = t->com[3 * (int64_t)k] - xi;
            float dy = t->com[3 * (int64_t)k + 1] - yi;
            float dz = t->com[3 * (int64_t)k + 2] - zi;
            if (per) {
                dx = wrap_d(dx, p->domain[0], hx);
                dy = wrap_d(dy, p->domain[1], hy);
                dz = wrap_d(dz, p->domain[2], hz);
            }
            float r2 = dx * dx + dy * dy + dz * dz + eps2;
            float sz = t->size[k];
            if (sz * sz < thetaSq * r2) {
                float inv = 1.0f / sqrtf(r2);
                float inv3 = inv * inv * inv;
                float fm = Gf * pm * gmass * inv3;
                fx += dx * fm; fy += dy * fm; fz += dz * fm;
                absf += fabs((double)fm) * sqrt((double)dx * dx + (double)dy * dy + (double)dz * dz);
                cnt++;
                if (use_temp) {
                    uint32_t c = t->end[k] - t->start[k];
                    if (c > 0) {
                        float avg = t->temp[k] / (float)c;
                        float diff = avg - ti;
                        float dist = 0.0f;
                        if (r2 > 1e-16f) dist = 1.0f / inv;
                        if (dist > 1e-8f) ti += p->heat_cond * diff / dist * p->dt;
                    }
                }
                k += t->next[k] + 1;
            } else if (node_is_leaf(t, k)) {
                for (uint32_t j = t->start[k]; j < t->end[k]; j++) {
                    if ((int64_t)j == i) continue;
                    float ddx = x[j] - xi, ddy = y[j] - yi, ddz = z[j] - zi;
                    if (per) {
                        ddx = wrap_d(ddx, p->domain[0], hx);
                        ddy = wrap_d(ddy, p->domain[1], hy);
                        ddz = wrap_d(ddz, p->domain[2], hz);
                    }
                    float rr = ddx * ddx + ddy * ddy + ddz * ddz + eps2;
                    float inv = 1.0f / sqrtf(rr);
                    float inv3 = inv * inv * inv;
                    float fm = Gf * pm * m[j] * inv3;
                    fx += ddx * fm; fy += ddy * fm; fz += ddz * fm;
                    absf += fabs((double)fm) * sqrt((double)ddx * ddx + (double)ddy * ddy + (double)ddz * ddz);
                    cnt++;
                    if (use_temp) {
                        float diff = told[j] - ti;
                        float dist = 0.0f;
                        if (rr > 1e-16f) dist = 1.0f / inv;
                        if (dist > 1e-8f) ti += p->heat_cond * diff / dist * p->dt;
                    }
                }
                k += t->next[k] + 1;
            } else {
                ++k;
            }
        }
        ax[i] = fx / m[i];
        ay[i] = fy / m[i];
        az[i] = fz / m[i];
        if (told) temp[i] = ti;
        if (inter) inter[i] = cnt;
        if (cond) {
            double net = sqrt((double)fx * fx + (double)fy * fy + (double)fz * fz);
            cond[i] = net > 0 ? (float)(absf / net) : INFINITY;
        }
    }
    free(told);
}

/* ------------------------------------------------------------------ */
/* AVX2 walk: physics.cpp:207-352 / physics3D.cpp:255-414.  The leaf   */
/* body runs 8 sources at a time with the approximate reciprocal square */
/* root and drops the self term by the test r^2 != eps2; the remainder  */
/* loop is scalar with 1/sqrtf and an index test.  Periodic wrapping    */
/* and temperature are not applied in the vector body, as in the        */
/* reference.                                                           */
/* ------------------------------------------------------------------ */
__attribute__((target("avx2,fma")))
void or_walk2d_avx2(int64_t n, const float *x, const float *y, const float *m,
                    const or_tree *t, const or_params *p, float *ax, float *ay, int nthreads) {
    const uint32_t ncount = (uint32_t)t->count;
    const float thetaSq = p->theta * p->theta;
    const float eps2 = p->eps2;
    const float Gf = p->G;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        float fx = 0.0f, fy = 0.0f;
        const float pm = m[i], xi = x[i], yi = y[i];
        uint32_t k = 0;
        while (k < ncount) {
            float gmass = t->mass[k];
            if (gmass <= 0.0f) { k += t->next[k] + 1; continue; }
            float dx = t->com[2 * (int64_t)k] - xi;
            float dy = t->com[2 * (int64_t)k + 1] - yi;
            float r2 = dx * dx + dy * dy + eps2;
            float sz = t->size[k];
            if (sz * sz < thetaSq * r2) {
                float inv = 1.0f / sqrtf(r2);
                float fm = Gf * pm * gmass * (inv * inv * inv);
                fx += dx * fm;
                fy += dy * fm;
                k += t->next[k] + 1;
            } else if (node_is_leaf(t, k)) {
                const __m256 vxi = _mm256_set1_ps(xi), vyi = _mm256_set1_ps(yi);
                const __m256 veps = _mm256_set1_ps(eps2), vgm = _mm256_set1_ps(Gf * pm);
                __m256 sx = _mm256_setzero_ps(), sy = _mm256_setzero_ps();
                uint32_t j = t->start[k];
                const uint32_t e = t->end[k];
                for (; j + 7 < e; j += 8) {
                    __m256 ddx = _mm256_sub_ps(_mm256_loadu_ps(x + j), vxi);
                    __m256 ddy = _mm256_sub_ps(_mm256_loadu_ps(y + j), vyi);
                    __m256 rr = _mm256_add_ps(_mm256_add_ps(_mm256_mul_ps(ddx, ddx),
                                                            _mm256_mul_ps(ddy, ddy)), veps);
                    __m256 inv = _mm256_rsqrt_ps(rr);
                    __m256 inv3 = _mm256_mul_ps(_mm256_mul_ps(inv, inv), inv);
                    __m256 fm = _mm256_mul_ps(_mm256_mul_ps(vgm, _mm256_loadu_ps(m + j)), inv3);
                    fm = _mm256_and_ps(fm, _mm256_cmp_ps(rr, veps, _CMP_NEQ_OQ));
                    sx = _mm256_add_ps(sx, _mm256_mul_ps(ddx, fm));
                    sy = _mm256_add_ps(sy, _mm256_mul_ps(ddy, fm));
                }
                float bx[8], by[8];
                _mm256_storeu_ps(bx, sx);
                _mm256_storeu_ps(by, sy);
                for (int l = 0; l < 8; l++) { fx += bx[l]; fy += by[l]; }
                for (; j < e; j++) {
                    if ((int64_t)j == i) continue;
                    float ddx = x[j] - xi, ddy = y[j] - yi;
                    float rr = ddx * ddx + ddy * ddy + eps2;
                    float inv = 1.0f / sqrtf(rr);
                    float fm = Gf * pm * m[j] * (inv * inv * inv);
                    fx += ddx * fm;
                    fy += ddy * fm;
                }
                k += t->next[k] + 1;
            } else {
                ++k;
            }
        }
        ax[i] = fx / m[i];
        ay[i] = fy / m[i];
    }
}

__attribute__((target("avx2,fma")))
void or_walk3d_avx2(int64_t n, const float *x, const float *y, const float *z, const float *m,
                    const or_tree *t, const or_params *p, float *ax, float *ay, float *az,
                    int nthreads) {
    const uint32_t ncount = (uint32_t)t->count;
    const float thetaSq = p->theta * p->theta;
    const float eps2 = p->eps2;
    const float Gf = p->G;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        const float pm = m[i], xi = x[i], yi = y[i], zi = z[i];
        uint32_t k = 0;
        while (k < ncount) {
            float gmass = t->mass[k];
            if (gmass <= 0.0f) { k += t->next[k] + 1; continue; }
            float dx = t->com[3 * (int64_t)k] - xi;
            float dy = t->com[3 * (int64_t)k + 1] - yi;
            float dz = t->com[3 * (int64_t)k + 2] - zi;
            float r2 = dx * dx + dy * dy + dz * dz + eps2;
            float sz = t->size[k];
            if (sz * sz < thetaSq * r2) {
                float inv = 1.0f / sqrtf(r2);
                float fm = Gf * pm * gmass * (inv * inv * inv);
                fx += dx * fm; fy += dy * fm; fz += dz * fm;
                k += t->next[k] + 1;
            } else if (node_is_leaf(t, k)) {
                const __m256 vxi = _mm256_set1_ps(xi), vyi = _mm256_set1_ps(yi);
                const __m256 vzi = _mm256_set1_ps(zi);
                const __m256 veps = _mm256_set1_ps(eps2), vgm = _mm256_set1_ps(Gf * pm);
                __m256 sx = _mm256_setzero_ps(), sy = _mm256_setzero_ps(), sz8 = _mm256_setzero_ps();
                uint32_t j = t->start[k];
                const uint32_t e = t->end[k];
                for (; j + 7 < e; j += 8) {
                    __m256 ddx = _mm256_sub_ps(_mm256_loadu_ps(x + j), vxi);
                    __m256 ddy = _mm256_sub_ps(_mm256_loadu_ps(y + j), vyi);
                    __m256 ddz = _mm256_sub_ps(_mm256_loadu_ps(z + j), vzi);
                    __m256 rr = _mm256_add_ps(_mm256_add_ps(_mm256_add_ps(
                        _mm256_mul_ps(ddx, ddx), _mm256_mul_ps(ddy, ddy)), _mm256_mul_ps(ddz, ddz)), veps);
                    __m256 inv = _mm256_rsqrt_ps(rr);
                    __m256 inv3 = _mm256_mul_ps(_mm256_mul_ps(inv, inv), inv);
                    __m256 fm = _mm256_mul_ps(_mm256_mul_ps(vgm, _mm256_loadu_ps(m + j)), inv3);
                    fm = _mm256_and_ps(fm, _mm256_cmp_ps(rr, veps, _CMP_NEQ_OQ));
                    sx = _mm256_add_ps(sx, _mm256_mul_ps(ddx, fm));
                    sy = _mm256_add_ps(sy, _mm256_mul_ps(ddy, fm));
                    sz8 = _mm256_add_ps(sz8, _mm256_mul_ps(ddz, fm));
                }
                float bx[8], by[8], bz[8];
                _mm256_storeu_ps(bx, sx);
                _mm256_storeu_ps(by, sy);
                _mm256_storeu_ps(bz, sz8);
                for (int l = 0; l < 8; l++) { fx += bx[l]; fy += by[l]; fz += bz[l]; }
                for (; j < e; j++) {
                    if ((int64_t)j == i) continue;
                    float ddx = x[j] - xi, ddy = y[j] - yi, ddz = z[j] - zi;
                    float rr = ddx * ddx + ddy * ddy + ddz * ddz + eps2;
                    float inv = 1.0f / sqrtf(rr);
                    float fm = Gf * pm * m[j] * (inv * inv * inv);
                    fx += ddx * fm; fy += ddy * fm; fz += ddz * fm;
                }
                k += t->next[k] + 1;
            } else {
                ++k;
            }
        }
        ax[i] = fx / m[i];
        ay[i] = fy / m[i];
        az[i] = fz / m[i];
    }
}

/* ------------------------------------------------------------------ */
/* direct sum: physics.cpp:392-434, 3D physics3D.cpp:416-469 (scalar   */
/* form; softening un-squared, self term included since d = 0 adds      */
/* nothing; the result is the acceleration, no heat exchange)           */
/* ------------------------------------------------------------------ */
void or_naive2d(int64_t n, const float *x, const float *y, const float *m,
                const or_params *p, float *ax, float *ay, int nthreads) {
    const float soft = p->naive_soft, G = p->G;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        float sx = 0.0f, sy = 0.0f;
        const float xi = x[i], yi = y[i];
        for (int64_t j = 0; j < n; j++) {
            float dx = x[j] - xi, dy = y[j] - yi;
            if (p->periodic) {
                dx = wrap_d(dx, p->domain[0], p->domain[0] * 0.5f);
                dy = wrap_d(dy, p->domain[1], p->domain[1] * 0.5f);
            }
            float r2 = dx * dx + dy * dy + soft;
            float inv = 1.0f / sqrtf(r2);
            float f = G * m[j] * (inv * inv * inv);
            sx += dx * f;
            sy += dy * f;
        }
        ax[i] = sx;
        ay[i] = sy;
    }
}

void or_naive3d(int64_t n, const float *x, const float *y, const float *z, const float *m,
                const or_params *p, float *ax, float *ay, float *az, int nthreads) {
    const float soft = p->naive_soft, G = p->G;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        float sx = 0.0f, sy = 0.0f, sz = 0.0f;
        const float xi = x[i], yi = y[i], zi = z[i];
        for (int64_t j = 0; j < n; j++) {
            float dx = x[j] - xi, dy = y[j] - yi, dz = z[j] - zi;
            if (p->periodic) {   /* physics3D.cpp:449-453 */
                dx = wrap_d(dx, p->domain[0], p->domain[0] * 0.5f);
                dy = wrap_d(dy, p->domain[1], p->domain[1] * 0.5f);
                dz = wrap_d(dz, p->domain[2], p->domain[2] * 0.5f);
            }
            float r2 = dx * dx + dy * dy + dz * dz + soft;
            float inv = 1.0f / sqrtf(r2);
            float f = G * m[j] * (inv * inv * inv);
            sx += dx * f; sy += dy * f; sz += dz * f;
        }
        ax[i] = sx; ay[i] = sy; az[i] = sz;
    }
}

void or_direct_f64(int dims, int64_t n, const float *x, const float *y, const float *z,
                   const float *m, double G, double eps2, int64_t nt, const int64_t *idx,
                   double *ax, double *ay, double *az, int nthreads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
    for (int64_t k = 0; k < nt; k++) {
        const int64_t i = idx[k];
        double sx = 0, sy = 0, sz = 0;
        const double xi = x[i], yi = y[i], zi = dims == 3 ? z[i] : 0.0;
        for (int64_t j = 0; j < n; j++) {
            if (j == i) continue;
            double dx = (double)x[j] - xi, dy = (double)y[j] - yi;
            double dz = dims == 3 ? (double)z[j] - zi : 0.0;
            double r2 = dx * dx + dy * dy + dz * dz + eps2;
            double f = G * (double)m[j] / (r2 * sqrt(r2));
            sx += dx * f; sy += dy * f; sz += dz * f;
        }
        ax[k] = sx; ay[k] = sy;
        if (az) az[k] = sz;
    }
}

/* ------------------------------------------------------------------ */
/* leapfrog halves: physics.cpp:1069-1125, physics3D.cpp:740-804,      */
/* :1158-1168.  Pinned particles are skipped.  The SPH velocity clamp   */
/* (isSPHEnabled) is outside the gravity path and not restated.         */
/* ------------------------------------------------------------------ */
void or_integrate_start(int dims, int64_t n, float *x, float *y, float *z,
                        float *vx, float *vy, float *vz, const float *ax, const float *ay,
                        const float *az, float *pvx, float *pvy, float *pvz,
                        const uint8_t *pinned, const or_params *p) {
    const float dt = p->dt, h = dt * 0.5f;
    for (int64_t i = 0; i < n; i++) {
        if (pinned && pinned[i]) continue;
        if (pvx) { pvx[i] = vx[i]; pvy[i] = vy[i]; if (dims == 3 && pvz) pvz[i] = vz[i]; }
        vx[i] += ax[i] * h;
        vy[i] += ay[i] * h;
        if (dims == 3) vz[i] += az[i] * h;
        x[i] += vx[i] * dt;
        y[i] += vy[i] * dt;
        if (dims == 3) z[i] += vz[i] * dt;
        if (p->periodic) {
            if (dims == 2) {
                /* physics.cpp:1104-1110: domain [0, size) */
                if (x[i] < 0.0f) x[i] += p->domain[0];
                else if (x[i] >= p->domain[0]) x[i] -= p->domain[0];
                if (y[i] < 0.0f) y[i] += p->domain[1];
                else if (y[i] >= p->domain[1]) y[i] -= p->domain[1];
            } else {
                /* physics3D.cpp:785-802: domain [-size/2, size/2) */
                float *c[3] = {x, y, z};
                for (int a = 0; a < 3; a++) {
                    float hd = p->domain[a] * 0.5f;
                    if (c[a][i] < -hd) c[a][i] += p->domain[a];
                    else if (c[a][i] >= hd) c[a][i] -= p->domain[a];
                }
            }
        }
    }
}

void or_integrate_end(int dims, int64_t n, float *vx, float *vy, float *vz,
                      const float *ax, const float *ay, const float *az,
                      const uint8_t *pinned, const or_params *p) {
    const float h = p->dt * 0.5f;
    for (int64_t i = 0; i < n; i++) {
        if (pinned && pinned[i]) continue;
        vx[i] += ax[i] * h;
        vy[i] += ay[i] * h;
        if (dims == 3) vz[i] += az[i] * h;
    }
}

/* ------------------------------------------------------------------ */
/* one frame: globalLogic.cpp:1155-1370 (2D) / :1584-1719 (3D)         */
/* ------------------------------------------------------------------ */
static void gather_f(float *a, const uint32_t *perm, int64_t n, float *tmp) {
    if (!a) return;
    for (int64_t k = 0; k < n; k++) tmp[k] = a[perm[k]];
    memcpy(a, tmp, sizeof(float) * (size_t)n);
}

int or_frame(const or_params *p, int64_t n, float *x, float *y, float *z,
             float *vx, float *vy, float *vz, float *ax, float *ay, float *az,
             float *m, uint32_t *id, float *pvx, float *pvy, float *pvz,
             float *temp, uint8_t *pinned, int walk, int nthreads,
             double *stage_ms, uint64_t *interactions, int64_t *nodes) {
    const int d3 = p->dims == 3;
    double t0 = now_ms(), tt[8] = {0};
    if (n <= 0) return 0;
    /* integrateStart (dt != 0 in every configuration used here) */
    or_integrate_start(p->dims, n, x, y, z, vx, vy, vz, ax, ay, az, pvx, pvy, pvz, pinned, p);
    double t1 = now_ms();
    float bb[4];
    if (d3) or_bbox3d(n, x, y, z, bb); else or_bbox2d(n, x, y, bb);
    double t2 = now_ms();
    uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    float *tmp = (float *)malloc(sizeof(float) * (size_t)n);
    if (!keys || !perm || !tmp) { free(keys); free(perm); free(tmp); return -1; }
    if (d3) or_keys3d(n, x, y, z, bb, keys); else or_keys2d(n, x, y, bb, keys);
    double t3 = now_ms();
    or_sort_perm(n, keys, perm);
    float *arrs[] = {x, y, z, vx, vy, vz, ax, ay, az, m, pvx, pvy, pvz, temp};
    for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); a++) {
        if (!d3 && (arrs[a] == z || arrs[a] == vz || arrs[a] == az || arrs[a] == pvz)) continue;
        gather_f(arrs[a], perm, n, tmp);
    }
    if (id) {
        uint32_t *ti = (uint32_t *)tmp;
        for (int64_t k = 0; k < n; k++) ti[k] = id[perm[k]];
        memcpy(id, ti, sizeof(uint32_t) * (size_t)n);
    }
    if (pinned) {
        uint8_t *tp = (uint8_t *)tmp;
        for (int64_t k = 0; k < n; k++) tp[k] = pinned[perm[k]];
        memcpy(pinned, tp, (size_t)n);
    }
    double t4 = now_ms();
    or_tree tree;
    int64_t cap = (d3 ? 8 : 4) * n + 64;
    if (or_tree_alloc(&tree, p->dims, cap)) { free(keys); free(perm); free(tmp); return -1; }
    int rc = d3 ? or_build_octree(&tree, n, x, y, z, m, p->temp_enabled ? temp : NULL, bb,
                                  p->leaf_cap, p->size_gate, p->min_size)
                : or_build_quadtree(&tree, n, x, y, m, p->temp_enabled ? temp : NULL, bb,
                                    p->leaf_cap, p->size_gate, p->min_size);
    double t5 = now_ms();
    uint32_t *inter = interactions ? (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n) : NULL;
    for (int64_t i = 0; i < n; i++) { ax[i] = 0.0f; ay[i] = 0.0f; if (d3) az[i] = 0.0f; }
    if ((walk == 2 && n < 5000) || (walk == 0 && n < (int64_t)p->direct_below)) {
        if (d3) or_naive3d(n, x, y, z, m, p, ax, ay, az, nthreads);
        else or_naive2d(n, x, y, m, p, ax, ay, nthreads);
    } else if (walk >= 1) {
        if (d3) or_walk3d_avx2(n, x, y, z, m, &tree, p, ax, ay, az, nthreads);
        else or_walk2d_avx2(n, x, y, m, &tree, p, ax, ay, nthreads);
    } else {
        if (d3) or_walk3d(n, x, y, z, m, temp, &tree, p, ax, ay, az, inter, NULL, nthreads);
        else or_walk2d(n, x, y, m, temp, &tree, p, ax, ay, inter, NULL, nthreads);
    }
    double t6 = now_ms();
    or_integrate_end(p->dims, n, vx, vy, vz, ax, ay, az, pinned, p);
    double t7 = now_ms();
    if (interactions) {
        uint64_t s = 0;
        if (walk == 0) for (int64_t i = 0; i < n; i++) s += inter[i];
        *interactions = s;
        free(inter);
    }
    if (nodes) *nodes = tree.count;
    tt[0] = t1 - t0; tt[1] = t2 - t1; tt[2] = t3 - t2; tt[3] = t4 - t3;
    tt[4] = t5 - t4; tt[5] = t6 - t5; tt[6] = t7 - t6; tt[7] = t7 - t0;
    if (stage_ms) memcpy(stage_ms, tt, sizeof(tt));
    or_tree_free(&tree);
    free(keys); free(perm); free(tmp);
    return rc;
}

/* ------------------------------------------------------------------ */
/* SPH neighbour grid: SPH::newGridGPU (SPH.h:533-590)                  */
/* ------------------------------------------------------------------ */
/* int(floor(v)) of the shader; out of the int range (undefined there)  */
/* it saturates, NaN gives 0                                            */
static int32_t floor_to_i32(float v) {
    if (v != v) return 0;
    const double f = floor((double)v);
    if (f >= 2147483647.0) return INT32_MAX;
    if (f <= -2147483648.0) return INT32_MIN;
    return (int32_t)f;
}

void or_sph_grid(int64_t n, const float *x, const float *y, float cell, uint32_t table,
                 uint32_t *keys, uint32_t *index, int32_t *cell_x, int32_t *cell_y,
                 uint32_t *offsets) {
    /* neighborSearchCompute (:130-151): posToCellCoord, hashCell; the int
       products wrap modulo 2^32 */
    for (int64_t i = 0; i < n; i++) {
        const int32_t cx = floor_to_i32(x[i] / cell), cy = floor_to_i32(y[i] / cell);
        keys[i] = (((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u)) % table;
        index[i] = (uint32_t)i;
        cell_x[i] = cx;
        cell_y[i] = cy;
    }
    /* gpuBitonicSort (:337-367) with bitonicSortCompute (:272-295): stages
       over the next power of two; a compare-exchange whose right index is
       past the end is skipped */
    uint32_t p2 = 1;
    while (p2 < (uint64_t)n) p2 <<= 1;
    int stages = 0;
    while ((1u << stages) < p2) stages++;
    for (int stage = 0; stage < stages; stage++) {
        for (int step = 0; step <= stage; step++) {
            const uint32_t gw = 1u << (stage - step), gh = 2 * gw - 1;
            for (uint32_t t = 0; t < p2 / 2; t++) {
                const uint32_t h = t & (gw - 1);
                const uint32_t l = h + (gh + 1) * (t / gw);
                const uint32_t r = l + (step == 0 ? gh - 2 * h : (gh + 1) / 2);
                if (r >= (uint64_t)n) continue;
                if (keys[l] > keys[r]) {
                    uint32_t tk = keys[l]; keys[l] = keys[r]; keys[r] = tk;
                    uint32_t ti = index[l]; index[l] = index[r]; index[r] = ti;
                    int32_t tx = cell_x[l]; cell_x[l] = cell_x[r]; cell_x[r] = tx;
                    int32_t ty = cell_y[l]; cell_y[l] = cell_y[r]; cell_y[r] = ty;
                }
            }
        }
    }
    /* offsetsResetCompute (:465-469) and offsetCompute (:386-399) */
    for (uint32_t k = 0; k < table; k++) offsets[k] = 0xFFFFFFFFu;
    for (int64_t i = 0; i < n; i++) {
        const uint32_t prev = i == 0 ? table : keys[i - 1];
        if (keys[i] != prev && keys[i] < table) offsets[keys[i]] = (uint32_t)i;
    }
}

/* ------------------------------------------------------------------ */
/* trajectory preview: ParticlesSpawning::predictTrajectory            */
/* (particlesSpawning.cpp:443-500, 3D :1000-1060) with the walk it     */
/* calls, Physics::calculateForceFromGridOld (physics.cpp:4-90, 3D     */
/* physics3D.cpp:49-120): leaves are taken whole (never opened), a     */
/* one-particle leaf within 0.001 of the probe on every axis is        */
/* skipped, softening is added squared in 2D and 3D (eps2 here).       */
/* ------------------------------------------------------------------ */
static void old_force(const or_tree *t, const float *pp[3], const or_params *p, float eps2,
                      const float pos[3], float pmass, float F[3]) {
    const int D = t->dims;
    const float thetaSq = p->theta * p->theta;
    F[0] = F[1] = F[2] = 0.0f;
    uint32_t k = 0;
    const uint32_t count = (uint32_t)t->count;
    while (k < count) {
        const float gm = t->mass[k];
        if (gm <= 0.0f) { k += t->next[k] + 1; continue; }
        float d[3] = {0, 0, 0};
        for (int a = 0; a < D; a++) {
            d[a] = t->com[(int64_t)k * D + a] - pos[a];
            if (p->periodic) {
                const float h = p->domain[a] * 0.5f;
                d[a] -= p->domain[a] * (float)((d[a] > h) - (d[a] < -h));
            }
        }
        float r2 = d[0] * d[0] + d[1] * d[1];
        if (D == 3) r2 = r2 + d[2] * d[2];
        r2 = r2 + eps2;
        const int leaf = node_is_leaf(t, k);
        const float sz = t->size[k];
        if ((sz * sz < thetaSq * r2) || leaf) {
            if (t->end[k] - t->start[k] == 1) {
                const uint32_t j = t->start[k];
                int near = 1;
                for (int a = 0; a < D; a++) near = near && fabsf(pp[a][j] - pos[a]) < 0.001f;
                if (near) { k += t->next[k] + 1; continue; }
            }
            const float inv = 1.0f / sqrtf(r2);
            const float inv3 = inv * inv * inv;
            const float fm = p->G * pmass * gm * inv3;
            for (int a = 0; a < D; a++) F[a] += d[a] * fm;
            k += t->next[k] + 1;
        } else {
            ++k;
        }
    }
}

void or_predict_trajectory(const or_tree *t, const float *x, const float *y, const float *z,
                           const or_params *p, float eps2, int64_t nprobes, const float *pos,
                           const float *vel, const float *mass, int32_t steps, float *path,
                           int nthreads) {
    const int D = t->dims;
    const float *pp[3] = {x, y, z};
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int64_t q = 0; q < nprobes; q++) {
        float ps[3] = {0, 0, 0}, v[3] = {0, 0, 0}, F[3], acc[3];
        for (int a = 0; a < D; a++) { ps[a] = pos[q * D + a]; v[a] = vel[q * D + a]; }
        const float m = mass[q], h = p->dt * 0.5f;
        for (int32_t s = 0; s < steps; s++) {
            old_force(t, pp, p, eps2, ps, m, F);
            for (int a = 0; a < D; a++) {
                acc[a] = F[a] / m;
                v[a] += acc[a] * h;
            }
            for (int a = 0; a < D; a++) ps[a] += v[a] * p->dt;
            if (p->periodic) {
                for (int a = 0; a < D; a++) {
                    const float lo = D == 2 ? 0.0f : -p->domain[a] * 0.5f;
                    const float hi = D == 2 ? p->domain[a] : p->domain[a] * 0.5f;
                    if (ps[a] < lo) ps[a] += p->domain[a];
                    else if (ps[a] >= hi) ps[a] -= p->domain[a];
                }
            }
            old_force(t, pp, p, eps2, ps, m, F);
            for (int a = 0; a < D; a++) {
                acc[a] = F[a] / m;
                v[a] += acc[a] * h;
            }
            for (int a = 0; a < D; a++) path[((int64_t)q * steps + s) * D + a] = ps[a];
        }
    }
}

/* ------------------------------------------------------------------ */
/* gravity field display (include/Physics/field.h): cells of           */
/* initializeCells (:59-80), the compute shader fieldGravityCompute    */
/* (:106-160) and the fragment shader's colour map (:165-222), in      */
/* single precision, each operation rounded on its own, GLSL round()   */
/* taken as roundf (halves away from zero).                            */
/* ------------------------------------------------------------------ */
static uint32_t unorm8(float v) {
    v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    return (uint32_t)lrintf(v * 255.0f);
}

int or_gravity_field(int64_t n, const float *x, const float *y, const float *m, float G,
                     float dom_x, float dom_y, int periodic, int res, float softness,
                     float threshold, float stretch, float exposure, int two_color,
                     const float low[3], const float high[3], float *strength, uint32_t *rgba,
                     int *amount_x, int *amount_y, int nthreads) {
    const float cell = (dom_x >= dom_y ? dom_y : dom_x) / (float)res;
    const int ax = (int)(dom_x / cell), ay = (int)(dom_y / cell);
    *amount_x = ax;
    *amount_y = ay;
    const float soft2 = softness * softness;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int c = 0; c < ax * ay; c++) {
        const int i = c / ay, j = c % ay;
        const float cx = (float)i * cell, cy = (float)j * cell;
        float force = 0.0f;
        for (int64_t k = 0; k < n; k++) {
            float dx = x[k] - cx, dy = y[k] - cy;
            if (periodic) {
                dx = dx - dom_x * roundf(dx / dom_x);
                dy = dy - dom_y * roundf(dy / dom_y);
            }
            const float d2 = dx * dx + dy * dy + soft2;
            const float dist = sqrtf(d2);
            if (dist > 0.0001f) force = force + G * (m[k] * 10.0f) / (dist * dist);
        }
        if (strength) strength[c] = force;
        if (!rgba) continue;
        const float cl = fminf(fmaxf(force, 0.0f), threshold);
        const float nrm = cl / threshold;
        const float s = logf(1.0f + nrm * stretch) / logf(1.0f + stretch);
        float col[3];
        if (two_color) {
            for (int a = 0; a < 3; a++) {
                const float base = low[a] * (1.0f - s) + high[a] * s;
                col[a] = base * s * exposure;
            }
        } else {
            const float h = (1.0f - s) * 240.0f / 360.0f;
            const float K[3] = {1.0f, 2.0f / 3.0f, 1.0f / 3.0f};
            for (int a = 0; a < 3; a++) {
                const float f = h + K[a];
                const float pp = fabsf((f - floorf(f)) * 6.0f - 3.0f);
                float t = pp - 1.0f;
                t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
                col[a] = s * t;
            }
        }
        rgba[c] = unorm8(col[0]) | (unorm8(col[1]) << 8) | (unorm8(col[2]) << 16) | (255u << 24);
    }
    return 0;
}


/* FP64 potential energy by direct summation: -1/2 G sum_i sum_{j != i}
 * m_i m_j / sqrt(|x_i - x_j|^2 + eps2) (the accuracy reference of the energy
 * pass; not in the reference). */
double or_potential_f64(int dims, int64_t n, const float *x, const float *y, const float *z,
                        const float *m, double G, double eps2, int nthreads) {
    double e = 0.0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : e) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        double s = 0.0;
        for (int64_t j = 0; j < n; j++) {
            if (j == i) continue;
            const double dx = (double)x[j] - x[i], dy = (double)y[j] - y[i];
            const double dz = dims == 3 ? (double)z[j] - z[i] : 0.0;
            s += (double)m[j] / sqrt(dx * dx + dy * dy + dz * dz + eps2);
        }
        e += (double)m[i] * s;
    }
    return -0.5 * G * e;
}
