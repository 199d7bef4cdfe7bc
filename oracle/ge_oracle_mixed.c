/*
 * ge_oracle_mixed.c -- CPU statement of the mixed-precision tree walk.
 * TEST INFRASTRUCTURE ONLY (the checker of GE_PREC_MIXED).
 *
 * The mixed mode has no counterpart in the reference: it keeps the
 * reference's tree (quadtree.cpp:5-292, the same nodes and particle ranges as
 * or_build_quadtree / or_build_octree) and its pre-order walk
 * (physics.cpp:91-205, physics3D.cpp:131-253), and changes what a node
 * contributes:
 *   - mass, centre of mass and second moments about it, in FP64: a leaf sums
 *     its particles in index order, an internal node combines its children in
 *     child-slot order with the parallel-axis rule (the same operations, each
 *     product-sum a correctly rounded fma, as the device pass);
 *   - opening test b^2 < |d|^2 + eps2 in FP32 with b = size / theta +
 *     |com - cell centre| (b^2 rounded to FP32 from FP64), d = FP32(com) - x;
 *   - an accepted node adds the monopole and quadrupole of the softened
 *     kernel:  G [ M d / r^3 - 3 I d / r^5 - 1.5 tr(I) d / r^5
 *                  + 7.5 (d.I.d) d / r^7 ],  r^2 = |d|^2 + eps2,
 *     here evaluated in FP64 with d = com - x in FP64;
 *   - a leaf that is opened adds G m_j d / r^3 for its particles j != i
 *     with m_j != 0, in FP64.
 * The device evaluates the same interaction list in FP32 with a Kahan sum.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ge_oracle.h"

#define EMPTY UINT32_MAX

static int is_leaf(const or_tree *t, int64_t k) {
    const int nq = 1 << t->dims;
    for (int q = 0; q < nq; q++)
        if (t->child[k * nq + q] != EMPTY) return 0;
    return 1;
}

/* second-moment slot of (a, b): 2D xx xy yy; 3D xx yy zz xy xz yz */
static int mom_index(int D, int a, int b) {
    if (D == 2) return 1 + D + a + b;
    if (a == b) return 1 + D + a;
    return 1 + D + 2 + a + b;
}

int or_moments_mixed(const or_tree *t, const float *x, const float *y, const float *z,
                     const float *m, double *mom) {
    const int D = t->dims, R = D == 2 ? 6 : 10, nq = 1 << D;
    const float *pos[3] = {x, y, z};
    for (int64_t k = t->count - 1; k >= 0; k--) {   /* children follow parents in pre-order */
        double *r = mom + k * R;
        for (int w = 0; w < R; w++) r[w] = 0.0;
        if (is_leaf(t, k)) {
            for (uint32_t j = t->start[k]; j < t->end[k]; j++) {
                const double mj = m[j];
                r[0] += mj;
                for (int a = 0; a < D; a++) r[1 + a] = fma(mj, (double)pos[a][j], r[1 + a]);
            }
            if (r[0] > 0.0) {
                for (int a = 0; a < D; a++) r[1 + a] /= r[0];
                for (uint32_t j = t->start[k]; j < t->end[k]; j++) {
                    const double mj = m[j];
                    double d[3];
                    for (int a = 0; a < D; a++) d[a] = (double)pos[a][j] - r[1 + a];
                    for (int a = 0; a < D; a++)
                        for (int b = a; b < D; b++) {
                            const int w = mom_index(D, a, b);
                            r[w] = fma(mj * d[a], d[b], r[w]);
                        }
                }
            }
        } else {
            for (int q = 0; q < nq; q++) {
                const uint32_t c = t->child[k * nq + q];
                if (c == EMPTY) continue;
                const double *cr = mom + (int64_t)c * R;
                r[0] += cr[0];
                for (int a = 0; a < D; a++) r[1 + a] = fma(cr[0], cr[1 + a], r[1 + a]);
            }
            if (r[0] > 0.0) {
                for (int a = 0; a < D; a++) r[1 + a] /= r[0];
                for (int q = 0; q < nq; q++) {
                    const uint32_t c = t->child[k * nq + q];
                    if (c == EMPTY) continue;
                    const double *cr = mom + (int64_t)c * R;
                    if (!(cr[0] > 0.0)) continue;
                    double d[3];
                    for (int a = 0; a < D; a++) d[a] = cr[1 + a] - r[1 + a];
                    for (int a = 0; a < D; a++)
                        for (int b = a; b < D; b++) {
                            const int w = mom_index(D, a, b);
                            r[w] += fma(cr[0] * d[a], d[b], cr[w]);
                        }
                }
            }
        }
    }
    return 0;
}

/* periodic image shift of one FP32 offset: physics.cpp:118-121 */
static float wrap_k(float d, float half) { return (float)((d > half) - (d < -half)); }

void or_walk_mixed(int64_t n, const float *x, const float *y, const float *z, const float *m,
                   const or_tree *t, const or_params *p, double *ax, double *ay, double *az,
                   uint32_t *inter, int nthreads) {
    const int D = t->dims, R = D == 2 ? 6 : 10;
    double *mom = (double *)malloc(sizeof(double) * (size_t)(t->count > 0 ? t->count : 1) * R);
    float *b2 = (float *)malloc(sizeof(float) * (size_t)(t->count > 0 ? t->count : 1));
    float *hi = (float *)malloc(sizeof(float) * (size_t)(t->count > 0 ? t->count : 1) * 3);
    if (!mom || !b2 || !hi) { free(mom); free(b2); free(hi); return; }
    or_moments_mixed(t, x, y, z, m, mom);
    const double inv_theta = 1.0 / (double)p->theta;
    for (int64_t k = 0; k < t->count; k++) {
        const double *r = mom + k * R;
        const double half = 0.5 * (double)t->size[k];
        double del2 = 0.0;
        for (int a = 0; a < D; a++) {
            hi[k * 3 + a] = (float)r[1 + a];
            const double dc = r[1 + a] - ((double)t->pos[k * D + a] + half);
            del2 = fma(dc, dc, del2);
        }
        const double b = fma((double)t->size[k], inv_theta, sqrt(del2));
        b2[k] = (float)(b * b);
    }
    const float *pos[3] = {x, y, z};
    const double G = p->G, eps2d = p->eps2;
    const float eps2 = p->eps2;
    const uint32_t count = (uint32_t)t->count;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        double f[3] = {0, 0, 0};
        uint32_t cnt = 0;
        float xi[3] = {x[i], y[i], D == 3 ? z[i] : 0.0f};
        uint32_t k = 0;
        while (k < count) {
            const double *r = mom + (int64_t)k * R;
            if (!(r[0] > 0.0)) { k += t->next[k] + 1; continue; }
            float df[3], sh[3] = {0, 0, 0};
            float r2 = 0.0f;
            for (int a = 0; a < D; a++) {
                df[a] = hi[(int64_t)k * 3 + a] - xi[a];
                if (p->periodic) {
                    sh[a] = wrap_k(df[a], p->domain[a] * 0.5f);
                    df[a] = df[a] - p->domain[a] * sh[a];
                }
            }
            r2 = df[0] * df[0] + df[1] * df[1];
            if (D == 3) r2 = r2 + df[2] * df[2];
            r2 = r2 + eps2;
            if (b2[k] < r2) {
                double d[3] = {0, 0, 0}, rr = eps2d;
                for (int a = 0; a < D; a++) {
                    d[a] = r[1 + a] - (double)xi[a] - (double)p->domain[a] * sh[a];
                    rr += d[a] * d[a];
                }
                const double inv = 1.0 / sqrt(rr), inv2 = inv * inv, inv3 = inv2 * inv;
                const double inv5 = inv3 * inv2, inv7 = inv5 * inv2;
                double I[3][3] = {{0}};
                for (int a = 0; a < D; a++)
                    for (int b = a; b < D; b++) I[a][b] = I[b][a] = (double)(float)r[mom_index(D, a, b)];
                double Id[3] = {0, 0, 0}, dId = 0.0, tr = 0.0;
                for (int a = 0; a < D; a++) {
                    for (int b = 0; b < D; b++) Id[a] += I[a][b] * d[b];
                    dId += d[a] * Id[a];
                    tr += I[a][a];
                }
                const double M = (double)(float)r[0];
                const double cm = M * inv3 - 1.5 * tr * inv5 + 7.5 * dId * inv7;
                for (int a = 0; a < D; a++) f[a] += cm * d[a] - 3.0 * Id[a] * inv5;
                cnt++;
                k += t->next[k] + 1;
            } else if (is_leaf(t, k)) {
                for (uint32_t j = t->start[k]; j < t->end[k]; j++) {
                    if ((int64_t)j == i || m[j] == 0.0f) continue;
                    double d[3] = {0, 0, 0}, rr = eps2d;
                    for (int a = 0; a < D; a++) {
                        float dj = pos[a][j] - xi[a];
                        if (p->periodic) dj = dj - p->domain[a] * wrap_k(dj, p->domain[a] * 0.5f);
                        d[a] = (double)dj;
                        rr += d[a] * d[a];
                    }
                    const double inv = 1.0 / sqrt(rr), fm = (double)m[j] * inv * inv * inv;
                    for (int a = 0; a < D; a++) f[a] += fm * d[a];
                    cnt++;
                }
                k += t->next[k] + 1;
            } else {
                k++;
            }
        }
        ax[i] = G * f[0];
        ay[i] = G * f[1];
        if (D == 3 && az) az[i] = G * f[2];
        if (inter) inter[i] = cnt;
    }
    free(mom); free(b2); free(hi);
}

/* Groups of the group walk: each particle belongs to exactly one node of at
 * most GS particles whose parent holds more (or that is the root); runs of
 * such nodes that are adjacent children of one parent are packed into one
 * group while the run holds at most GS particles; a leaf of more than GS
 * particles is cut into GS-particle pieces.  A sparse child (mean spacing
 * more than four times its parent's: (s / S)^D C > 4^D c) is split down its
 * subtree, depth first with an explicit stack of 256 entries, into leaves and
 * nodes dense enough by the same reference (the node whole when the stack is
 * full).  ranges receives {start, end}. */
static void push_range(int64_t *ranges, int64_t *ng, int64_t a, int64_t b) {
    ranges[2 * *ng] = a;
    ranges[2 * *ng + 1] = b;
    (*ng)++;
}

static int sparse_node(int D, float s, int64_t c, float S, int64_t C) {
    const double r = (double)s / (double)S;
    const double rd = D == 2 ? r * r : r * r * r;
    return rd * (double)C > (D == 2 ? 16.0 : 64.0) * (double)c;
}

static void split_sparse(const or_tree *t, int64_t node, float S, int64_t C, int64_t *ranges,
                         int64_t *ng) {
    enum { kStack = 256 };
    const int D = t->dims, nq = 1 << D;
    int64_t stack[kStack];
    int top = 0;
    stack[top++] = node;
    while (top > 0) {
        const int64_t k = stack[--top];
        const int64_t a = t->start[k], b = t->end[k];
        if (b <= a) continue;
        int nc = 0;
        for (int q = 0; q < nq; q++) nc += t->child[k * nq + q] != EMPTY;
        if (is_leaf(t, k) || !sparse_node(D, t->size[k], b - a, S, C) || top + nc > kStack) {
            push_range(ranges, ng, a, b);
            continue;
        }
        for (int q = nq - 1; q >= 0; q--)
            if (t->child[k * nq + q] != EMPTY) stack[top++] = t->child[k * nq + q];
    }
}

static void make_groups(const or_tree *t, int64_t k, int64_t GS, int is_root, int64_t *ranges,
                        int64_t *ng) {
    const int nq = 1 << t->dims;
    const int64_t a = t->start[k], b = t->end[k];
    if (b - a <= GS) {
        if (is_root && b > a) push_range(ranges, ng, a, b);
        return;
    }
    if (is_leaf(t, k)) {
        for (int64_t s = a; s < b; s += GS) push_range(ranges, ng, s, s + GS < b ? s + GS : b);
        return;
    }
    int64_t ra = 0, rb = 0;
    for (int q = 0; q < nq; q++) {
        const uint32_t c = t->child[k * nq + q];
        if (c == EMPTY) continue;
        const int64_t ca = t->start[c], cb = t->end[c];
        if (cb - ca > GS) {
            if (rb > ra) push_range(ranges, ng, ra, rb);
            ra = rb = 0;
            make_groups(t, c, GS, 0, ranges, ng);
            continue;
        }
        if (!is_leaf(t, c) && sparse_node(t->dims, t->size[c], cb - ca, t->size[k], b - a)) {
            if (rb > ra) push_range(ranges, ng, ra, rb);
            ra = rb = 0;
            split_sparse(t, c, t->size[k], b - a, ranges, ng);
            continue;
        }
        if (rb > ra && rb == ca && cb - ra <= GS) {
            rb = cb;
        } else {
            if (rb > ra) push_range(ranges, ng, ra, rb);
            ra = ca;
            rb = cb;
        }
    }
    if (rb > ra) push_range(ranges, ng, ra, rb);
}

/* Group walk (the mixed mode with group_size > 0): the groups above; a node
 * is accepted for the whole group when
 * b^2 < eps2 + sum_a max(lo_a - com_a, com_a - hi_a, 0)^2 (FP32, fused
 * multiply-adds in axis order, [lo, hi] the group's bounding box); an opened
 * leaf contributes its particles.  The interaction set is evaluated in FP64
 * for each member (the particle itself skipped). */
static void group_visit(const or_tree *t, const double *mom, const float *b2, const float *hi,
                        int64_t k, const float lo_b[3], const float hi_b[3], float eps2,
                        int64_t *nodes, int64_t *nn, int64_t *leaves, int64_t *nl) {
    const int D = t->dims, R = D == 2 ? 6 : 10, nq = 1 << D;
    if (!(mom[k * R] > 0.0)) return;
    float dm = eps2;
    for (int a = 0; a < D; a++) {
        const float c = hi[k * 3 + a];
        const float e = fmaxf(fmaxf(lo_b[a] - c, c - hi_b[a]), 0.0f);
        dm = fmaf(e, e, dm);
    }
    if (b2[k] < dm) { nodes[(*nn)++] = k; return; }
    if (is_leaf(t, k)) { leaves[(*nl)++] = k; return; }
    for (int q = 0; q < nq; q++) {
        const uint32_t c = t->child[k * nq + q];
        if (c != EMPTY) group_visit(t, mom, b2, hi, c, lo_b, hi_b, eps2, nodes, nn, leaves, nl);
    }
}

void or_walk_group(int64_t n, const float *x, const float *y, const float *z, const float *m,
                   const or_tree *t, const or_params *p, int group_size, double *ax, double *ay,
                   double *az, uint32_t *inter, int nthreads) {
    const int D = t->dims, R = D == 2 ? 6 : 10;
    const int64_t cnt = t->count > 0 ? t->count : 1;
    double *mom = (double *)malloc(sizeof(double) * (size_t)cnt * R);
    float *b2 = (float *)malloc(sizeof(float) * (size_t)cnt);
    float *hi = (float *)malloc(sizeof(float) * (size_t)cnt * 3);
    if (!mom || !b2 || !hi) { free(mom); free(b2); free(hi); return; }
    or_moments_mixed(t, x, y, z, m, mom);
    const double inv_theta = 1.0 / (double)p->theta;
    for (int64_t k = 0; k < t->count; k++) {
        const double *r = mom + k * R;
        const double half = 0.5 * (double)t->size[k];
        double del2 = 0.0;
        for (int a = 0; a < D; a++) {
            hi[k * 3 + a] = (float)r[1 + a];
            const double dc = r[1 + a] - ((double)t->pos[k * D + a] + half);
            del2 = fma(dc, dc, del2);
        }
        const double b = fma((double)t->size[k], inv_theta, sqrt(del2));
        b2[k] = (float)(b * b);
    }
    const float *pos[3] = {x, y, z};
    const int64_t GS = group_size;
    int64_t *ranges = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(n > 0 ? n : 1));
    int64_t ngroups = 0;
    if (!ranges) { free(mom); free(b2); free(hi); return; }
    if (t->count > 0) make_groups(t, 0, GS, 1, ranges, &ngroups);
    const double G = p->G, eps2d = p->eps2;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int64_t g = 0; g < ngroups; g++) {
        const int64_t i0 = ranges[2 * g], i1 = ranges[2 * g + 1];
        float lo_b[3] = {INFINITY, INFINITY, INFINITY}, hi_b[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = i0; i < i1; i++)
            for (int a = 0; a < D; a++) {
                lo_b[a] = fminf(lo_b[a], pos[a][i]);
                hi_b[a] = fmaxf(hi_b[a], pos[a][i]);
            }
        int64_t *nodes = (int64_t *)malloc(sizeof(int64_t) * (size_t)cnt);
        int64_t *leaves = (int64_t *)malloc(sizeof(int64_t) * (size_t)cnt);
        int64_t nn = 0, nl = 0;
        if (nodes && leaves && t->count > 0)
            group_visit(t, mom, b2, hi, 0, lo_b, hi_b, p->eps2, nodes, &nn, leaves, &nl);
        for (int64_t i = i0; i < i1; i++) {
            double f[3] = {0, 0, 0};
            uint32_t c = 0;
            for (int64_t u = 0; u < nn; u++) {
                const double *r = mom + nodes[u] * R;
                double d[3] = {0, 0, 0}, rr = eps2d;
                for (int a = 0; a < D; a++) {
                    d[a] = r[1 + a] - (double)pos[a][i];
                    rr += d[a] * d[a];
                }
                const double inv = 1.0 / sqrt(rr), inv2 = inv * inv, inv3 = inv2 * inv;
                const double inv5 = inv3 * inv2, inv7 = inv5 * inv2;
                double I[3][3] = {{0}};
                for (int a = 0; a < D; a++)
                    for (int b = a; b < D; b++) I[a][b] = I[b][a] = (double)(float)r[mom_index(D, a, b)];
                double Id[3] = {0, 0, 0}, dId = 0.0, tr = 0.0;
                for (int a = 0; a < D; a++) {
                    for (int b = 0; b < D; b++) Id[a] += I[a][b] * d[b];
                    dId += d[a] * Id[a];
                    tr += I[a][a];
                }
                const double M = (double)(float)r[0];
                const double cm = M * inv3 - 1.5 * tr * inv5 + 7.5 * dId * inv7;
                for (int a = 0; a < D; a++) f[a] += cm * d[a] - 3.0 * Id[a] * inv5;
                c++;
            }
            for (int64_t u = 0; u < nl; u++) {
                const int64_t k = leaves[u];
                for (uint32_t j = t->start[k]; j < t->end[k]; j++) {
                    if ((int64_t)j == i) continue;
                    double d[3] = {0, 0, 0}, rr = eps2d;
                    for (int a = 0; a < D; a++) {
                        d[a] = (double)pos[a][j] - (double)pos[a][i];
                        rr += d[a] * d[a];
                    }
                    const double inv = 1.0 / sqrt(rr), fm = (double)m[j] * inv * inv * inv;
                    for (int a = 0; a < D; a++) f[a] += fm * d[a];
                    c++;
                }
            }
            ax[i] = G * f[0];
            ay[i] = G * f[1];
            if (D == 3 && az) az[i] = G * f[2];
            if (inter) inter[i] = c;
        }
        free(nodes);
        free(leaves);
    }
    free(ranges);
    free(mom); free(b2); free(hi);
}
