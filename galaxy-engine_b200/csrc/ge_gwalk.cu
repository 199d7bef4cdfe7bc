// ge_gwalk.cu -- the group walk of the mixed-precision mode.
//
// No counterpart in the reference: its walk (physics.cpp:91-205,
// physics3D.cpp:131-253) is one traversal per particle.  Here one warp walks
// the tree once for a group of at most GS = 32 x PPL particles that share a
// small cell of the tree (k_make_groups):
//   * the group's bounding box decides the opening test for all of them: a
//     node is accepted when b^2 < dmin^2 + eps2, dmin the distance from its
//     centre of mass to the box and b the node's opening radius (ge_moments.cu),
//     which is at least as strict as every member's own test;
//   * up to 32 candidate nodes are tested at once, one per lane, taken from a
//     per-warp work stack in shared memory (moved to the warp's stack in
//     global memory when it outgrows it);
//   * accepted nodes (centre of mass, mass, second moments) and the
//     particles of opened leaves are staged in shared memory and, when a list
//     fills up or the walk ends, every lane evaluates them for its own
//     particles (monopole + softened quadrupole for nodes, the softened pair
//     force for particles; the particle itself is skipped);
//   * each lane sums a list pass in FP32 and adds that sum to its running
//     total with Kahan compensation.
// Which nodes a particle interacts with depends only on its group, not on the
// traversal order, so the interaction set is deterministic; only the FP32
// summation order within a list pass follows the traversal.
#include <cfloat>

#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kGWWarps = 4;
constexpr int kGWThreads = kGWWarps * 32;
constexpr int kGWNodes = 64;           // staged accepted nodes per warp
constexpr int kGWParts = 64;           // staged leaf particles per warp
constexpr uint32_t kGWStack = 2048;    // work stack entries per warp (global memory)
// the work stack lives in shared memory while it fits (the deepest measured
// stacks: ~170 entries in 2D, ~800 in 3D at theta 0.5, ~1400 at theta 0.3)
// and moves to the warp's global stack when it would not
template <int D> struct GWShared { static constexpr uint32_t value = D == 2 ? 256u : 1024u; };
constexpr int kMetaGroupCtr = 10;      // tree meta word: next group to walk
constexpr int kMetaGroupCount = 11;    // tree meta word: groups made
constexpr int kMetaSlotsW = 9;         // tree meta word: node slots of the last build

template <int D>
struct GWSmem {
    // an accepted node, staged: c = (hi - o) + lo, its centre of mass from
    // the group's centre o; J = 7.5 I, its second moments; t = -1.5 tr(I)
    float4 nA[kGWNodes];   // 2D {c.x, c.y, m, Jxx}; 3D {c.x, c.y, c.z, m}
    float4 nB[kGWNodes];   // 2D {Jxy, Jyy, t, 0}; 3D {Jxx, Jyz, t, 0}
    float4 nC[D == 3 ? kGWNodes : 1];   // 3D {Jyy, Jzz, Jxy, Jxz}
    float4 pA[kGWParts];   // {x - o, m}
    uint32_t pI[kGWParts]; // particle slot
};

__device__ __forceinline__ float rsqrt_fast(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <int D, int PPL>
struct GroupState {
    float x[PPL][3];
    float f[PPL][3], fc[PPL][3];   // running sums and their Kahan compensation
    float u[PPL], uc[PPL];         // potential pass: sum of m / r terms (phi = -G u)
    uint32_t idx[PPL];
    bool act[PPL];
    unsigned long long count;
};

// accepted nodes: monopole + quadrupole of the softened kernel (with POT,
// the potential instead: M / r + 1.5 (d.I.d) / r^5 - 0.5 tr(I) / r^3).  The
// moments are staged as J = 7.5 I with t = -1.5 tr(I), so that
//   a = (M / r^3 + (d.J.d / r^2 + t) / r^5) d - 0.4 (J d) / r^5.
template <int D, int PPL, bool POT = false>
__device__ __forceinline__ void flush_nodes(const GWSmem<D> &sm, int nl, GroupState<D, PPL> &g,
                                            float eps2, bool count) {
    float acc[PPL][3], pu[PPL];
#pragma unroll
    for (int k = 0; k < PPL; k++) {
        pu[k] = 0.0f;
#pragma unroll
        for (int a = 0; a < 3; a++) acc[k][a] = 0.0f;
    }
    for (int j = 0; j < nl; j++) {
        const float4 A = sm.nA[j], B = sm.nB[j];
        const float4 C = D == 3 ? sm.nC[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float tq = B.z;
        const float m = D == 2 ? A.z : A.w;
        const float jxx = D == 2 ? A.w : B.x;
        const float jxy = D == 2 ? B.x : C.z;
        const float jyy = D == 2 ? B.y : C.x;
#pragma unroll
        for (int k = 0; k < PPL; k++) {
            float d[3];
            d[0] = A.x - g.x[k][0];
            d[1] = A.y - g.x[k][1];
            d[2] = D == 3 ? A.z - g.x[k][2] : 0.0f;
            float rr = __fmaf_rn(d[1], d[1], eps2);
            if (D == 3) rr = __fmaf_rn(d[2], d[2], rr);
            rr = __fmaf_rn(d[0], d[0], rr);
            const float inv = rsqrt_fast(rr);
            const float inv2 = inv * inv, inv3 = inv2 * inv, inv5 = inv3 * inv2;
            float Jd[3];
            if (D == 2) {
                Jd[0] = __fmaf_rn(jxx, d[0], jxy * d[1]);
                Jd[1] = __fmaf_rn(jxy, d[0], jyy * d[1]);
                Jd[2] = 0.0f;
            } else {
                const float jzz = C.y, jxz = C.w, jyz = B.y;
                Jd[0] = __fmaf_rn(jxx, d[0], __fmaf_rn(jxy, d[1], jxz * d[2]));
                Jd[1] = __fmaf_rn(jxy, d[0], __fmaf_rn(jyy, d[1], jyz * d[2]));
                Jd[2] = __fmaf_rn(jxz, d[0], __fmaf_rn(jyz, d[1], jzz * d[2]));
            }
            float dJd = __fmaf_rn(d[1], Jd[1], d[0] * Jd[0]);
            if (D == 3) dJd = __fmaf_rn(d[2], Jd[2], dJd);
            if (POT) {   // 1.5 d.I.d = 0.2 d.J.d, -0.5 tr = t / 3
                pu[k] += m * inv + 0.2f * dJd * inv5 + (tq * (1.0f / 3.0f)) * inv3;
                continue;
            }
            const float q = __fmaf_rn(dJd, inv2, tq);
            const float cm = __fmaf_rn(q, inv5, m * inv3);
            const float ci = -0.4f * inv5;
#pragma unroll
            for (int a = 0; a < D; a++) acc[k][a] = __fmaf_rn(ci, Jd[a], __fmaf_rn(cm, d[a], acc[k][a]));
        }
    }
#pragma unroll
    for (int k = 0; k < PPL; k++) {
        if (POT) kahan_add(g.u[k], g.uc[k], pu[k]);
#pragma unroll
        for (int a = 0; a < D; a++)
            if (!POT) kahan_add(g.f[k][a], g.fc[k][a], acc[k][a]);
        if (count && g.act[k]) g.count += (unsigned long long)nl;
    }
}

// particles of opened leaves: the softened pair force (with POT, m / r), the
// particle itself skipped
template <int D, int PPL, bool POT = false>
__device__ __forceinline__ void flush_parts(const GWSmem<D> &sm, int pl, GroupState<D, PPL> &g,
                                            float eps2, bool count) {
    float acc[PPL][3], pu[PPL];
    uint32_t self_hits = 0;
#pragma unroll
    for (int k = 0; k < PPL; k++) {
        pu[k] = 0.0f;
#pragma unroll
        for (int a = 0; a < 3; a++) acc[k][a] = 0.0f;
    }
    if (!POT && !count && eps2 > 0.0f) {
        // the particle's own term is exactly zero (d = 0: its staged offset
        // is its own offset, bit for bit), so no pair needs the test
        for (int j = 0; j < pl; j++) {
            const float4 P = sm.pA[j];
#pragma unroll
            for (int k = 0; k < PPL; k++) {
                float d[3];
                d[0] = P.x - g.x[k][0];
                d[1] = P.y - g.x[k][1];
                d[2] = D == 3 ? P.z - g.x[k][2] : 0.0f;
                float rr = __fmaf_rn(d[1], d[1], eps2);
                if (D == 3) rr = __fmaf_rn(d[2], d[2], rr);
                rr = __fmaf_rn(d[0], d[0], rr);
                const float inv = rsqrt_fast(rr);
                const float fm = P.w * (inv * inv * inv);
#pragma unroll
                for (int a = 0; a < D; a++) acc[k][a] = __fmaf_rn(d[a], fm, acc[k][a]);
            }
        }
    } else
    for (int j = 0; j < pl; j++) {
        const float4 P = sm.pA[j];
        const uint32_t pj = sm.pI[j];
#pragma unroll
        for (int k = 0; k < PPL; k++) {
            float d[3];
            d[0] = P.x - g.x[k][0];
            d[1] = P.y - g.x[k][1];
            d[2] = D == 3 ? P.z - g.x[k][2] : 0.0f;
            float rr = d[0] * d[0] + d[1] * d[1] + eps2;
            if (D == 3) rr += d[2] * d[2];
            const float inv = rsqrt_fast(rr);
            const bool self = pj == g.idx[k];
            self_hits += (self && g.act[k]) ? 1u : 0u;
            if (POT) {
                pu[k] += self ? 0.0f : P.w * inv;
                continue;
            }
            const float fm = self ? 0.0f : P.w * (inv * inv * inv);
#pragma unroll
            for (int a = 0; a < D; a++) acc[k][a] += d[a] * fm;
        }
    }
#pragma unroll
    for (int k = 0; k < PPL; k++) {
        if (POT) kahan_add(g.u[k], g.uc[k], pu[k]);
#pragma unroll
        for (int a = 0; a < D; a++)
            if (!POT) kahan_add(g.f[k][a], g.fc[k][a], acc[k][a]);
        if (count && g.act[k]) g.count += (unsigned long long)pl;
    }
    if (count) g.count -= self_hits;
}

// Groups: every particle belongs to exactly one node that holds at most GS
// particles while its parent holds more (or that is its simulation's root);
// runs of such nodes that are adjacent children of one parent are packed
// into one group while the run holds at most GS particles.  A group is then
// a contiguous particle range inside one cell (its parent's), so its
// bounding box stays compact.  A leaf of more than GS particles (a cell at
// the minimum size) is cut into GS-particle pieces.  A sparse child (below)
// is split down its subtree instead.  The groups depend only on the tree, so
// a simulation forms the same groups alone and in a batch.
__device__ __forceinline__ void emit_group(const Tree &t, uint32_t a, uint32_t b) {
    const uint32_t k = atomicAdd(&t.meta[kMetaGroupCount], 1u);
    t.grp[k] = make_uint2(a, b);
}

// A node of c particles and cell size s is sparse, relative to a parent of
// C particles and size S, when its particles' mean spacing is more than four
// times the parent's: (s / S)^D C > 4^D c.  A group made of it would have a
// box far larger than the matter around it warrants (halo and tidal-tail
// particles in a cell beside a dense disk: one such group of 57 particles
// spread over 6 x 10 units opened ~11,000 particles for every member and
// held one warp for 3.5 ms), so it is split down its subtree, depth first
// with a stack of 256 entries, into nodes dense enough by the same reference,
// or leaves (the node whole when the stack is full).
template <int D>
__device__ __forceinline__ bool sparse_node(float s, uint32_t c, float S, uint32_t C) {
    const double r = (double)s / (double)S;
    const double rd = D == 2 ? r * r : r * r * r;
    return rd * (double)C > (D == 2 ? 16.0 : 64.0) * (double)c;
}

template <int D>
__device__ void emit_split(const Tree &t, uint32_t node, float S, uint32_t C) {
    constexpr int kStack = 256;
    uint32_t stack[kStack];
    int top = 0;
    stack[top++] = node;
    while (top > 0) {
        const uint32_t k = stack[--top];
        const uint4 inf = __ldcg(&t.info[k]);
        if (inf.w <= inf.z) continue;
        const int nc = __popc(inf.y);
        // a leaf, a node dense enough, or (stack full) the node whole
        if (!inf.y || !sparse_node<D>(__ldcg(&t.cell[k]).w, inf.w - inf.z, S, C) ||
            top + nc > kStack) {
            emit_group(t, inf.z, inf.w);
            continue;
        }
        for (int q = nc - 1; q >= 0; q--) stack[top++] = inf.x + (uint32_t)q;
    }
}

template <int D>
__global__ void k_make_groups(Tree t, uint32_t GS) {
    dep_wait();
    const uint32_t slots = __ldcg(&t.meta[kMetaSlotsW]);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < slots; k += stride) {
        const uint4 inf = __ldcg(&t.info[k]);
        if (inf.w <= inf.z) continue;   // hole
        const uint32_t cnt = inf.w - inf.z;
        if (cnt <= GS) {
            if (__ldcg(&t.aux[k]).z == kEmpty) emit_group(t, inf.z, inf.w);   // a small root
            continue;
        }
        if (!inf.y) {   // a leaf larger than a group
            for (uint32_t a = inf.z; a < inf.w; a += GS) emit_group(t, a, min(a + GS, inf.w));
            continue;
        }
        const int nc = __popc(inf.y);
        const float S = __ldcg(&t.cell[k]).w;
        uint32_t ra = 0, rb = 0;   // current run of small adjacent children
        for (int c = 0; c < nc; c++) {
            const uint32_t ck = inf.x + (uint32_t)c;
            const uint4 ci = __ldcg(&t.info[ck]);
            const uint32_t cc = ci.w - ci.z;
            if (cc > GS) {
                if (rb > ra) emit_group(t, ra, rb);
                ra = rb = 0;
                continue;
            }
            if (ci.y && sparse_node<D>(__ldcg(&t.cell[ck]).w, cc, S, cnt)) {
                if (rb > ra) emit_group(t, ra, rb);
                ra = rb = 0;
                emit_split<D>(t, ck, S, cnt);
                continue;
            }
            if (rb > ra && rb == ci.z && (ci.w - ra) <= GS) {
                rb = ci.w;
            } else {
                if (rb > ra) emit_group(t, ra, rb);
                ra = ci.z;
                rb = ci.w;
            }
        }
        if (rb > ra) emit_group(t, ra, rb);
    }
}

template <int D, int PPL, bool COUNT, bool POT = false>
__global__ void __launch_bounds__(kGWThreads)
k_group_walk(State s, StepParams p, Segs sg_tab, Tree t, int integrate_end,
             unsigned long long *inter, uint32_t *err, double *epot = nullptr) {
    dep_wait();
    __shared__ GWSmem<D> smem[kGWWarps];
    __shared__ uint32_t s_stack[kGWWarps][GWShared<D>::value];
    GWSmem<D> &sm = smem[threadIdx.x >> 5];
    uint32_t *stk = s_stack[threadIdx.x >> 5];
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t *wl = t.wl + (size_t)gwarp * kGWStack;
    const uint32_t ngroups = __ldcg(&t.meta[kMetaGroupCount]);
    const float eps2 = p.eps2;
    const float *pos[3] = {s.x, s.y, s.z};
    GroupState<D, PPL> g;
    g.count = 0;
    while (true) {
        uint32_t grp = 0;
        if (lane == 0) grp = atomicAdd(&t.meta[kMetaGroupCtr], 1u);
        grp = __shfl_sync(0xffffffffu, grp, 0);
        if (grp >= ngroups) break;
        const uint2 range = __ldcg(&t.grp[grp]);
        const uint32_t base = range.x, seg_end = range.y;
        const uint32_t sg = sg_tab.seg_of ? sg_tab.seg_of[base] : 0u;
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
#pragma unroll
        for (int k = 0; k < PPL; k++) {
            const uint32_t i = base + (uint32_t)k * 32u + lane;
            g.idx[k] = i;
            g.act[k] = i < seg_end;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                g.x[k][a] = (g.act[k] && a < D) ? pos[a][i] : 0.0f;
                g.f[k][a] = 0.0f;
                g.fc[k][a] = 0.0f;
            }
            g.u[k] = 0.0f;
            g.uc[k] = 0.0f;
            if (g.act[k]) {
#pragma unroll
                for (int a = 0; a < D; a++) {
                    lo[a] = fminf(lo[a], g.x[k][a]);
                    hi[a] = fmaxf(hi[a], g.x[k][a]);
                }
            }
        }
#pragma unroll
        for (int a = 0; a < D; a++)
            for (int o = 16; o > 0; o >>= 1) {
                lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
                hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
            }
        // the list terms are evaluated from the group's centre o: members
        // and staged sources are stored as offsets from it (the opening test
        // keeps the absolute box)
        float oc[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int a = 0; a < D; a++) oc[a] = 0.5f * (lo[a] + hi[a]);
#pragma unroll
        for (int k = 0; k < PPL; k++)
#pragma unroll
            for (int a = 0; a < D; a++) g.x[k][a] -= oc[a];
        int nl = 0, pl = 0;
        uint32_t top = 1;
        bool spilled = false;   // warp-uniform: the stack is in wl (global)
        if (lane == 0) stk[0] = sg;   // the simulation's root node slot
        __syncwarp();
        bool overflow = false;
        while (top > 0) {
            const uint32_t take = min(top, 32u);
            top -= take;
            const uint32_t c = lane < take ? (spilled ? __ldcg(&wl[top + lane]) : stk[top + lane])
                                           : kEmpty;
            __syncwarp();
            int kind = 0;   // 1 accepted node, 2 opened leaf, 3 opened internal node
            float4 A = make_float4(0.f, 0.f, 0.f, 0.f);
            uint4 inf = make_uint4(0u, 0u, 0u, 0u);
            if (c != kEmpty) {
                A = __ldg(&t.gw[c]);
                inf = __ldg(&t.info[c]);
                const float m = D == 2 ? A.z : A.w;
                const float b2 = D == 2 ? A.w : __ldg(&t.gq2[c]).y;
                if (m > 0.0f) {
                    const float com[3] = {A.x, A.y, A.z};
                    float dm = eps2;
#pragma unroll
                    for (int a = 0; a < D; a++) {
                        const float e = fmaxf(fmaxf(lo[a] - com[a], com[a] - hi[a]), 0.0f);
                        dm = __fmaf_rn(e, e, dm);
                    }
                    kind = b2 < dm ? 1 : (inf.y ? 3 : 2);
                }
            }
            // 1. accepted nodes into the node list
            const unsigned accb = __ballot_sync(0xffffffffu, kind == 1);
            if (nl + __popc(accb) > kGWNodes) {
                flush_nodes<D, PPL, POT>(sm, nl, g, eps2, COUNT);
                nl = 0;
                __syncwarp();
            }
            if (kind == 1) {
                const int q = nl + __popc(accb & lt);
                float4 Bq = __ldg(&t.gq0[c]);
                float4 Cq = D == 3 ? __ldg(&t.gq1[c]) : make_float4(0.f, 0.f, 0.f, 0.f);
                float Eq = __ldg(&t.gq2[c]).x;
                // staged for flush_nodes: J = 7.5 I and t = -1.5 tr(I)
                float tr;
                if (D == 2) {   // {lo.x, lo.y, Ixx, Ixy}, Iyy
                    tr = Bq.z + Eq;
                    Bq.z *= 7.5f; Bq.w *= 7.5f; Eq *= 7.5f;
                } else {        // {lo.xyz, Ixx}, {Iyy, Izz, Ixy, Ixz}, Iyz
                    tr = Bq.w + Cq.x + Cq.y;
                    Bq.w *= 7.5f; Cq.x *= 7.5f; Cq.y *= 7.5f; Cq.z *= 7.5f; Cq.w *= 7.5f; Eq *= 7.5f;
                }
                const float cx = (A.x - oc[0]) + Bq.x, cy = (A.y - oc[1]) + Bq.y;
                if (D == 2) {
                    sm.nA[q] = make_float4(cx, cy, A.z, Bq.z);
                    sm.nB[q] = make_float4(Bq.w, Eq, -1.5f * tr, 0.0f);
                } else {
                    sm.nA[q] = make_float4(cx, cy, (A.z - oc[2]) + Bq.z, A.w);
                    sm.nB[q] = make_float4(Bq.w, Eq, -1.5f * tr, 0.0f);
                    sm.nC[q] = Cq;
                }
            }
            nl += __popc(accb);
            // 2. children of opened internal nodes onto the work stack
            const uint32_t nch = kind == 3 ? (uint32_t)__popc(inf.y) : 0u;
            uint32_t incl = nch;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (unsigned)o) incl += v;
            }
            const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
            if (!spilled && top + tot > GWShared<D>::value) {   // warp-uniform: move to wl
                for (uint32_t q = lane; q < top; q += 32) wl[q] = stk[q];
                spilled = true;
                __syncwarp();
            }
            if (top + tot > kGWStack) {   // warp-uniform
                overflow = true;
                break;
            }
            if (spilled)
                for (uint32_t q = 0; q < nch; q++) wl[top + incl - nch + q] = inf.x + q;
            else
                for (uint32_t q = 0; q < nch; q++) stk[top + incl - nch + q] = inf.x + q;
            top += tot;
            // 3. particles of opened leaves into the particle list
            uint32_t pc = kind == 2 ? inf.w - inf.z : 0u;
            uint32_t pbeg = inf.z;
            unsigned pend = __ballot_sync(0xffffffffu, pc > 0u);
            while (pend) {
                uint32_t pin = pc;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xffffffffu, pin, o);
                    if (lane >= (unsigned)o) pin += v;
                }
                const uint32_t ptot = __shfl_sync(0xffffffffu, pin, 31);
                if (pl + ptot <= (uint32_t)kGWParts) {
                    for (uint32_t j = 0; j < pc; j++) {
                        const uint32_t q = pl + pin - pc + j, src = pbeg + j;
                        sm.pA[q] = make_float4(s.x[src] - oc[0], s.y[src] - oc[1],
                                               D == 3 ? s.z[src] - oc[2] : 0.0f, s.m[src]);
                        sm.pI[q] = src;
                    }
                    pl += (int)ptot;
                    break;
                }
                // does not fit: flush, then move the first pending leaf in
                // list-sized chunks
                __syncwarp();
                flush_parts<D, PPL, POT>(sm, pl, g, eps2, COUNT);
                __syncwarp();
                const int L = __ffs(pend) - 1;
                const uint32_t lb = __shfl_sync(0xffffffffu, pbeg, L);
                const uint32_t lc = __shfl_sync(0xffffffffu, pc, L);
                const uint32_t chunk = min(lc, (uint32_t)kGWParts);
                for (uint32_t j = lane; j < chunk; j += 32) {
                    sm.pA[j] = make_float4(s.x[lb + j] - oc[0], s.y[lb + j] - oc[1],
                                           D == 3 ? s.z[lb + j] - oc[2] : 0.0f, s.m[lb + j]);
                    sm.pI[j] = lb + j;
                }
                pl = (int)chunk;
                if ((int)lane == L) {
                    pbeg += chunk;
                    pc -= chunk;
                }
                __syncwarp();
                pend = __ballot_sync(0xffffffffu, pc > 0u);
            }
            __syncwarp();
        }
        if (overflow) {
            if (lane == 0) set_err(err, kErrStack);
            nl = 0;
            pl = 0;
        }
        __syncwarp();
        if (nl) flush_nodes<D, PPL, POT>(sm, nl, g, eps2, COUNT);
        if (pl) flush_parts<D, PPL, POT>(sm, pl, g, eps2, COUNT);
        __syncwarp();
        if (POT) {   // potential pass: sum_i m_i u_i in FP64, nothing written to the state
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < PPL; k++)
                if (g.act[k]) v += (double)s.m[g.idx[k]] * ((double)g.u[k] - (double)g.uc[k]);
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) atomicAdd(epot, v);
            continue;
        }
        // results and the fused second half kick
#pragma unroll
        for (int k = 0; k < PPL; k++) {
            if (!g.act[k]) continue;
            const uint32_t i = g.idx[k];
            float a3[3];
#pragma unroll
            for (int a = 0; a < D; a++) a3[a] = p.G * (g.f[k][a] - g.fc[k][a]);
            s.ax[i] = a3[0];
            s.ay[i] = a3[1];
            if (D == 3) s.az[i] = a3[2];
            if (integrate_end && !(s.pinned && s.pinned[i])) {
                float *vel[3] = {s.vx, s.vy, s.vz};
                if (s.kvx) {
                    float *kv[3] = {s.kvx, s.kvy, s.kvz};
#pragma unroll
                    for (int a = 0; a < D; a++) kahan_add(vel[a][i], kv[a][i], fmul(a3[a], p.half_dt));
                } else {
#pragma unroll
                    for (int a = 0; a < D; a++) vel[a][i] = fadd(vel[a][i], fmul(a3[a], p.half_dt));
                }
            }
        }
    }
    if (COUNT) {
        unsigned long long v = g.count;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(inter, v);
    }
}

static int grid_blocks(int n) {
    int b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    return b < 1 ? 1 : b;
}

template <int D, int PPL, bool COUNT>
static int resident_blocks() {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_group_walk<D, PPL, COUNT>,
                                                      kGWThreads, 0) != cudaSuccess)
        return 0;
    return per_sm;
}

template <int D>
static int most_resident() {
    int m = resident_blocks<D, 1, false>();
    m = max(m, resident_blocks<D, 2, false>());
    m = max(m, resident_blocks<D, 4, false>());
    m = max(m, resident_blocks<D, 1, true>());
    m = max(m, resident_blocks<D, 2, true>());
    m = max(m, resident_blocks<D, 4, true>());
    return m;
}

// Warps the group walk keeps resident (its work stacks are sized for them).
int group_walk_warps(int dims, int num_sms) {
    const int per_sm = dims == 2 ? most_resident<2>() : most_resident<3>();
    return per_sm * num_sms * kGWWarps;
}

uint32_t group_walk_stack_entries() { return kGWStack; }

template <int D, int PPL, bool COUNT>
static cudaError_t gw_launch(const State &s, const StepParams &p, const Segs &g, const Tree &t,
                             int ie, unsigned long long *inter, uint32_t *err, cudaStream_t st) {
    cudaError_t e = launch_dep(k_make_groups<D>, grid_blocks(p.n), 256, st, t, 32u * PPL);
    if (e != cudaSuccess) return e;
    // one work stack per warp bounds the grid; groups number at most n
    int blocks = (int)(t.wl_warps / kGWWarps);
    const int64_t want = ((int64_t)p.n + kGWWarps - 1) / kGWWarps;
    if (blocks > want) blocks = (int)want;
    if (blocks < 1) blocks = 1;
    double *no_pot = nullptr;
    return launch_dep(k_group_walk<D, PPL, COUNT>, blocks, kGWThreads, st, s, p, g, t, ie, inter, err,
                      no_pot);
}

template <int D>
static cudaError_t gw_dims(const State &s, const StepParams &p, const Segs &g, const Tree &t,
                           int ie, unsigned long long *inter, uint32_t *err, cudaStream_t st) {
    if (inter) {
        if (p.group_size >= 128) return gw_launch<D, 4, true>(s, p, g, t, ie, inter, err, st);
        if (p.group_size >= 64) return gw_launch<D, 2, true>(s, p, g, t, ie, inter, err, st);
        return gw_launch<D, 1, true>(s, p, g, t, ie, inter, err, st);
    }
    if (p.group_size >= 128) return gw_launch<D, 4, false>(s, p, g, t, ie, inter, err, st);
    if (p.group_size >= 64) return gw_launch<D, 2, false>(s, p, g, t, ie, inter, err, st);
    return gw_launch<D, 1, false>(s, p, g, t, ie, inter, err, st);
}

template <int D, int PPL>
static cudaError_t gw_pot(const State &s, const StepParams &p, const Segs &g, const Tree &t,
                          uint32_t *err, double *epot, cudaStream_t st) {
    k_make_groups<D><<<grid_blocks(p.n), 256, 0, st>>>(t, 32u * PPL);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int blocks = (int)(t.wl_warps / kGWWarps);
    const int64_t want = ((int64_t)p.n + kGWWarps - 1) / kGWWarps;
    if (blocks > want) blocks = (int)want;
    if (blocks < 1) blocks = 1;
    k_group_walk<D, PPL, false, true><<<blocks, kGWThreads, 0, st>>>(s, p, g, t, 0, nullptr, err,
                                                                     epot);
    return cudaGetLastError();
}

cudaError_t launch_group_potential(int dims, const State &s, const StepParams &p, const Segs &g,
                                   const Tree &t, uint32_t *counter, uint32_t *err, double *epot,
                                   cudaStream_t st) {
    if (!t.wl || !t.grp || t.wl_warps < (uint32_t)kGWWarps) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(counter, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(epot, 0, sizeof(double), st)) != cudaSuccess) return e;
    return dims == 2 ? gw_pot<2, 1>(s, p, g, t, err, epot, st) : gw_pot<3, 1>(s, p, g, t, err, epot, st);
}

cudaError_t launch_group_walk(int dims, const State &s, const StepParams &p, const Segs &g,
                              const Tree &t, bool integrate_end, unsigned long long *inter_count,
                              uint32_t *counter, uint32_t *err, cudaStream_t st) {
    if (!t.wl || !t.grp || t.wl_warps < (uint32_t)kGWWarps) return cudaErrorInvalidValue;
    // counter[0]: next group to walk, counter[1]: groups made
    cudaError_t e = cudaMemsetAsync(counter, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const int ie = integrate_end ? 1 : 0;
    return dims == 2 ? gw_dims<2>(s, p, g, t, ie, inter_count, err, st)
                     : gw_dims<3>(s, p, g, t, ie, inter_count, err, st);
}

}  // namespace ge
