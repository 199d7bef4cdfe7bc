// ge_tree_dev.cuh -- device helpers shared by the tree builds (ge_tree.cu,
// ge_kbuild.cu): the exact std::partition_point emulation, the leaf rule,
// leaf sums and the cell arithmetic of Node::subGridMaker.
#pragma once
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

// std::partition_point(v + first, v + first + len, [mid](float a){ return a < mid; })
// emulated by G consecutive lanes.  Lane j (1 <= j < G) of the group stands for
// node j of the search's decision tree (heap order; child 2j when the probe is
// false, 2j+1 when true); one round evaluates all of them and walks log2(G)
// steps.  All 32 lanes call this together; groups may differ in their
// arguments (len 0 for a group with nothing to search).  With SH the values
// are a shared-memory copy: element j is v[j - off].
template <int G, bool SH = false>
__device__ __forceinline__ uint32_t group_partition_point(const float *__restrict__ v,
                                                          uint32_t first, uint32_t len,
                                                          float mid, uint32_t off = 0u) {
    constexpr int DEPTH = (G == 32) ? 5 : (G == 16) ? 4 : (G == 8) ? 3 : (G == 4) ? 2 : 1;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gl = lane & (G - 1u);
    const unsigned gbase = lane & ~(G - 1u);
    while (__any_sync(0xffffffffu, len > 0)) {
        bool pred = false;
        if (len > 0 && gl > 0) {
            uint32_t f = first, l = len;
            const int depth = 31 - __clz(gl);
            for (int b = depth - 1; b >= 0 && l > 0; --b) {
                uint32_t half = l >> 1;
                if ((gl >> b) & 1u) { f += half + 1; l -= half + 1; }
                else { l = half; }
            }
            if (l > 0) pred = (SH ? v[f + (l >> 1) - off] : __ldg(v + f + (l >> 1))) < mid;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, pred) >> gbase;
        unsigned j = 1;
#pragma unroll
        for (int st = 0; st < DEPTH; st++) {
            if (len == 0) break;
            uint32_t half = len >> 1;
            unsigned b = (bal >> j) & 1u;
            if (b) { first += half + 1; len -= half + 1; }
            else { len = half; }
            j = 2 * j + b;
        }
    }
    return first;
}

// Cut points of one node per group of G lanes: Node::subGridMaker (y, then x
// in each half) / subGridMaker3D (z, then y in each half, then x in each
// quarter).  Every lane of the group ends with the group's b[0..Q].  With SH
// the coordinates are shared-memory copies of particles [off, off + len).
template <int D, int G, bool SH = false>
__device__ __forceinline__ void cut_group_v(const float *px, const float *py, const float *pz,
                                            uint32_t off, uint32_t st, uint32_t en,
                                            const float *mid, uint32_t *b) {
    constexpr int Q = 1 << D;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gl = lane & (G - 1u), gbase = lane & ~(G - 1u);
    b[0] = st; b[Q] = en;
    if (D == 2) {
        b[2] = group_partition_point<G, SH>(py, st, en - st, mid[1], off);
        const bool lo = gl < G / 2;
        const uint32_t f = lo ? st : b[2];
        const uint32_t l = lo ? b[2] - st : en - b[2];
        const uint32_t r = group_partition_point<G / 2, SH>(px, f, l, mid[0], off);
        b[1] = __shfl_sync(0xffffffffu, r, gbase);
        b[3] = __shfl_sync(0xffffffffu, r, gbase + G / 2);
    } else {
        b[4] = group_partition_point<G, SH>(pz, st, en - st, mid[2], off);
        const bool lo = gl < G / 2;
        uint32_t f = lo ? st : b[4];
        uint32_t l = lo ? b[4] - st : en - b[4];
        uint32_t r = group_partition_point<G / 2, SH>(py, f, l, mid[1], off);
        b[2] = __shfl_sync(0xffffffffu, r, gbase);
        b[6] = __shfl_sync(0xffffffffu, r, gbase + G / 2);
        const unsigned g4 = gl / (G / 4);
        const uint32_t a0 = g4 == 0 ? st : (g4 == 1 ? b[2] : (g4 == 2 ? b[4] : b[6]));
        const uint32_t a1 = g4 == 0 ? b[2] : (g4 == 1 ? b[4] : (g4 == 2 ? b[6] : en));
        r = group_partition_point<G / 4, SH>(px, a0, a1 - a0, mid[0], off);
        b[1] = __shfl_sync(0xffffffffu, r, gbase);
        b[3] = __shfl_sync(0xffffffffu, r, gbase + G / 4);
        b[5] = __shfl_sync(0xffffffffu, r, gbase + 2 * (G / 4));
        b[7] = __shfl_sync(0xffffffffu, r, gbase + 3 * (G / 4));
    }
}

template <int D, int G>
__device__ __forceinline__ void cut_group(const State &s, uint32_t st, uint32_t en,
                                          const float *mid, uint32_t *b) {
    cut_group_v<D, G>(s.x, s.y, s.z, 0u, st, en, mid, b);
}

// std::partition_point over predicate bits held in a register (bit r is the
// predicate of element r), GNU probe sequence, positions relative to bit 0
__device__ __forceinline__ uint32_t bits_partition_point(uint32_t bits, uint32_t first,
                                                         uint32_t len) {
    while (len > 0) {
        const uint32_t half = len >> 1;
        const uint32_t probe = first + half;
        if ((bits >> probe) & 1u) { first = probe + 1; len -= half + 1; }
        else { len = half; }
    }
    return first;
}

template <int D>
__device__ __forceinline__ bool is_leaf(const StepParams &p, uint32_t cnt, float size) {
    // quadtree.cpp:16 / :120 with the leaf capacity and size gate parameterised
    return ((cnt <= p.leaf_cap && size <= p.size_gate) || cnt == 1u) || size <= p.min_size;
}

// computeLeafMass / computeLeafMass3D: sequential sums in the reference's order
template <int D>
__device__ __forceinline__ float4 leaf_mass(const State &s, uint32_t st, uint32_t en) {
    float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t i = st; i < en; i++) {
        const float mi = s.m[i];
        gm = fadd(gm, mi);
        c[0] = fadd(c[0], fmul(s.x[i], mi));
        c[1] = fadd(c[1], fmul(s.y[i], mi));
        if (D == 3) c[2] = fadd(c[2], fmul(s.z[i], mi));
    }
    if (gm > 0.0f) {
        c[0] = fdiv(c[0], gm); c[1] = fdiv(c[1], gm);
        if (D == 3) c[2] = fdiv(c[2], gm);
    }
    return make_float4(c[0], c[1], c[2], gm);
}

template <int D>
__device__ __forceinline__ void put_walk(Tree &t, uint32_t k, float4 cm, float size) {
    const float s2 = fmul(size, size);
    if (D == 2) t.walk[k] = make_float4(cm.x, cm.y, cm.w, s2);
    else { t.walk[k] = make_float4(cm.x, cm.y, cm.z, cm.w); t.size2[k] = s2; }
}
// Corner of child slot q of a cell (Node::subGridMaker newPos).
template <int D>
__device__ __forceinline__ float4 child_cell(float4 cell, float half, unsigned q) {
    float4 cc;
    cc.x = fadd(cell.x, (q & 1u) ? half : 0.0f);
    cc.y = fadd(cell.y, (q & 2u) ? half : 0.0f);
    cc.z = D == 3 ? fadd(cell.z, (q & 4u) ? half : 0.0f) : 0.0f;
    cc.w = half;
    return cc;
}
}  // namespace ge
