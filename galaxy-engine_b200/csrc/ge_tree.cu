// ge_tree.cu -- quadtree / octree construction with mass and centre of mass,
// and the depth-first walk layout.
//
// Reference: Node::Node, Node::subGridMaker, computeLeafMass, computeInternalMass
// (GalaxyEngine/src/Physics/quadtree.cpp:5-88, include/Physics/quadtree.h:31-111)
// and the octree analogues (quadtree.cpp:109-271, quadtree.h:134-179).
//
// The reference builds recursively: a node over the Morton-sorted range
// [start, end) is a leaf when ((count <= 4 && size <= 2) || count == 1 ||
// size <= 1e-6); otherwise the range is cut by std::partition_point on float
// midpoint compares (y then x; z then y then x in 3D) and one child is made
// per non-empty quadrant.  Every cut point here is found with the exact probe
// sequence of std::partition_point (the GNU halving search), so the cut points
// agree with the reference even where float compares disagree with the Morton
// order and a range is not partitioned.
//
// One cooperative launch, three phases:
//  1. Nodes of more than kSmallNode particles are split level by level
//     (bounded grid barrier between levels).  A group of G lanes cuts one
//     node: G-1 lanes probe the G-1 nodes of the next log2(G) levels of the
//     search's decision tree per round.  Smaller non-leaf nodes are queued.
//  2. Each queued node's whole subtree is built by one warp without further
//     barriers: lane l holds particle start + l, the predicates of all its
//     particles against a node's midpoint come from one ballot, and the
//     searches run on those bits.
//  3. The depth-first walk layout (ge_internal.h) is scattered from the node
//     ranges: pre(k) = C(start) + level, successor = C(end) + level - same_end,
//     with C the prefix count of node ends.
// A node's mass and centre of mass are computed as soon as its last child is
// final (a per-node pending count), always reading the children in the
// reference's x-major subGrids order with the reference's rounding, so the
// sums are bit-identical to the reference's whatever order nodes finish in.
#include <cfloat>
#include <cuda/atomic>

#include "ge_device.cuh"
#include "ge_internal.h"
#include "ge_tree_dev.cuh"

namespace ge {

constexpr int kBuildThreads = 256;
constexpr int kMaxBuildBlocks = 4 * kBuildThreads;   // blocks of the cooperative build (chunk offsets in shared memory)
constexpr uint32_t kSmallNode = 32;

// meta[] words used by the build
constexpr int kMetaNodes = 0, kMetaLevels = 1, kMetaBarCount = 2, kMetaBarGen = 3,
              kMetaSmall = 5, kMetaP2Alloc = 6, kMetaTimeline = 7, kMetaReal = 8, kMetaSlots = 9,
              kMetaP2Task = 12, kMetaDone = 15, kMetaBuildId = 16;
constexpr uint32_t kChunk = 256;   // node slots a warp takes at a time in phase 2
// keyed builds: exact-rebuild roots and phase-1 nodes of at most kBlockRootMax
// particles are rebuilt by one block each
#ifndef GE_BLOCK_ROOT_MAX
#define GE_BLOCK_ROOT_MAX 2048
#endif
constexpr uint32_t kBlockRootMax = GE_BLOCK_ROOT_MAX;
constexpr int kBlkList = (int)(kBlockRootMax / kSmallNode);
constexpr int kKmBlockQ = 33;   // key meta word: phase-1 nodes handed to the blocks
constexpr int kKmBlockTake = 34;   // key meta word: next block root to take
constexpr int kKmProdDone = 64;    // key meta word (a cache line of its own): blocks done queueing

// Bounded grid-wide barrier for a cooperative launch (all blocks resident).
__device__ __forceinline__ void grid_barrier(uint32_t *bar_count, uint32_t *bar_gen,
                                             uint32_t *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t *vgen = bar_gen;
        uint32_t gen = *vgen;
        __threadfence();
        uint32_t arrived = atomicAdd(bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(bar_count, 0u);
            __threadfence();
            atomicAdd(bar_gen, 1u);
        } else {
            uint32_t spins = 0;
            while (*vgen == gen) {
                if (++spins > kSpinLimit) { set_err(err, kErrSpin); break; }
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// Build timeline: one globaltimer stamp per grid barrier (thread 0 only).
__device__ __forceinline__ void stamp(Tree &t) {
    unsigned long long ns;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ns));
    const uint32_t i = t.meta[7];
    if (i < (uint32_t)kTimeline) {
        t.tl[i] = ns;
        t.meta[7] = i + 1;
    }
}


// computeInternalMass / computeInternalMass3D: children read in the
// reference's subGrids[x][y]([z]) order, x outermost
template <int D>
__device__ __forceinline__ float4 combine_children(const Tree &t, uint4 inf) {
    constexpr int Q = 1 << D;
    float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kk = 0; kk < Q; kk++) {
        unsigned q;
        if (D == 2) q = ((kk >> 1) & 1) | ((kk & 1) << 1);
        else q = ((kk >> 2) & 1) | (((kk >> 1) & 1) << 1) | ((kk & 1) << 2);
        if (!((inf.y >> q) & 1u)) continue;
        const uint32_t ci = inf.x + __popc(inf.y & ((1u << q) - 1u));
        const float4 cw = __ldcg(&t.walk[ci]);
        const float cm = D == 2 ? cw.z : cw.w;
        gm = fadd(gm, cm);
        c[0] = fadd(c[0], fmul(cw.x, cm));
        c[1] = fadd(c[1], fmul(cw.y, cm));
        if (D == 3) c[2] = fadd(c[2], fmul(cw.z, cm));
    }
    if (gm > 0.0f) {
        c[0] = fdiv(c[0], gm); c[1] = fdiv(c[1], gm);
        if (D == 3) c[2] = fdiv(c[2], gm);
    }
    return make_float4(c[0], c[1], c[2], gm);
}

// Node k's mass is final: tell its parent.  The child that completes a
// parent's set combines the parent (in the reference's child order, so the
// result does not depend on which child came last) and carries on upward.
template <int D>
__device__ __forceinline__ void finish_upward(Tree &t, uint32_t k) {
    // the decrement releases this node's mass to the parent's last child,
    // whose decrement acquires every sibling's (one release sequence per counter).
    // An ancestor's links and cell were written before any of its children
    // existed, so they are read ahead: the next ancestor's while this one's
    // counter and children are on their way, which leaves two round trips
    // (counter, children) per level.
    uint32_t par = __ldcg(&t.aux[k]).z;
    if (par == kEmpty) return;
    uint4 inf = __ldcg(&t.info[par]);
    float size = __ldcg(&t.cell[par]).w;
    uint32_t next = __ldcg(&t.aux[par]).z;
    while (true) {
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> pend(t.pend[par]);
        if (pend.fetch_sub(1u, cuda::memory_order_acq_rel) != 1u) break;
        uint4 inf2 = make_uint4(0u, 0u, 0u, 0u);
        float size2 = 0.0f;
        uint32_t next2 = kEmpty;
        if (next != kEmpty) {
            inf2 = __ldcg(&t.info[next]);
            size2 = __ldcg(&t.cell[next]).w;
            next2 = __ldcg(&t.aux[next]).z;
        }
        put_walk<D>(t, par, combine_children<D>(t, inf), size);
        if (next == kEmpty) break;
        par = next;
        inf = inf2;
        size = size2;
        next = next2;
    }
}


// Write node k's children (slots in increasing q from `first`) and its own
// child links; the pending count is set atomically before any child can finish.
template <int D>
__device__ __forceinline__ void emit_children(Tree &t, uint32_t k, uint32_t first, uint32_t mask,
                                              const uint32_t *b, float4 cell, float half,
                                              uint4 inf, uint4 ax) {
    constexpr int Q = 1 << D;
    uint32_t ci = first;
#pragma unroll
    for (int q = 0; q < Q; q++) {
        if (!((mask >> q) & 1u)) continue;
        t.cell[ci] = child_cell<D>(cell, half, (unsigned)q);
        t.info[ci] = make_uint4(0u, 0u, b[q], b[q + 1]);
        atomicAdd(&t.endcnt[b[q + 1]], 1u);   // the walk layout's end counts
        // same-end ancestors: the child ends where its parent ends
        t.aux[ci] = make_uint4(ax.x + 1u, b[q + 1] == inf.w ? ax.y + 1u : 0u, k, 0u);
        ci++;
    }
    t.info[k] = make_uint4(first, mask, inf.z, inf.w);
    atomicExch(&t.pend[k], (uint32_t)__popc(mask));
    __threadfence();
}

// Chains.  A node whose particles all lie in one quadrant of its cell has one
// child with the same range; nearly coincident particles make long chains of
// such nodes (one per halving of the cell) before the range splits.  The
// quadrant of every particle at a level follows from the range's bounding
// box: the compares p < mid are monotone in p, so all particles agree when the
// box's two corners do (partition_point then returns the range's start or
// end, whatever the order inside).  A chain is therefore written in one go,
// level by level in the reference's float arithmetic, and only its last node
// (a leaf, or a node that splits) is left to the level loops.

// Bounding box of particles [st, en) (coordinates px/py/pz, element j at
// index j - off) by the G lanes of a group; every lane of the group gets it.
// `nan` is set when some coordinate is NaN (no chain is taken then).  All 32
// lanes call this; lanes with act false contribute nothing.
template <int D, int G>
__device__ __forceinline__ void group_bbox(const float *px, const float *py, const float *pz,
                                           uint32_t off, uint32_t st, uint32_t en, bool act,
                                           float *mn, float *mx, bool &nan) {
    const unsigned gl = threadIdx.x & (G - 1u);
    const float *pc[3] = {px, py, pz};
    bool bad = false;
#pragma unroll
    for (int a = 0; a < D; a++) { mn[a] = FLT_MAX; mx[a] = -FLT_MAX; }
    if (act)
        for (uint32_t j = st + gl; j < en; j += G)
#pragma unroll
            for (int a = 0; a < D; a++) {
                const float v = pc[a][j - off];
                bad |= v != v;
                mn[a] = fminf(mn[a], v);
                mx[a] = fmaxf(mx[a], v);
            }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
        for (int a = 0; a < D; a++) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
        bad |= __shfl_xor_sync(0xffffffffu, (int)bad, o) != 0;
    }
    nan = bad;
}

// The quadrant of the cell (corner + half) that holds every particle of a
// box, or -1 when the box straddles a midpoint.
template <int D>
__device__ __forceinline__ int box_quadrant(float4 cell, float half, const float *mn,
                                            const float *mx) {
    const float c[3] = {cell.x, cell.y, cell.z};
    int q = 0;
#pragma unroll
    for (int a = 0; a < D; a++) {
        const float mid = fadd(c[a], half);
        const bool lo = mn[a] < mid, hi = mx[a] < mid;
        if (lo != hi) return -1;
        q |= (lo ? 0 : 1) << a;
    }
    return q;
}

// Chain below a node's single child c (cell `cell`, depth `depth`): how many
// more single-child levels follow before a node that is a leaf or splits;
// `cell` becomes that last node's cell.
template <int D>
__device__ __forceinline__ uint32_t chain_length(const StepParams &p, uint32_t cnt, float4 &cell,
                                                 uint32_t depth, const float *mn,
                                                 const float *mx) {
    uint32_t j = 0;
    while (depth + j + 2u < (uint32_t)kMaxLevels && !is_leaf<D>(p, cnt, cell.w)) {
        const float half = fmul(cell.w, 0.5f);
        const int q = box_quadrant<D>(cell, half, mn, mx);
        if (q < 0) break;
        cell = child_cell<D>(cell, half, (unsigned)q);
        j++;
    }
    return j;
}

// Write the chain: c (slot `first`, already written as a fresh child) and the
// j nodes below it in slots first + 1 .. first + j, each the single child of
// the one before; the last is left fresh (info.y = 0) for the level loops.
// Returns the last node's cell.
template <int D>
__device__ __forceinline__ float4 write_chain(Tree &t, uint32_t first, uint32_t j, uint32_t st,
                                              uint32_t en, float4 cell, uint4 cax,
                                              const float *mn, const float *mx) {
    for (uint32_t i = 0; i < j; i++) {
        const uint32_t k = first + i;
        const float half = fmul(cell.w, 0.5f);
        const unsigned q = (unsigned)box_quadrant<D>(cell, half, mn, mx);
        cell = child_cell<D>(cell, half, q);
        t.cell[k + 1] = cell;
        t.info[k + 1] = make_uint4(0u, 0u, st, en);
        atomicAdd(&t.endcnt[en], 1u);
        t.aux[k + 1] = make_uint4(cax.x + i + 1u, cax.y + i + 1u, k, 0u);
        t.info[k] = make_uint4(k + 1, 1u << q, st, en);
        t.pend[k] = 1u;
    }
    return cell;
}

// Phase 1 work of one node per group of G lanes.
template <int D, int G>
__device__ __forceinline__ void split_level_node(const State &s, const StepParams &p, Tree &t,
                                                 uint32_t k, bool valid, uint32_t level_end,
                                                 uint32_t *lvl_alloc, uint32_t *err,
                                                 uint32_t bid, bool defer = false,
                                                 uint32_t *handoff = nullptr) {
    constexpr int Q = 1 << D;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gl = lane & (G - 1u);
    uint4 inf = make_uint4(0, 0, 0, 0), ax = make_uint4(0, 0, 0, 0);
    float4 cell = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
        // written by other blocks during the previous level: read through L2
        inf = __ldcg(&t.info[k]);
        cell = __ldcg(&t.cell[k]);
        ax = __ldcg(&t.aux[k]);
        valid = inf.y == 0u;   // a chain's inner node is written whole already
    }
    const uint32_t cnt = inf.w - inf.z;
    const bool leaf = valid && is_leaf<D>(p, cnt, cell.w);
    const bool small = valid && !leaf && cnt <= kSmallNode;
    // with handoff (keyed), a node that one block can rebuild is listed for
    // the blocks after the level loop
    const bool block = handoff && valid && !leaf && !small && cnt <= kBlockRootMax;
    const bool split = valid && !leaf && !small && !block;
    const float half = fmul(cell.w, 0.5f);
    const float mid[3] = {fadd(cell.x, half), fadd(cell.y, half), fadd(cell.z, half)};
    uint32_t b[Q + 1];
    cut_group<D, G>(s, split ? inf.z : 0u, split ? inf.w : 0u, mid, b);
    uint32_t mask = 0;
    if (split) {
#pragma unroll
        for (int q = 0; q < Q; q++) mask |= (b[q + 1] > b[q] ? 1u : 0u) << q;
    }
    // a single child: the chain below it (every lane of the group computes
    // it; the box is read for ranges of at most 64 particles per lane)
    const bool single = split && __popc(mask) == 1 && cnt <= 64u * G;
    uint32_t j = 0;
    float mn[3], mx[3];
    const float4 c1 = child_cell<D>(cell, half, single ? (unsigned)(__ffs(mask) - 1) : 0u);
    if (__any_sync(0xffffffffu, single)) {
        bool nan;
        group_bbox<D, G>(s.x, s.y, s.z, 0u, inf.z, inf.w, single, mn, mx, nan);
        float4 cend = c1;
        if (single && !nan) j = chain_length<D>(p, cnt, cend, ax.x + 1u, mn, mx);
    }
    const bool leader = gl == 0;
    if (leader && leaf) {
        put_walk<D>(t, k, leaf_mass<D>(s, inf.z, inf.w), cell.w);
        if (defer) t.kdone[atomicAdd(&t.kmeta[7], 1u)] = k;   // upward after the rebuilds
        else finish_upward<D>(t, k);
        atomicMax(&t.meta[kMetaLevels], ax.x + 1u);
    }
    // queue the small subtrees and the block roots (one atomic per warp each)
    {
        const unsigned qb = __ballot_sync(0xffffffffu, leader && small);
        uint32_t qbase = 0;
        if (lane == 0 && qb) qbase = atomicAdd(&t.meta[kMetaSmall], (uint32_t)__popc(qb));
        qbase = __shfl_sync(0xffffffffu, qbase, 0);
        if (leader && small) t.small[qbase + __popc(qb & ((1u << lane) - 1u))] = make_uint2(k, bid);
        const unsigned bb = __ballot_sync(0xffffffffu, leader && block);
        uint32_t bbase = 0;
        if (lane == 0 && bb) bbase = atomicAdd(&t.kmeta[kKmBlockQ], (uint32_t)__popc(bb));
        bbase = __shfl_sync(0xffffffffu, bbase, 0);
        if (leader && block) handoff[bbase + __popc(bb & ((1u << lane) - 1u))] = k;
    }
    // children of the split nodes (one atomic per warp)
    const uint32_t nch = (leader && split) ? (uint32_t)__popc(mask) + j : 0u;
    uint32_t incl = nch;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += v;
    }
    const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t base = 0;
    if (lane == 0 && tot) base = atomicAdd(lvl_alloc, tot);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (nch) {
        const uint32_t first = level_end + base + incl - nch;
        if ((uint64_t)first + nch > (uint64_t)t.cap) {
            set_err(err, kErrNodeCap);
        } else {
            emit_children<D>(t, k, first, mask, b, cell, half, inf, ax);
            if (j) {
                write_chain<D>(t, first, j, inf.z, inf.w, c1,
                               make_uint4(ax.x + 1u, ax.y + 1u, k, 0u), mn, mx);
                __threadfence();
            }
        }
    }
}

// Keyed build: an exact-rebuild root of up to kBlockRootMax particles is
// rebuilt by one block, level by level with block barriers.  The block's
// level lists hold only its nodes of more than kSmallNode particles (at most
// count / (kSmallNode + 1) per level); a child that is a leaf is summed and
// passed upward at once, a small one goes to the subtree queue (phase 2).
// Children's slots come from *alloc above `base`.  The root's coordinates are
// staged in shared memory (sx[a][j - off]), so the searches' probes are
// shared-memory loads.

// The block's shared state during an exact rebuild: the root's particles
// (coordinates and masses), the current and next level's nodes (slot, range,
// cell, level and same-end count), and the root's deferred leaves and small
// subtrees (bit 31), published with one atomic per kind when the buffer
// fills or the root is done.
constexpr int kBlkOut = 512;
template <int D>
struct BlockSmem {
    float x[D][kBlockRootMax];
    float m[kBlockRootMax];
    uint32_t node[2][kBlkList];
    uint4 inf[2][kBlkList];
    float4 cell[2][kBlkList];
    uint2 ax[2][kBlkList];
    uint32_t out[kBlkOut];
    uint32_t cnt[2], mcur, nout, maxlev, bad;
    // the block's slots: a chunk [anext, aend) of the phase-2 pool (used up
    // to aused), `real` slots used in all, a hole range to zero
    uint32_t anext, aend, aused, real, hole_a, hole_b;
    uint32_t r0;   // the block's current root (list position)
};
constexpr uint32_t kBlkChunk = 512;   // slots a block takes at a time (at least)

// computeLeafMass / computeLeafMass3D over staged particles (the same
// sequential sums as leaf_mass)
template <int D>
__device__ __forceinline__ float4 leaf_mass_smem(const BlockSmem<D> &b, uint32_t st, uint32_t en) {
    float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t i = st; i < en; i++) {
        const float mi = b.m[i];
        gm = fadd(gm, mi);
        c[0] = fadd(c[0], fmul(b.x[0][i], mi));
        c[1] = fadd(c[1], fmul(b.x[1][i], mi));
        if (D == 3) c[2] = fadd(c[2], fmul(b.x[D - 1][i], mi));
    }
    if (gm > 0.0f) {
        c[0] = fdiv(c[0], gm); c[1] = fdiv(c[1], gm);
        if (D == 3) c[2] = fdiv(c[2], gm);
    }
    return make_float4(c[0], c[1], c[2], gm);
}

// Publish the block's buffered leaves and small subtrees (one thread, after a
// block barrier: the fence makes the block's node writes visible before the
// entries that lead other warps to them).
template <int D>
__device__ __forceinline__ void flush_block_out(Tree &t, BlockSmem<D> &sb, uint32_t bid) {
    __threadfence();
    uint32_t nl = 0, ns = 0;
    for (uint32_t q = 0; q < sb.nout; q++) (sb.out[q] >> 31 ? ns : nl)++;
    uint32_t bl = nl ? atomicAdd(&t.kmeta[7], nl) : 0u;
    uint32_t bs = ns ? atomicAdd(&t.meta[kMetaSmall], ns) : 0u;
    for (uint32_t q = 0; q < sb.nout; q++) {
        const uint32_t v = sb.out[q];
        if (v >> 31) t.small[bs++] = make_uint2(v & 0x7FFFFFFFu, bid);
        else t.kdone[bl++] = v;
    }
    sb.nout = 0u;
}

// Level-loop work of one node of a block rebuild (list entry e of the current
// level) per group of G lanes.  Children's slots come from the block's chunk
// (or the pool *alloc above `base`); the searches probe the staged
// coordinates.  Children that are not
// leaves and hold more than kSmallNode particles go to the next level's list;
// leaves and small subtrees to the block's buffer.  No fence: the next level
// reads the lists after a block barrier, and everything else reads these
// nodes after a grid barrier.
template <int D, int G>
__device__ __forceinline__ void rebuild_level_node(const StepParams &p, Tree &t, BlockSmem<D> &sb,
                                                   int cur, uint32_t e, bool valid, uint32_t base,
                                                   uint32_t *alloc, uint32_t *err, uint32_t off) {
    constexpr int Q = 1 << D;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gl = lane & (G - 1u);
    uint32_t k = 0;
    uint4 inf = make_uint4(0, 0, 0, 0);
    uint2 ax = make_uint2(0u, 0u);
    float4 cell = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
        k = sb.node[cur][e];
        inf = sb.inf[cur][e];
        cell = sb.cell[cur][e];
        ax = sb.ax[cur][e];
    }
    const float half = fmul(cell.w, 0.5f);
    const float mid[3] = {fadd(cell.x, half), fadd(cell.y, half), fadd(cell.z, half)};
    uint32_t b[Q + 1];
    cut_group_v<D, G, true>(sb.x[0], sb.x[1], sb.x[D - 1], off, valid ? inf.z : 0u,
                            valid ? inf.w : 0u, mid, b);
    uint32_t mask = 0;
    if (valid) {
#pragma unroll
        for (int q = 0; q < Q; q++) mask |= (b[q + 1] > b[q] ? 1u : 0u) << q;
    }
    // a single child: the chain below it (every lane of the group computes it)
    const bool single = valid && __popc(mask) == 1;
    uint32_t j = 0;
    float mn[3], mx[3];
    const float4 c1 = child_cell<D>(cell, half, single ? (unsigned)(__ffs(mask) - 1) : 0u);
    float4 cend = c1;
    if (__any_sync(0xffffffffu, single)) {
        bool nan;
        group_bbox<D, G>(sb.x[0], sb.x[1], sb.x[D - 1], off, inf.z, inf.w, single, mn, mx, nan);
        if (single && !nan) j = chain_length<D>(p, inf.w - inf.z, cend, ax.x + 1u, mn, mx);
    }
    const bool leader = valid && gl == 0;
    const uint32_t nch = leader ? (uint32_t)__popc(mask) + j : 0u;
    uint32_t incl = nch;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += v;
    }
    const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
    // slots from the block's chunk, or exactly tot from the pool when the
    // chunk cannot hold them (chains)
    uint32_t wbase = 0;
    if (lane == 0 && tot) {
        const uint32_t a = atomicAdd(&sb.anext, tot);
        if (a + tot <= sb.aend && a + tot > a) {
            wbase = a;
            atomicMax(&sb.aused, a + tot);
        } else {
            wbase = base + atomicAdd(alloc, tot);
        }
        atomicAdd(&sb.real, tot);
    }
    wbase = __shfl_sync(0xffffffffu, wbase, 0);
    uint32_t first = wbase + incl - nch;
    first = __shfl_sync(0xffffffffu, first, lane & ~(G - 1u));
    const bool ok = (uint64_t)wbase + tot <= (uint64_t)t.cap;
    if (!ok && lane == 0) {
        set_err(err, kErrNodeCap);
        sb.bad = 1u;
    }
    if (leader && ok) {
        t.info[k] = make_uint4(first, mask, inf.z, inf.w);
        t.pend[k] = (uint32_t)__popc(mask);
        if (j) {   // the chain's first node (write_chain writes and counts the rest)
            t.cell[first] = c1;
            t.aux[first] = make_uint4(ax.x + 1u, ax.y + 1u, k, 0u);
            atomicAdd(&t.endcnt[inf.w], 1u);
        }
        if (j)
            write_chain<D>(t, first, j, inf.z, inf.w, c1, make_uint4(ax.x + 1u, ax.y + 1u, k, 0u),
                           mn, mx);
    }
    // the group's lane q writes child q (a chain's last node for a single child)
    if (valid && ok && gl < (unsigned)Q && ((mask >> gl) & 1u)) {
        const uint32_t lo = b[gl], hi = b[gl + 1], cnt = hi - lo;
        const uint32_t c = first + __popc(mask & ((1u << gl) - 1u)) + j;
        const float4 cc = j ? cend : child_cell<D>(cell, half, gl);
        const uint32_t lvl = ax.x + 1u + j;
        const uint32_t same = hi == inf.w ? ax.y + 1u + j : 0u;
        t.cell[c] = cc;
        t.info[c] = make_uint4(0u, 0u, lo, hi);
        if (!j) atomicAdd(&t.endcnt[hi], 1u);
        t.aux[c] = make_uint4(lvl, same, j ? first + j - 1u : k, 0u);
        if (is_leaf<D>(p, cnt, cc.w)) {
            // its upward pass waits for the end of the rebuilds, so that no
            // level of this loop waits for a chain up the whole tree
            put_walk<D>(t, c, leaf_mass_smem<D>(sb, lo - off, hi - off), cc.w);
            sb.out[atomicAdd(&sb.nout, 1u)] = c;
            atomicMax(&sb.maxlev, lvl + 1u);
        } else if (cnt <= kSmallNode) {
            sb.out[atomicAdd(&sb.nout, 1u)] = c | 0x80000000u;
        } else {
            const uint32_t q = atomicAdd(&sb.cnt[cur ^ 1], 1u);
            sb.node[cur ^ 1][q] = c;
            sb.inf[cur ^ 1][q] = make_uint4(0u, 0u, lo, hi);
            sb.cell[cur ^ 1][q] = cc;
            sb.ax[cur ^ 1][q] = make_uint2(lvl, same);
        }
    }
}

// Phase-2 node allocation per warp: slots come from the shared counter in
// chunks of kChunk; the unused tail of a chunk becomes holes (empty range),
// which the layout skips.  `real` counts the slots actually used.
struct WarpAlloc {
    uint32_t next, end, real;
};

__device__ __forceinline__ void mark_holes(Tree &t, uint32_t a, uint32_t b) {
    const unsigned lane = threadIdx.x & 31u;
    if (b > (uint32_t)t.cap) b = (uint32_t)t.cap;
    for (uint32_t k = a + lane; k < b; k += 32) t.info[k] = make_uint4(0u, 0u, 0u, 0u);
}

// First of cnt consecutive node slots (warp-uniform; all lanes call), or
// kEmpty when the node array is full.
__device__ __forceinline__ uint32_t walloc(Tree &t, WarpAlloc &a, uint32_t cnt, uint32_t base,
                                           uint32_t *err) {
    if (a.next + cnt > a.end) {
        mark_holes(t, a.next, a.end);
        const uint32_t want = cnt > kChunk ? cnt : kChunk;
        uint32_t g = 0;
        if ((threadIdx.x & 31u) == 0) g = atomicAdd(&t.meta[kMetaP2Alloc], want);
        g = __shfl_sync(0xffffffffu, g, 0);
        a.next = base + g;
        a.end = a.next + want;
        if ((uint64_t)a.end > (uint64_t)t.cap) {
            if ((threadIdx.x & 31u) == 0) set_err(err, kErrNodeCap);
            a.end = a.next;
            return kEmpty;
        }
    }
    const uint32_t r = a.next;
    a.next += cnt;
    a.real += cnt;
    return r;
}

// Phase 2: the whole subtree of queued node R (2..kSmallNode particles) by one
// warp.  Lane l holds particle start + l and follows the node containing it.
template <int D>
__device__ void build_small_subtree(const State &s, const StepParams &p, Tree &t, uint32_t R,
                                    uint32_t node_base, WarpAlloc &wa, uint32_t *err) {
    constexpr int Q = 1 << D;
    const unsigned lane = threadIdx.x & 31u;
    const uint4 rinf = __ldcg(&t.info[R]);
    const uint4 rax = __ldcg(&t.aux[R]);
    const uint32_t st = rinf.z, en = rinf.w;
    const uint32_t pidx = st + lane;
    const bool act = pidx < en;
    float pos[3] = {0.f, 0.f, 0.f}, pm = 0.f;
    if (act) {
        pos[0] = s.x[pidx]; pos[1] = s.y[pidx];
        if (D == 3) pos[2] = s.z[pidx];
        pm = s.m[pidx];
    }
    uint32_t nid = R, na = st, nb = en, lev = rax.x, same_end = rax.y;
    float4 cell = __ldcg(&t.cell[R]);
    bool done = !act;
    uint32_t maxlev = 0;
    for (int it = 0; __any_sync(0xffffffffu, !done); it++) {
        if (it > kMaxLevels) { if (lane == 0) set_err(err, kErrDepth); break; }
        const uint32_t cnt = nb - na;
        const bool leader = !done && pidx == na;
        const bool leaf = !done && is_leaf<D>(p, cnt, cell.w);
        // leaves: sequential sums over the leaf's particles, in particle order
        if (__any_sync(0xffffffffu, leaf)) {
            float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll 4
            for (int j = 0; j < 32; j++) {
                const float xj = __shfl_sync(0xffffffffu, pos[0], j);
                const float yj = __shfl_sync(0xffffffffu, pos[1], j);
                const float zj = __shfl_sync(0xffffffffu, pos[2], j);
                const float mj = __shfl_sync(0xffffffffu, pm, j);
                const uint32_t pj = st + (uint32_t)j;
                if (leaf && leader && pj >= na && pj < nb) {
                    gm = fadd(gm, mj);
                    c[0] = fadd(c[0], fmul(xj, mj));
                    c[1] = fadd(c[1], fmul(yj, mj));
                    if (D == 3) c[2] = fadd(c[2], fmul(zj, mj));
                }
            }
            if (leaf && leader) {
                if (gm > 0.0f) {
                    c[0] = fdiv(c[0], gm); c[1] = fdiv(c[1], gm);
                    if (D == 3) c[2] = fdiv(c[2], gm);
                }
                put_walk<D>(t, nid, make_float4(c[0], c[1], c[2], gm), cell.w);
                finish_upward<D>(t, nid);
                maxlev = max(maxlev, lev);
            }
            done = done || leaf;
        }
        // the remaining nodes: predicates of every particle against its node's
        // midpoint, one ballot per axis, then the searches on those bits
        const float half = fmul(cell.w, 0.5f);
        const bool live = !done;
        const unsigned bx = __ballot_sync(0xffffffffu, live && pos[0] < fadd(cell.x, half));
        const unsigned by = __ballot_sync(0xffffffffu, live && pos[1] < fadd(cell.y, half));
        const unsigned bz = D == 3 ? __ballot_sync(0xffffffffu, live && pos[2] < fadd(cell.z, half)) : 0u;
        uint32_t b[Q + 1];
        const uint32_t r0 = na - st, len = nb - na;
        b[0] = na; b[Q] = nb;
        if (D == 2) {
            const uint32_t r2 = bits_partition_point(by, r0, len);
            b[2] = st + r2;
            b[1] = st + bits_partition_point(bx, r0, r2 - r0);
            b[3] = st + bits_partition_point(bx, r2, r0 + len - r2);
        } else {
            const uint32_t r4 = bits_partition_point(bz, r0, len);
            const uint32_t r2 = bits_partition_point(by, r0, r4 - r0);
            const uint32_t r6 = bits_partition_point(by, r4, r0 + len - r4);
            b[4] = st + r4; b[2] = st + r2; b[6] = st + r6;
            b[1] = st + bits_partition_point(bx, r0, r2 - r0);
            b[3] = st + bits_partition_point(bx, r2, r4 - r2);
            b[5] = st + bits_partition_point(bx, r4, r6 - r4);
            b[7] = st + bits_partition_point(bx, r6, r0 + len - r6);
        }
        uint32_t mask = 0;
#pragma unroll
        for (int q = 0; q < Q; q++) mask |= (b[q + 1] > b[q] ? 1u : 0u) << q;
        // allocation: node leaders' child counts, one atomic per warp
        const uint32_t nch = (live && leader) ? (uint32_t)__popc(mask) : 0u;
        uint32_t incl = nch;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += v;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        if (tot == 0) continue;
        const uint32_t base = walloc(t, wa, tot, node_base, err);
        if (base == kEmpty) break;
        const uint32_t myfirst = base + incl - nch;
        if (live && leader) {
            emit_children<D>(t, nid, myfirst, mask, b, cell, half, make_uint4(0, 0, na, nb),
                             make_uint4(lev, same_end, 0, 0));
        }
        // every live lane moves to the child that holds its particle
        const uint32_t first = __shfl_sync(0xffffffffu, myfirst, (int)((na - st) & 31u));
        if (live) {
            unsigned q = 0;
#pragma unroll
            for (int qq = 1; qq < Q; qq++) if (pidx >= b[qq]) q = (unsigned)qq;
            const uint32_t cnb = b[q + 1];
            nid = first + __popc(mask & ((1u << q) - 1u));
            cell = child_cell<D>(cell, half, q);
            same_end = cnb == nb ? same_end + 1u : 0u;
            na = b[q];
            nb = cnb;
            lev++;
        }
    }
    for (int o = 16; o > 0; o >>= 1) maxlev = max(maxlev, __shfl_xor_sync(0xffffffffu, maxlev, o));
    if (lane == 0) atomicMax(&t.meta[kMetaLevels], maxlev + 1u);
}

// Phase 2, fast form: the subtree of queued node R is built in shared memory
// (nodes, cells, masses), then allocated with one atomic and written out.
// Lane l holds particle start + l; sm.p keeps them for the leaf sums.  Returns
// false, with nothing written, when the subtree has more than kSubMax nodes
// (long single-child chains of nearly coincident particles); the caller then
// builds it with build_small_subtree.
constexpr int kSubMax = 64;

struct SubTreeSmem {
    float4 p[32];            // particles {x, y, z, m}
    float4 cell[kSubMax];
    float4 cm[kSubMax];      // {com.x, com.y, com.z, mass}
    uint4 node[kSubMax];     // {a | b << 8 | mask << 16, first child, parent, level | same_end << 16}
    uint32_t lvl[kSubMax + 1];
};

// The upward mass pass from R (finish_upward) is left to the caller, which
// runs those of up to 32 subtrees at once, one per lane.
template <int D>
__device__ bool build_small_subtree_smem(const State &s, const StepParams &p, Tree &t,
                                         uint32_t R, uint32_t node_base, SubTreeSmem &sm,
                                         WarpAlloc &wa, uint32_t *err) {
    constexpr int Q = 1 << D;
    const unsigned lane = threadIdx.x & 31u;
    const uint4 rinf = __ldcg(&t.info[R]);
    const uint4 rax = __ldcg(&t.aux[R]);
    const float4 rcell = __ldcg(&t.cell[R]);
    const uint32_t st = rinf.z, cnt = rinf.w - rinf.z;
    const bool act = lane < cnt;
    float pos[3] = {0.f, 0.f, 0.f};
    if (act) {
        pos[0] = s.x[st + lane]; pos[1] = s.y[st + lane];
        if (D == 3) pos[2] = s.z[st + lane];
        sm.p[lane] = make_float4(pos[0], pos[1], pos[2], s.m[st + lane]);
    }
    if (lane == 0) {
        sm.cell[0] = rcell;
        sm.node[0] = make_uint4(cnt << 8, 0u, kEmpty, rax.x | (rax.y << 16));
        sm.cm[0] = make_float4(0.f, 0.f, 0.f, 0.f);
        sm.lvl[0] = 0;
        sm.lvl[1] = 1;
    }
    __syncwarp();
    uint32_t loc = 0, na = 0, nb = cnt, lev = rax.x, se = rax.y, count = 1;
    int nlv = 1;   // local levels made so far
    float4 cell = rcell;
    bool done = !act;
    uint32_t maxlev = 0;
    for (int it = 0; __any_sync(0xffffffffu, !done); it++) {
        if (it > kMaxLevels) { if (lane == 0) set_err(err, kErrDepth); return true; }
        const bool leader = !done && lane == na;
        const bool leaf = !done && is_leaf<D>(p, nb - na, cell.w);
        if (leaf && leader) {
            // computeLeafMass: sequential sums in particle order
            float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
            for (uint32_t j = na; j < nb; j++) {
                const float4 q = sm.p[j];
                gm = fadd(gm, q.w);
                c[0] = fadd(c[0], fmul(q.x, q.w));
                c[1] = fadd(c[1], fmul(q.y, q.w));
                if (D == 3) c[2] = fadd(c[2], fmul(q.z, q.w));
            }
            if (gm > 0.0f) {
                c[0] = fdiv(c[0], gm); c[1] = fdiv(c[1], gm);
                if (D == 3) c[2] = fdiv(c[2], gm);
            }
            sm.cm[loc] = make_float4(c[0], c[1], c[2], gm);
            maxlev = max(maxlev, lev);
        }
        done = done || leaf;
        const float half = fmul(cell.w, 0.5f);
        const bool live = !done;
        const unsigned bx = __ballot_sync(0xffffffffu, live && pos[0] < fadd(cell.x, half));
        const unsigned by = __ballot_sync(0xffffffffu, live && pos[1] < fadd(cell.y, half));
        const unsigned bz = D == 3 ? __ballot_sync(0xffffffffu, live && pos[2] < fadd(cell.z, half)) : 0u;
        uint32_t b[Q + 1];
        const uint32_t len = nb - na;
        b[0] = na; b[Q] = nb;
        if (D == 2) {
            b[2] = bits_partition_point(by, na, len);
            b[1] = bits_partition_point(bx, na, b[2] - na);
            b[3] = bits_partition_point(bx, b[2], nb - b[2]);
        } else {
            b[4] = bits_partition_point(bz, na, len);
            b[2] = bits_partition_point(by, na, b[4] - na);
            b[6] = bits_partition_point(by, b[4], nb - b[4]);
            b[1] = bits_partition_point(bx, na, b[2] - na);
            b[3] = bits_partition_point(bx, b[2], b[4] - b[2]);
            b[5] = bits_partition_point(bx, b[4], b[6] - b[4]);
            b[7] = bits_partition_point(bx, b[6], nb - b[6]);
        }
        uint32_t mask = 0;
#pragma unroll
        for (int q = 0; q < Q; q++) mask |= (b[q + 1] > b[q] ? 1u : 0u) << q;
        const uint32_t nch = (live && leader) ? (uint32_t)__popc(mask) : 0u;
        uint32_t incl = nch;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += v;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        if (tot == 0) break;
        if (count + tot > (uint32_t)kSubMax || nlv + 1 > kSubMax) return false;
        const uint32_t myfirst = count + incl - nch;
        if (live && leader) {
            uint4 nd = sm.node[loc];
            nd.x |= mask << 16;
            nd.y = myfirst;
            sm.node[loc] = nd;
            uint32_t ci = myfirst;
#pragma unroll
            for (int q = 0; q < Q; q++) {
                if (!((mask >> q) & 1u)) continue;
                sm.cell[ci] = child_cell<D>(cell, half, (unsigned)q);
                const uint32_t cse = b[q + 1] == nb ? se + 1u : 0u;
                sm.node[ci] = make_uint4(b[q] | (b[q + 1] << 8), 0u, loc, (lev + 1u) | (cse << 16));
                sm.cm[ci] = make_float4(0.f, 0.f, 0.f, 0.f);
                ci++;
            }
        }
        count += tot;
        nlv++;
        if (lane == 0) sm.lvl[nlv] = count;
        __syncwarp();
        const uint32_t first = __shfl_sync(0xffffffffu, myfirst, (int)(na & 31u));
        if (live) {
            unsigned q = 0;
#pragma unroll
            for (int qq = 1; qq < Q; qq++) if (lane >= b[qq]) q = (unsigned)qq;
            const uint32_t cnb = b[q + 1];
            loc = first + __popc(mask & ((1u << q) - 1u));
            cell = child_cell<D>(cell, half, q);
            se = cnb == nb ? se + 1u : 0u;
            na = b[q];
            nb = cnb;
            lev++;
        }
    }
    __syncwarp();
    // computeInternalMass, deepest local level first, children in x-major order
    for (int L = nlv - 1; L >= 0; --L) {
        const uint32_t j = sm.lvl[L] + lane;
        if (j < sm.lvl[L + 1]) {
            const uint4 nd = sm.node[j];
            const uint32_t mask = nd.x >> 16;
            if (mask) {
                float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int kk = 0; kk < Q; kk++) {
                    unsigned q;
                    if (D == 2) q = ((kk >> 1) & 1) | ((kk & 1) << 1);
                    else q = ((kk >> 2) & 1) | (((kk >> 1) & 1) << 1) | ((kk & 1) << 2);
                    if (!((mask >> q) & 1u)) continue;
                    const float4 cw = sm.cm[nd.y + __popc(mask & ((1u << q) - 1u))];
                    gm = fadd(gm, cw.w);
                    c[0] = fadd(c[0], fmul(cw.x, cw.w));
                    c[1] = fadd(c[1], fmul(cw.y, cw.w));
                    if (D == 3) c[2] = fadd(c[2], fmul(cw.z, cw.w));
                }
                if (gm > 0.0f) {
                    c[0] = fdiv(c[0], gm); c[1] = fdiv(c[1], gm);
                    if (D == 3) c[2] = fdiv(c[2], gm);
                }
                sm.cm[j] = make_float4(c[0], c[1], c[2], gm);
            }
        }
        __syncwarp();
    }
    // allocate and write out: local node 0 is R itself
    const uint32_t base = walloc(t, wa, count - 1u, node_base, err);
    if (base == kEmpty) return true;
    for (uint32_t j = lane; j < count; j += 32) {
        const uint4 nd = sm.node[j];
        const uint32_t a = nd.x & 0xFFu, bb = (nd.x >> 8) & 0xFFu, mask = nd.x >> 16;
        const uint32_t gid = j == 0 ? R : base + j - 1u;
        const uint32_t gfirst = mask ? base + nd.y - 1u : 0u;
        t.info[gid] = make_uint4(gfirst, mask, st + a, st + bb);
        const float4 cl = sm.cell[j];
        if (j > 0) {
            t.cell[gid] = cl;
            const uint32_t gpar = nd.z == 0 ? R : base + nd.z - 1u;
            t.aux[gid] = make_uint4(nd.w & 0xFFFFu, nd.w >> 16, gpar, 0u);
            atomicAdd(&t.endcnt[st + bb], 1u);   // the walk layout's end counts
        }
        put_walk<D>(t, gid, sm.cm[j], cl.w);
    }
    for (int o = 16; o > 0; o >>= 1) maxlev = max(maxlev, __shfl_xor_sync(0xffffffffu, maxlev, o));
    __syncwarp();
    if (lane == 0) atomicMax(&t.meta[kMetaLevels], maxlev + 1u);
    return true;
}

// The walk-layout entries of node slot k (and of its particles when it is a
// leaf), from its fields and the end counts C(start) = ez, C(end) = ew.
template <int D>
__device__ __forceinline__ void scatter_entry(const State &s, const Segs &g, Tree &t, uint32_t k,
                                              uint4 inf, uint4 ax, float4 w, float size2,
                                              uint32_t ez, uint32_t ew, uint32_t total,
                                              uint32_t *err, bool packed, int extras) {
    const uint32_t me = ez + ax.x + inf.z;
    const uint32_t skip = ew + ax.x - ax.y + inf.w;
    if (me >= total || skip > total) {   // cannot happen for a consistent tree
        set_err(err, kErrDepth);
        return;
    }
    if (extras & kLayoutEntry) t.aux[k].w = me;   // the node's entry
    if (extras & kLayoutRange) t.nrange[k] = make_uint2(me, skip);   // its layout range
    if (k < (uint32_t)g.S) {   // a segment's root: where its particles' walks start and end
        g.root_begin[k] = me;
        g.root_end[k] = skip;
    }
    const float nm = D == 2 ? w.z : w.w;
    const bool massless = nm <= 0.0f;
    if (massless) {
        // gridMass <= 0: the reference skips the whole subtree.  As a source
        // it is accepted by every test (size^2 = -2; particles have -1),
        // carries no mass (the walk makes no interaction with a massless
        // node) and leads to its successor.
        t.src[me] = D == 2 ? make_float4(w.x, w.y, 0.0f,
                                         packed ? __uint_as_float(pack_entry_word(kPackMassless, skip))
                                                : -2.0f)
                           : make_float4(w.x, w.y, w.z, 0.0f);
        if (D == 3) ((uint2 *)t.link)[me] = make_uint2(skip, __float_as_uint(-2.0f));
        else if (!packed) ((uint32_t *)t.link)[me] = skip;
    } else {
        t.src[me] = D == 2 && packed ? make_float4(w.x, w.y, w.z, __uint_as_float(pack_entry_word(ax.x, skip)))
                                     : w;
        if (D == 3) ((uint2 *)t.link)[me] = make_uint2(skip, __float_as_uint(size2));
        else if (!packed) ((uint32_t *)t.link)[me] = skip;
    }
    if (inf.y) return;
    // a leaf: its particles follow it, four at a time (loads before stores)
    for (uint32_t j0 = inf.z; j0 < inf.w; j0 += 4u) {
        float px[4], py[4], pz[4], pm[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t j = j0 + q;
            const bool in = j < inf.w && !massless;
            px[q] = in ? s.x[j] : 0.0f;
            py[q] = in ? s.y[j] : 0.0f;
            pz[q] = in && D == 3 ? s.z[j] : 0.0f;
            pm[q] = in ? s.m[j] : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t j = j0 + q;
            if (j >= inf.w) break;
            const uint32_t e = me + 1 + (j - inf.z);
            t.slot_of[j] = e;
            if (massless) continue;   // never reached by the walk
            if (D == 2) {
                t.src[e] = make_float4(px[q], py[q], pm[q],
                                       packed ? __uint_as_float(pack_entry_word(kPackParticle, e + 1))
                                              : -1.0f);
                if (!packed) ((uint32_t *)t.link)[e] = e + 1;
            } else {
                t.src[e] = make_float4(px[q], py[q], pz[q], pm[q]);
                ((uint2 *)t.link)[e] = make_uint2(e + 1, __float_as_uint(-1.0f));
            }
        }
    }
}

template <int D>
__global__ void __launch_bounds__(kBuildThreads, D == 2 ? 3 : 2)
k_build(State s, StepParams p, Segs g, Tree t, uint32_t *err, int keyed) {
    dep_wait();
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nthreads = gridDim.x * blockDim.x;
    const uint32_t gwarp = gtid >> 5, nwarps = nthreads >> 5;
    const uint32_t n = (uint32_t)p.n;
    uint32_t *bar_count = t.meta + kMetaBarCount, *bar_gen = t.meta + kMetaBarGen;
    // the block rebuilds' staged coordinates, then phase 2's per-warp subtrees
    constexpr size_t kSharedBytes = sizeof(SubTreeSmem) * (kBuildThreads / 32) >
                                            sizeof(BlockSmem<D>)
                                        ? sizeof(SubTreeSmem) * (kBuildThreads / 32)
                                        : sizeof(BlockSmem<D>);
    __shared__ __align__(16) unsigned char s_shared[kSharedBytes];

    // Keyed: the key passes (ge_kbuild.cu) wrote key_nodes nodes in slots
    // [0, key_nodes), the segment roots first; pend holds each node's child
    // bits (bit 31: an exact-rebuild root), aux.w marks exact-rebuild roots
    // (1) and nodes whose mass is already final (2: every leaf, and the nodes
    // inside one emit tile).  Phase 0 turns the bits into child masks and, for
    // the other nodes, counts the children still pending; nodes with none are
    // listed to be combined after the exact rebuilds (phases 1, 2).
    uint32_t lb = 0, le = (uint32_t)g.S, front = (uint32_t)g.S;
    uint32_t key_nodes = 0;   // keyed: slots [0, key_nodes) hold the key passes' nodes
    const uint32_t *list = nullptr;
    // counters of this build (read only after the first grid barrier)
    if (gtid == 0) {
        t.meta[kMetaNodes] = 0u; t.meta[kMetaLevels] = 0u;
        t.meta[kMetaSmall] = 0u; t.meta[kMetaP2Alloc] = 0u; t.meta[kMetaTimeline] = 0u;
        t.meta[kMetaReal] = 0u; t.meta[kMetaSlots] = 0u; t.meta[kMetaP2Task] = 0u;
        t.meta[kMetaBigRoot] = 0u; t.meta[kMetaDone] = 0u; t.kmeta[kKmProdDone] = 0u;
        const uint32_t id = t.meta[kMetaBuildId] + 1u;   // read after the first grid barrier
        t.meta[kMetaBuildId] = id ? id : 1u;
        stamp(t);
    }
    for (uint32_t i = gtid; i < (uint32_t)kMaxLevels + 2u; i += nthreads) t.lvl_alloc[i] = 0u;
    // keyed: the emit pass wrote the key nodes' end counts (every entry)
    if (!keyed)
        for (uint32_t i = gtid; i <= n; i += nthreads) t.endcnt[i] = 0u;
    if (keyed) {
        key_nodes = *(volatile uint32_t *)&t.kmeta[3];
        if ((int64_t)key_nodes > t.cap) return;   // the emit pass set kErrNodeCap
        for (uint32_t k = gtid; k < key_nodes; k += nthreads) {
            const uint32_t pv = __ldcg(&t.pend[k]);
            const uint32_t mask = pv & 0xFFu;
            const bool exact = pv >> 31;
            const bool done = __ldcg(&t.aux[k]).w & 2u;
            reinterpret_cast<uint32_t *>(t.info)[4 * (size_t)k + 1] = exact ? 0u : mask;
            uint32_t pending = 0;
            if (!exact && !done) {
                const uint32_t first = __ldcg(&t.info[k]).x;
                const uint32_t nch = (uint32_t)__popc(mask);
                for (uint32_t c = 0; c < nch; c++) pending += (__ldcg(&t.aux[first + c]).w & 2u) ? 0u : 1u;
            }
            t.pend[k] = pending;
            const bool ready = !exact && !done && pending == 0u;
            // combined after the exact rebuilds: list them (slot_of is free
            // until the layout)
            const unsigned lbits = __ballot_sync(__activemask(), ready);
            if (ready) {
                const int leader = __ffs(lbits) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(&t.kmeta[5], (uint32_t)__popc(lbits));
                base = __shfl_sync(lbits, base, leader);
                t.slot_of[base + __popc(lbits & ((1u << lane) - 1u))] = k;
            }
        }
        if (gtid == 0) atomicMax(&t.meta[kMetaLevels], *(volatile uint32_t *)&t.kmeta[4]);
        grid_barrier(bar_count, bar_gen, err);
        if (gtid == 0) stamp(t);
        list = t.kroots;
        le = *(volatile uint32_t *)&t.kmeta[1];
        front = key_nodes;
    } else {
        // one root per segment (seeded by the box kernel): nodes 0 .. S-1
        for (uint32_t r = gtid; r < (uint32_t)g.S; r += nthreads)
            t.aux[r] = make_uint4(0u, 0u, kEmpty, 0u);
    }

    // ---- phase 1: nodes of more than kSmallNode particles, level by level ----
    // the first level is the segment roots (or, keyed, the exact-rebuild roots,
    // by list: those of at most kBlockRootMax particles go to the block list,
    // the small ones to the subtree queue); children go to slots from `front` on
    int L = 0;
    if (gtid == 0) t.level[0] = lb;
    if (!keyed) {   // the roots' links above
        grid_barrier(bar_count, bar_gen, err);
        if (gtid == 0) stamp(t);
        // the roots' ends (every other node's end is counted where it is made;
        // the key passes count the key nodes')
        for (uint32_t r = gtid; r < (uint32_t)g.S; r += nthreads) {
            const uint32_t e = __ldcg(&t.info[r]).w;
            if (e) atomicAdd(&t.endcnt[e], 1u);
        }
    }
    const uint32_t nroots0 = le;   // keyed: the key passes' exact-rebuild roots
    const uint32_t bid = *(volatile uint32_t *)&t.meta[kMetaBuildId];   // this build's id
    while (true) {
        if (le - lb <= nwarps) {
            for (uint32_t k = lb + gwarp; k < le; k += nwarps) {
                const uint32_t node = list ? __ldcg(&list[k]) : k;
                split_level_node<D, 32>(s, p, t, node, true, front, &t.lvl_alloc[L], err, bid, keyed,
                                        keyed ? t.kroots + nroots0 : nullptr);
            }
        } else {
            for (uint32_t kb = lb + gwarp * 4; kb < le; kb += nwarps * 4) {
                const uint32_t k = kb + (lane >> 3);
                const uint32_t node = list && k < le ? __ldcg(&list[k]) : k;
                const bool valid = k < le;
                split_level_node<D, 8>(s, p, t, node, valid, front, &t.lvl_alloc[L], err, bid, keyed,
                                       keyed ? t.kroots + nroots0 : nullptr);
            }
        }
        grid_barrier(bar_count, bar_gen, err);
        if (gtid == 0) stamp(t);
        const uint32_t cnt = *(volatile uint32_t *)&t.lvl_alloc[L];
        const uint32_t e = *(volatile uint32_t *)err;
        if (cnt == 0 || (e & (kErrNodeCap | kErrSpin))) break;
        if (L + 1 >= kMaxLevels) {
            if (gtid == 0) set_err(err, kErrDepth);
            break;
        }
        lb = front;
        le = front + cnt;
        front = le;
        list = nullptr;
        L++;
        if (gtid == 0) t.level[L] = lb;
    }
    le = front;   // phase-1 slots end here
    if (gtid == 0) {
        t.level[L + 1] = le;
        if (!keyed) atomicMax(&t.meta[kMetaLevels], (uint32_t)(L + 1));
    }
    if ((*(volatile uint32_t *)err) & (kErrNodeCap | kErrSpin | kErrDepth)) return;

    if (keyed) {
        // exact-rebuild roots of up to kBlockRootMax particles: a block each
        // (shares its memory with phase 2's subtrees)
        BlockSmem<D> &sb = *reinterpret_cast<BlockSmem<D> *>(s_shared);
        // the nodes of 33 .. kBlockRootMax particles that phase 1 handed over
        // (its first level is the key passes' exact-rebuild roots)
        const uint32_t nblk = *(volatile uint32_t *)&t.kmeta[kKmBlockQ];
        // slots come from phase 2's pool (above the phase-1 slots)
        const uint32_t xbase = le;
        uint32_t *xalloc = &t.meta[kMetaP2Alloc];
        const unsigned w = threadIdx.x >> 5, W = kBuildThreads / 32;
        if (threadIdx.x == 0) {
            sb.nout = 0u; sb.maxlev = 0u; sb.bad = 0u;
            sb.anext = sb.aend = sb.aused = 0u; sb.real = 0u; sb.hole_a = sb.hole_b = 0u;
        }
        // roots taken one at a time from a counter (their costs differ)
        while (true) {
            __syncthreads();
            if (threadIdx.x == 0) sb.r0 = atomicAdd(&t.kmeta[kKmBlockTake], 1u);
            __syncthreads();
            const uint32_t r = sb.r0;
            if (r >= nblk) break;
            const uint32_t root = __ldcg(&t.kroots[nroots0 + r]);
            const uint4 ri = __ldcg(&t.info[root]);
            const uint32_t cnt = ri.w - ri.z;
            if (threadIdx.x == 0) {
                const uint4 rx = __ldcg(&t.aux[root]);
                sb.node[0][0] = root;
                sb.inf[0][0] = ri;
                sb.cell[0][0] = __ldcg(&t.cell[root]);
                sb.ax[0][0] = make_uint2(rx.x, rx.y);
                sb.cnt[0] = 1u;
                if ((*(volatile uint32_t *)err) & kErrNodeCap) sb.bad = 1u;
            }
            for (uint32_t j = threadIdx.x; j < cnt; j += blockDim.x) {
                sb.x[0][j] = s.x[ri.z + j];
                sb.x[1][j] = s.y[ri.z + j];
                if (D == 3) sb.x[D - 1][j] = s.z[ri.z + j];
                sb.m[j] = s.m[ri.z + j];
            }
            int cur = 0;
            for (int it = 0; it < kMaxLevels; it++) {
                if (threadIdx.x == 0) {   // one decision for the whole block
                    sb.cnt[cur ^ 1] = 0u;
                    sb.hole_a = sb.hole_b = 0u;
                    sb.mcur = sb.bad ? 0u : sb.cnt[cur];
                    if (sb.nout + sb.mcur * (1u << D) > (uint32_t)kBlkOut) flush_block_out<D>(t, sb, bid);
                    // a fresh chunk when this level's children may not fit (the
                    // old chunk's unused tail becomes holes)
                    const uint32_t need = sb.mcur * (1u << D);
                    if (sb.mcur && sb.aend - sb.aused < need) {
                        sb.hole_a = sb.aused;
                        sb.hole_b = sb.aend;
                        const uint32_t want = need > kBlkChunk / 2 ? 2u * need : kBlkChunk;
                        const uint32_t g = xbase + atomicAdd(xalloc, want);
                        if ((uint64_t)g + want > (uint64_t)t.cap) {
                            set_err(err, kErrNodeCap);
                            sb.bad = 1u;
                            sb.mcur = 0u;
                            sb.anext = sb.aend = sb.aused = 0u;
                        } else {
                            sb.anext = sb.aused = g;
                            sb.aend = g + want;
                        }
                    }
                }
                __syncthreads();
                const uint32_t m = sb.mcur;
                for (uint32_t q = sb.hole_a + threadIdx.x; q < sb.hole_b; q += blockDim.x)
                    t.info[q] = make_uint4(0u, 0u, 0u, 0u);
                if (m == 0u) break;
                if (m <= W) {
                    for (uint32_t j = w; j < m; j += W)
                        rebuild_level_node<D, 32>(p, t, sb, cur, j, true, xbase, xalloc, err, ri.z);
                } else {
                    for (uint32_t jb = w * 4; jb < m; jb += W * 4) {
                        const uint32_t j = jb + (lane >> 3);
                        rebuild_level_node<D, 8>(p, t, sb, cur, j, j < m, xbase, xalloc, err, ri.z);
                    }
                }
                __syncthreads();
                cur ^= 1;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            flush_block_out<D>(t, sb, bid);
            if (sb.maxlev) atomicMax(&t.meta[kMetaLevels], sb.maxlev);
            if (sb.real) atomicAdd(&t.meta[kMetaReal], sb.real);
            sb.hole_a = sb.aused;
            sb.hole_b = sb.aend;
        }
        __syncthreads();
        for (uint32_t q = sb.hole_a + threadIdx.x; q < sb.hole_b; q += blockDim.x)
            t.info[q] = make_uint4(0u, 0u, 0u, 0u);
    }

    // this block queues nothing more (its entries and nodes are visible first)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&t.kmeta[kKmProdDone], 1u);
    }

    // ---- phase 2: queued small subtrees, one warp each, no barriers --------
    // A warp claims queue positions from a counter and takes each one's entry
    // once it is written (an entry of this build carries its id), while other
    // blocks may still be rebuilding and queueing; it stops at a position
    // past the final count, known once every block has finished queueing.
    // poll(task): its entry (1), nothing yet (0), or the queue is final and
    // ends before it, or the build failed (2).  Lane 0.
    constexpr uint32_t kNotYet = 0xFFFFFFFEu;
    auto poll = [&](uint32_t task) -> uint32_t {
        if (task < t.small_cap) {
            const uint2 e = __ldcv(&t.small[task]);
            if (e.y == bid) {
                __threadfence();   // the subtree's nodes were written before its entry
                return e.x;
            }
        }
        if (*(volatile uint32_t *)&t.kmeta[kKmProdDone] == gridDim.x) {
            __threadfence();
            if (task >= *(volatile uint32_t *)&t.meta[kMetaSmall]) return kEmpty;
        }
        if ((*(volatile uint32_t *)err) & (kErrNodeCap | kErrSpin | kErrDepth)) return kEmpty;
        return kNotYet;
    };
    // the listed key nodes whose children are all final (known since phase
    // 0): combined and passed upward 32 at a time, by warps waiting for
    // queue entries or done with them
    const uint32_t nready = keyed ? *(volatile uint32_t *)&t.kmeta[5] : 0u;
    uint32_t *ready_ctr = &t.kmeta[kKeyMetaWords - 2];   // zeroed with the key passes' words
    auto climb_ready = [&]() -> bool {   // false when none are left
        uint32_t b = 0;
        if (lane == 0) b = atomicAdd(ready_ctr, 32u);
        b = __shfl_sync(0xffffffffu, b, 0);
        if (b >= nready) return false;
        const uint32_t idx = b + lane;
        if (idx < nready) {
            const uint32_t cur = __ldcg(&t.slot_of[idx]);
            put_walk<D>(t, cur, combine_children<D>(t, __ldcg(&t.info[cur])),
                        __ldcg(&t.cell[cur]).w);
            finish_upward<D>(t, cur);
        }
        __syncwarp();
        return true;
    };
    {
        SubTreeSmem &sm = reinterpret_cast<SubTreeSmem *>(s_shared)[threadIdx.x >> 5];
        WarpAlloc wa{0u, 0u, 0u};
        // tasks are taken from a counter (their costs differ); lane j holds the
        // j-th finished subtree root whose upward pass is still to run, and the
        // warp runs 32 of them at once, so their atomics' round trips overlap
        uint32_t held = kEmpty, nheld = 0;
        uint32_t task = 0;
        if (lane == 0) task = atomicAdd(&t.meta[kMetaP2Task], 1u);
        bool ready_left = nready > 0;
        uint32_t ns = 32, spins = 0;
        while (true) {
            uint32_t R = 0;
            if (lane == 0) R = poll(task);
            R = __shfl_sync(0xffffffffu, R, 0);
            if (R == kEmpty) break;
            if (R == kNotYet) {
                if (ready_left && (ready_left = climb_ready())) continue;
                if (++spins > kSpinLimit) {
                    if (lane == 0) set_err(err, kErrSpin);
                    break;
                }
                if (lane == 0) __nanosleep(ns);
                if (ns < 256) ns *= 2;
                continue;
            }
            ns = 32;
            if (lane == 0) task = atomicAdd(&t.meta[kMetaP2Task], 1u);
            if (build_small_subtree_smem<D>(s, p, t, R, le, sm, wa, err)) {
                if (lane == nheld) held = R;
                if (++nheld == 32u) {
                    __syncwarp();
                    finish_upward<D>(t, held);
                    held = kEmpty;
                    nheld = 0;
                }
            } else {
                build_small_subtree<D>(s, p, t, R, le, wa, err);   // passes its own leaves upward
            }
            __syncwarp();
        }
        __syncwarp();
        if (held != kEmpty) finish_upward<D>(t, held);
        mark_holes(t, wa.next, wa.end);
        if (lane == 0 && wa.real) atomicAdd(&t.meta[kMetaReal], wa.real);
        while (ready_left && (ready_left = climb_ready())) {
        }
    }
    if (keyed) {
        // the exact rebuilds' deferred leaves (already summed), upward from
        // each, 32 at a time (the list is final once the queue is)
        const uint32_t ndone = *(volatile uint32_t *)&t.kmeta[7];
        uint32_t *take = &t.kmeta[kKeyMetaWords - 1];   // zeroed with the key passes' words
        while (true) {
            uint32_t b = 0;
            if (lane == 0) b = atomicAdd(take, 32u);
            b = __shfl_sync(0xffffffffu, b, 0);
            if (b >= ndone) break;
            if (b + lane < ndone) finish_upward<D>(t, __ldcg(&t.kdone[b + lane]));
            __syncwarp();
        }
    }
    // root sizes whose square is not a normal float rule out packed entries
    for (uint32_t sg = gtid; sg < (uint32_t)g.S; sg += nthreads)
        if (!(g.box[sg].w < 1e19f)) atomicOr(&t.meta[kMetaBigRoot], 1u);
    grid_barrier(bar_count, bar_gen, err);
    if (gtid == 0) stamp(t);
    // slots in use (phase-2 holes included) and real nodes (the walk's extent)
    uint32_t slots = le + *(volatile uint32_t *)&t.meta[kMetaP2Alloc];
    if (slots > (uint32_t)t.cap) slots = (uint32_t)t.cap;
    const uint32_t nodes = le + *(volatile uint32_t *)&t.meta[kMetaReal];
    if (gtid == 0) {
        t.meta[kMetaNodes] = nodes;
        t.meta[kMetaSlots] = slots;
    }
    if ((*(volatile uint32_t *)err) & (kErrNodeCap | kErrSpin | kErrDepth)) return;

    // ---- phase 3: depth-first walk layout ------------------------------------
    // endcnt holds the histogram of range ends: the key nodes' from the emit
    // pass (or zeroed above), every other node's added where it was made
    // inclusive scan of endcnt[0..n] in place, by block chunks; each chunk's
    // offset (the earlier chunks' total) is added where the scatter reads it:
    //   C(e) = endcnt[e] + s_boff[e / chunk]
    __shared__ uint32_t s_boff[kMaxBuildBlocks];
    const uint32_t chunk = (n + 1 + gridDim.x - 1) / gridDim.x;
    {
        constexpr int W = kBuildThreads / 32;
        __shared__ uint32_t s_w[W];
        const uint32_t total = n + 1;
        const uint32_t c0 = min(blockIdx.x * chunk, total);
        const uint32_t c1 = min(c0 + chunk, total);
        uint32_t carry = 0;
        for (uint32_t base = c0; base < c1; base += blockDim.x) {
            const uint32_t i = base + threadIdx.x;
            const uint32_t v = i < c1 ? __ldcg(&t.endcnt[i]) : 0u;
            uint32_t incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (unsigned)o) incl += u;
            }
            if (lane == 31) s_w[threadIdx.x >> 5] = incl;
            __syncthreads();
            uint32_t wpre = 0, btot = 0;
            for (int w = 0; w < W; w++) {
                if (w < (int)(threadIdx.x >> 5)) wpre += s_w[w];
                btot += s_w[w];
            }
            if (i < c1) t.endcnt[i] = carry + wpre + incl;
            carry += btot;
            __syncthreads();
        }
        if (threadIdx.x == 0) t.blocksum[blockIdx.x] = carry;
        grid_barrier(bar_count, bar_gen, err);
        if (gtid == 0) stamp(t);
        // exclusive prefix of the chunk totals, in every block: thread j sums
        // chunks [4j, 4j + 4), then a block scan of those sums
        static_assert(kMaxBuildBlocks == 4 * kBuildThreads, "four chunks per thread");
        uint32_t v4[4], s4 = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t b2 = 4u * threadIdx.x + q;
            v4[q] = b2 < gridDim.x ? __ldcg(&t.blocksum[b2]) : 0u;
            s4 += v4[q];
        }
        uint32_t incl = s4;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += u;
        }
        if (lane == 31) s_w[threadIdx.x >> 5] = incl;
        __syncthreads();
        uint32_t run = incl - s4;
        for (int w = 0; w < (int)(threadIdx.x >> 5); w++) run += s_w[w];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            s_boff[4u * threadIdx.x + q] = run;
            run += v4[q];
        }
        __syncthreads();
    }
    if (gtid == 0) stamp(t);
    // scatter nodes and the particles of leaves into the walk layout, in which
    // each leaf's particles follow the leaf: with C(e) the number of nodes
    // whose range ends at or before e,
    //   entry of node k      = C(start) + level + start
    //   subtree successor    = C(end) + level - same_end + end
    //   entry of particle j  = entry of its leaf + 1 + (j - start)
    const uint32_t total = nodes + n;
    // 2D, not rewritten by the moment pass: packed entries when every level
    // and successor fits the word and every size^2 is a normal float (a node
    // of size <= min_size is a leaf, so sizes stay >= min_size / 2, or the
    // tree is one leaf; root sizes below 1e19), where quartering L times is
    // the exponent minus 2L
    const bool packed = D == 2 && !p.mixed && p.min_size >= 1e-18f &&
                        *(volatile uint32_t *)&t.meta[kMetaBigRoot] == 0u &&
                        *(volatile uint32_t *)&t.meta[kMetaLevels] <= kPackMaxLevel + 1u &&
                        total < (1u << kPackSkipBits);
    if (gtid == 0) t.meta[kMetaWalkPacked] = packed ? 1u : 0u;
    // two slots per round: both slots' loads are issued before either's stores
    for (uint32_t k0 = gtid; k0 < slots; k0 += 2u * nthreads) {
        const uint32_t kk[2] = {k0, k0 + nthreads};
        uint4 inf[2], ax[2];
        float4 wv[2];
        float s2[2];
        uint32_t ez[2], ew[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const bool in = kk[u] < slots;
            inf[u] = in ? __ldcg(&t.info[kk[u]]) : make_uint4(0u, 0u, 0u, 0u);
            ax[u] = in ? __ldcg(&t.aux[kk[u]]) : make_uint4(0u, 0u, 0u, 0u);
            wv[u] = in ? __ldcg(&t.walk[kk[u]]) : make_float4(0.f, 0.f, 0.f, 0.f);
            s2[u] = in && D == 3 ? __ldcg(&t.size2[kk[u]]) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {   // holes have an empty range ending at 0
            ez[u] = inf[u].w ? __ldcg(&t.endcnt[inf[u].z]) + s_boff[inf[u].z / chunk] : 0u;
            ew[u] = inf[u].w ? __ldcg(&t.endcnt[inf[u].w]) + s_boff[inf[u].w / chunk] : 0u;
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            if (inf[u].w == 0u) continue;
            scatter_entry<D>(s, g, t, kk[u], inf[u], ax[u], wv[u], s2[u], ez[u], ew[u], total, err,
                             packed, p.layout_extras);
        }
    }
    // the last block to finish stamps the end of the build
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&t.meta[kMetaDone], 1u) == gridDim.x - 1u) stamp(t);
    }
}

static int g_build_blocks[2] = {0, 0};

int build_grid_blocks(int dims, int num_sms);

// Node slots the build may leave unused: each warp's last phase-2 chunk and
// each block's last block-rebuild chunk.
int64_t build_node_slack(int dims, int num_sms) {
    const int64_t blk = 2 * (int64_t)kBlkList * (dims == 2 ? 4 : 8);
    return (int64_t)build_grid_blocks(dims, num_sms) *
           ((kBuildThreads / 32) * kChunk + (blk > kBlkChunk ? blk : kBlkChunk));
}

int build_grid_blocks(int dims, int num_sms) {
    const int di = dims == 2 ? 0 : 1;
    if (g_build_blocks[di] == 0) {
        if (num_sms < 1) return 0;
        int per_sm = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, dims == 2 ? (const void *)k_build<2> : (const void *)k_build<3>,
            kBuildThreads, 0);
        if (e != cudaSuccess || per_sm < 1) return 0;
        // at most three blocks per SM: every block joins every grid barrier, so
        // more blocks lengthen the barriers; more warps hide the latency of
        // the subtree phase
        int b = (per_sm < 3 ? per_sm : 3) * num_sms;
        if (b > kMaxBuildBlocks) b = kMaxBuildBlocks - kMaxBuildBlocks % num_sms;
        g_build_blocks[di] = b;
    }
    return g_build_blocks[di];
}

cudaError_t launch_build(int dims, const State &s, const StepParams &p, const Segs &g, Tree &t,
                         uint32_t *err, int num_sms, cudaStream_t st, bool keyed) {
    // the kernel zeroes its own counters, level allocation and end histogram
    const int blocks = build_grid_blocks(dims, num_sms);
    if (blocks < 1) return cudaErrorLaunchOutOfResources;
    State sc = s;
    StepParams pc = p;
    Segs gc = g;
    Tree tc = t;
    uint32_t *ec = err;
    int kc = keyed ? 1 : 0;
    void *args[] = {&sc, &pc, &gc, &tc, &ec, &kc};
    const void *kern = dims == 2 ? (const void *)k_build<2> : (const void *)k_build<3>;
    // cooperative, and launched while the previous kernel drains (dep_wait);
    // a runtime that refuses the pair gets the plain cooperative launch
    static bool pair_ok = true;
    if (pair_ok) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(blocks);
        cfg.blockDim = dim3(kBuildThreads);
        cfg.stream = st;
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 2;
        const cudaError_t e = cudaLaunchKernelExC(&cfg, kern, args);
        if (e == cudaSuccess) return e;
        (void)cudaGetLastError();   // a launch-configuration error is not sticky
        pair_ok = false;
    }
    return cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(kBuildThreads), args, 0, st);
}

}  // namespace ge
