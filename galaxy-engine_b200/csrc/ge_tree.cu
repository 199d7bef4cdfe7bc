// ge_tree.cu -- quadtree / octree construction with mass and centre of mass.
//
// Reference: Node::Node, Node::subGridMaker, computeLeafMass, computeInternalMass
// (GalaxyEngine/src/Physics/quadtree.cpp:5-88, include/Physics/quadtree.h:31-111)
// and the octree analogues (quadtree.cpp:109-271, quadtree.h:134-179).
//
// The reference builds recursively: a node over the Morton-sorted range
// [start, end) is a leaf when ((count <= 4 && size <= 2) || count == 1 ||
// size <= 1e-6); otherwise the range is cut by std::partition_point on
// float midpoint compares (y then x; z then y then x in 3D) and one child is
// made per non-empty quadrant.  This kernel makes the same nodes level by
// level: one warp per node evaluates the three (seven) partition points with
// the exact probe sequence of std::partition_point (GNU halving search),
// resolving log2(G) halving steps per round with G-1 lanes probing the G-1
// nodes of the next levels of the search's decision tree.  Because the probes
// are the reference's own, the cut points agree with the reference even where
// the float compares disagree with the Morton order and the range is not
// partitioned.  Children of a level are allocated by one atomic per block
// per batch of nodes; levels are separated by a bounded grid barrier inside
// one cooperative launch, and masses / centres of mass are then combined
// bottom-up, level by level, reading children in the reference's x-major
// subGrids order so every float sum rounds exactly as the reference's does.
#include <cfloat>

#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kBuildThreads = 256;
constexpr int kBuildWarps = kBuildThreads / 32;

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
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// std::partition_point(v + first, v + first + len, [mid](float a){ return a < mid; })
// emulated by G consecutive lanes.  Lane j (1 <= j < G) of the group stands
// for node j of the search's decision tree (heap order; child 2j when the
// probe is false, 2j+1 when true); one round evaluates all of them and walks
// log2(G) steps.  All 32 lanes must call this together; groups may differ in
// their arguments.
template <int G>
__device__ __forceinline__ uint32_t group_partition_point(const float *__restrict__ v,
                                                          uint32_t first, uint32_t len,
                                                          float mid) {
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
            if (l > 0) pred = __ldg(v + f + (l >> 1)) < mid;
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

template <int D>
__device__ __forceinline__ const float *axis_ptr(const State &s, int a) {
    return a == 0 ? s.x : (a == 1 ? s.y : s.z);
}

template <int D>
__global__ void __launch_bounds__(kBuildThreads)
k_build(State s, StepParams p, Tree t, uint32_t *err) {
    constexpr int Q = 1 << D;
    __shared__ uint32_t s_cnt[kBuildWarps], s_off[kBuildWarps], s_base;
    const int warp = threadIdx.x >> 5;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t cap = (uint32_t)t.cap;
    uint32_t *bar_count = t.meta + 2, *bar_gen = t.meta + 3;

    uint32_t lb = 0, le = 1;
    int L = 0;
    if (gtid == 0) t.level[0] = 0;
    while (true) {
        for (uint32_t kb = lb + blockIdx.x * kBuildWarps; kb < le;
             kb += gridDim.x * kBuildWarps) {
            const uint32_t k = kb + warp;
            const bool valid = k < le;
            uint32_t mask = 0, bnd[Q + 1];
            float4 cell = make_float4(0.f, 0.f, 0.f, 0.f);
            uint32_t st = 0, en = 0;
            bool leaf = true;
            if (valid) {
                // written by other blocks in the previous level: read through L2
                const uint4 inf = __ldcg(&t.info[k]);
                cell = __ldcg(&t.cell[k]);
                st = inf.z; en = inf.w;
                const uint32_t cnt = en - st;
                const float size = cell.w;
                leaf = ((cnt <= p.leaf_cap && size <= p.size_gate) || cnt == 1u) ||
                       size <= p.min_size;
            }
            const float half = fmul(cell.w, 0.5f);
            if (!leaf) {
                // children cut points, exactly as Node::subGridMaker[3D]
                const float midx = fadd(cell.x, half), midy = fadd(cell.y, half);
                bnd[0] = st; bnd[Q] = en;
                if (D == 2) {
                    bnd[2] = group_partition_point<32>(s.y, st, en - st, midy);
                    const uint32_t f = lane < 16 ? st : bnd[2];
                    const uint32_t l = lane < 16 ? bnd[2] - st : en - bnd[2];
                    const uint32_t r = group_partition_point<16>(s.x, f, l, midx);
                    bnd[1] = __shfl_sync(0xffffffffu, r, 0);
                    bnd[3] = __shfl_sync(0xffffffffu, r, 16);
                } else {
                    const float midz = fadd(cell.z, half);
                    bnd[4] = group_partition_point<32>(s.z, st, en - st, midz);
                    uint32_t f = lane < 16 ? st : bnd[4];
                    uint32_t l = lane < 16 ? bnd[4] - st : en - bnd[4];
                    uint32_t r = group_partition_point<16>(s.y, f, l, midy);
                    bnd[2] = __shfl_sync(0xffffffffu, r, 0);
                    bnd[6] = __shfl_sync(0xffffffffu, r, 16);
                    const unsigned g = lane >> 3;
                    f = bnd[2 * g];
                    l = bnd[2 * g + 2] - bnd[2 * g];
                    r = group_partition_point<8>(s.x, f, l, midx);
                    bnd[1] = __shfl_sync(0xffffffffu, r, 0);
                    bnd[3] = __shfl_sync(0xffffffffu, r, 8);
                    bnd[5] = __shfl_sync(0xffffffffu, r, 16);
                    bnd[7] = __shfl_sync(0xffffffffu, r, 24);
                }
#pragma unroll
                for (int q = 0; q < Q; q++) mask |= (bnd[q + 1] > bnd[q] ? 1u : 0u) << q;
            } else if (valid && lane == 0) {
                // computeLeafMass: sequential sums in the reference's order
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
                const float s2 = fmul(cell.w, cell.w);
                if (D == 2) t.walk[k] = make_float4(c[0], c[1], gm, s2);
                else { t.walk[k] = make_float4(c[0], c[1], c[2], gm); t.size2[k] = s2; }
            }
            const uint32_t nch = (uint32_t)__popc(mask);
            if (lane == 0) s_cnt[warp] = valid ? nch : 0u;
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t tot = 0;
                for (int w = 0; w < kBuildWarps; w++) { s_off[w] = tot; tot += s_cnt[w]; }
                s_base = tot ? atomicAdd(&t.lvl_alloc[L], tot) : 0u;
            }
            __syncthreads();
            if (valid && nch) {
                const uint32_t first = le + s_base + s_off[warp];
                if ((uint64_t)first + nch > cap) {
                    if (lane == 0) set_err(err, kErrNodeCap);
                } else {
                    if (lane < (unsigned)Q && ((mask >> lane) & 1u)) {
                        const unsigned q = lane;
                        const uint32_t ci = first + __popc(mask & ((1u << q) - 1u));
                        float4 cc;
                        cc.x = fadd(cell.x, (q & 1u) ? half : 0.0f);
                        cc.y = fadd(cell.y, (q & 2u) ? half : 0.0f);
                        cc.z = D == 3 ? fadd(cell.z, (q & 4u) ? half : 0.0f) : 0.0f;
                        cc.w = half;
                        t.cell[ci] = cc;
                        t.info[ci] = make_uint4(0u, 0u, bnd[q], bnd[q + 1]);
                    }
                    if (lane == 0) t.info[k] = make_uint4(first, mask, st, en);
                }
            }
            __syncthreads();
        }
        grid_barrier(bar_count, bar_gen, err);
        const uint32_t cnt = *(volatile uint32_t *)&t.lvl_alloc[L];
        const uint32_t e = *(volatile uint32_t *)err;
        if (cnt == 0 || (e & (kErrNodeCap | kErrSpin))) break;
        if (L + 1 >= kMaxLevels) {
            if (gtid == 0) set_err(err, kErrDepth);
            break;
        }
        lb = le;
        le = le + cnt;
        L++;
        if (gtid == 0) t.level[L] = lb;
    }
    const int nlev = L + 1;
    if (gtid == 0) {
        t.level[nlev] = le;
        t.meta[0] = le;
        t.meta[1] = (uint32_t)nlev;
    }
    // bottom-up: computeInternalMass[3D] with children read in subGrids[x][y]([z])
    // order, x outermost
    for (int lev = nlev - 2; lev >= 0; --lev) {
        const uint32_t a = __ldcg(&t.level[lev]), b = __ldcg(&t.level[lev + 1]);
        for (uint32_t k = a + gtid; k < b; k += gridDim.x * blockDim.x) {
            const uint4 inf = __ldcg(&t.info[k]);
            const uint32_t mask = inf.y;
            if (!mask) continue;
            float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int kk = 0; kk < Q; kk++) {
                unsigned q;
                if (D == 2) q = ((kk >> 1) & 1) | ((kk & 1) << 1);
                else q = ((kk >> 2) & 1) | (((kk >> 1) & 1) << 1) | ((kk & 1) << 2);
                if (!((mask >> q) & 1u)) continue;
                const uint32_t ci = inf.x + __popc(mask & ((1u << q) - 1u));
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
            const float size = __ldcg(&t.cell[k]).w;
            const float s2 = fmul(size, size);
            if (D == 2) t.walk[k] = make_float4(c[0], c[1], gm, s2);
            else { t.walk[k] = make_float4(c[0], c[1], c[2], gm); t.size2[k] = s2; }
        }
        grid_barrier(bar_count, bar_gen, err);
    }
}

static int g_build_blocks[2] = {0, 0};

cudaError_t launch_build(int dims, const State &s, const StepParams &p, Tree &t, uint32_t *err,
                         int num_sms, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(t.lvl_alloc, 0, sizeof(uint32_t) * (kMaxLevels + 2), st);
    if (e != cudaSuccess) return e;
    const int di = dims == 2 ? 0 : 1;
    if (g_build_blocks[di] == 0) {
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, dims == 2 ? (const void *)k_build<2> : (const void *)k_build<3>,
            kBuildThreads, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorLaunchOutOfResources;
        g_build_blocks[di] = per_sm * num_sms;
    }
    int blocks = g_build_blocks[di];
    // every block takes part in each grid barrier: more blocks than the widest
    // level needs only lengthen the barriers
    int want = (p.n + 31) / 32;
    if (want > num_sms * 4) want = num_sms * 4;
    if (want < 1) want = 1;
    if (blocks > want) blocks = want;
    State sc = s;
    StepParams pc = p;
    Tree tc = t;
    uint32_t *ec = err;
    void *args[] = {&sc, &pc, &tc, &ec};
    return cudaLaunchCooperativeKernel(dims == 2 ? (const void *)k_build<2> : (const void *)k_build<3>,
                                       dim3(blocks), dim3(kBuildThreads), args, 0, st);
}

}  // namespace ge
