// ge_moments.cu -- FP64 node moments for the mixed-precision mode.
//
// GE_PREC_MIXED keeps the reference's tree (same nodes, same particle ranges)
// but replaces what each node tells the walk:
//   * mass and centre of mass summed in FP64 from the particles, the centre
//     stored as a double-float pair (FP32 value + FP32 remainder), so the
//     walk's offset d = com - x is formed to about one FP32 rounding of d
//     itself instead of one rounding of the (much larger) coordinates;
//   * the second moments about the centre of mass, for a quadrupole term
//     with the softened kernel's own derivatives;
//   * an opening radius b = size / theta + |com - cell centre| (the opening
//     test b^2 < |d|^2 + eps2 also accounts for how far the centre of mass
//     sits from the cell centre), stored where the other modes keep size^2.
// The reference has no counterpart: its nodes carry only the FP32 mass and
// centre of mass (quadtree.h:53-92, computeLeafMass / computeInternalMass).
//
// Every product-sum is an explicit fused multiply-add (or an explicit
// unfused product), so the FP64 moments do not depend on the compiler's
// contraction choices.
//
// One launch, no waits: every leaf sums its particles, then the last child
// of each node to finish (a per-node counter of children still pending)
// combines the children's moments with the parallel-axis rule and carries on
// upward, so a node is written once, after all of its children.
#include <cuda/atomic>

#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kMomThreads = 256;
constexpr int kMetaSlotsWord = 9;   // node slots of the last build (tree meta word)

__global__ void k_pend_init(Tree t) {
    dep_wait();
    const uint32_t slots = __ldcg(&t.meta[kMetaSlotsWord]);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < slots; k += stride) {
        const uint4 inf = __ldcg(&t.info[k]);
        t.pend[k] = (inf.w > inf.z) ? (uint32_t)__popc(inf.y) : 0u;
    }
}

// A node's moments into its walk entry.
template <int D>
__device__ void write_entry(const Tree &t, uint32_t k, const double *r, double inv_theta) {
    const double M = r[0];
    if (!(M > 0.0)) {
        // massless: the walk layout already holds an accepted entry without
        // mass; the group walk skips a node of mass 0
        if (t.gw) t.gw[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float4 cell = __ldcg(&t.cell[k]);
    const double half = 0.5 * (double)cell.w;
    const double cc[3] = {(double)cell.x + half, (double)cell.y + half, (double)cell.z + half};
    double del2 = 0.0;
    float hi[3] = {0.f, 0.f, 0.f}, lo[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < D; a++) {
        const double c = r[1 + a];
        hi[a] = (float)c;
        lo[a] = (float)(c - (double)hi[a]);
        const double dc = c - cc[a];
        del2 = __fma_rn(dc, dc, del2);
    }
    const double b = __fma_rn((double)cell.w, inv_theta, sqrt(del2));
    const float b2 = (float)__dmul_rn(b, b);
    if (t.gw) {   // per node slot, for the group walk
        if (D == 2) {
            t.gw[k] = make_float4(hi[0], hi[1], (float)M, b2);
            t.gq0[k] = make_float4(lo[0], lo[1], (float)r[3], (float)r[4]);
            t.gq2[k] = make_float2((float)r[5], 0.0f);
        } else {
            t.gw[k] = make_float4(hi[0], hi[1], hi[2], (float)M);
            t.gq0[k] = make_float4(lo[0], lo[1], lo[2], (float)r[4]);
            t.gq1[k] = make_float4((float)r[5], (float)r[6], (float)r[7], (float)r[8]);
            t.gq2[k] = make_float2((float)r[9], b2);
        }
    }
    if (!t.mq0) return;
    const uint32_t e = __ldcg(&t.aux[k]).w;
    if (D == 2) {
        t.src[e] = make_float4(hi[0], hi[1], (float)M, b2);
        t.mq0[e] = make_float4(lo[0], lo[1], (float)r[3], (float)r[4]);
        t.mq2[e] = (float)r[5];
    } else {
        t.src[e] = make_float4(hi[0], hi[1], hi[2], (float)M);
        ((uint2 *)t.link)[e].y = __float_as_uint(b2);
        t.mq0[e] = make_float4(lo[0], lo[1], lo[2], (float)r[4]);
        t.mq1[e] = make_float4((float)r[5], (float)r[6], (float)r[7], (float)r[8]);
        t.mq2[e] = (float)r[9];
    }
}

// second-moment index of the pair (a, b): 2D xx xy yy; 3D xx yy zz xy xz yz
template <int D>
__device__ __forceinline__ int mom_index(int a, int b) {
    if (D == 2) return 1 + D + a + b;
    if (a == b) return 1 + D + a;
    return 1 + D + 2 + a + b;   // xy -> 3, xz -> 4, yz -> 5 (after the diagonal)
}

template <int D>
__global__ void __launch_bounds__(kMomThreads)
k_moments(State s, Tree t, double inv_theta, uint32_t *err) {
    dep_wait();
    constexpr int R = MomWords<D>::value;
    const uint32_t slots = __ldcg(&t.meta[kMetaSlotsWord]);
    const uint32_t stride = gridDim.x * blockDim.x;
    const float *pos[3] = {s.x, s.y, s.z};
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < slots; k += stride) {
        const uint4 inf = __ldcg(&t.info[k]);
        if (inf.w <= inf.z || inf.y != 0u) continue;   // holes and internal nodes
        double r[R];
#pragma unroll
        for (int q = 0; q < R; q++) r[q] = 0.0;
        for (uint32_t j = inf.z; j < inf.w; j++) {
            const double mj = s.m[j];
            r[0] += mj;
#pragma unroll
            for (int a = 0; a < D; a++) r[1 + a] = __fma_rn(mj, (double)pos[a][j], r[1 + a]);
        }
        if (r[0] > 0.0) {
#pragma unroll
            for (int a = 0; a < D; a++) r[1 + a] /= r[0];
            for (uint32_t j = inf.z; j < inf.w; j++) {
                const double mj = s.m[j];
                double d[3];
#pragma unroll
                for (int a = 0; a < D; a++) d[a] = (double)pos[a][j] - r[1 + a];
#pragma unroll
                for (int a = 0; a < D; a++)
#pragma unroll
                    for (int b = a; b < D; b++) {
                        const int w = mom_index<D>(a, b);
                        r[w] = __fma_rn(__dmul_rn(mj, d[a]), d[b], r[w]);
                    }
            }
        }
        double *rec = t.mom + (size_t)k * R;
#pragma unroll
        for (int q = 0; q < R; q++) rec[q] = r[q];
        write_entry<D>(t, k, r, inv_theta);
        // upward: the last child of each node to finish combines its children
        uint32_t node = k;
        for (int lev = 0; lev < kMaxLevels; lev++) {
            const uint32_t par = __ldcg(&t.aux[node]).z;
            if (par == kEmpty) break;
            cuda::atomic_ref<uint32_t, cuda::thread_scope_device> pc(t.pend[par]);
            if (pc.fetch_sub(1u, cuda::memory_order_acq_rel) != 1u) break;
            const uint4 pinf = __ldcg(&t.info[par]);
            const int nc = __popc(pinf.y);
            double q[R];
#pragma unroll
            for (int w = 0; w < R; w++) q[w] = 0.0;
            for (int c = 0; c < nc; c++) {
                const double *cr = t.mom + (size_t)(pinf.x + (uint32_t)c) * R;
                const double mc = __ldcg(&cr[0]);
                q[0] += mc;
#pragma unroll
                for (int a = 0; a < D; a++) q[1 + a] = __fma_rn(mc, __ldcg(&cr[1 + a]), q[1 + a]);
            }
            if (q[0] > 0.0) {
#pragma unroll
                for (int a = 0; a < D; a++) q[1 + a] /= q[0];
                for (int c = 0; c < nc; c++) {
                    const double *cr = t.mom + (size_t)(pinf.x + (uint32_t)c) * R;
                    const double mc = __ldcg(&cr[0]);
                    if (!(mc > 0.0)) continue;
                    double d[3];
#pragma unroll
                    for (int a = 0; a < D; a++) d[a] = __ldcg(&cr[1 + a]) - q[1 + a];
#pragma unroll
                    for (int a = 0; a < D; a++)
#pragma unroll
                        for (int b = a; b < D; b++) {
                            const int w = mom_index<D>(a, b);
                            q[w] += __fma_rn(__dmul_rn(mc, d[a]), d[b], __ldcg(&cr[w]));
                        }
                }
            }
            double *prec = t.mom + (size_t)par * R;
#pragma unroll
            for (int w = 0; w < R; w++) prec[w] = q[w];
            write_entry<D>(t, par, q, inv_theta);
            node = par;
            if (lev + 1 == kMaxLevels) set_err(err, kErrDepth);
        }
    }
}

cudaError_t launch_moments(int dims, const State &s, const StepParams &p, Tree &t, uint32_t *err,
                           int num_sms, cudaStream_t st) {
    const int blocks = num_sms * 8;
    cudaError_t e = launch_dep(k_pend_init, blocks, kMomThreads, st, t);
    if (e != cudaSuccess) return e;
    const double inv_theta = 1.0 / (double)p.theta;   // theta = 0: every node is opened
    if (dims == 2) return launch_dep(k_moments<2>, blocks, kMomThreads, st, s, t, inv_theta, err);
    return launch_dep(k_moments<3>, blocks, kMomThreads, st, s, t, inv_theta, err);
}

}  // namespace ge
