// ge_walk.cu -- the theta-criterion tree walk with softened force.
//
// Reference: Physics::calculateForceFromGrid (GalaxyEngine/src/Physics/physics.cpp:91-205)
// and Physics3D::calculateForceFromGrid3D (physics3D.cpp:131-253).  Per
// particle i the reference scans the pre-order node array: a node of zero mass
// is skipped; with d = com - x_i and r2 = |d|^2 + eps2 the node is accepted as
// a monopole when size^2 < theta^2 * r2; otherwise a leaf is summed directly
// over its particles j != i; otherwise the walk descends.  acc_i = F_i / m_i.
//
// Warp-cooperative form: the 32 particles of a warp are consecutive in Morton
// order and share one depth-first traversal stack in shared memory whose
// entries carry the mask of lanes that still have to examine the node.  Every
// lane applies the reference's own opening test (computed with the reference's
// rounding, no contraction), so each particle's interaction set is exactly the
// reference's; children are pushed in reverse slot order, so each lane also
// meets its nodes in the reference's pre-order and accumulates in that order.
//   GE_PREC_EXACT : every interaction with the reference's rounding
//                   (1/sqrtf, three products, no FMA): bit-identical results.
//   GE_PREC_FAST  : rsqrt and FMA for the force terms, G applied once.
// integrateEnd (physics.cpp:1114-1125) is fused into the epilogue.
#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kWalkThreads = 128;
constexpr int kWalkWarps = kWalkThreads / 32;

template <int D>
struct WalkStack { static constexpr int size = D == 2 ? 512 : 1024; };

__device__ __forceinline__ float wrap_d(float d, float dom, float hd) {
    // d -= domain * ((d > half) - (d < -half))   (physics.cpp:118-121)
    const int k = (int)(d > hd) - (int)(d < -hd);
    return fsub(d, fmul(dom, (float)k));
}

template <int D, int MODE, bool COUNT>
__global__ void __launch_bounds__(kWalkThreads)
k_walk(State s, StepParams p, Tree t, int integrate_end, unsigned long long *inter,
       uint32_t *err) {
    constexpr int SS = WalkStack<D>::size;
    __shared__ uint2 stk_all[kWalkWarps][SS];
    const int warp = threadIdx.x >> 5;
    const unsigned lane = threadIdx.x & 31u;
    uint2 *stk = stk_all[warp];
    const int n = p.n;
    const float eps2 = p.eps2, th2 = p.theta2, G = p.G;
    unsigned long long my_count = 0;

    for (int gw = blockIdx.x * kWalkWarps + warp; gw * 32 < n; gw += gridDim.x * kWalkWarps) {
        const int i = gw * 32 + (int)lane;
        const bool active = i < n;
        float pi[3] = {0.f, 0.f, 0.f};
        float mi = 1.0f;
        if (active) {
            pi[0] = s.x[i]; pi[1] = s.y[i];
            if (D == 3) pi[2] = s.z[i];
            mi = s.m[i];
        }
        const float gm_i = MODE == GE_PREC_EXACT ? fmul(G, mi) : 0.0f;   // Gf * pmass
        float f[3] = {0.f, 0.f, 0.f};
        uint32_t cnt = 0;
        int sp = 1;
        const unsigned amask = __ballot_sync(0xffffffffu, active);
        if (lane == 0) stk[0] = make_uint2(0u, amask);
        __syncwarp();
        while (sp > 0) {
            --sp;
            const uint2 e = stk[sp];
            __syncwarp();
            const uint32_t node = e.x;
            const bool mine = (e.y >> lane) & 1u;
            const float4 A = __ldg(&t.walk[node]);
            const float nm = D == 2 ? A.z : A.w;
            if (nm <= 0.0f) continue;   // gridMass <= 0: skip the subtree
            const uint4 B = __ldg(&t.info[node]);
            const float s2 = D == 2 ? A.w : __ldg(&t.size2[node]);
            float d[3];
            d[0] = fsub(A.x, pi[0]);
            d[1] = fsub(A.y, pi[1]);
            if (D == 3) d[2] = fsub(A.z, pi[2]);
            if (p.periodic) {
#pragma unroll
                for (int a = 0; a < D; a++) d[a] = wrap_d(d[a], p.domain[a], p.half_domain[a]);
            }
            float r2 = fadd(fmul(d[0], d[0]), fmul(d[1], d[1]));
            if (D == 3) r2 = fadd(r2, fmul(d[2], d[2]));
            r2 = fadd(r2, eps2);
            const bool accept = mine && (s2 < fmul(th2, r2));
            if (accept) {
                if (MODE == GE_PREC_EXACT) {
                    const float inv = fdiv(1.0f, __fsqrt_rn(r2));
                    const float inv3 = fmul(fmul(inv, inv), inv);
                    const float fm = fmul(fmul(gm_i, nm), inv3);
#pragma unroll
                    for (int a = 0; a < D; a++) f[a] = fadd(f[a], fmul(d[a], fm));
                } else {
                    const float inv = rsqrtf(r2);
                    const float fm = nm * (inv * inv * inv);
#pragma unroll
                    for (int a = 0; a < D; a++) f[a] = fmaf(d[a], fm, f[a]);
                }
                if (COUNT) cnt++;
            }
            const unsigned open = __ballot_sync(0xffffffffu, mine && !accept);
            if (!open) continue;
            if (B.y == 0u) {
                // leaf: direct sum over its particles, j != i
                const bool me = (open >> lane) & 1u;
                for (uint32_t j = B.z; j < B.w; j++) {
                    float pj[3];
                    pj[0] = __ldg(&s.x[j]); pj[1] = __ldg(&s.y[j]);
                    if (D == 3) pj[2] = __ldg(&s.z[j]);
                    const float mj = __ldg(&s.m[j]);
                    if (me && (int)j != i) {
                        float q[3];
#pragma unroll
                        for (int a = 0; a < D; a++) q[a] = fsub(pj[a], pi[a]);
                        if (p.periodic) {
#pragma unroll
                            for (int a = 0; a < D; a++)
                                q[a] = wrap_d(q[a], p.domain[a], p.half_domain[a]);
                        }
                        float rr = fadd(fmul(q[0], q[0]), fmul(q[1], q[1]));
                        if (D == 3) rr = fadd(rr, fmul(q[2], q[2]));
                        rr = fadd(rr, eps2);
                        if (MODE == GE_PREC_EXACT) {
                            const float inv = fdiv(1.0f, __fsqrt_rn(rr));
                            const float inv3 = fmul(fmul(inv, inv), inv);
                            const float fm = fmul(fmul(gm_i, mj), inv3);
#pragma unroll
                            for (int a = 0; a < D; a++) f[a] = fadd(f[a], fmul(q[a], fm));
                        } else {
                            const float inv = rsqrtf(rr);
                            const float fm = mj * (inv * inv * inv);
#pragma unroll
                            for (int a = 0; a < D; a++) f[a] = fmaf(q[a], fm, f[a]);
                        }
                        if (COUNT) cnt++;
                    }
                }
            } else {
                // descend: push the children in reverse slot order (first child on top)
                const int nc = __popc(B.y);
                if (sp + nc > SS) {
                    if (lane == 0) set_err(err, kErrStack);
                    break;
                }
                if ((int)lane < nc) stk[sp + nc - 1 - (int)lane] = make_uint2(B.x + lane, open);
                sp += nc;
                __syncwarp();
            }
        }
        if (active) {
            float acc[3];
#pragma unroll
            for (int a = 0; a < D; a++)
                acc[a] = MODE == GE_PREC_EXACT ? fdiv(f[a], mi) : G * f[a];
            s.ax[i] = acc[0]; s.ay[i] = acc[1];
            if (D == 3) s.az[i] = acc[2];
            if (integrate_end && !(s.pinned && s.pinned[i])) {
                s.vx[i] = fadd(s.vx[i], fmul(acc[0], p.half_dt));
                s.vy[i] = fadd(s.vy[i], fmul(acc[1], p.half_dt));
                if (D == 3) s.vz[i] = fadd(s.vz[i], fmul(acc[2], p.half_dt));
            }
        }
        if (COUNT) my_count += cnt;
        __syncwarp();
    }
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) my_count += __shfl_xor_sync(0xffffffffu, my_count, o);
        if (lane == 0 && my_count) atomicAdd(inter, my_count);
    }
}

template <int D, int MODE, bool COUNT>
static cudaError_t walk_one(const State &s, const StepParams &p, const Tree &t, int ie,
                            unsigned long long *inter, uint32_t *err, cudaStream_t st) {
    int warps = (p.n + 31) / 32;
    int blocks = (warps + kWalkWarps - 1) / kWalkWarps;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    k_walk<D, MODE, COUNT><<<blocks, kWalkThreads, 0, st>>>(s, p, t, ie, inter, err);
    return cudaGetLastError();
}

cudaError_t launch_walk(int dims, int precision, const State &s, const StepParams &p,
                        const Tree &t, bool integrate_end, unsigned long long *inter_count,
                        uint32_t *err, cudaStream_t st) {
    const int ie = integrate_end ? 1 : 0;
    const bool cnt = inter_count != nullptr;
    const bool exact = precision == GE_PREC_EXACT;
#define GE_WALK(Dv, Mv)                                                                   \
    return cnt ? walk_one<Dv, Mv, true>(s, p, t, ie, inter_count, err, st)                \
               : walk_one<Dv, Mv, false>(s, p, t, ie, nullptr, err, st)
    if (dims == 2) {
        if (exact) GE_WALK(2, GE_PREC_EXACT);
        GE_WALK(2, GE_PREC_FAST);
    } else {
        if (exact) GE_WALK(3, GE_PREC_EXACT);
        GE_WALK(3, GE_PREC_FAST);
    }
#undef GE_WALK
}

}  // namespace ge
