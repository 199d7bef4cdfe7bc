// ge_direct.cu -- the O(N^2) direct sum the application runs instead of the
// tree walk for small simulations.
//
// Reference: Physics::naiveGravity (GalaxyEngine/src/Physics/physics.cpp:392-434)
// and Physics3D::naiveGravity3D (physics3D.cpp:416-469), selected by the frame
// for fewer than 5000 particles or with myVar.naive (globalLogic.cpp:1321-1346,
// 3D :1677-1702).  Per particle i, over every j of the simulation in order
// (the self term included: d = 0 adds exactly zero):
//   d = x_j - x_i (wrapped when periodic), r2 = |d|^2 + softening (un-squared),
//   inv = 1 / sqrt(r2), acc_i += d * ((G * m_j) * (inv * inv * inv)).
// The result is the acceleration itself (no division by m_i) and the pass
// exchanges no heat.  integrateEnd (physics.cpp:1114-1125) is fused.
//   GE_PREC_EXACT : the scalar form's rounding (correctly rounded sqrt and
//                   division, no contraction): bit-identical to it.
//   GE_PREC_FAST  : approximate reciprocal square root and FMA accumulation.
// A block takes kDirectTile particles of one simulation and streams that
// simulation's particles through shared memory in order, so every thread
// accumulates in the reference's j order.
#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

namespace {

__device__ __forceinline__ float wrap_dd(float d, float dom, float hd) {
    // d -= domain * ((d > half) - (d < -half))   (physics.cpp:416-419)
    const int k = (int)(d > hd) - (int)(d < -hd);
    return fsub(d, fmul(dom, (float)k));
}

__device__ __forceinline__ float rsqrt_fast(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <int D, int MODE, bool PER>
__global__ void __launch_bounds__(kDirectTile)
k_direct(State s, StepParams p, Segs g, const uint2 *__restrict__ tiles, int integrate_end) {
    __shared__ float4 sj[kDirectTile];   // {x, y, z, G * m}
    const uint2 tile = tiles[blockIdx.x];
    const uint32_t lo = seg_lo(g, tile.x), hi = seg_hi(g, tile.x, (uint32_t)p.n);
    const uint32_t i = tile.y + threadIdx.x;
    const bool own = i < hi;
    float pi[3] = {0.f, 0.f, 0.f};
    if (own) {
        pi[0] = s.x[i]; pi[1] = s.y[i];
        if (D == 3) pi[2] = s.z[i];
    }
    const float soft = p.direct_eps2;
    float acc[3] = {0.f, 0.f, 0.f};
    for (uint32_t base = lo; base < hi; base += kDirectTile) {
        const uint32_t j = base + threadIdx.x;
        if (j < hi)
            sj[threadIdx.x] = make_float4(s.x[j], s.y[j], D == 3 ? s.z[j] : 0.0f,
                                          fmul(p.G, s.m[j]));
        __syncthreads();
        const uint32_t cnt = min((uint32_t)kDirectTile, hi - base);
        if (own) {
            for (uint32_t t = 0; t < cnt; t++) {
                const float4 q = sj[t];
                float d[3] = {fsub(q.x, pi[0]), fsub(q.y, pi[1]), D == 3 ? fsub(q.z, pi[2]) : 0.f};
                if (PER) {
#pragma unroll
                    for (int a = 0; a < D; a++) d[a] = wrap_dd(d[a], p.domain[a], p.half_domain[a]);
                }
                float r2 = fadd(fmul(d[0], d[0]), fmul(d[1], d[1]));
                if (D == 3) r2 = fadd(r2, fmul(d[2], d[2]));
                r2 = fadd(r2, soft);
                if (MODE == GE_PREC_EXACT) {
                    const float inv = fdiv(1.0f, __fsqrt_rn(r2));
                    const float f = fmul(q.w, fmul(fmul(inv, inv), inv));
#pragma unroll
                    for (int a = 0; a < D; a++) acc[a] = fadd(acc[a], fmul(d[a], f));
                } else {
                    const float inv = rsqrt_fast(r2);
                    const float f = q.w * (inv * inv * inv);
#pragma unroll
                    for (int a = 0; a < D; a++) acc[a] = fmaf(d[a], f, acc[a]);
                }
            }
        }
        __syncthreads();
    }
    if (!own) return;
    s.ax[i] = acc[0]; s.ay[i] = acc[1];
    if (D == 3) s.az[i] = acc[2];
    if (integrate_end && !(s.pinned && s.pinned[i])) {
        s.vx[i] = fadd(s.vx[i], fmul(acc[0], p.half_dt));
        s.vy[i] = fadd(s.vy[i], fmul(acc[1], p.half_dt));
        if (D == 3) s.vz[i] = fadd(s.vz[i], fmul(acc[2], p.half_dt));
    }
}

template <int D, int MODE>
cudaError_t direct_mode(const State &s, const StepParams &p, const Segs &g, const uint2 *tiles,
                        int64_t ntiles, int ie, cudaStream_t st) {
    if (p.periodic)
        k_direct<D, MODE, true><<<(unsigned)ntiles, kDirectTile, 0, st>>>(s, p, g, tiles, ie);
    else
        k_direct<D, MODE, false><<<(unsigned)ntiles, kDirectTile, 0, st>>>(s, p, g, tiles, ie);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_direct(int dims, int precision, const State &s, const StepParams &p,
                          const Segs &g, const uint2 *tiles, int64_t ntiles, bool integrate_end,
                          cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
    const int ie = integrate_end ? 1 : 0;
    const bool exact = precision == GE_PREC_EXACT;
    if (dims == 2)
        return exact ? direct_mode<2, GE_PREC_EXACT>(s, p, g, tiles, ntiles, ie, st)
                     : direct_mode<2, GE_PREC_FAST>(s, p, g, tiles, ntiles, ie, st);
    return exact ? direct_mode<3, GE_PREC_EXACT>(s, p, g, tiles, ntiles, ie, st)
                 : direct_mode<3, GE_PREC_FAST>(s, p, g, tiles, ntiles, ie, st);
}

}  // namespace ge
