// ge_predict.cu -- trajectory preview of probe particles on the resident tree.
//
// ParticlesSpawning::predictTrajectory (particlesSpawning.cpp:443-500, 3D
// :1000-1060) steps one probe particle against the frame's tree without
// rebuilding it: each step computes the force at the probe's position with
// the older walk Physics::calculateForceFromGridOld (physics.cpp:4-90;
// physics3D.cpp:49-120), kicks half a step, drifts (with the periodic wrap),
// computes the force again, kicks the other half and records the position.
// That walk never opens a leaf (a leaf is taken whole by its mass and centre
// of mass), skips a one-particle leaf within 0.001 of the probe on every
// axis, and adds the softening squared in 2D and 3D.  Here one thread runs
// one probe over the walk layout of the last build, with the reference's
// rounding for every operation, so many probes cost one launch.
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kPredThreads = 64;

// size^2 of entry k (-1 for a particle); rs_bits: the simulation's root
// size^2, for the packed 2D layout
__device__ __forceinline__ float entry_s2(const Tree &t, int D, uint32_t k, bool packed,
                                          uint32_t rs_bits) {
    if (D == 3) return __uint_as_float(__ldg(&((const uint2 *)t.link)[k]).y);
    const float4 A = __ldg(&t.src[k]);
    if (!packed) return A.w;
    const uint32_t wb = __float_as_uint(A.w);
    if (packed_particle(wb)) return -1.0f;
    if (packed_accepts(wb)) return -2.0f;   // a massless node
    return packed_size2(wb, rs_bits);
}
// successor of entry k (A = its src word): packed 2D entries carry it in
// their fourth word's low bits (no link array is written then)
__device__ __forceinline__ uint32_t entry_skip(const Tree &t, int D, uint32_t k, bool packed,
                                               float4 A) {
    if (D == 2 && packed) return __float_as_uint(A.w) & ((1u << kPackSkipBits) - 1u);
    return D == 2 ? __ldg(&((const uint32_t *)t.link)[k]) : __ldg(&((const uint2 *)t.link)[k]).x;
}

template <int D>
__device__ void old_force(const Tree &t, const StepParams &p, uint32_t begin, uint32_t end,
                          float eps2, const float *pos, float pmass, float *F, bool packed,
                          uint32_t rs_bits) {
    F[0] = F[1] = F[2] = 0.0f;
    uint32_t k = begin;
    while (k < end) {
        const float4 A = __ldg(&t.src[k]);
        const uint32_t skip = entry_skip(t, D, k, packed, A);
        const uint32_t nxt = max(k + 1, skip);   // always moves forward
        const float gm = D == 2 ? A.z : A.w;
        if (!(gm > 0.0f)) { k = nxt; continue; }   // gridMass <= 0: skip the subtree
        const float com[3] = {A.x, A.y, A.z};
        float d[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int a = 0; a < D; a++) {
            d[a] = fsub(com[a], pos[a]);
            if (p.periodic) {
                const int s = (int)(d[a] > p.half_domain[a]) - (int)(d[a] < -p.half_domain[a]);
                d[a] = fsub(d[a], fmul(p.domain[a], (float)s));
            }
        }
        float r2 = fadd(fmul(d[0], d[0]), fmul(d[1], d[1]));
        if (D == 3) r2 = fadd(r2, fmul(d[2], d[2]));
        r2 = fadd(r2, eps2);
        // a leaf's particles follow it in the layout (size^2 = -1)
        const bool leaf = k + 1 < skip && entry_s2(t, D, k + 1, packed, rs_bits) == -1.0f;
        const float s2 = entry_s2(t, D, k, packed, rs_bits);
        if (s2 < fmul(p.theta2, r2) || leaf) {
            if (leaf && skip - k - 1 == 1u) {   // one particle: skip it when it sits on the probe
                const float4 o = __ldg(&t.src[k + 1]);
                const float op[3] = {o.x, o.y, o.z};
                bool near = true;
#pragma unroll
                for (int a = 0; a < D; a++) near = near && fabsf(fsub(op[a], pos[a])) < 0.001f;
                if (near) { k = nxt; continue; }
            }
            const float inv = fdiv(1.0f, __fsqrt_rn(r2));
            const float inv3 = fmul(fmul(inv, inv), inv);
            const float fm = fmul(fmul(fmul(p.G, pmass), gm), inv3);
#pragma unroll
            for (int a = 0; a < D; a++) F[a] = fadd(F[a], fmul(d[a], fm));
            k = nxt;
        } else {
            ++k;
        }
    }
}

template <int D>
__global__ void __launch_bounds__(kPredThreads)
k_predict(Tree t, StepParams p, const float4 *box, uint32_t begin, uint32_t end, float eps2,
          int nprobes, const float *__restrict__ pos, const float *__restrict__ vel,
          const float *__restrict__ mass, int steps, float *__restrict__ path) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nprobes) return;
    const bool packed = D == 2 && __ldg(&t.meta[kMetaWalkPacked]) != 0u;
    const float rs = packed ? __ldg(box).w : 0.0f;   // the simulation's root size
    const uint32_t rs_bits = __float_as_uint(fmul(rs, rs));
    float ps[3] = {0.f, 0.f, 0.f}, v[3] = {0.f, 0.f, 0.f}, F[3];
#pragma unroll
    for (int a = 0; a < D; a++) { ps[a] = pos[q * D + a]; v[a] = vel[q * D + a]; }
    const float m = mass[q], h = fmul(p.dt, 0.5f);
    for (int s = 0; s < steps; s++) {
        old_force<D>(t, p, begin, end, eps2, ps, m, F, packed, rs_bits);
#pragma unroll
        for (int a = 0; a < D; a++) v[a] = fadd(v[a], fmul(fdiv(F[a], m), h));
#pragma unroll
        for (int a = 0; a < D; a++) ps[a] = fadd(ps[a], fmul(v[a], p.dt));
        if (p.periodic) {
#pragma unroll
            for (int a = 0; a < D; a++) {
                // particlesSpawning.cpp:478-484 (2D: [0, size)), :1031-1047 (3D: [-size/2, size/2))
                const float lo = D == 2 ? 0.0f : -p.half_domain[a];
                const float hi = D == 2 ? p.domain[a] : p.half_domain[a];
                if (ps[a] < lo) ps[a] = fadd(ps[a], p.domain[a]);
                else if (ps[a] >= hi) ps[a] = fsub(ps[a], p.domain[a]);
            }
        }
        old_force<D>(t, p, begin, end, eps2, ps, m, F, packed, rs_bits);
#pragma unroll
        for (int a = 0; a < D; a++) v[a] = fadd(v[a], fmul(fdiv(F[a], m), h));
#pragma unroll
        for (int a = 0; a < D; a++) path[((size_t)q * steps + s) * D + a] = ps[a];
    }
}

cudaError_t launch_predict(int dims, const Tree &t, const StepParams &p, const float4 *box,
                           uint32_t begin,
                           uint32_t end, float eps2, int nprobes, const float *pos,
                           const float *vel, const float *mass, int steps, float *path,
                           cudaStream_t st) {
    const int blocks = (nprobes + kPredThreads - 1) / kPredThreads;
    if (blocks < 1) return cudaSuccess;
    if (dims == 2)
        k_predict<2><<<blocks, kPredThreads, 0, st>>>(t, p, box, begin, end, eps2, nprobes, pos,
                                                     vel, mass, steps, path);
    else
        k_predict<3><<<blocks, kPredThreads, 0, st>>>(t, p, box, begin, end, eps2, nprobes, pos,
                                                     vel, mass, steps, path);
    return cudaGetLastError();
}

}  // namespace ge
