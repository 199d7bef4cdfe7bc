// ge_walk.cu -- the theta-criterion tree walk with softened force.
//
// Reference: Physics::calculateForceFromGrid (GalaxyEngine/src/Physics/physics.cpp:91-205)
// and Physics3D::calculateForceFromGrid3D (physics3D.cpp:131-253).  Per
// particle i the reference scans the pre-order node array: a node of zero mass
// is skipped; with d = com - x_i and r2 = |d|^2 + eps2 the node is accepted as
// a monopole when size^2 < theta^2 * r2; otherwise a leaf is summed directly
// over its particles j != i; otherwise the walk descends.  acc_i = F_i / m_i.
//
// Here every particle walks the depth-first layout built with the tree
// (ge_internal.h) with no stack: each step loads one entry and its skip
// target, evaluates the reference's opening test with the reference's
// rounding (so the interaction set is exactly the reference's), interacts if
// accepted and goes to the skip target, else to the next entry (the first
// child, or a leaf's first particle).  A leaf's particles follow the leaf as
// entries of their own with size^2 = -1, which every test accepts, so the
// direct sum over a leaf is the same loop body (the self term j == i is
// skipped as in the reference); a node of zero mass is laid out as an accepted
// entry without mass, so its subtree is skipped as in the reference.
// Sources are met in the reference's pre-order, so each particle accumulates
// in the reference's order.
//   GE_PREC_EXACT : every interaction with the reference's rounding
//                   (1/sqrtf, products in the reference's order, no FMA):
//                   bit-identical accelerations.
//   GE_PREC_FAST  : approximate reciprocal square root (MUFU, flush-to-zero)
//                   and FMA for the force terms, G applied once.
//   GE_PREC_MIXED : the node entries written by the moment pass
//                   (ge_moments.cu): opening radius instead of size, the
//                   double-float centre of mass, a quadrupole term, and
//                   Kahan-compensated sums of the acceleration terms.
// integrateEnd (physics.cpp:1114-1125) is fused into the epilogue.  A
// simulation below params.direct_below is skipped here (ge_direct.cu).
#include <type_traits>

#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

// threads per block: 1024 in 3D, where a block's particles (consecutive in
// Morton order, on one SM) share more of their longer walks through L1
// (3.70 -> 3.42 ms for the 1M Plummer walk against 256); 256 in 2D (no gain)
template <int D> constexpr int walk_threads() { return D == 2 ? 256 : 1024; }

__device__ __forceinline__ float wrap_d(float d, float dom, float hd) {
    // d -= domain * ((d > half) - (d < -half))   (physics.cpp:118-121)
    const int k = (int)(d > hd) - (int)(d < -hd);
    return fsub(d, fmul(dom, (float)k));
}

__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// skip target and size^2 of an entry: 2D link = skip (size^2 in the source),
// 3D link = {skip, size^2 bits}
__device__ __forceinline__ uint32_t link_skip(uint32_t l) { return l; }
__device__ __forceinline__ uint32_t link_skip(const uint2 &l) { return l.x; }
__device__ __forceinline__ float link_s2(uint32_t, float in_src) { return in_src; }
__device__ __forceinline__ float link_s2(const uint2 &l, float) { return __uint_as_float(l.y); }

template <int D> struct LinkOf;
template <> struct LinkOf<2> { using T = uint32_t; };
template <> struct LinkOf<3> { using T = uint2; };

template <int D, int MODE, bool COUNT, bool PER, bool POS_EPS, bool TEMP = false>
__global__ void __launch_bounds__(walk_threads<D>())
k_walk(State s, StepParams p, Segs g, Tree t, int integrate_end, unsigned long long *inter,
       uint32_t *err) {
    dep_wait();
    using LT = typename LinkOf<D>::T;
    constexpr bool kSelfTest = MODE != GE_PREC_FAST || COUNT || !POS_EPS || TEMP;
    const LT *__restrict__ link = (const LT *)t.link;
    const float4 *__restrict__ src = t.src;
    const int n = p.n;
    const float eps2 = p.eps2, th2 = p.theta2, G = p.G;
    const int i = p.i0 + blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long my_count = 0;
    // particles of simulations that take the direct sum are left to it
    const bool walks = i < n && !(g.direct && __ldg(&g.direct[g.seg_of ? __ldg(&g.seg_of[i]) : 0u]));
    if (walks) {
        float pi[3];
        pi[0] = s.x[i]; pi[1] = s.y[i];
        pi[2] = D == 3 ? s.z[i] : 0.0f;
        const float mi = s.m[i];
        const float gm_i = fmul(G, mi);   // Gf * pmass (exact mode)
        const uint32_t self = kSelfTest ? __ldg(&t.slot_of[i]) : kEmpty;
        float f[3] = {0.f, 0.f, 0.f};
        float fc[3] = {0.f, 0.f, 0.f};   // Kahan compensation (MIXED)
        float ti = TEMP ? __ldg(&t.tv[self]) : 0.0f;   // own temperature, accumulated in walk order
        // the walk of the particle's own segment: its root to the root's successor
        const uint32_t sg = g.seg_of ? __ldg(&g.seg_of[i]) : 0u;
        uint32_t k = __ldg(&g.root_begin[sg]);
        const uint32_t end = __ldg(&g.root_end[sg]);
        uint32_t cnt = 0;
        // 2D packed entries: one load per step (the successor and the level
        // in the fourth word); the root size of the particle's simulation
        const bool packed = D == 2 && MODE != GE_PREC_MIXED && __ldg(&t.meta[kMetaWalkPacked]) != 0u;
        const float rs = packed ? __ldg(&g.box[sg]).w : 0.0f;
        const uint32_t rs2_bits = __float_as_uint(fmul(rs, rs));   // the root's size^2
        // the loop once per layout, chosen here rather than at every step
        auto walk_range = [&](auto pk) {
            constexpr bool PK = decltype(pk)::value && D == 2 && MODE != GE_PREC_MIXED;
            while (k < end) {
                const float4 A = __ldg(&src[k]);
                const float m = D == 2 ? A.z : A.w;
                float s2;          // a node's size^2 (plain layout: -1 particle, -2 massless)
                uint32_t nxt_skip;
                bool part;         // a particle's entry
                bool always = false;   // packed: a particle or a massless node
                if constexpr (PK) {
                    const uint32_t wb = __float_as_uint(A.w);
                    always = packed_accepts(wb);
                    part = packed_particle(wb);
                    s2 = packed_size2(wb, rs2_bits);   // not used for marked entries
                    nxt_skip = wb & ((1u << kPackSkipBits) - 1u);   // a particle's: k + 1
                } else {
                    const LT L = __ldg(&link[k]);
                    s2 = link_s2(L, A.w);
                    nxt_skip = link_skip(L);
                    part = s2 == -1.0f;
                }
                float d[3];
                d[0] = fsub(A.x, pi[0]);
                d[1] = fsub(A.y, pi[1]);
                d[2] = D == 3 ? fsub(A.z, pi[2]) : 0.0f;
                if (PER) {
    #pragma unroll
                    for (int a = 0; a < D; a++) d[a] = wrap_d(d[a], p.domain[a], p.half_domain[a]);
                }
                float r2 = fadd(fmul(d[0], d[0]), fmul(d[1], d[1]));
                if (D == 3) r2 = fadd(r2, fmul(d[2], d[2]));
                r2 = fadd(r2, eps2);
                // MIXED entries hold the squared opening radius, which already
                // includes 1 / theta
                bool acc;
                if constexpr (PK) acc = always || s2 < fmul(th2, r2);   // as -1 / -2 would
                else acc = MODE == GE_PREC_MIXED ? s2 < r2 : s2 < fmul(th2, r2);
                if (kSelfTest) {
                    // heat exchange (physics.cpp:145-158, 183-191): an accepted node
                    // with mass, or any other particle of an opened leaf (massless
                    // ones included); the others' temperatures as before the walk
                    if (TEMP && acc && k != self && (m != 0.0f || part)) {
                        float inv;
                        if (MODE == GE_PREC_EXACT) inv = fdiv(1.0f, __fsqrt_rn(r2));
                        else inv = rsqrt_approx(r2);
                        const float dist = r2 > 1e-16f ? fdiv(1.0f, inv) : 0.0f;
                        if (dist > 1e-8f) {
                            const float diff = fsub(__ldg(&t.tv[k]), ti);
                            ti = fadd(ti, fmul(fdiv(fmul(p.heat_cond, diff), dist), p.dt));
                        }
                    }
                    if (acc && m != 0.0f && k != self) {
                        if (MODE == GE_PREC_MIXED) {
                            float term[3];
                            if (s2 >= 0.0f) {
                                // node: centre of mass = hi + lo, then monopole +
                                // quadrupole of the softened kernel:
                                //   m d / r^3 - 3 I d / r^5 - 1.5 tr(I) d / r^5
                                //   + 7.5 (d.I.d) d / r^7,   r^2 = |d|^2 + eps2
                                const float4 B = __ldg(&t.mq0[k]);
                                d[0] += B.x; d[1] += B.y;
                                if (D == 3) d[2] += B.z;
                                float rr = d[0] * d[0] + d[1] * d[1] + eps2;
                                if (D == 3) rr += d[2] * d[2];
                                const float inv = rsqrt_approx(rr);
                                const float inv2 = inv * inv, inv3 = inv2 * inv, inv5 = inv3 * inv2;
                                const float inv7 = inv5 * inv2;
                                float Id[3], tr;
                                if (D == 2) {
                                    const float ixx = B.z, ixy = B.w, iyy = __ldg(&t.mq2[k]);
                                    Id[0] = ixx * d[0] + ixy * d[1];
                                    Id[1] = ixy * d[0] + iyy * d[1];
                                    Id[2] = 0.0f;
                                    tr = ixx + iyy;
                                } else {
                                    const float4 C = __ldg(&t.mq1[k]);   // {Iyy, Izz, Ixy, Ixz}
                                    const float ixx = B.w, iyz = __ldg(&t.mq2[k]);
                                    Id[0] = ixx * d[0] + C.z * d[1] + C.w * d[2];
                                    Id[1] = C.z * d[0] + C.x * d[1] + iyz * d[2];
                                    Id[2] = C.w * d[0] + iyz * d[1] + C.y * d[2];
                                    tr = ixx + C.x + C.y;
                                }
                                float dId = d[0] * Id[0] + d[1] * Id[1];
                                if (D == 3) dId += d[2] * Id[2];
                                const float cm = m * inv3 - 1.5f * tr * inv5 + 7.5f * dId * inv7;
                                const float ci = -3.0f * inv5;
    #pragma unroll
                                for (int a = 0; a < D; a++) term[a] = cm * d[a] + ci * Id[a];
                            } else {
                                const float inv = rsqrt_approx(r2);
                                const float fm = m * (inv * inv * inv);
    #pragma unroll
                                for (int a = 0; a < D; a++) term[a] = d[a] * fm;
                            }
    #pragma unroll
                            for (int a = 0; a < D; a++) {   // Kahan summation
                                const float y = fsub(term[a], fc[a]);
                                const float tt = fadd(f[a], y);
                                fc[a] = fsub(fsub(tt, f[a]), y);
                                f[a] = tt;
                            }
                        } else if (MODE == GE_PREC_EXACT) {
                            const float inv = fdiv(1.0f, __fsqrt_rn(r2));
                            const float inv3 = fmul(fmul(inv, inv), inv);
                            const float fm = fmul(fmul(gm_i, m), inv3);
    #pragma unroll
                            for (int a = 0; a < D; a++) f[a] = fadd(f[a], fmul(d[a], fm));
                        } else {
                            const float inv = rsqrt_approx(r2);
                            const float fm = m * (inv * inv * inv);
    #pragma unroll
                            for (int a = 0; a < D; a++) f[a] = fmaf(d[a], fm, f[a]);
                        }
                        if (COUNT) cnt++;
                    }
                } else {
                    // eps2 > 0: the self term (d = 0) and massless sources add exactly
                    // zero, so no test is needed for them
                    const float inv = rsqrt_approx(r2);
                    const float fm = acc ? m * (inv * inv * inv) : 0.0f;
    #pragma unroll
                    for (int a = 0; a < D; a++) f[a] = fmaf(d[a], fm, f[a]);
                }
                // a valid skip lies past k; max() keeps k increasing whatever the
                // layout holds, so the walk ends within end - begin entries (a
                // packed particle's own successor is k + 1)
                if constexpr (PK) k = max(k + 1, acc ? nxt_skip : k + 1);
                else k = max(k + 1, acc && !part ? nxt_skip : k + 1);
            }
        };
        if (packed) walk_range(std::true_type{});
        else walk_range(std::false_type{});
        float a3[3];
#pragma unroll
        for (int a = 0; a < D; a++)
            a3[a] = MODE == GE_PREC_EXACT ? fdiv(f[a], mi)
                  : MODE == GE_PREC_MIXED ? G * fsub(f[a], fc[a]) : G * f[a];
        s.ax[i] = a3[0]; s.ay[i] = a3[1];
        if (D == 3) s.az[i] = a3[2];
        if (TEMP) s.temp[i] = ti;
        if (integrate_end && !(s.pinned && s.pinned[i])) {
            if (MODE == GE_PREC_MIXED && s.kvx) {
                float *vel[3] = {s.vx, s.vy, s.vz}, *kv[3] = {s.kvx, s.kvy, s.kvz};
#pragma unroll
                for (int a = 0; a < D; a++) kahan_add(vel[a][i], kv[a][i], fmul(a3[a], p.half_dt));
            } else {
                s.vx[i] = fadd(s.vx[i], fmul(a3[0], p.half_dt));
                s.vy[i] = fadd(s.vy[i], fmul(a3[1], p.half_dt));
                if (D == 3) s.vz[i] = fadd(s.vz[i], fmul(a3[2], p.half_dt));
            }
        }
        my_count = cnt;
    }
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) my_count += __shfl_xor_sync(0xffffffffu, my_count, o);
        if ((threadIdx.x & 31) == 0 && my_count) atomicAdd(inter, my_count);
    }
}

template <int D, int MODE, bool COUNT, bool PER, bool POS_EPS, bool TEMP = false>
static cudaError_t walk_one(const State &s, const StepParams &p, const Segs &g, const Tree &t,
                            int ie, unsigned long long *inter, uint32_t *err, cudaStream_t st) {
    constexpr int kWalkThreads = walk_threads<D>();
    const int blocks = (p.n - p.i0 + kWalkThreads - 1) / kWalkThreads;
    return launch_dep(k_walk<D, MODE, COUNT, PER, POS_EPS, TEMP>, blocks < 1 ? 1 : blocks,
                      kWalkThreads, st, s, p, g, t, ie, inter, err);
}

template <int D, int MODE, bool PER>
static cudaError_t walk_eps(const State &s, const StepParams &p, const Segs &g, const Tree &t,
                            int ie, unsigned long long *inter, uint32_t *err, cudaStream_t st) {
    if constexpr (MODE != GE_PREC_MIXED)
        if (s.temp && t.tv) {   // heat exchange (counting included)
            if (inter) return walk_one<D, MODE, true, PER, false, true>(s, p, g, t, ie, inter, err, st);
            return walk_one<D, MODE, false, PER, false, true>(s, p, g, t, ie, nullptr, err, st);
        }
    if (inter) return walk_one<D, MODE, true, PER, false>(s, p, g, t, ie, inter, err, st);
    if constexpr (MODE != GE_PREC_MIXED)   // MIXED always tests for the particle itself
        if (p.eps2 > 0.0f)
            return walk_one<D, MODE, false, PER, true>(s, p, g, t, ie, nullptr, err, st);
    return walk_one<D, MODE, false, PER, false>(s, p, g, t, ie, nullptr, err, st);
}

template <int D, int MODE>
static cudaError_t walk_mode(const State &s, const StepParams &p, const Segs &g, const Tree &t,
                             int ie, unsigned long long *inter, uint32_t *err, cudaStream_t st) {
    if (p.periodic) return walk_eps<D, MODE, true>(s, p, g, t, ie, inter, err, st);
    return walk_eps<D, MODE, false>(s, p, g, t, ie, inter, err, st);
}

cudaError_t launch_walk(int dims, int precision, const State &s, const StepParams &p,
                        const Segs &g, const Tree &t, bool integrate_end,
                        unsigned long long *inter_count, uint32_t *err, int num_sms,
                        cudaStream_t st) {
    const int ie = integrate_end ? 1 : 0;
    const bool exact = precision == GE_PREC_EXACT;
    // (the warp walk stages a particle's own term with its leaf, which adds
    // zero only with eps2 > 0)
    if (p.walk_kind == 1 && precision == GE_PREC_FAST && !p.periodic && !(s.temp && t.tv) &&
        p.eps2 > 0.0f)
        return launch_warp_walk(dims, s, p, g, t, integrate_end, inter_count, err, num_sms, st);
    if (precision == GE_PREC_MIXED)
        return dims == 2 ? walk_mode<2, GE_PREC_MIXED>(s, p, g, t, ie, inter_count, err, st)
                         : walk_mode<3, GE_PREC_MIXED>(s, p, g, t, ie, inter_count, err, st);
    if (dims == 2)
        return exact ? walk_mode<2, GE_PREC_EXACT>(s, p, g, t, ie, inter_count, err, st)
                     : walk_mode<2, GE_PREC_FAST>(s, p, g, t, ie, inter_count, err, st);
    return exact ? walk_mode<3, GE_PREC_EXACT>(s, p, g, t, ie, inter_count, err, st)
                 : walk_mode<3, GE_PREC_FAST>(s, p, g, t, ie, inter_count, err, st);
}

}  // namespace ge
