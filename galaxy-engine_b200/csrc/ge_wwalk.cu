// ge_wwalk.cu -- warp-cooperative tree walk (GE_PREC_FAST) that keeps the
// reference's per-particle interaction set.
//
// Reference: Physics::calculateForceFromGrid (GalaxyEngine/src/Physics/
// physics.cpp:91-205) and Physics3D::calculateForceFromGrid3D (physics3D.cpp:
// 131-253).  For every particle i the reference visits the tree in pre-order:
// a node of zero mass is skipped; a node with size^2 < theta^2 * r^2 (r^2 =
// |com - x_i|^2 + eps2, the reference's rounding) is taken as a monopole;
// otherwise a leaf's particles j != i are summed directly and an inner node is
// opened.  acc_i = G * sum m d / r^3.
//
// Here the 32 lanes of a warp hold 32 Morton-consecutive particles of one
// simulation and walk the node tree together, 32 nodes per round from a work
// stack in shared memory.  Each node is decided for all 32 particles at once
// against the warp's bounding box with the same IEEE operations as the
// per-particle test: d = com - x is monotone in x, and the squares, sums and
// the product with theta^2 are monotone in d, so the box's nearest and
// farthest points bound every lane's r^2 *as the lane itself rounds it*:
//   size^2 <  theta^2 * r2(nearest)   -> every lane takes the monopole;
//   size^2 >= theta^2 * r2(farthest)  -> every lane opens the node;
// a node in between is "near": its subtree is walked by every lane for its
// own particle (the per-particle walk over the depth-first layout, from the
// node's entry to its successor), which applies the reference's test lane by
// lane.  So each particle's set of monopoles and leaf particles is exactly the
// reference's.  Monopoles that every lane takes, and the particles of leaves
// that every lane opens, are staged in a source list in shared memory and
// evaluated by every lane for its own particle (sources broadcast): rsqrt +
// FMA per term, as the per-particle FAST walk.  The order of the terms
// differs from the reference's pre-order (FAST accuracy, not bit-exact).
// A particle's own term, staged with its leaf, adds exactly zero because
// eps2 > 0 (the launcher sends eps2 == 0 to the per-particle walk).
//
// A warp whose stack would outgrow shared memory finishes its particles with
// the per-particle walk from the root.  The kernel is persistent: warps take
// chunks of 32 particles from a counter; a chunk lies inside one simulation
// and is counted from the simulation's first particle, so a simulation's
// results are the same alone and in a batch.  Simulations taking the direct
// sum are skipped.
#include <cfloat>

#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kWWWarps = 4;                 // warps per block
constexpr int kWWThreads = kWWWarps * 32;
// shared memory per warp stays small (2.3 KB): the per-lane near walks read
// the layout through L1, which takes what shared memory leaves
constexpr uint32_t kWWStack = 256;          // stack nodes per warp
constexpr int kWWList = 64;                 // staged sources per warp
constexpr int kWWNear = 32;                 // near subtrees per warp
constexpr uint32_t kWWLeafRegs = 4;         // leaf particles prefetched into registers
constexpr unsigned kFull = 0xffffffffu;

struct WWSmem {
    uint32_t stk[kWWStack];                 // node slots
    float4 src[kWWList];                    // 2D {x, y, m, -}   3D {x, y, z, m}
    uint2 near[kWWNear];                    // {first entry, successor} in the depth-first layout
};

__device__ __forceinline__ float ww_rsqrt(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, unsigned lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(kFull, v, o);
        if (lane >= (unsigned)o) v += u;
    }
    return v;
}

// r^2 with the reference's rounding: ((dx*dx + dy*dy) (+ dz*dz)) + eps2
template <int D>
__device__ __forceinline__ float ref_r2(const float (&d)[3], float eps2) {
    float r2 = fadd(fmul(d[0], d[0]), fmul(d[1], d[1]));
    if (D == 3) r2 = fadd(r2, fmul(d[2], d[2]));
    return fadd(r2, eps2);
}

// every lane's force from the staged sources
template <int D>
__device__ __forceinline__ void eval_list(const WWSmem &sm, int nl, const float (&pi)[3],
                                          float eps2, float (&f)[3]) {
#pragma unroll 4
    for (int e = 0; e < nl; e++) {
        const float4 S = sm.src[e];
        const float d0 = S.x - pi[0], d1 = S.y - pi[1];
        const float d2 = D == 3 ? S.z - pi[2] : 0.0f;
        float r2 = fmaf(d1, d1, fmaf(d0, d0, eps2));
        if (D == 3) r2 = fmaf(d2, d2, r2);
        const float inv = ww_rsqrt(r2);
        const float fm = (D == 2 ? S.z : S.w) * (inv * inv * inv);
        f[0] = fmaf(d0, fm, f[0]);
        f[1] = fmaf(d1, fm, f[1]);
        if (D == 3) f[2] = fmaf(d2, fm, f[2]);
    }
}

// One entry of the depth-first layout: its position/mass word, size^2 (nodes),
// subtree successor, and whether it is a particle.
template <int D>
__device__ __forceinline__ void layout_entry(const Tree &t, uint32_t k, bool packed,
                                             uint32_t rs2_bits, float4 &A, float &s2,
                                             uint32_t &skip, bool &part) {
    A = __ldg(&t.src[k]);
    if (D == 2 && packed) {
        const uint32_t wb = __float_as_uint(A.w);
        part = packed_particle(wb);   // (massless nodes: mass 0, accepted below)
        s2 = packed_size2(wb, rs2_bits);
        skip = wb & ((1u << kPackSkipBits) - 1u);
    } else if (D == 2) {
        s2 = A.w;
        skip = __ldg(&((const uint32_t *)t.link)[k]);
        part = s2 == -1.0f;
    } else {
        const uint2 L = __ldg(&((const uint2 *)t.link)[k]);
        s2 = __uint_as_float(L.y);
        skip = L.x;
        part = s2 == -1.0f;
    }
}

// The per-particle walk of particle pi over the depth-first layout ranges
// rng[0..nr) one after another (subtrees, or [root, end) for a whole walk):
// the reference's test per entry, FAST arithmetic.  COUNT: the particle's own
// entry (self) and massless sources are left out of the force and the count;
// otherwise they add exactly zero (eps2 > 0).
template <int D, bool COUNT>
__device__ __forceinline__ void walk_ranges(const Tree &t, const uint2 *rng, int nr,
                                            const float (&pi)[3], uint32_t self, bool packed,
                                            uint32_t rs2_bits, float eps2, float th2,
                                            float (&f)[3], uint32_t &cnt) {
    int it = 0;
    uint32_t k = 0u, end = 0u;
    while (true) {
        if (k >= end) {   // this range is done: straight on to the next one
            if (it == nr) break;
            const uint2 r = rng[it++];
            k = r.x;
            end = r.y;
        }
        float4 A;
        float s2;
        uint32_t skip;
        bool part;
        layout_entry<D>(t, k, packed, rs2_bits, A, s2, skip, part);
        const float m = D == 2 ? A.z : A.w;
        float d[3] = {fsub(A.x, pi[0]), fsub(A.y, pi[1]), D == 3 ? fsub(A.z, pi[2]) : 0.0f};
        const float r2 = ref_r2<D>(d, eps2);
        const bool acc = part || m <= 0.0f || s2 < fmul(th2, r2);
        const float inv = ww_rsqrt(r2);
        float fm = m * (inv * inv * inv);
        bool take = acc;
        if (COUNT) {
            take = acc && m != 0.0f && k != self;
            cnt += take ? 1u : 0u;
        }
        fm = take ? fm : 0.0f;
#pragma unroll
        for (int a = 0; a < D; a++) f[a] = fmaf(d[a], fm, f[a]);
        // a valid successor lies past k; max() keeps k increasing whatever
        // the layout holds
        k = max(k + 1, acc && !part ? skip : k + 1);
    }
}

template <int D, bool COUNT>
// 12 blocks per SM: 48 resident warps (the near walks are latency-bound)
__global__ void __launch_bounds__(kWWThreads, 12)
k_warp_walk(State s, StepParams p, Segs g, Tree t, int integrate_end,
            unsigned long long *inter, uint32_t *ctr) {
    dep_wait();
    __shared__ WWSmem smem[kWWWarps];
    WWSmem &sm = smem[threadIdx.x >> 5];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt = (1u << lane) - 1u;
    const int n = p.n, i0 = p.i0;
    // chunks of 32 particles, each inside one simulation and counted from the
    // simulation's first particle: one simulation, chunks from p.i0; several,
    // 128 chunks per sort tile (4096 particles of one simulation, its tiles
    // counted from its first particle)
    const bool multi = g.tile_seg != nullptr;
    const uint32_t nchunks = multi ? (uint32_t)g.tiles * (uint32_t)(kSortTile / 32)
                                   : (uint32_t)((n - i0 + 31) / 32);
    const float eps2 = p.eps2, th2 = p.theta2;
    const float *pos[3] = {s.x, s.y, s.z};
    const bool packed = D == 2 && __ldcg(&t.meta[kMetaWalkPacked]) != 0u;
    unsigned long long my_count = 0;
    while (true) {
        uint32_t c = kEmpty;   // the next chunk
        if (lane == 0) {
            c = atomicAdd(&ctr[0], 1u);
            if (c >= nchunks) c = kEmpty;
        }
        c = __shfl_sync(kFull, c, 0);
        if (c == kEmpty) break;
        int base, iend;
        uint32_t sg = 0;
        if (multi) {
            const uint32_t tile = c / (uint32_t)(kSortTile / 32);
            sg = __ldg(&g.tile_seg[tile]);
            base = (int)(__ldg(&g.off[sg]) + (tile - __ldg(&g.tile_base[sg])) * (uint32_t)kSortTile +
                         (c % (uint32_t)(kSortTile / 32)) * 32u);
            iend = (int)__ldg(&g.off[sg + 1]);
            if (base >= iend) continue;   // past the simulation's last particle
        } else {
            base = i0 + (int)c * 32;
            iend = n;
        }
        const int i = base + (int)lane;
        const bool valid = i < iend && !(g.direct && __ldg(&g.direct[sg]));
        if (!__any_sync(kFull, valid)) continue;
        float pi[3] = {0.0f, 0.0f, 0.0f};
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
#pragma unroll
        for (int a = 0; a < D; a++) {
            if (valid) {
                pi[a] = pos[a][i];
                lo[a] = hi[a] = pi[a];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo[a] = fminf(lo[a], __shfl_xor_sync(kFull, lo[a], o));
                hi[a] = fmaxf(hi[a], __shfl_xor_sync(kFull, hi[a], o));
            }
        }
        const uint32_t rs2 = packed ? __float_as_uint(fmul(__ldg(&g.box[sg]).w, __ldg(&g.box[sg]).w)) : 0u;
        const uint32_t self = COUNT && valid ? __ldg(&t.slot_of[i]) : kEmpty;
        float f[3] = {0.0f, 0.0f, 0.0f};
        uint32_t cnt = 0;           // COUNT: this lane's interactions in the near walks
        uint32_t list_total = 0;    // COUNT: staged sources with mass, warp-uniform
        uint32_t self_staged = 0;   // COUNT: whether this lane's own particle was staged
        int nl = 0, nn = 0;
        // the simulation's root (node slot s is the root of simulation s)
        uint32_t top = 1;
        if (lane == 0) sm.stk[0] = sg;
        __syncwarp();
        bool fallback = false;
        while (top > 0) {
            const uint32_t take = min(top, 32u);
            top -= take;
            const uint32_t nd = lane < take ? sm.stk[top + lane] : kEmpty;
            __syncwarp();
            // 0: nothing (empty lane, massless node), 1: every lane takes the
            // monopole, 2: every lane opens it, 3: near (lane by lane)
            int kind = 0;
            float4 W = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            uint4 inf = make_uint4(0u, 0u, 0u, 0u);
            uint2 rng = make_uint2(0u, 0u);
            if (nd != kEmpty) {
                W = __ldg(&t.walk[nd]);
                inf = __ldg(&t.info[nd]);
                rng = __ldg(&t.nrange[nd]);
                const float s2 = D == 2 ? W.w : __ldg(&t.size2[nd]);
                if ((D == 2 ? W.z : W.w) > 0.0f) {   // gridMass <= 0: skipped (physics.cpp:108-111)
                    const float com[3] = {W.x, W.y, W.z};
                    float en[3], ef[3];
#pragma unroll
                    for (int a = 0; a < D; a++) {
                        // every lane's d = com - x lies in [dh, dl]
                        const float dl = fsub(com[a], lo[a]), dh = fsub(com[a], hi[a]);
                        en[a] = fmaxf(dh, 0.0f) + fminf(dl, 0.0f);   // nearest: one term is 0
                        ef[a] = fmaxf(dl, -dh);                      // farthest |d|
                    }
                    const float r2n = ref_r2<D>(en, eps2), r2f = ref_r2<D>(ef, eps2);
                    kind = s2 < fmul(th2, r2n) ? 1 : (s2 < fmul(th2, r2f) ? 3 : 2);
                }
            }
            const bool leaf = inf.y == 0u;
            // the particles of a leaf every lane opens: the first few into
            // registers now, so their loads overlap the bookkeeping below
            const uint32_t lcnt = (kind == 2 && leaf) ? inf.w - inf.z : 0u;
            float4 lp[kWWLeafRegs];
#pragma unroll
            for (uint32_t q = 0; q < kWWLeafRegs; q++) {
                const uint32_t j = inf.z + q;
                lp[q] = q < lcnt ? (D == 2 ? make_float4(__ldg(&s.x[j]), __ldg(&s.y[j]), __ldg(&s.m[j]), 0.0f)
                                           : make_float4(__ldg(&s.x[j]), __ldg(&s.y[j]), __ldg(&s.z[j]),
                                                         __ldg(&s.m[j])))
                                 : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
            // children of nodes every lane opens onto the stack
            const uint32_t nch = (kind == 2 && !leaf) ? (uint32_t)__popc(inf.y) : 0u;
            const uint32_t incl = warp_incl_scan(nch, lane);
            const uint32_t tot = __shfl_sync(kFull, incl, 31);
            if (top + tot > kWWStack) {   // warp-uniform
                fallback = true;
                break;
            }
            for (uint32_t q = 0; q < nch; q++) sm.stk[top + incl - nch + q] = inf.x + q;
            top += tot;
            // near nodes: their layout range, walked lane by lane
            const bool nr = kind == 3;
            const unsigned nb = __ballot_sync(kFull, nr);
            if (nb) {
                if (nn + __popc(nb) > kWWNear) {
                    __syncwarp();
                    walk_ranges<D, COUNT>(t, sm.near, nn, pi, self, packed, rs2, eps2, th2, f, cnt);
                    nn = 0;
                    __syncwarp();
                }
                if (nr) sm.near[nn + __popc(nb & lt)] = rng;
                nn += __popc(nb);
            }
            // staged sources: monopoles every lane takes, and the particles
            // of leaves every lane opens
            uint32_t pc = kind == 1 ? 1u : lcnt;
            uint32_t pj = 0;
            while (__any_sync(kFull, pc != 0u)) {
                const uint32_t pin = warp_incl_scan(pc, lane);
                const uint32_t ptot = __shfl_sync(kFull, pin, 31);
                uint32_t space = (uint32_t)(kWWList - nl);
                if (space == 0u) {
                    __syncwarp();
                    eval_list<D>(sm, nl, pi, eps2, f);
                    nl = 0;
                    space = kWWList;
                    __syncwarp();
                }
                const uint32_t excl = pin - pc;
                const uint32_t tk = excl >= space ? 0u : min(pc, space - excl);
                for (uint32_t u = 0; u < tk; u++) {
                    const uint32_t slot = (uint32_t)nl + excl + u;
                    if (kind == 1) {
                        sm.src[slot] = W;   // 2D {x, y, m, size^2}: w unused
                    } else {
                        const uint32_t q = pj++;
                        float4 v;
                        if (q < kWWLeafRegs) {
                            v = lp[0];
#pragma unroll
                            for (uint32_t r = 1; r < kWWLeafRegs; r++) v = q == r ? lp[r] : v;
                        } else {
                            const uint32_t j = inf.z + q;
                            v = D == 2 ? make_float4(s.x[j], s.y[j], s.m[j], 0.0f)
                                       : make_float4(s.x[j], s.y[j], s.z[j], s.m[j]);
                        }
                        sm.src[slot] = v;
                    }
                }
                pc -= tk;
                nl += (int)min(ptot, space);
            }
            if (COUNT) {
                // every staged source counts for every lane, except massless
                // particles (no interaction) and a lane's own particle
                uint32_t massless = 0, mine = 0;
                for (uint32_t j = inf.z; j < inf.z + lcnt; j++) {
                    const bool z = s.m[j] == 0.0f;
                    massless += z ? 1u : 0u;
                    const uint32_t rel = j - (uint32_t)base;
                    if (rel < 32u && !z) mine |= 1u << rel;
                }
                uint32_t tsum = (kind == 1 ? 1u : 0u) + lcnt - massless;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) tsum += __shfl_xor_sync(kFull, tsum, o);
                list_total += tsum;
                self_staged |= (__reduce_or_sync(kFull, mine) >> lane) & 1u;
            }
        }
        __syncwarp();
        if (fallback) {
            // the stack would outgrow shared memory: these particles walk the
            // whole tree one by one (everything staged so far is dropped)
            f[0] = f[1] = f[2] = 0.0f;
            cnt = 0;
            list_total = 0;
            self_staged = 0;
            if (lane == 0) atomicAdd(ctr + 1, 1u);
            const uint2 whole = make_uint2(__ldg(&g.root_begin[sg]), __ldg(&g.root_end[sg]));
            if (valid) walk_ranges<D, COUNT>(t, &whole, 1, pi, self, packed, rs2, eps2, th2, f, cnt);
        } else {
            if (nl) eval_list<D>(sm, nl, pi, eps2, f);
            if (nn) walk_ranges<D, COUNT>(t, sm.near, nn, pi, self, packed, rs2, eps2, th2, f, cnt);
        }
        __syncwarp();
        if (valid) {
            float a3[3];
#pragma unroll
            for (int a = 0; a < D; a++) a3[a] = p.G * f[a];
            s.ax[i] = a3[0];
            s.ay[i] = a3[1];
            if (D == 3) s.az[i] = a3[2];
            if (integrate_end && !(s.pinned && s.pinned[i])) {
                s.vx[i] = fadd(s.vx[i], fmul(a3[0], p.half_dt));
                s.vy[i] = fadd(s.vy[i], fmul(a3[1], p.half_dt));
                if (D == 3) s.vz[i] = fadd(s.vz[i], fmul(a3[2], p.half_dt));
            }
            if (COUNT) my_count += cnt + list_total - self_staged;
        }
    }
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) my_count += __shfl_xor_sync(kFull, my_count, o);
        if (lane == 0 && my_count) atomicAdd(inter, my_count);
    }
}

// Blocks of the persistent walk that one wave holds on this device.
template <int D, bool COUNT>
static int ww_wave(int num_sms) {
    static int per_sm = -1;
    if (per_sm < 0) {
        int v = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_warp_walk<D, COUNT>, kWWThreads, 0) !=
            cudaSuccess)
            v = 0;
        per_sm = v;
    }
    return per_sm * num_sms;
}

template <int D, bool COUNT>
static cudaError_t ww_launch(const State &s, const StepParams &p, const Segs &g, const Tree &t,
                             int ie, unsigned long long *inter, int num_sms, cudaStream_t st) {
    const int64_t chunks = g.tile_seg ? g.tiles * (kSortTile / 32) : (p.n - p.i0 + 31) / 32;
    const int wave = ww_wave<D, COUNT>(num_sms);
    if (wave < 1) return cudaErrorLaunchOutOfResources;
    int64_t blocks = (chunks + kWWWarps - 1) / kWWWarps;
    if (blocks > wave) blocks = wave;
    if (blocks < 1) blocks = 1;
    return launch_dep(k_warp_walk<D, COUNT>, (unsigned)blocks, kWWThreads, st, s, p, g, t, ie,
                      inter, t.wctr);
}

cudaError_t launch_warp_walk(int dims, const State &s, const StepParams &p, const Segs &g,
                             const Tree &t, bool integrate_end, unsigned long long *inter_count,
                             uint32_t *err, int num_sms, cudaStream_t st) {
    static_assert(kSortTile % 32 == 0, "chunks tile the sort tiles");
    (void)err;
    if (p.n <= p.i0) return cudaSuccess;
    if (g.tile_seg && p.i0 != 0) return cudaErrorInvalidValue;   // ranges: one simulation only
    // the chunk counter and the fallback count, zeroed in stream order
    cudaError_t e = launch_zero(t.wctr, kWWCtrWords, st);
    if (e != cudaSuccess) return e;
    const int ie = integrate_end ? 1 : 0;
    if (dims == 2)
        return inter_count ? ww_launch<2, true>(s, p, g, t, ie, inter_count, num_sms, st)
                           : ww_launch<2, false>(s, p, g, t, ie, nullptr, num_sms, st);
    return inter_count ? ww_launch<3, true>(s, p, g, t, ie, inter_count, num_sms, st)
                       : ww_launch<3, false>(s, p, g, t, ie, nullptr, num_sms, st);
}

}  // namespace ge
