// ge_integrate.cu -- leapfrog halves and the bounding boxes.
//
// integrateStart (GalaxyEngine/src/Physics/physics.cpp:1069-1112,
// physics3D.cpp:740-804) is fused with boundingBox (globalLogic.cpp:1083-1099,
// :1460-1477): the drift writes the positions the box is taken over, so one
// pass reads x, v, a once and writes x, v.  Min and max are exact in any
// order; each segment (independent simulation) keeps its own min/max as
// order-preserving integer words updated with atomics, one update per block
// when a block lies inside one segment.  A second small kernel then applies
// the reference's float formula for the square (cubic) root box of every
// segment, seeds each segment's root node and resets the words.
#include <cfloat>

#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kBoxBatch = 4;    // particles of a thread loaded together, before any store

// float <-> unsigned with the same order (negative floats reversed)
__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// pos, vel, acc: particle i's, already loaded
template <int D>
__device__ __forceinline__ void kick_drift(const State &s, const StepParams &p, int i,
                                           float *pos, float *vel, const float *acc) {
    if (s.pvx) {
        s.pvx[i] = vel[0]; s.pvy[i] = vel[1];
        if (D == 3) s.pvz[i] = vel[2];
    }
    if (s.kx) {
        // GE_PREC_MIXED: both updates Kahan-compensated
        float *kp[3] = {s.kx, s.ky, s.kz}, *kv[3] = {s.kvx, s.kvy, s.kvz};
#pragma unroll
        for (int a = 0; a < D; a++) {
            float cv = kv[a][i], cp = kp[a][i];
            kahan_add(vel[a], cv, fmul(acc[a], p.half_dt));
            kahan_add(pos[a], cp, fmul(vel[a], p.dt));
            kv[a][i] = cv;
            kp[a][i] = cp;
        }
    } else {
#pragma unroll
        for (int a = 0; a < D; a++) {
            vel[a] = fadd(vel[a], fmul(acc[a], p.half_dt));   // vel += acc * halfDt
            pos[a] = fadd(pos[a], fmul(vel[a], p.dt));         // pos += vel * dt
        }
    }
    if (p.periodic) {
        if (D == 2) {
            // physics.cpp:1104-1110: domain [0, size)
#pragma unroll
            for (int a = 0; a < 2; a++) {
                if (pos[a] < 0.0f) pos[a] = fadd(pos[a], p.domain[a]);
                else if (pos[a] >= p.domain[a]) pos[a] = fsub(pos[a], p.domain[a]);
            }
        } else {
            // physics3D.cpp:785-802: domain [-size/2, size/2)
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (pos[a] < -p.half_domain[a]) pos[a] = fadd(pos[a], p.domain[a]);
                else if (pos[a] >= p.half_domain[a]) pos[a] = fsub(pos[a], p.domain[a]);
            }
        }
    }
    s.x[i] = pos[0]; s.y[i] = pos[1];
    s.vx[i] = vel[0]; s.vy[i] = vel[1];
    if (D == 3) { s.z[i] = pos[2]; s.vz[i] = vel[2]; }
}

template <int D>
__global__ void __launch_bounds__(kBBoxThreads)
k_kick_drift_box(State s, StepParams p, int kick, Segs g) {
    dep_wait();
    const uint32_t n = (uint32_t)p.n;
    constexpr uint32_t TILE = kBBoxThreads * kBoxItems;
    __shared__ float s_lo[kBBoxThreads / 32][3], s_hi[kBBoxThreads / 32][3];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * TILE; base < n; base += gridDim.x * TILE) {
        const uint32_t last = min(base + TILE, n) - 1;
        const uint32_t seg0 = g.seg_of ? g.seg_of[base] : 0u;
        const bool one = !g.seg_of || g.seg_of[last] == seg0;
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
#pragma unroll 1
        for (int it0 = 0; it0 < kBoxItems; it0 += kBoxBatch) {
          // the batch's loads first: stores to the state arrays would
          // otherwise keep the next particle's loads behind them
          float pos[kBoxBatch][3], vel[kBoxBatch][3], acc[kBoxBatch][3];
          bool mv[kBoxBatch];
#pragma unroll
          for (int u = 0; u < kBoxBatch; u++) {
            const uint32_t i = base + (it0 + u) * kBBoxThreads + threadIdx.x;
            mv[u] = false;
            pos[u][0] = pos[u][1] = pos[u][2] = 0.0f;
            vel[u][0] = vel[u][1] = vel[u][2] = 0.0f;
            acc[u][0] = acc[u][1] = acc[u][2] = 0.0f;
            if (i < n) {
                pos[u][0] = s.x[i]; pos[u][1] = s.y[i];
                if (D == 3) pos[u][2] = s.z[i];
                mv[u] = kick && !(s.pinned && s.pinned[i]);
                if (kick) {
                    vel[u][0] = s.vx[i]; vel[u][1] = s.vy[i];
                    acc[u][0] = s.ax[i]; acc[u][1] = s.ay[i];
                    if (D == 3) { vel[u][2] = s.vz[i]; acc[u][2] = s.az[i]; }
                }
            }
          }
#pragma unroll
          for (int u = 0; u < kBoxBatch; u++) {
            const uint32_t i = base + (it0 + u) * kBBoxThreads + threadIdx.x;
            if (i >= n) break;
            if (mv[u]) kick_drift<D>(s, p, (int)i, pos[u], vel[u], acc[u]);
            if (one) {
#pragma unroll
                for (int a = 0; a < D; a++) {
                    lo[a] = ref_min(lo[a], pos[u][a]);
                    hi[a] = ref_max(hi[a], pos[u][a]);
                }
            } else {
                // the tile straddles segments: update this particle's segment
                const uint32_t sg = g.seg_of[i];
#pragma unroll
                for (int a = 0; a < D; a++) {
                    atomicMin(&g.boxmm[sg * 6 + a], f2o(pos[u][a]));
                    atomicMax(&g.boxmm[sg * 6 + 3 + a], f2o(pos[u][a]));
                }
            }
          }
        }
        if (one) {   // uniform across the block
#pragma unroll
            for (int a = 0; a < D; a++) {
                for (int o = 16; o > 0; o >>= 1) {
                    lo[a] = ref_min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
                    hi[a] = ref_max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
                }
            }
            if (lane == 0)
                for (int a = 0; a < D; a++) { s_lo[w][a] = lo[a]; s_hi[w][a] = hi[a]; }
            __syncthreads();
            if (threadIdx.x < D) {
                const int a = threadIdx.x;
                float l = FLT_MAX, h = -FLT_MAX;
                for (int ww = 0; ww < kBBoxThreads / 32; ww++) {
                    l = ref_min(l, s_lo[ww][a]);
                    h = ref_max(h, s_hi[ww][a]);
                }
                atomicMin(&g.boxmm[seg0 * 6 + a], f2o(l));
                atomicMax(&g.boxmm[seg0 * 6 + 3 + a], f2o(h));
            }
            __syncthreads();
        }
    }
}

// Per segment: boundingBox() / boundingBox3D() from the min/max, root node
// seeding, and the min/max words reset for the next step.
template <int D>
__global__ void k_finalize_boxes(Segs g, Tree t, uint32_t n) {
    dep_wait();
    const int sgi = blockIdx.x * blockDim.x + threadIdx.x;
    if (sgi >= g.S) return;
    const uint32_t sg = (uint32_t)sgi;
    float l[3], h[3];
    for (int a = 0; a < 3; a++) {
        l[a] = a < D ? o2f(g.boxmm[sg * 6 + a]) : 0.0f;
        h[a] = a < D ? o2f(g.boxmm[sg * 6 + 3 + a]) : 0.0f;
        g.boxmm[sg * 6 + a] = 0xFFFFFFFFu;       // identity of min
        g.boxmm[sg * 6 + 3 + a] = 0u;            // identity of max
    }
    float size = ref_max(fsub(h[0], l[0]), fsub(h[1], l[1]));
    if (D == 3) size = ref_max(size, fsub(h[2], l[2]));
    const float half = fmul(size, 0.5f);
    float4 bb;
    bb.x = fsub(fmul(fadd(l[0], h[0]), 0.5f), half);
    bb.y = fsub(fmul(fadd(l[1], h[1]), 0.5f), half);
    bb.z = D == 3 ? fsub(fmul(fadd(l[2], h[2]), 0.5f), half) : 0.0f;
    bb.w = size;
    g.box[sg] = bb;
    // root node of segment sg: cell = box, particle range = the segment
    t.cell[sg] = bb;
    t.info[sg] = make_uint4(0u, 0u, seg_lo(g, sg), seg_hi(g, sg, n));
}

__global__ void k_reset_boxmm(uint32_t *boxmm, int S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S * 6) boxmm[i] = (i % 6) < 3 ? 0xFFFFFFFFu : 0u;
}

template <int D>
__global__ void k_integrate_end(State s, StepParams p) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        if (s.pinned && s.pinned[i]) continue;
        if (s.kvx) {
            kahan_add(s.vx[i], s.kvx[i], fmul(s.ax[i], p.half_dt));
            kahan_add(s.vy[i], s.kvy[i], fmul(s.ay[i], p.half_dt));
            if (D == 3) kahan_add(s.vz[i], s.kvz[i], fmul(s.az[i], p.half_dt));
            continue;
        }
        s.vx[i] = fadd(s.vx[i], fmul(s.ax[i], p.half_dt));
        s.vy[i] = fadd(s.vy[i], fmul(s.ay[i], p.half_dt));
        if (D == 3) s.vz[i] = fadd(s.vz[i], fmul(s.az[i], p.half_dt));
    }
}

// largest s in [0, S) with tab[s] <= v (tab ascending, tab[0] = 0)
__device__ __forceinline__ uint32_t upper_seg(const uint32_t *tab, int S, uint32_t v) {
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&tab[mid]) <= v) lo = mid;
        else hi = mid - 1;
    }
    return (uint32_t)lo;
}

__global__ void k_seg_tables(const uint32_t *off, const uint32_t *tile_base, int S, int n,
                             int64_t tiles, uint32_t *seg_of, uint32_t *tile_seg) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
        seg_of[i] = upper_seg(off, S, (uint32_t)i);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tiles; i += stride)
        tile_seg[i] = upper_seg(tile_base, S, (uint32_t)i);
}

cudaError_t launch_seg_tables(const uint32_t *off, const uint32_t *tile_base, int S, int n,
                              int64_t tiles, uint32_t *seg_of, uint32_t *tile_seg,
                              cudaStream_t st) {
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    k_seg_tables<<<blocks, 256, 0, st>>>(off, tile_base, S, n, tiles, seg_of, tile_seg);
    return cudaGetLastError();
}

cudaError_t launch_reset_boxes(const Segs &g, cudaStream_t st) {
    const int cnt = g.S * 6;
    k_reset_boxmm<<<(cnt + 255) / 256, 256, 0, st>>>(g.boxmm, g.S);
    return cudaGetLastError();
}

cudaError_t launch_kick_drift_bbox(int dims, const State &s, const StepParams &p, bool kick_drift,
                                   const Segs &g, SortScratch &ss, Tree &t, cudaStream_t st) {
    const int blocks = ss.box_blocks;
    const int kd = kick_drift ? 1 : 0;
    cudaError_t e = dims == 2 ? launch_dep(k_kick_drift_box<2>, blocks, kBBoxThreads, st, s, p, kd, g)
                              : launch_dep(k_kick_drift_box<3>, blocks, kBBoxThreads, st, s, p, kd, g);
    if (e != cudaSuccess) return e;
    const int fb = (g.S + 127) / 128;
    const uint32_t nn = (uint32_t)p.n;
    return dims == 2 ? launch_dep(k_finalize_boxes<2>, fb, 128, st, g, t, nn)
                     : launch_dep(k_finalize_boxes<3>, fb, 128, st, g, t, nn);
}

cudaError_t launch_integrate_end(int dims, const State &s, const StepParams &p, cudaStream_t st) {
    int blocks = (p.n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    if (dims == 2) k_integrate_end<2><<<blocks, 256, 0, st>>>(s, p);
    else k_integrate_end<3><<<blocks, 256, 0, st>>>(s, p);
    return cudaGetLastError();
}

}  // namespace ge
