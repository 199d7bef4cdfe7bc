// ge_integrate.cu -- leapfrog halves and the bounding box.
//
// integrateStart (GalaxyEngine/src/Physics/physics.cpp:1069-1112,
// physics3D.cpp:740-804) is fused with boundingBox (globalLogic.cpp:1083-1099,
// :1460-1477): the drift writes the positions the box is taken over, so one
// pass reads x, v, a once and writes x, v.  The min/max reduction is exact in
// any order; the last block to finish applies the reference's float formula
// for the square (cubic) root box and seeds the root node of the tree.
#include <cfloat>

#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

template <int D>
__global__ void __launch_bounds__(kBBoxThreads)
k_kick_drift_bbox(State s, StepParams p, int kick, float4 *part, uint32_t *ctr, float4 *bbox,
                  Tree t) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    const int n = p.n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float pos[3], vel[3], acc[3];
        pos[0] = s.x[i]; pos[1] = s.y[i];
        if (D == 3) pos[2] = s.z[i];
        if (kick && !(s.pinned && s.pinned[i])) {
            vel[0] = s.vx[i]; vel[1] = s.vy[i];
            acc[0] = s.ax[i]; acc[1] = s.ay[i];
            if (D == 3) { vel[2] = s.vz[i]; acc[2] = s.az[i]; }
            if (s.pvx) {
                s.pvx[i] = vel[0]; s.pvy[i] = vel[1];
                if (D == 3) s.pvz[i] = vel[2];
            }
#pragma unroll
            for (int a = 0; a < D; a++) {
                vel[a] = fadd(vel[a], fmul(acc[a], p.half_dt));   // vel += acc * halfDt
                pos[a] = fadd(pos[a], fmul(vel[a], p.dt));         // pos += vel * dt
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
#pragma unroll
        for (int a = 0; a < D; a++) {
            lo[a] = ref_min(lo[a], pos[a]);
            hi[a] = ref_max(hi[a], pos[a]);
        }
    }
    // block reduction
#pragma unroll
    for (int a = 0; a < D; a++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = ref_min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = ref_max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    __shared__ float s_lo[kBBoxThreads / 32][3], s_hi[kBBoxThreads / 32][3];
    __shared__ int s_last;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        for (int a = 0; a < D; a++) { s_lo[w][a] = lo[a]; s_hi[w][a] = hi[a]; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int ww = 1; ww < kBBoxThreads / 32; ww++)
            for (int a = 0; a < D; a++) {
                lo[a] = ref_min(lo[a], s_lo[ww][a]);
                hi[a] = ref_max(hi[a], s_hi[ww][a]);
            }
        part[2 * blockIdx.x] = make_float4(lo[0], lo[1], D == 3 ? lo[2] : 0.0f, 0.0f);
        part[2 * blockIdx.x + 1] = make_float4(hi[0], hi[1], D == 3 ? hi[2] : 0.0f, 0.0f);
        __threadfence();
        s_last = (atomicAdd(ctr, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    // last block: fold the partials
    __threadfence();
    float l[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, h[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        float4 a = __ldcg(&part[2 * b]), c = __ldcg(&part[2 * b + 1]);
        l[0] = ref_min(l[0], a.x); l[1] = ref_min(l[1], a.y); l[2] = ref_min(l[2], a.z);
        h[0] = ref_max(h[0], c.x); h[1] = ref_max(h[1], c.y); h[2] = ref_max(h[2], c.z);
    }
    for (int a = 0; a < 3; a++) {
        for (int o = 16; o > 0; o >>= 1) {
            l[a] = ref_min(l[a], __shfl_xor_sync(0xffffffffu, l[a], o));
            h[a] = ref_max(h[a], __shfl_xor_sync(0xffffffffu, h[a], o));
        }
    }
    __syncthreads();
    if (lane == 0) {
        for (int a = 0; a < 3; a++) { s_lo[w][a] = l[a]; s_hi[w][a] = h[a]; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int ww = 1; ww < kBBoxThreads / 32; ww++)
            for (int a = 0; a < 3; a++) {
                l[a] = ref_min(l[a], s_lo[ww][a]);
                h[a] = ref_max(h[a], s_hi[ww][a]);
            }
        float size = ref_max(fsub(h[0], l[0]), fsub(h[1], l[1]));
        if (D == 3) size = ref_max(size, fsub(h[2], l[2]));
        float half = fmul(size, 0.5f);
        float4 bb;
        bb.x = fsub(fmul(fadd(l[0], h[0]), 0.5f), half);
        bb.y = fsub(fmul(fadd(l[1], h[1]), 0.5f), half);
        bb.z = D == 3 ? fsub(fmul(fadd(l[2], h[2]), 0.5f), half) : 0.0f;
        bb.w = size;
        *bbox = bb;
        // root node of the tree: cell = box, particle range [0, n)
        t.cell[0] = bb;
        t.info[0] = make_uint4(0u, 0u, 0u, (uint32_t)n);
        *ctr = 0u;
    }
}

template <int D>
__global__ void k_integrate_end(State s, StepParams p) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        if (s.pinned && s.pinned[i]) continue;
        s.vx[i] = fadd(s.vx[i], fmul(s.ax[i], p.half_dt));
        s.vy[i] = fadd(s.vy[i], fmul(s.ay[i], p.half_dt));
        if (D == 3) s.vz[i] = fadd(s.vz[i], fmul(s.az[i], p.half_dt));
    }
}

cudaError_t launch_kick_drift_bbox(int dims, const State &s, const StepParams &p, bool kick_drift,
                                   SortScratch &ss, Tree &t, uint32_t *err, cudaStream_t st) {
    (void)err;
    int blocks = ss.bbox_blocks;
    if (dims == 2)
        k_kick_drift_bbox<2><<<blocks, kBBoxThreads, 0, st>>>(s, p, kick_drift, ss.bbox_part,
                                                              ss.bbox_ctr, ss.bbox, t);
    else
        k_kick_drift_bbox<3><<<blocks, kBBoxThreads, 0, st>>>(s, p, kick_drift, ss.bbox_part,
                                                              ss.bbox_ctr, ss.bbox, t);
    return cudaGetLastError();
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
