// ge_diag.cu -- FP64 diagnostics: direct-sum accelerations for sampled
// particles (the accuracy reference every result is stated against) and
// energy / momentum sums.
//
// The direct sum adds eps2 to r^2 exactly as the tree walk does and skips
// j == i; it does not use the tree.  One thread per sampled target, sources
// staged through shared memory in tiles.
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kDiagThreads = 256;

template <int D>
__global__ void __launch_bounds__(kDiagThreads)
k_direct_f64(State s, int n, Segs g, const uint32_t *__restrict__ idx, int nt, double G,
             double eps2, double *__restrict__ out) {
    __shared__ float4 tile[kDiagThreads];
    __shared__ uint32_t s_lo, s_hi;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = t < nt;
    uint32_t i = ok ? idx[t] : 0u;
    if (i >= (uint32_t)n) i = 0u;
    // sources: the target's own segment; the block walks the union of its
    // targets' segments
    const uint32_t sg = g.seg_of ? g.seg_of[i] : 0u;
    const uint32_t lo = seg_lo(g, sg), hi = seg_hi(g, sg, (uint32_t)n);
    if (threadIdx.x == 0) { s_lo = 0xFFFFFFFFu; s_hi = 0u; }
    __syncthreads();
    if (ok) { atomicMin(&s_lo, lo); atomicMax(&s_hi, hi); }
    __syncthreads();
    const int blo = (int)s_lo, bhi = (int)s_hi;
    const double xi = s.x[i], yi = s.y[i], zi = D == 3 ? (double)s.z[i] : 0.0;
    double a[3] = {0.0, 0.0, 0.0};
    for (int base = blo; base < bhi; base += kDiagThreads) {
        const int j = base + threadIdx.x;
        __syncthreads();
        if (j < bhi) tile[threadIdx.x] = make_float4(s.x[j], s.y[j], D == 3 ? s.z[j] : 0.0f, s.m[j]);
        __syncthreads();
        const int cnt = min(kDiagThreads, bhi - base);
        for (int k = 0; k < cnt; k++) {
            const uint32_t jj = (uint32_t)(base + k);
            if (jj == i || jj < lo || jj >= hi) continue;
            const float4 q = tile[k];
            const double dx = (double)q.x - xi, dy = (double)q.y - yi;
            const double dz = D == 3 ? (double)q.z - zi : 0.0;
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            const double rs = rsqrt(r2);
            const double f = (double)q.w * rs * rs * rs;
            a[0] += dx * f;
            a[1] += dy * f;
            a[2] += dz * f;
        }
    }
    if (ok) {
        out[(size_t)t * D + 0] = G * a[0];
        out[(size_t)t * D + 1] = G * a[1];
        if (D == 3) out[(size_t)t * D + 2] = G * a[2];
    }
}

cudaError_t launch_direct_f64(int dims, const State &s, int n, const Segs &g, const uint32_t *idx,
                              int nt, double G, double eps2, double *out, cudaStream_t st) {
    const int blocks = (nt + kDiagThreads - 1) / kDiagThreads;
    if (blocks < 1) return cudaSuccess;
    if (dims == 2)
        k_direct_f64<2><<<blocks, kDiagThreads, 0, st>>>(s, n, g, idx, nt, G, eps2, out);
    else k_direct_f64<3><<<blocks, kDiagThreads, 0, st>>>(s, n, g, idx, nt, G, eps2, out);
    return cudaGetLastError();
}

// Kinetic energy, momentum and mass in FP64 (one block-level reduction per
// block, then atomics on doubles): out = {E_kin, p_x, p_y, p_z, M}.
template <int D>
__global__ void k_sums_f64(State s, int n, double *out) {
    double v[5] = {0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double m = s.m[i], vx = s.vx[i], vy = s.vy[i], vz = D == 3 ? (double)s.vz[i] : 0.0;
        v[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        v[1] += m * vx;
        v[2] += m * vy;
        v[3] += m * vz;
        v[4] += m;
    }
    for (int k = 0; k < 5; k++) {
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&out[k], v[k]);
    }
}

cudaError_t launch_sums_f64(int dims, const State &s, int n, double *out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, 5 * sizeof(double), st);
    if (e != cudaSuccess) return e;
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    if (dims == 2) k_sums_f64<2><<<blocks, 256, 0, st>>>(s, n, out);
    else k_sums_f64<3><<<blocks, 256, 0, st>>>(s, n, out);
    return cudaGetLastError();
}

}  // namespace ge
