// ge_aos.cu -- the reference's particle records (array of structures) in and
// out of the resident structure-of-arrays state.
//
// Reference: the records are ParticlePhysics / ParticlePhysics3D and
// ParticleRendering / ParticleRendering3D (GalaxyEngine/include/Particles/
// particle.h:5-277); Physics::flattenParticles (src/Physics/physics.cpp:
// 354-390) copies their gravity members into SoA vectors before the walk and
// Physics::readFlattenBack (:542-565) copies them back.  Here the records
// travel to the device as they are (one contiguous copy), k_aos_in takes the
// members out into the state, and after the frame k_aos_out writes the
// updated members back into each particle's own record (its index before the
// frame's Morton sort), so the caller's arrays keep their order.
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

__device__ __forceinline__ float rd(const unsigned char *r, int off) {
    return *reinterpret_cast<const float *>(r + off);
}
__device__ __forceinline__ void wr(unsigned char *r, int off, float v) {
    *reinterpret_cast<float *>(r + off) = v;
}

template <int D>
__global__ void __launch_bounds__(256)
k_aos_in(const unsigned char *__restrict__ phys, const unsigned char *__restrict__ rend,
         AosLayout L, int n, State s) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const unsigned char *r = phys + (size_t)k * L.stride;
        float *pos[3] = {s.x, s.y, s.z}, *vel[3] = {s.vx, s.vy, s.vz}, *acc[3] = {s.ax, s.ay, s.az};
        float *pv[3] = {s.pvx, s.pvy, s.pvz};
#pragma unroll
        for (int a = 0; a < D; a++) {
            pos[a][k] = rd(r, L.off_pos + 4 * a);
            const float v = rd(r, L.off_vel + 4 * a);
            vel[a][k] = v;
            acc[a][k] = rd(r, L.off_acc + 4 * a);
            if (pv[0]) pv[a][k] = v;   // as ge_upload: prevVel starts at the velocity
        }
        s.m[k] = rd(r, L.off_mass);
        s.id[k] = *reinterpret_cast<const uint32_t *>(r + L.off_id);
        if (s.temp && L.off_temp >= 0) s.temp[k] = rd(r, L.off_temp);
        if (s.pinned && rend) s.pinned[k] = rend[(size_t)k * L.r_stride + L.r_off_pinned] ? 1 : 0;
    }
}

template <int D>
__global__ void __launch_bounds__(256)
k_aos_out(unsigned char *__restrict__ phys, AosLayout L, int n, State s,
          const uint64_t *__restrict__ keys, const uint32_t *__restrict__ vals) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        // the slot each particle held before the frame's sort = its record
        uint32_t j = D == 2 ? (uint32_t)(keys[k] & 0x0FFFFFFFull) : vals[k];
        if (j >= (uint32_t)n) continue;   // only after a failed sort (error word set)
        unsigned char *r = phys + (size_t)j * L.stride;
        const float *pos[3] = {s.x, s.y, s.z}, *vel[3] = {s.vx, s.vy, s.vz},
                    *acc[3] = {s.ax, s.ay, s.az}, *pv[3] = {s.pvx, s.pvy, s.pvz};
#pragma unroll
        for (int a = 0; a < D; a++) {
            wr(r, L.off_pos + 4 * a, pos[a][k]);
            wr(r, L.off_vel + 4 * a, vel[a][k]);
            wr(r, L.off_acc + 4 * a, acc[a][k]);
            if (pv[0] && L.off_prev_vel >= 0) wr(r, L.off_prev_vel + 4 * a, pv[a][k]);
        }
        if (s.temp && L.off_temp >= 0) wr(r, L.off_temp, s.temp[k]);
    }
}

static int aos_grid(int n) {
    int b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return b < 1 ? 1 : b;
}

cudaError_t launch_aos_in(int dims, const unsigned char *phys, const unsigned char *rend,
                          const AosLayout &L, int n, const State &s, cudaStream_t st) {
    if (dims == 2) k_aos_in<2><<<aos_grid(n), 256, 0, st>>>(phys, rend, L, n, s);
    else k_aos_in<3><<<aos_grid(n), 256, 0, st>>>(phys, rend, L, n, s);
    return cudaGetLastError();
}

cudaError_t launch_aos_out(int dims, unsigned char *phys, const AosLayout &L, int n,
                           const State &s, const SortScratch &ss, cudaStream_t st) {
    if (dims == 2) k_aos_out<2><<<aos_grid(n), 256, 0, st>>>(phys, L, n, s, ss.keys[0], ss.vals[0]);
    else k_aos_out<3><<<aos_grid(n), 256, 0, st>>>(phys, L, n, s, ss.keys[0], ss.vals[0]);
    return cudaGetLastError();
}

}  // namespace ge
