// ge_temp.cu -- node temperatures for the walk's heat exchange.
//
// The reference sums the particles' temperatures into every node while it
// builds the tree: a leaf adds its particles in particle order
// (computeLeafMass, include/Physics/quadtree.h:53-66; 3D :159-170), an
// internal node adds its children in subGrids[x][y]([z]) order
// (computeInternalMass, quadtree.h:69-86; 3D quadtree.cpp:227-243), and the
// walk uses gridTemp / count as the node's temperature
// (physics.cpp:145-158, physics3D.cpp:190-201).  Here the same FP32 sums run
// after the build, bottom-up like the moment pass (the last child of a node
// to finish adds up its siblings), and each node's walk entry receives its
// average; each particle's entry receives its own temperature.  Both are the
// values before the walk, which the walk then reads.
#include <cuda/atomic>

#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kTempThreads = 256;
constexpr int kMetaSlotsT = 9;   // tree meta word: node slots of the last build

__global__ void k_temp_pend_init(Tree t) {
    const uint32_t slots = __ldcg(&t.meta[kMetaSlotsT]);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < slots; k += stride) {
        const uint4 inf = __ldcg(&t.info[k]);
        t.pend[k] = (inf.w > inf.z) ? (uint32_t)__popc(inf.y) : 0u;
    }
}

__global__ void k_particle_temps(State s, Tree t, uint32_t n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
        t.tv[t.slot_of[j]] = s.temp[j];
}

__device__ __forceinline__ void put_node_temp(const Tree &t, uint32_t k, float gt, uint32_t cnt) {
    t.ntemp[k] = gt;
    t.tv[__ldcg(&t.aux[k]).w] = fdiv(gt, (float)cnt);   // gridTemp / count
}

template <int D>
__global__ void __launch_bounds__(kTempThreads) k_node_temps(State s, Tree t) {
    constexpr int Q = 1 << D;
    const uint32_t slots = __ldcg(&t.meta[kMetaSlotsT]);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < slots; k += stride) {
        const uint4 inf = __ldcg(&t.info[k]);
        if (inf.w <= inf.z || inf.y != 0u) continue;   // holes and internal nodes
        float gt = 0.0f;
        for (uint32_t j = inf.z; j < inf.w; j++) gt = fadd(gt, s.temp[j]);
        put_node_temp(t, k, gt, inf.w - inf.z);
        uint32_t node = k;
        for (int lev = 0; lev < kMaxLevels; lev++) {
            const uint32_t par = __ldcg(&t.aux[node]).z;
            if (par == kEmpty) break;
            cuda::atomic_ref<uint32_t, cuda::thread_scope_device> pc(t.pend[par]);
            if (pc.fetch_sub(1u, cuda::memory_order_acq_rel) != 1u) break;
            const uint4 pinf = __ldcg(&t.info[par]);
            float sum = 0.0f;
#pragma unroll
            for (int kk = 0; kk < Q; kk++) {
                // x-major order of subGrids[x][y]([z]): child slot q has x in bit 0
                unsigned q;
                if (D == 2) q = ((kk >> 1) & 1) | ((kk & 1) << 1);
                else q = ((kk >> 2) & 1) | (((kk >> 1) & 1) << 1) | ((kk & 1) << 2);
                if (!((pinf.y >> q) & 1u)) continue;
                sum = fadd(sum, __ldcg(&t.ntemp[pinf.x + __popc(pinf.y & ((1u << q) - 1u))]));
            }
            put_node_temp(t, par, sum, pinf.w - pinf.z);
            node = par;
        }
    }
}

cudaError_t launch_node_temps(int dims, const State &s, const StepParams &p, Tree &t,
                              int num_sms, cudaStream_t st) {
    const int blocks = num_sms * 8;
    k_temp_pend_init<<<blocks, kTempThreads, 0, st>>>(t);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_particle_temps<<<blocks, kTempThreads, 0, st>>>(s, t, (uint32_t)p.n);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (dims == 2) k_node_temps<2><<<blocks, kTempThreads, 0, st>>>(s, t);
    else k_node_temps<3><<<blocks, kTempThreads, 0, st>>>(s, t);
    return cudaGetLastError();
}

}  // namespace ge
