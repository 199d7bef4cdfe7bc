// ge_sph.cu -- the SPH neighbour grid: hashed cell keys of the particles,
// entries sorted by key, and the first entry of every key.
//
// Reference: SPH::newGridGPU (GalaxyEngine/include/Physics/SPH.h:533-590), GL
// compute shaders run in order:
//   neighborSearchCompute (:101-152): cell = (int(floor(x / cellSize)),
//     int(floor(y / cellSize))); key = (uint(cx * 73856093) ^ uint(cy * 19349663))
//     % hashTableSize (int products wrap modulo 2^32); entry i = {key, i, cx, cy};
//   bitonicSortCompute (:247-296) driven by gpuBitonicSort (:337-367): the
//     entries sorted by key (a compare-exchange network over the next power
//     of two; equal keys end in the network's order);
//   offsetsResetCompute + offsetCompute (:369-400, :455-470, gpuOffsets
//     :503-531): offsets[key] = first entry of the key, UINT32_MAX for keys
//     that no particle has.
// Here the sort is this library's stable one-sweep radix pass (ge_sort.cu)
// over the words (key << 28 | i): the sorted keys and the offsets are the
// reference's exactly, and a key's entries come in increasing particle
// order (the bitonic network leaves them in an order of its own; no
// consumer depends on it).  The division is IEEE (correctly rounded) and the
// float-to-int conversion saturates (the shader's is undefined out of range).
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

namespace {

constexpr int kGridThreads = 256;
constexpr int kRadixG = 256;

__device__ __forceinline__ void cell_of(float x, float y, float cell, int32_t &cx, int32_t &cy) {
    cx = __float2int_rd(fdiv(x, cell));
    cy = __float2int_rd(fdiv(y, cell));
}

__device__ __forceinline__ uint32_t hash_cell(int32_t cx, int32_t cy, uint32_t table) {
    return (((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u)) % table;
}

// words (key << 28 | i) of particles [lo, lo + n) and the digit histograms of
// the sort's passes; clears the passes' look-back words and tile counters
__global__ void __launch_bounds__(kGridThreads)
k_cell_keys(const float *__restrict__ x, const float *__restrict__ y, uint32_t lo, int n,
            float cell, uint32_t table, int passes, uint64_t *words, uint32_t *hist,
            uint32_t *status, int64_t status_words, uint32_t *tile_ctr) {
    __shared__ uint32_t sh[3][kRadixG];
    for (int k = threadIdx.x; k < 3 * kRadixG; k += blockDim.x) (&sh[0][0])[k] = 0u;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < status_words;
         k += (int64_t)gridDim.x * blockDim.x)
        status[k] = 0u;
    if (blockIdx.x == 0 && threadIdx.x < 8) tile_ctr[threadIdx.x] = 0u;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int32_t cx, cy;
        cell_of(x[lo + i], y[lo + i], cell, cx, cy);
        const uint64_t key = hash_cell(cx, cy, table);
        words[i] = (key << 28) | (uint64_t)i;
        for (int ps = 0; ps < passes; ps++) atomicAdd(&sh[ps][(key >> (8 * ps)) & 0xFFu], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < passes * kRadixG; k += blockDim.x) {
        const uint32_t c = (&sh[0][0])[k];
        if (c) atomicAdd(&hist[k], c);
    }
}

__global__ void k_cell_out(const uint64_t *__restrict__ words, int n, const float *__restrict__ x,
                           const float *__restrict__ y, uint32_t lo, float cell, uint32_t table,
                           uint32_t *keys, uint32_t *index, int32_t *cell_x, int32_t *cell_y,
                           uint32_t *offsets) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint64_t w = words[k];
        const uint32_t key = (uint32_t)(w >> 28), i = (uint32_t)(w & 0x0FFFFFFFull);
        if (i >= (uint32_t)n || key >= table) continue;   // only after a failed sort (error word set)
        keys[k] = key;
        index[k] = i;
        int32_t cx, cy;
        cell_of(x[lo + i], y[lo + i], cell, cx, cy);
        cell_x[k] = cx;
        cell_y[k] = cy;
        if (k == 0 || (uint32_t)(words[k - 1] >> 28) != key) offsets[key] = (uint32_t)k;
    }
}

}  // namespace

int sph_grid_passes(uint32_t table) {
    return table <= 256u ? 1 : table <= 65536u ? 2 : 3;
}

cudaError_t launch_sph_grid(const State &s, uint32_t lo, int n, float cell, uint32_t table,
                            SortScratch &ss, uint32_t *err, uint32_t *keys, uint32_t *index,
                            int32_t *cell_x, int32_t *cell_y, uint32_t *offsets, int num_sms,
                            cudaStream_t st) {
    const int passes = sph_grid_passes(table);
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    cudaError_t e = cudaMemsetAsync(ss.hist, 0, sizeof(uint32_t) * kRadixG * passes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(offsets, 0xFF, sizeof(uint32_t) * table, st);
    if (e != cudaSuccess) return e;
    int blocks = (n + kGridThreads - 1) / kGridThreads;
    if (blocks > num_sms * 8) blocks = num_sms * 8;
    if (blocks < 1) blocks = 1;
    k_cell_keys<<<blocks, kGridThreads, 0, st>>>(s.x, s.y, lo, n, cell, table, passes, ss.keys[0],
                                                 ss.hist, ss.status, passes * tiles * kRadixG,
                                                 ss.tile_ctr);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int cur = 0;
    if ((e = launch_radix_words(ss.keys, n, 28, passes, ss.hist, ss.status, ss.tile_ctr, err, &cur,
                                st)) != cudaSuccess)
        return e;
    k_cell_out<<<blocks, kGridThreads, 0, st>>>(ss.keys[cur], n, s.x, s.y, lo, cell, table, keys,
                                                index, cell_x, cell_y, offsets);
    return cudaGetLastError();
}

}  // namespace ge
