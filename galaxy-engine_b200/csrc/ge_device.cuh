// ge_device.cuh -- shared device helpers for the Barnes-Hut step kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

// First statement of a kernel launched with launch_dep: wait until the kernel
// before it in the stream has finished and its writes are visible (a no-op
// when the launch was an ordinary one).
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

namespace ge {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kMaxLevels = 192;          // tree depth limit (size halves per level)
constexpr uint32_t kSpinLimit = 1u << 22; // bounded device-side waits

// device error word bits (ctx->d_err); the host turns them into ge_status
enum : uint32_t {
    kErrNodeCap = 1u,     // node array full
    kErrDepth = 2u,       // more than kMaxLevels levels
    kErrStack = 4u,       // walk stack overflow
    kErrSpin = 8u,        // a bounded wait gave up
};

// IEEE single operations that must not be contracted into FMA: the tree
// arithmetic and the opening test reproduce the reference's own rounding.
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// glm::min / glm::max on one component: (b < a) ? b : a and (a < b) ? b : a
__device__ __forceinline__ float ref_min(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float ref_max(float a, float b) { return (a < b) ? b : a; }

// v += t with Kahan compensation c (the running error of v, subtracted from
// the next addend)
__device__ __forceinline__ void kahan_add(float &v, float &c, float t) {
    const float y = fsub(t, c);
    const float s = fadd(v, y);
    c = fsub(fsub(s, v), y);
    v = s;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ void set_err(uint32_t *err, uint32_t bit) {
    if (err) atomicOr(err, bit);
}

// Interleave helpers for Morton keys (bit b of v -> bit 2b / 3b).
__device__ __forceinline__ uint64_t spread2(uint64_t v) {
    v &= 0x3FFFFull;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
}
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x001F00000000FFFFull;
    v = (v | (v << 16)) & 0x001F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// Morton::scaleToGrid (morton.cpp:3-10) and scaleToGrid3D (:67-75) with the
// same IEEE operations: clamp, (p - lo) / (hi - lo), * scale, truncate.
__device__ __forceinline__ uint64_t scale_to_grid(float p, float lo, float hi, float scale,
                                                  uint64_t qmax) {
    if (hi <= lo) return 0;
    float c = (p < lo) ? lo : ((hi < p) ? hi : p);
    float u = fdiv(fsub(c, lo), fsub(hi, lo));
    uint64_t q = __float2ull_rz(fmul(u, scale));
    return q < qmax ? q : qmax;
}

}  // namespace ge
