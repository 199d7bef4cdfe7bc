// ge_field.cu -- the gravity field display, as CUDA.
//
// The reference draws a "gravity field" over the 2D domain with two GL
// shaders (include/Physics/field.h): a compute shader (fieldGravityCompute,
// field.h:106-160) gives every cell the sum over the particles of
// G * (10 m_j) / dist^2, dist^2 = |p_j - cell corner|^2 + softness^2 (the
// minimum image when periodic, only for dist > 1e-4), and a fragment shader
// (fieldFragmentShader, field.h:165-222) maps that strength to a colour:
// clamp to [0, threshold], normalise, stretch s = log(1 + n k) / log(1 + k),
// then either mix(low, high, s) * s * exposure or an HSV ramp (hue
// (1 - s) * 240 degrees, value s).  The cells are laid out as
// Field::initializeCells (field.h:59-80): size = min(domain) / res, index
// j + i * amountY, corner (i, j) * size.  This box has no graphics stack, so
// both shaders run here as one kernel over the resident particles; the
// picture is an RGBA8 buffer (one pixel per cell) instead of a window.
// Every operation is the IEEE single operation in the shaders' order.
#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kFieldThreads = 256;

__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

__device__ __forceinline__ uint32_t to_unorm8(float v) {
    return (uint32_t)__float2int_rn(fmul(clamp01(v), 255.0f));
}

__global__ void __launch_bounds__(kFieldThreads)
k_field(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ m,
        uint32_t lo, uint32_t hi, int amount_x, int amount_y, float cell, float G, float soft2,
        int periodic, float dom_x, float dom_y, ge_field_params fp, float *__restrict__ strength,
        uint32_t *__restrict__ rgba) {
    __shared__ float3 tile[kFieldThreads];
    const int cells = amount_x * amount_y;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = c < cells;
    const int ci = ok ? c / amount_y : 0, cj = ok ? c % amount_y : 0;
    const float cx = fmul((float)ci, cell), cy = fmul((float)cj, cell);
    float force = 0.0f;
    for (uint32_t base = lo; base < hi; base += kFieldThreads) {
        __syncthreads();
        const uint32_t j = base + threadIdx.x;
        if (j < hi) tile[threadIdx.x] = make_float3(x[j], y[j], m[j]);
        __syncthreads();
        const int cnt = (int)min((uint32_t)kFieldThreads, hi - base);
        for (int k = 0; k < cnt; k++) {
            const float3 q = tile[k];
            float dx = fsub(q.x, cx), dy = fsub(q.y, cy);
            if (periodic) {   // d -= domainSize * round(d / domainSize)
                dx = fsub(dx, fmul(dom_x, roundf(fdiv(dx, dom_x))));
                dy = fsub(dy, fmul(dom_y, roundf(fdiv(dy, dom_y))));
            }
            const float d2 = fadd(fadd(fmul(dx, dx), fmul(dy, dy)), soft2);
            const float dist = __fsqrt_rn(d2);
            if (dist > 0.0001f)
                force = fadd(force, fdiv(fmul(G, fmul(q.z, 10.0f)), fmul(dist, dist)));
        }
    }
    if (!ok) return;
    if (strength) strength[c] = force;
    if (!rgba) return;
    const float clamped = fminf(fmaxf(force, 0.0f), fp.threshold);
    const float nrm = fdiv(clamped, fp.threshold);
    const float s = fdiv(logf(fadd(1.0f, fmul(nrm, fp.stretch))), logf(fadd(1.0f, fp.stretch)));
    float col[3];
    if (fp.two_color) {
        for (int a = 0; a < 3; a++) {
            // mix(low, high, s) = low * (1 - s) + high * s
            const float base = fadd(fmul(fp.color_low[a], fsub(1.0f, s)), fmul(fp.color_high[a], s));
            col[a] = fmul(fmul(base, s), fp.exposure);
        }
    } else {
        // hsv2rgb(vec3(hue / 360, 1, s)), hue = (1 - s) * 240
        const float h = fdiv(fmul(fsub(1.0f, s), 240.0f), 360.0f);
        const float K[3] = {1.0f, 2.0f / 3.0f, 1.0f / 3.0f};
        for (int a = 0; a < 3; a++) {
            const float f = fadd(h, K[a]);
            const float fr = fsub(f, floorf(f));
            const float pp = fabsf(fsub(fmul(fr, 6.0f), 3.0f));
            const float t = clamp01(fsub(pp, 1.0f));
            col[a] = fmul(s, t);   // c.z * mix(K.xxx, t, c.y) with c.y = 1
        }
    }
    rgba[c] = to_unorm8(col[0]) | (to_unorm8(col[1]) << 8) | (to_unorm8(col[2]) << 16) | (255u << 24);
}

cudaError_t launch_field(const State &s, uint32_t lo, uint32_t hi, int amount_x, int amount_y,
                         float cell, float G, float soft2, int periodic, float dom_x, float dom_y,
                         const ge_field_params &fp, float *strength, uint32_t *rgba,
                         cudaStream_t st) {
    const int cells = amount_x * amount_y;
    const int blocks = (cells + kFieldThreads - 1) / kFieldThreads;
    if (blocks < 1) return cudaSuccess;
    k_field<<<blocks, kFieldThreads, 0, st>>>(s.x, s.y, s.m, lo, hi, amount_x, amount_y, cell, G,
                                              soft2, periodic, dom_x, dom_y, fp, strength, rgba);
    return cudaGetLastError();
}

}  // namespace ge
