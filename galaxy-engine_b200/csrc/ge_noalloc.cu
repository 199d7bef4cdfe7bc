// ge_noalloc.cu -- 2D Morton-key sort that allocates no device memory.
//
// Callers that cannot allocate device memory use this entry point: for
// example a host application whose device memory is carved up front into a
// fixed arena under its own accounting, or a frame loop that must not call
// cudaMalloc / cudaFree (both can synchronise the whole device and stall
// the frame).  They pass device buffers for the inputs and outputs; every
// temporary the sort needs (box min/max words, packed keys in two ping-pong
// buffers, digit histograms, look-back words) lives in one file-scope
// __device__ array of fixed size, which each GPU that loads the library
// holds until the process exits.
//
// The work is the same as ge_compute_morton_keys + ge_sort_by_morton_key on
// a context (bounding box, Morton keys, stable radix sort) and runs the same
// kernels; only the scratch differs.
#include <mutex>

#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {
namespace {

constexpr int64_t kNoAllocMaxN = GE_NOALLOC_MAX_N;
constexpr int64_t kNoAllocTiles = (kNoAllocMaxN + kSortTile - 1) / kSortTile;

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
// byte offsets inside the scratch array
constexpr size_t kOffKeys0 = 0;
constexpr size_t kOffKeys1 = kOffKeys0 + align256(sizeof(uint64_t) * kNoAllocMaxN);
constexpr size_t kOffHist = kOffKeys1 + align256(sizeof(uint64_t) * kNoAllocMaxN);
// digit histograms and look-back words: the sort's words per segment / tile
constexpr size_t kOffStatus = kOffHist + align256(sizeof(uint32_t) * kSortDigitWords);
constexpr size_t kOffTileCtr = kOffStatus + align256(sizeof(uint32_t) * kSortDigitWords * kNoAllocTiles);
constexpr size_t kOffBox = kOffTileCtr + align256(sizeof(uint32_t) * 8);
constexpr size_t kOffBoxMM = kOffBox + align256(sizeof(float4));
constexpr size_t kOffRootCell = kOffBoxMM + align256(sizeof(uint32_t) * 6);
constexpr size_t kOffRootInfo = kOffRootCell + align256(sizeof(float4));
constexpr size_t kOffErr = kOffRootInfo + align256(sizeof(uint4));
constexpr size_t kScratchBytes = kOffErr + align256(sizeof(uint32_t));

// All calls on a device share this array (about 5.1 MB).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
static unsigned char *g_scratch_dev[kMaxDevices];
static int g_sms_dev[kMaxDevices];   // SM count of each device (sizes the box grid)
static std::mutex g_scratch_mu;

// Device address of the scratch array on the current device, and that
// device's SM count.  In host code the array's name is only a host-side
// stand-in, so the address must come from cudaGetSymbolAddress, made once per
// device with that device current.
cudaError_t scratch_for_current_device(unsigned char **out, int *sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_dev[dev]) {
        int count = 0;
        e = cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_sms_dev[dev] = count > 0 ? count : 1;
        g_scratch_dev[dev] = (unsigned char *)p;
    }
    *out = g_scratch_dev[dev];
    *sms = g_sms_dev[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace ge

using namespace ge;

extern "C" int ge_morton_sort_2d_noalloc(int64_t n, const float *d_x, const float *d_y,
                                         uint32_t *d_perm, uint64_t *d_keys, void *stream) {
    if (n < 1 || !d_x || !d_y || !d_perm) return GE_ERR_ARG;
    if (n > kNoAllocMaxN) return GE_ERR_CAPACITY;
    unsigned char *base = nullptr;
    int sms = 0;
    if (scratch_for_current_device(&base, &sms) != cudaSuccess) return GE_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;

    SortScratch ss{};
    ss.keys[0] = (uint64_t *)(base + kOffKeys0);
    ss.keys[1] = (uint64_t *)(base + kOffKeys1);
    ss.vals[0] = ss.vals[1] = nullptr;
    ss.hist = (uint32_t *)(base + kOffHist);
    ss.status = (uint32_t *)(base + kOffStatus);
    ss.tile_ctr = (uint32_t *)(base + kOffTileCtr);
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    // the box grid as a context sizes it: one block per kBBoxThreads *
    // kBoxItems particles, at most four per SM
    int64_t blocks = (n + kBBoxThreads * kBoxItems - 1) / (kBBoxThreads * kBoxItems);
    if (blocks > (int64_t)sms * 4) blocks = (int64_t)sms * 4;
    ss.box_blocks = (int)(blocks < 1 ? 1 : blocks);
    uint32_t *err = (uint32_t *)(base + kOffErr);

    // one segment: every particle belongs to it, so no segment tables
    Segs g{};
    g.S = 1;
    g.tiles = tiles;
    g.box = (float4 *)(base + kOffBox);
    g.boxmm = (uint32_t *)(base + kOffBoxMM);

    Tree t{};
    t.cell = (float4 *)(base + kOffRootCell);   // the box kernel seeds a root node here
    t.info = (uint4 *)(base + kOffRootInfo);
    t.cap = 1;

    State s{};
    s.x = const_cast<float *>(d_x);
    s.y = const_cast<float *>(d_y);
    StepParams p{};
    p.n = (int)n;

    // the array keeps the previous call's contents (zero before the first):
    // set what must start at a known value -- the min/max words and the error
    // word; the key launch clears the histograms, look-back words and tile
    // counters itself
    if (launch_reset_boxes(g, st) != cudaSuccess) return GE_ERR_CUDA;
    if (cudaMemsetAsync(err, 0, sizeof(uint32_t), st) != cudaSuccess) return GE_ERR_CUDA;
    if (launch_kick_drift_bbox(2, s, p, false, g, ss, t, st) != cudaSuccess) return GE_ERR_CUDA;
    if (launch_keys(2, s, (int)n, g, ss, st) != cudaSuccess) return GE_ERR_CUDA;
    if (launch_sort(2, (int)n, g, ss, err, st) != cudaSuccess) return GE_ERR_CUDA;
    if (launch_perm_out(2, (int)n, ss, d_perm, st) != cudaSuccess) return GE_ERR_CUDA;
    if (d_keys && launch_keys_out(2, (int)n, ss, d_keys, st) != cudaSuccess) return GE_ERR_CUDA;
    uint32_t h_err = 0;
    if (cudaMemcpyAsync(&h_err, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return GE_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return GE_ERR_CUDA;
    return h_err ? GE_ERR_TIMEOUT : GE_OK;
}
