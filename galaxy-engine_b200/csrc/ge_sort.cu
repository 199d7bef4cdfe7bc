// ge_sort.cu -- Morton keys, stable LSD radix sort, state permutation.
//
// Reference: Morton::computeMortonKeys[3D] (GalaxyEngine/src/Physics/morton.cpp:27-38,
// :92-112) and Morton::sortParticlesByMortonKey[3D] (:40-63, :114-138).
//
// Keys are bit-exact with the reference: the same IEEE single operations
// (clamp, subtract, divide, scale, truncate) and the same interleave.  The
// reference sorts with std::sort, whose order among equal keys is
// unspecified; this sort is stable, so equal keys keep their current order.
//
// 2D keys use 36 bits.  They are packed with the particle's current index as
// (key << 28) | index, so each pass moves one 8-byte word per particle
// (N < 2^28).  3D keys use 63 bits and travel with a separate 32-bit index.
// Digits are 9 bits wide: 4 passes in 2D, 7 in 3D.  The other callers' words
// (the SPH grid's) sort by 8-bit digits.
//
// Each pass is one kernel: a tile of 4096 keys is ranked in shared memory
// (warp-private digit counters; the lanes of equal digits found by one ballot
// per digit bit), the tile's per-digit counts are published, and the exclusive
// prefix over earlier tiles is found by decoupled look-back on per-tile
// status words (bounded waits).  Digit histograms of every pass are computed
// once, by the key kernel.
#include "ge_device.cuh"
#include "ge_internal.h"

namespace ge {

constexpr int kKeyBits = 9;                  // digit width of the Morton key passes
constexpr int kKeyRadix = 1 << kKeyBits;
constexpr int kWordBits = 8;                 // digit width of launch_radix_words
constexpr int kSortThreads = 512;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItems = kSortTile / kSortThreads;  // 8
constexpr uint32_t kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kValMask = (1u << 30) - 1;

__host__ __device__ constexpr int key_passes(int dims) { return dims == 2 ? 4 : 7; }

// The lanes whose BITS-bit digit equals this lane's, among the lanes with
// `valid` set: one ballot per digit bit (the same mask as __match_any_sync
// over the digits, for valid lanes; an invalid lane's mask is not used).
template <int BITS>
__device__ __forceinline__ unsigned digit_peers(uint32_t d, bool valid) {
    unsigned m = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < BITS; b++) {
        const bool bit = (d >> b) & 1u;
        const unsigned bb = __ballot_sync(0xffffffffu, bit);
        m &= bit ? bb : ~bb;
    }
    return m;
}
static_assert(4 * kKeyBits == 36 && 7 * kKeyBits == 63, "passes cover the key bits");
static_assert(7 * kKeyRadix <= kSortDigitWords, "hist / status words per segment / tile");
static_assert(kKeyRadix <= kSortThreads, "one thread per digit");
__host__ __device__ constexpr int key_shift0(int dims) { return dims == 2 ? 28 : 0; }

// Morton keys of every particle from its segment's root box, and the digit
// histograms of every pass per segment.  Each block covers a contiguous chunk
// of particles and accumulates in shared memory while its particles stay in
// one segment (one flush per segment change); a warp that straddles segments
// counts with global atomics instead.
template <int D>
__global__ void __launch_bounds__(256)
k_keys(State s, int n, Segs g, uint64_t *keys, uint32_t *vals, uint32_t *hist,
       uint32_t *status, int64_t status_words, uint32_t *tile_ctr) {
    dep_wait();
    constexpr int P = key_passes(D), S0 = key_shift0(D), R = kKeyRadix;
    __shared__ uint32_t sh[P][R];
    const int lane = threadIdx.x & 31;
    const size_t SH = (size_t)g.S * R;   // stride of one pass in hist
    for (int i = threadIdx.x; i < P * R; i += blockDim.x) (&sh[0][0])[i] = 0;
    // clear the look-back status words for this step's passes
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < status_words;
         i += (int64_t)gridDim.x * blockDim.x)
        status[i] = 0u;
    if (blockIdx.x == 0 && threadIdx.x < 8) tile_ctr[threadIdx.x] = 0u;
    __syncthreads();
    const int chunk = ((n + gridDim.x - 1) / gridDim.x + 255) & ~255;
    const int c0 = blockIdx.x * chunk, c1 = min(c0 + chunk, n);
    int cur = -1;   // segment the shared histogram belongs to (block-uniform)
    for (int base = c0; base < c1; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const bool ok = i < c1;
        const uint32_t sg = ok && g.seg_of ? g.seg_of[i] : 0u;
        // one segment for the whole block tile?
        const int tlast = min(base + (int)blockDim.x, c1) - 1;
        const uint32_t s_first = g.seg_of ? g.seg_of[base] : 0u;
        const uint32_t s_last = g.seg_of ? g.seg_of[tlast] : 0u;
        const bool uni = s_first == s_last;
        if (uni && (int)s_first != cur) {
            __syncthreads();
            if (cur >= 0)
                for (int k = threadIdx.x; k < P * R; k += blockDim.x) {
                    const uint32_t c = (&sh[0][0])[k];
                    if (c) atomicAdd(&hist[(k / R) * SH + (size_t)cur * R + (k % R)], c);
                }
            __syncthreads();
            for (int k = threadIdx.x; k < P * R; k += blockDim.x) (&sh[0][0])[k] = 0;
            __syncthreads();
            cur = (int)s_first;
        }
        uint64_t word = 0;
        if (ok) {
            const float4 bb = g.box[sg];
            float hx, hy, hz;
            if (D == 2) {
                const float ext = bb.w > 1e-6f ? bb.w : 1e-6f;   // std::max(posSize.z, 1e-6f)
                hx = fadd(bb.x, ext); hy = fadd(bb.y, ext); hz = 0.0f;
            } else {
                hx = fadd(bb.x, bb.w); hy = fadd(bb.y, bb.w); hz = fadd(bb.z, bb.w);
            }
            if (D == 2) {
                const uint64_t ix = scale_to_grid(s.x[i], bb.x, hx, 262144.0f, 262143ull);
                const uint64_t iy = scale_to_grid(s.y[i], bb.y, hy, 262144.0f, 262143ull);
                const uint64_t key = spread2(ix) | (spread2(iy) << 1);
                word = (key << 28) | (uint64_t)i;
                keys[i] = word;
            } else {
                const uint64_t ix = scale_to_grid(s.x[i], bb.x, hx, 2097151.0f, 2097151ull);
                const uint64_t iy = scale_to_grid(s.y[i], bb.y, hy, 2097151.0f, 2097151ull);
                const uint64_t iz = scale_to_grid(s.z[i], bb.z, hz, 2097151.0f, 2097151ull);
                word = spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2);
                keys[i] = word;
                vals[i] = (uint32_t)i;
            }
        }
#pragma unroll
        for (int ps = 0; ps < P; ps++) {
            const uint32_t d = ok ? (uint32_t)((word >> (S0 + kKeyBits * ps)) & (R - 1)) : (uint32_t)R;
            if (uni) {
                // a warp of one digit (the upper digits of nearly sorted keys)
                // adds once; the others count by digit groups
                if (__all_sync(0xffffffffu, d == __shfl_sync(0xffffffffu, d, 0) && ok)) {
                    if (lane == 0) atomicAdd(&sh[ps][d], 32u);
                } else {
                    const unsigned peers = digit_peers<kKeyBits>(d, ok);
                    if (ok && lane == __ffs(peers) - 1) atomicAdd(&sh[ps][d], (uint32_t)__popc(peers));
                }
            } else {
                const unsigned peers = __match_any_sync(
                    0xffffffffu, ok ? ((uint64_t)sg << 16) | d : ~0ull);
                if (ok && lane == __ffs(peers) - 1)
                    atomicAdd(&hist[ps * SH + (size_t)sg * R + d], (uint32_t)__popc(peers));
            }
        }
    }
    __syncthreads();
    if (cur >= 0)
        for (int k = threadIdx.x; k < P * R; k += blockDim.x) {
            const uint32_t c = (&sh[0][0])[k];
            if (c) atomicAdd(&hist[(k / R) * SH + (size_t)cur * R + (k % R)], c);
        }
}

// One stable counting pass over digit (word >> shift) & (2^BITS - 1), segment
// by segment: a tile belongs to one segment, its digit offsets start at the
// segment's first slot, and look-back stops at the segment's first tile.
template <bool PAIRS, int BITS>
__global__ void __launch_bounds__(kSortThreads)
k_radix_pass(const uint64_t *__restrict__ kin, uint64_t *__restrict__ kout,
             const uint32_t *__restrict__ vin, uint32_t *__restrict__ vout, int n, int shift,
             Segs g, const uint32_t *__restrict__ hist, uint32_t *status, uint32_t *tile_ctr,
             uint32_t *err, uint32_t spin_limit, uint32_t withhold_first) {
    dep_wait();
    constexpr int R = 1 << BITS;
    const uint32_t max_spins = spin_limit ? spin_limit : kSpinLimit;
    __shared__ uint32_t s_whist[kSortWarps][R];
    __shared__ uint32_t s_off[R];
    __shared__ uint32_t s_scan[kSortWarps];
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    for (int i = tid; i < kSortWarps * R; i += kSortThreads) (&s_whist[0][0])[i] = 0u;
    __syncthreads();
    const int tile = (int)s_tile;
    const uint32_t sg = g.tile_seg ? g.tile_seg[tile] : 0u;
    const int tile0 = g.tile_base ? (int)g.tile_base[sg] : 0;
    const uint32_t lo = seg_lo(g, sg), hi = seg_hi(g, sg, (uint32_t)n);
    // exclusive scan of this segment's digit counts (thread = digit)
    const uint32_t gcount = tid < R ? hist[(size_t)sg * R + tid] : 0u;
    uint32_t incl = gcount;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_scan[w] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (int ww = 0; ww < w; ww++) wbase += s_scan[ww];
    const uint32_t gexcl = lo + wbase + incl - gcount;
    const uint32_t tstart = lo + (uint32_t)(tile - tile0) * kSortTile;
    const int base = (int)tstart + w * 32 * kItems;

    uint64_t k[kItems];
    uint32_t v[kItems], rk[kItems], dg[kItems];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int it = 0; it < kItems; it++) {
        const int idx = base + it * 32 + lane;
        const bool ok = idx < (int)hi;
        k[it] = ok ? kin[idx] : 0ull;
        if (PAIRS) v[it] = ok ? vin[idx] : 0u;
        dg[it] = ok ? (uint32_t)((k[it] >> shift) & (R - 1)) : (uint32_t)R;
    }
#pragma unroll
    for (int it = 0; it < kItems; it++) {
        const uint32_t d = dg[it];
        const unsigned peers = digit_peers<BITS>(d, d < (uint32_t)R);
        uint32_t prev = 0;
        const int leader = __ffs(peers) - 1;
        if (d < (uint32_t)R && lane == leader) {
            prev = s_whist[w][d];
            s_whist[w][d] = prev + (uint32_t)__popc(peers);
        }
        prev = __shfl_sync(0xffffffffu, prev, leader);
        rk[it] = prev + (uint32_t)__popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps and the tile total
    if (tid < R) {
        const int d = tid;
        uint32_t sum = 0;
#pragma unroll
        for (int ww = 0; ww < kSortWarps; ww++) {
            const uint32_t c = s_whist[ww][d];
            s_whist[ww][d] = sum;
            sum += c;
        }
        volatile uint32_t *st = status;
        uint32_t excl = 0;
        if (tile == tile0) {
            // (withheld only under the test hook: the first tile of the whole
            // sort then never publishes, and every later wait on it is bounded)
            if (!(withhold_first && tile == 0)) st[(int64_t)tile * R + d] = kFlagInc | sum;
        } else {
            st[(int64_t)tile * R + d] = kFlagAgg | sum;
            // look back kLookBack tiles per round trip: the words are read at
            // once and consumed in order up to the first inclusive one (done)
            // or the first unpublished one (read again from there)
            constexpr int kLookBack = 2;
            int t = tile - 1;
            uint32_t spins = 0;
            bool done = false;
            while (!done && t >= tile0) {
                const int m = min(kLookBack, t - tile0 + 1);
                uint32_t wd[kLookBack];
#pragma unroll
                for (int j = 0; j < kLookBack; j++)
                    wd[j] = j < m ? st[(int64_t)(t - j) * R + d] : 0u;
                int j = 0;
                for (; j < m; j++) {
                    const uint32_t f = wd[j] & ~kValMask;
                    if (f == 0u) break;
                    excl += wd[j] & kValMask;
                    if (f == kFlagInc) { done = true; break; }
                }
                if (done) break;
                t -= j;
                if (j < m && ++spins > max_spins) { set_err(err, kErrSpin); break; }
            }
            st[(int64_t)tile * R + d] = kFlagInc | ((excl + sum) & kValMask);
        }
        s_off[d] = gexcl + excl;
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kItems; it++) {
        const uint32_t d = dg[it];
        if (d < (uint32_t)R) {
            const uint32_t pos = s_off[d] + s_whist[w][d] + rk[it];
            if (pos < hi) {   // always true unless a look-back wait gave up
                kout[pos] = k[it];
                if (PAIRS) vout[pos] = v[it];
            }
        }
    }
}

// Two particles per thread, both gathers issued before either's stores (the
// stores could alias the next particle's loads, which would keep them apart).
constexpr int kPermItems = 2;

template <int D>
__global__ void __launch_bounds__(256)
k_permute(const uint64_t *__restrict__ keys, const uint32_t *__restrict__ vals, int n, State in,
          State out, int with_acc) {
    dep_wait();
    constexpr int U = kPermItems;
    const int stride = gridDim.x * blockDim.x * U;
    for (int k0 = blockIdx.x * blockDim.x * U + threadIdx.x; k0 < n; k0 += stride) {
        int kk[U];
        uint32_t j[U];
        float x[U], y[U], z[U], vx[U], vy[U], vz[U], m[U], ax[U], ay[U], az[U];
        uint32_t id[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            kk[u] = k0 + u * (int)blockDim.x;
            j[u] = 0u;
            if (kk[u] < n) {
                j[u] = (D == 2) ? (uint32_t)(keys[kk[u]] & 0x0FFFFFFFull) : vals[kk[u]];
                if (j[u] >= (uint32_t)n) j[u] = (uint32_t)kk[u];   // only after a failed sort (error word set)
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (kk[u] >= n) continue;
            const uint32_t q = j[u];
            x[u] = in.x[q]; y[u] = in.y[q];
            vx[u] = in.vx[q]; vy[u] = in.vy[q];
            m[u] = in.m[q];
            id[u] = in.id[q];
            if (D == 3) { z[u] = in.z[q]; vz[u] = in.vz[q]; }
            if (with_acc) {
                ax[u] = in.ax[q]; ay[u] = in.ay[q];
                if (D == 3) az[u] = in.az[q];
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = kk[u];
            if (k >= n) continue;
            const uint32_t q = j[u];
            out.x[k] = x[u]; out.y[k] = y[u];
            out.vx[k] = vx[u]; out.vy[k] = vy[u];
            out.m[k] = m[u];
            out.id[k] = id[u];
            if (D == 3) { out.z[k] = z[u]; out.vz[k] = vz[u]; }
            if (with_acc) {
                out.ax[k] = ax[u]; out.ay[k] = ay[u];
                if (D == 3) out.az[k] = az[u];
            }
            if (in.pvx) {
                out.pvx[k] = in.pvx[q]; out.pvy[k] = in.pvy[q];
                if (D == 3) out.pvz[k] = in.pvz[q];
            }
            if (in.pinned) out.pinned[k] = in.pinned[q];
            if (in.temp) out.temp[k] = in.temp[q];
            if (in.kx) {
                out.kx[k] = in.kx[q]; out.ky[k] = in.ky[q];
                out.kvx[k] = in.kvx[q]; out.kvy[k] = in.kvy[q];
                if (D == 3) { out.kz[k] = in.kz[q]; out.kvz[k] = in.kvz[q]; }
            }
        }
    }
}

template <int D>
__global__ void k_perm_out(const uint64_t *keys, const uint32_t *vals, int n, uint32_t *perm,
                           uint64_t *kout) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        if (perm) perm[k] = (D == 2) ? (uint32_t)(keys[k] & 0x0FFFFFFFull) : vals[k];
        if (kout) kout[k] = (D == 2) ? (keys[k] >> 28) : keys[k];
    }
}

__global__ void __launch_bounds__(256) k_zero_words(uint32_t *w, int64_t count) {
    dep_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        w[i] = 0u;
}

cudaError_t launch_zero(uint32_t *w, int64_t count, cudaStream_t st) {
    if (count < 1) return cudaSuccess;
    int64_t blocks = (count + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    return launch_dep(k_zero_words, (unsigned)blocks, 256, st, w, count);
}

static int grid_for(int n, int threads, int cap) {
    int b = (n + threads - 1) / threads;
    if (b > cap) b = cap;
    return b < 1 ? 1 : b;
}

// Blocks of `threads` that one wave holds on this device (resident blocks per
// SM x SMs), found once per kernel; 0 if the query fails.
static int one_wave(const void *kernel, int threads) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess)
        return 0;
    return per_sm * sms;
}

cudaError_t launch_keys(int dims, const State &s, int n, const Segs &g, SortScratch &ss,
                        cudaStream_t st) {
    // one wave: every block takes one contiguous chunk of the particles
    static const int wave[2] = {one_wave((const void *)k_keys<2>, 256),
                                one_wave((const void *)k_keys<3>, 256)};
    const int w = wave[dims == 2 ? 0 : 1];
    const int blocks = grid_for(n, 256, w > 0 ? w : 148 * 4);
    const int64_t words = (int64_t)key_passes(dims) * g.tiles * kKeyRadix;
    cudaError_t e = launch_zero(ss.hist, (int64_t)key_passes(dims) * g.S * kKeyRadix, st);
    if (e != cudaSuccess) return e;
    if (dims == 2)
        return launch_dep(k_keys<2>, blocks, 256, st, s, n, g, ss.keys[0], ss.vals[0], ss.hist,
                          ss.status, words, ss.tile_ctr);
    return launch_dep(k_keys<3>, blocks, 256, st, s, n, g, ss.keys[0], ss.vals[0], ss.hist,
                      ss.status, words, ss.tile_ctr);
}

cudaError_t launch_sort(int dims, int n, const Segs &g, SortScratch &ss, uint32_t *err,
                        cudaStream_t st) {
    const int P = key_passes(dims), S0 = key_shift0(dims);
    const int tiles = (int)g.tiles;
    int cur = 0;
    for (int ps = 0; ps < P; ps++) {
        uint32_t *status = ss.status + (int64_t)ps * g.tiles * kKeyRadix;
        const uint32_t *hist = ss.hist + (size_t)ps * g.S * kKeyRadix;
        const int shift = S0 + kKeyBits * ps;
        const uint32_t *no_vin = nullptr;
        uint32_t *no_vout = nullptr;
        const cudaError_t e =
            dims == 2 ? launch_dep(k_radix_pass<false, kKeyBits>, tiles, kSortThreads, st,
                                   ss.keys[cur], ss.keys[cur ^ 1], no_vin, no_vout, n, shift, g,
                                   hist, status, ss.tile_ctr + ps, err, ss.spin_limit,
                                   ss.withhold_first)
                      : launch_dep(k_radix_pass<true, kKeyBits>, tiles, kSortThreads, st,
                                   ss.keys[cur], ss.keys[cur ^ 1], ss.vals[cur], ss.vals[cur ^ 1],
                                   n, shift, g, hist, status, ss.tile_ctr + ps, err,
                                   ss.spin_limit, ss.withhold_first);
        if (e != cudaSuccess) return e;
        cur ^= 1;
    }
    // an odd number of passes leaves the result in buffer 1: swap the roles
    if (cur == 1) {
        uint64_t *tk = ss.keys[0]; ss.keys[0] = ss.keys[1]; ss.keys[1] = tk;
        uint32_t *tv = ss.vals[0]; ss.vals[0] = ss.vals[1]; ss.vals[1] = tv;
    }
    return cudaSuccess;
}

cudaError_t launch_radix_words(uint64_t *const words[2], int n, int shift0, int passes,
                               const uint32_t *hist, uint32_t *status, uint32_t *tile_ctr,
                               uint32_t *err, int *result, cudaStream_t st) {
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    const Segs one{};   // a single range [0, n)
    int cur = 0;
    for (int ps = 0; ps < passes; ps++) {
        constexpr int R = 1 << kWordBits;
        k_radix_pass<false, kWordBits><<<(unsigned)(tiles < 1 ? 1 : tiles), kSortThreads, 0, st>>>(
            words[cur], words[cur ^ 1], nullptr, nullptr, n, shift0 + kWordBits * ps, one,
            hist + (size_t)ps * R, status + ps * tiles * R, tile_ctr + ps, err, 0u, 0u);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        cur ^= 1;
    }
    *result = cur;
    return cudaSuccess;
}

cudaError_t launch_permute(int dims, int n, const SortScratch &ss, const State &in,
                           const State &out, bool with_acc, cudaStream_t st) {
    int blocks = grid_for(n, 256 * kPermItems, 148 * 16);
    const int wa = with_acc ? 1 : 0;
    if (dims == 2) return launch_dep(k_permute<2>, blocks, 256, st, ss.keys[0], ss.vals[0], n, in, out, wa);
    return launch_dep(k_permute<3>, blocks, 256, st, ss.keys[0], ss.vals[0], n, in, out, wa);
}

cudaError_t launch_perm_out(int dims, int n, const SortScratch &ss, uint32_t *perm,
                            cudaStream_t st) {
    int blocks = grid_for(n, 256, 148 * 16);
    if (dims == 2) k_perm_out<2><<<blocks, 256, 0, st>>>(ss.keys[0], ss.vals[0], n, perm, nullptr);
    else k_perm_out<3><<<blocks, 256, 0, st>>>(ss.keys[0], ss.vals[0], n, perm, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_keys_out(int dims, int n, const SortScratch &ss, uint64_t *keys,
                            cudaStream_t st) {
    int blocks = grid_for(n, 256, 148 * 16);
    if (dims == 2) k_perm_out<2><<<blocks, 256, 0, st>>>(ss.keys[0], ss.vals[0], n, nullptr, keys);
    else k_perm_out<3><<<blocks, 256, 0, st>>>(ss.keys[0], ss.vals[0], n, nullptr, keys);
    return cudaGetLastError();
}

}  // namespace ge
