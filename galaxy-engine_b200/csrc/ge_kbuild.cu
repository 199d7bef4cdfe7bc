// ge_kbuild.cu -- the tree's nodes straight from the Morton keys, with exact
// rebuilds where the keys and the reference's float splits disagree.
//
// Reference: Node::Node / subGridMaker (GalaxyEngine/src/Physics/quadtree.cpp:5-88,
// octree :109-271): a node over the sorted range [start, end) is a leaf when
// ((count <= 4 && size <= 2) || count == 1 || size <= 1e-6); otherwise its range is
// cut by std::partition_point on float compares with the cell's midpoint (y,
// then x; z, then y, then x in 3D), one child per non-empty quadrant.
//
// The particles are sorted by Morton key, and the key's level-L digit (2 bits
// in 2D, 3 in 3D) names the quadrant of the particle's level-L cell.  Where
// every particle of a node compares with the node's midpoints exactly as its
// key digit says, the float predicates are monotone over the sorted range, so
// std::partition_point returns the key boundaries and the children are the
// key runs of the next level.  So the tree is built from the keys:
//   k_key_levels  delta(i) = the level at which particle i's key first differs
//                 from particle i-1's (-1 at a simulation's first particle);
//                 the node holding i at level L is the run of particles with
//                 delta >= L around i, so its count is known from a window of
//                 leaf_cap deltas on each side and the leaf level lambda(i)
//                 follows from the leaf rule; along its key path (the cells
//                 computed with the reference's float operations) every level
//                 where i's compares disagree with its digit is a suspect;
//   k_key_check   each suspect node's cut points are computed exactly (the
//                 partition_point probe sequence) and compared with the key
//                 boundaries; a node where they differ becomes an exact-rebuild
//                 root: its children are built by the top-down exact builder
//                 (ge_tree.cu), as is every node the keys cannot split (a run of
//                 equal keys that is not a leaf);
//   k_key_count / k_key_scan / k_key_emit   particle a starts the nodes of
//                 levels delta(a)+1 .. T(a) (T = its leaf level, or its exact
//                 root's level); node slots are laid out level by level, in
//                 start order within a level (so siblings are contiguous), from
//                 per-tile, per-level counts and their prefix sums.  Every node
//                 is written by the particle that starts it (cell, start, first
//                 child, parent, child bit in the parent) and by the particle
//                 that ends it (end, ancestors ending at the same place).
// The tree equals the reference's node for node (the exact rebuilds included)
// whatever the keys' rounding; the masses, the exact rebuilds and the walk
// layout follow in the build kernel (ge_tree.cu, keyed mode).
#include "ge_device.cuh"
#include "ge_internal.h"
#include "ge_tree_dev.cuh"

namespace ge {

namespace {

constexpr int kKT = 256;                   // threads of the key passes
constexpr int kHalo = kKeyMaxCap;          // window of the leaf-count test
// kmeta words
constexpr int kKmSus = 0, kKmRoots = 1, kKmOverflow = 2, kKmTotal = 3, kKmLevels = 4,
              kKmLevelTot = 8, kKmBig = 32;
// an exact-rebuild root of more particles than this is recorded in the large
// list and marked by the node-count pass (one thread per particle) instead of
// by the warp that found it
#ifndef GE_MARK_DIRECT
#define GE_MARK_DIRECT 4096
#endif
constexpr uint32_t kMarkDirect = GE_MARK_DIRECT;

template <int D> struct KeyBits;
template <> struct KeyBits<2> { static constexpr int B = 18, W = 36; };
template <> struct KeyBits<3> { static constexpr int B = 21, W = 63; };

template <int D>
__device__ __forceinline__ uint64_t key_at(const uint64_t *keys, uint32_t i) {
    return D == 2 ? (__ldg(&keys[i]) >> 28) : __ldg(&keys[i]);
}

// the level-L digit of a key (the quadrant / octant of the level-L cell)
template <int D>
__device__ __forceinline__ unsigned digit(uint64_t key, int L) {
    return (unsigned)(key >> (D * (KeyBits<D>::B - 1 - L))) & ((1u << D) - 1u);
}

// delta(j): first level at which the keys of j-1 and j differ; -1 at the
// first particle of a simulation and at j = n
template <int D>
__device__ __forceinline__ int delta_at(const Segs &g, const uint64_t *keys, int64_t j, int n) {
    if (j <= 0 || j >= n) return -1;
    const uint32_t sg = g.seg_of ? __ldg(&g.seg_of[j]) : 0u;
    if ((uint32_t)j == seg_lo(g, sg)) return -1;
    const uint64_t x = key_at<D>(keys, (uint32_t)j) ^ key_at<D>(keys, (uint32_t)j - 1u);
    if (x == 0) return KeyBits<D>::B;
    const int lead = KeyBits<D>::W - (64 - __clzll((long long)x));
    return lead / D;
}

// T(i): the deepest level of the key tree that holds particle i
__device__ __forceinline__ uint32_t key_depth(const Tree &t, uint32_t i) {
    const uint32_t l = t.klam[i], x = __ldcg(&t.kxr[i]);
    return l < x ? l : x;
}

template <int D>
__global__ void __launch_bounds__(kKT)
k_key_levels(State s, StepParams p, Segs g, const uint64_t *__restrict__ keys, Tree t) {
    dep_wait();
    constexpr int B = KeyBits<D>::B;
    __shared__ int8_t sd[kKT + 2 * kHalo + 1];
    __shared__ int s_lv[3];   // {segment, size-gate level, minimum-size level} of the block's first particle
    const int n = p.n;
    const int64_t base = (int64_t)blockIdx.x * kKT;
    for (int q = threadIdx.x; q < kKT + 2 * kHalo + 1; q += kKT)
        sd[q] = (int8_t)delta_at<D>(g, keys, base - kHalo + q, n);
    // parent child bits and counts are accumulated into pend by the emit pass
    {
        uint4 *p4 = reinterpret_cast<uint4 *>(t.pend);   // cudaMalloc: 16-byte aligned
        const int64_t n4 = t.cap / 4;
        for (int64_t k = (int64_t)blockIdx.x * kKT + threadIdx.x; k < n4;
             k += (int64_t)gridDim.x * kKT)
            p4[k] = make_uint4(0u, 0u, 0u, 0u);
        if (blockIdx.x == 0 && threadIdx.x < (unsigned)(t.cap - n4 * 4))
            t.pend[n4 * 4 + threadIdx.x] = 0u;
        if (blockIdx.x == 0)
            for (int q = threadIdx.x; q < kKeyBigHash; q += kKT) t.kbig_keys[q] = 0ull;
    }
    // first levels whose cells are no larger than the size gate / min size
    // (the sizes are exact halvings of the root's: w * 2^-L)
    auto first_level_at_most = [&](float w, float limit) {
        if (w != w) return 127;
        if (w <= limit) return 0;
        if (!(limit > 0.0f)) return 127;
        int L = max(0, ilogbf(w) - ilogbf(limit) - 1);
        while (L <= B && scalbnf(w, -L) > limit) L++;
        return L <= B ? L : 127;
    };
    if (threadIdx.x == 0 && base < n) {   // once per block, for its first particle's simulation
        const uint32_t s0 = g.seg_of ? g.seg_of[base] : 0u;
        const float w0 = g.box[s0].w;
        s_lv[0] = (int)s0;
        s_lv[1] = first_level_at_most(w0, p.size_gate);
        s_lv[2] = first_level_at_most(w0, p.min_size);
    }
    __syncthreads();
    const int64_t i = base + threadIdx.x;
    if (i >= n) return;
    auto dl = [&](int64_t j) { return (int)sd[j - base + kHalo]; };
    const uint32_t sg = g.seg_of ? g.seg_of[i] : 0u;
    const int64_t lo = seg_lo(g, sg), hi = seg_hi(g, sg, (uint32_t)n);
    const int cap = (int)p.leaf_cap;
    // count <= cap at level L  <=>  L > min over boundary pairs a <= i < e with
    // e - a <= cap of max(delta(a), delta(e)) (a boundary: delta < L)
    int best = 127, pm = 127;
    for (int tt = cap - 1; tt >= 0; --tt) {
        const int64_t r = i + 1 + (cap - 1 - tt);
        if (r <= hi) pm = min(pm, dl(r));
        const int64_t a = i - tt;
        if (a >= lo) best = min(best, max(dl(a), pm));
    }
    const int l_count = best == 127 ? 127 : best + 1;
    const int l_one = max(dl(i), dl(i + 1)) + 1;
    const float4 box = g.box[sg];
    const bool same = (int)sg == s_lv[0];
    const int l_gate = same ? s_lv[1] : first_level_at_most(box.w, p.size_gate);
    const int l_min = same ? s_lv[2] : first_level_at_most(box.w, p.min_size);
    int lam = min(min(max(l_count, l_gate), l_one), l_min);
    if (lam > B) lam = B + 1;
    t.kdl[i] = (uint8_t)(dl(i) + 1);
    t.klam[i] = (uint8_t)lam;
    t.kxr[i] = lam > B ? (uint32_t)B : kEmpty;
    // suspects: levels where the particle's compares disagree with its digits
    const uint64_t key = key_at<D>(keys, (uint32_t)i);
    float pos[3] = {s.x[i], s.y[i], D == 3 ? s.z[i] : 0.0f};
    float cor[3] = {box.x, box.y, box.z};
    float sz = box.w;
    const int levels = min(lam, B);
    for (int L = 0; L < levels; L++) {
        const float half = fmul(sz, 0.5f);
        const unsigned q = digit<D>(key, L);
        bool bad = false;
#pragma unroll
        for (int a = 0; a < D; a++) {
            const bool up = (q >> a) & 1u;
            bad |= (pos[a] < fadd(cor[a], half)) == up;
            cor[a] = fadd(cor[a], up ? half : 0.0f);
        }
        sz = half;
        if (bad) {
            const uint32_t k = atomicAdd(&t.kmeta[kKmSus], 1u);
            if (k < t.ksus_cap) t.ksus[k] = make_uint2((uint32_t)L, (uint32_t)i);
            else t.kmeta[kKmOverflow] = 1u;
        }
    }
}

// First j in [first, last) with pred(j) false, pred monotone (true then
// false), by groups of G lanes, each group with its own range and predicate:
// G probes per round narrow the range (G + 1)-fold; every lane of the warp
// must call it, and a group's lanes get the same result.
template <int G, typename F>
__device__ __forceinline__ uint32_t group_lower_bound(uint32_t first, uint32_t last, F pred) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gl = lane & (G - 1u), gbase = lane & ~(G - 1u);
    const unsigned gm = G == 32 ? 0xffffffffu : (1u << G) - 1u;
    while (__any_sync(0xffffffffu, last - first > (uint32_t)G)) {
        const bool act = last - first > (uint32_t)G;
        uint32_t q = 0;
        bool pv = false;
        if (act) {
            q = first + (uint32_t)(((uint64_t)(last - first) * (gl + 1u)) / (G + 1u));
            pv = pred(q);
        }
        const unsigned tc = __popc((__ballot_sync(0xffffffffu, pv) >> gbase) & gm);
        const uint32_t qa = __shfl_sync(0xffffffffu, q, gbase + (tc ? tc - 1u : 0u));
        const uint32_t qb = __shfl_sync(0xffffffffu, q, gbase + (tc < (unsigned)G ? tc : G - 1u));
        if (act) {
            const uint32_t nf = tc ? qa + 1u : first;
            last = tc < (unsigned)G ? qb + 1u : last;
            first = nf;
        }
    }
    const bool v = first + gl < last && pred(first + gl);
    return first + (uint32_t)__popc((__ballot_sync(0xffffffffu, v) >> gbase) & gm);
}

template <int D>
__global__ void __launch_bounds__(kKT)
k_key_check(State s, StepParams p, Segs g, const uint64_t *__restrict__ keys, Tree t) {
    dep_wait();
    constexpr int B = KeyBits<D>::B, Q = 1 << D;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t gwarp = (blockIdx.x * kKT + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kKT) >> 5;
    const uint32_t n = (uint32_t)p.n;
    if (*(volatile uint32_t *)&t.kmeta[kKmOverflow]) {
        // too many suspects to record: every simulation is rebuilt exactly
        for (uint32_t i = blockIdx.x * kKT + threadIdx.x; i < n; i += gridDim.x * kKT)
            t.kxr[i] = 0u;
        return;
    }
    const uint32_t ns = min(*(volatile uint32_t *)&t.kmeta[kKmSus], t.ksus_cap);
    for (uint32_t w = gwarp; w < ns; w += nwarps) {
        const uint2 sp = t.ksus[w];
        const int L = (int)sp.x;
        const uint32_t i = sp.y;
        if (__ldcg(&t.kxr[i]) <= (uint32_t)L) continue;   // inside a rebuild root already
        const uint32_t sg = g.seg_of ? g.seg_of[i] : 0u;
        const uint32_t lo = seg_lo(g, sg), hi = seg_hi(g, sg, n);
        const uint64_t ki = key_at<D>(keys, i);
        const int shift = D * (B - L);
        const uint64_t pre = ki >> shift;
        // the node's range: the run of keys that agree with ki on L digits (its
        // start by the low half-warp, its end by the high one, at once)
        const bool hi_half = lane >= 16u;
        const uint32_t r = group_lower_bound<16>(hi_half ? i + 1 : lo, hi_half ? hi : i, [&](uint32_t j) {
            const uint64_t v = key_at<D>(keys, j) >> shift;
            return hi_half ? v <= pre : v < pre;
        });
        const uint32_t a = __shfl_sync(0xffffffffu, r, 0);
        const uint32_t e = __shfl_sync(0xffffffffu, r, 16);
        // the node's cell along the key path
        const float4 box = g.box[sg];
        float cor[3] = {box.x, box.y, box.z};
        float sz = box.w;
        for (int l = 0; l < L; l++) {
            const float half = fmul(sz, 0.5f);
            const unsigned q = digit<D>(ki, l);
#pragma unroll
            for (int ax = 0; ax < D; ax++) cor[ax] = fadd(cor[ax], ((q >> ax) & 1u) ? half : 0.0f);
            sz = half;
        }
        const float half = fmul(sz, 0.5f);
        const float mid[3] = {fadd(cor[0], half), fadd(cor[1], half), fadd(cor[2], half)};
        uint32_t b[Q + 1];
        cut_group<D, 32>(s, a, e, mid, b);
        // is each cut the first particle of its digit value?  (digits are
        // sorted within the node: one look on each side of the cut decides)
        bool bad = false;
        if (lane > 0u && lane < (unsigned)Q) {
            uint32_t j = b[1];
#pragma unroll
            for (int q = 2; q < Q; q++) j = lane == (unsigned)q ? b[q] : j;
            if (j > a && digit<D>(key_at<D>(keys, j - 1), L) >= lane) bad = true;
            if (j < e && digit<D>(key_at<D>(keys, j), L) < lane) bad = true;
        }
        const bool differ = __any_sync(0xffffffffu, bad);
        if (!differ) continue;
        // a large root goes to the large list once (several suspects may find
        // it), unless the set or the list is full
        bool listed = false;
        if (e - a > kMarkDirect && lane == 0) {
            const unsigned long long key = (((unsigned long long)a << 8) | (unsigned)L) + 1ull;
            uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 40) & (kKeyBigHash - 1u);
            for (int probe = 0; probe < 32; probe++, h = (h + 1u) & (kKeyBigHash - 1u)) {
                const unsigned long long old = atomicCAS(&t.kbig_keys[h], 0ull, key);
                if (old == key) { listed = true; break; }   // recorded by another warp
                if (old == 0ull) {
                    const uint32_t k = atomicAdd(&t.kmeta[kKmBig], 1u);
                    if (k < (uint32_t)kKeyBigCap) {
                        t.kbig[k] = make_uint4((uint32_t)L, a, e, 0u);
                        listed = true;
                    }
                    break;
                }
            }
        }
        if (__shfl_sync(0xffffffffu, listed, 0)) continue;
        for (uint32_t j = a + lane; j < e; j += 32) atomicMin(&t.kxr[j], (uint32_t)L);
    }
}

// Node starts of every level, per tile (kKeyTile particles): ktile[L][tile]
template <int D>
__global__ void __launch_bounds__(kKT)
k_key_count(StepParams p, Tree t, int tiles) {
    dep_wait();
    constexpr int NL = KeyBits<D>::B + 1;
    constexpr uint32_t kTileBig = 32;
    __shared__ uint32_t sc[NL];
    __shared__ uint4 s_big[kTileBig];
    __shared__ uint32_t s_nb;
    if (threadIdx.x < NL) sc[threadIdx.x] = 0u;
    if (threadIdx.x == 0) s_nb = 0u;
    __syncthreads();
    const uint32_t a = blockIdx.x * kKeyTile + threadIdx.x;
    const bool valid = a < (uint32_t)p.n;
    // the large exact-rebuild roots that k_key_check listed instead of
    // marking: the ones over this tile are applied to kxr here
    const uint32_t nbig = min(t.kmeta[kKmBig], (uint32_t)kKeyBigCap);
    if (nbig) {   // block-uniform
        const uint32_t t0 = blockIdx.x * kKeyTile, t1 = t0 + kKeyTile;
        for (uint32_t q = threadIdx.x; q < nbig; q += kKT) {
            const uint4 b = t.kbig[q];
            if (b.y < t1 && b.z > t0) {
                const uint32_t k = atomicAdd(&s_nb, 1u);
                if (k < kTileBig) s_big[k] = b;
            }
        }
        __syncthreads();
        const uint32_t nb = s_nb;
        if (valid && nb) {
            uint32_t x = t.kxr[a];
            const uint32_t x0 = x;
            for (uint32_t q = 0; q < (nb <= kTileBig ? nb : nbig); q++) {
                const uint4 b = nb <= kTileBig ? s_big[q] : t.kbig[q];
                if (b.y <= a && a < b.z) x = min(x, b.x);
            }
            if (x != x0) t.kxr[a] = x;
        }
    }
    const uint32_t dl = valid ? t.kdl[a] : 1u, T = valid ? key_depth(t, a) : 0u;
#pragma unroll
    for (int L = 0; L < NL; L++) {
        const unsigned b = __ballot_sync(0xffffffffu, dl <= (uint32_t)L && (uint32_t)L <= T);
        if ((threadIdx.x & 31u) == 0 && b) atomicAdd(&sc[L], (uint32_t)__popc(b));
    }
    __syncthreads();
    if (threadIdx.x < NL) t.ktile[(size_t)threadIdx.x * tiles + blockIdx.x] = sc[threadIdx.x];
}

// one block per level: exclusive prefix of the tiles' counts, and the total
template <int D>
__global__ void __launch_bounds__(1024)
k_key_scan(Tree t, int tiles) {
    dep_wait();
    __shared__ uint32_t sw[32];
    __shared__ uint32_t s_carry;
    const int L = blockIdx.x;
    uint32_t *col = t.ktile + (size_t)L * tiles;
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0u;
    __syncthreads();
    for (int base = 0; base < tiles; base += 1024) {
        const int k = base + threadIdx.x;
        const uint32_t v = k < tiles ? col[k] : 0u;
        uint32_t incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += u;
        }
        if (lane == 31) sw[w] = incl;
        __syncthreads();
        if (w == 0) {
            const uint32_t x = sw[lane];
            uint32_t xi = x;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t u = __shfl_up_sync(0xffffffffu, xi, o);
                if (lane >= (unsigned)o) xi += u;
            }
            sw[lane] = xi - x;
        }
        __syncthreads();
        const uint32_t carry = s_carry;
        if (k < tiles) col[k] = carry + sw[w] + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = carry + sw[w] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) t.kmeta[kKmLevelTot + L] = s_carry;
}

// Node slots: level L's nodes are the slots from base[L] = the node count of
// the levels above, in the order of their first particles.  Per warp and
// level, the ballot of the particles that start a level-L node ranks them, so
// with off[L][w] = the level-L nodes started before the warp:
//   a starts (L, a)                   -> slot off[L][w] + popc(ballot & below a)
//   the level-L node holding a        -> off[L][w] + popc(ballot & up to a) - 1
//   the node holding a-1 ends at a (a a level-L boundary) -> slot off[L][w] + popc(ballot & below a) - 1
// Each particle then writes the few nodes it starts and ends.  Masses follow
// bottom-up, one thread per node of the tile and level.
template <int D>
__global__ void __launch_bounds__(kKT, 8)
k_key_emit(State s, StepParams p, Segs g, const uint64_t *__restrict__ keys, Tree t, int tiles,
           uint32_t *err) {
    dep_wait();
    constexpr int B = KeyBits<D>::B, NL = B + 1, W = kKT / 32, Q = 1 << D;
    __shared__ uint32_t s_bal[NL][W];      // per level and warp: the particles that start a node
    __shared__ uint32_t s_off[NL][W + 1];  // slot of each warp's first level-L node; [W] = end
    __shared__ uint8_t s_start[NL][kKT];   // the particle that starts the tile's j-th level-L node
    __shared__ uint32_t s_loc[NL][W];      // bit j: that node ends inside the tile
    __shared__ uint32_t s_total, s_maxT;
    __shared__ float4 s_leaf[kKT];         // leaf masses by the particle that starts the leaf
    __shared__ float4 s_walk[2][kKT];      // masses by level parity, by node within the tile
    __shared__ uint8_t s_done[2][kKT];
    __shared__ uint8_t s_lam[kKT], s_x[kKT], s_dlb[kKT];
    __shared__ float s_rs[kKT];            // root size of each particle's simulation
    __shared__ uint32_t s_cm[NL][kKT / 4]; // child masks of the nodes started in the tile (bytes)
    const uint32_t n = (uint32_t)p.n;
    const unsigned tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    const unsigned lt = (1u << lane) - 1u, le = lt | (1u << lane);
    const uint32_t a = blockIdx.x * kKeyTile + tid;
    const uint32_t w0 = blockIdx.x * kKeyTile;
    const bool valid = a < n;
    const uint32_t dl = valid ? t.kdl[a] : 1u;   // a starts the nodes of levels dl .. T
    const uint32_t T = valid ? key_depth(t, a) : 0u;
    const uint32_t Tp = valid && a > 0 ? key_depth(t, a - 1) : 0u;
    const uint32_t X = valid ? __ldcg(&t.kxr[a]) : kEmpty;
    const uint32_t lam = valid ? (uint32_t)t.klam[a] : 0u;
    const uint32_t dlb = valid ? dl : 0u;   // past the array's end: a boundary at every level
#pragma unroll
    for (int L = 0; L < NL; L++) {
        const unsigned b = __ballot_sync(0xffffffffu, dl <= (uint32_t)L && (uint32_t)L <= T);
        if (lane == 0) { s_bal[L][w] = b; s_loc[L][w] = 0u; }
    }
    for (int k = tid; k < NL * (kKT / 4); k += kKT) (&s_cm[0][0])[k] = 0u;
    s_lam[tid] = (uint8_t)lam;
    s_x[tid] = (uint8_t)min(X, 255u);
    s_dlb[tid] = (uint8_t)dlb;
    if (tid == 0) s_maxT = 0u;
    __syncthreads();
    if (w == 0) {   // lane L: level L's slots (NL <= 32)
        const uint32_t c = lane < (unsigned)NL ? t.kmeta[kKmLevelTot + lane] : 0u;
        const uint32_t kt = lane < (unsigned)NL ? t.ktile[(size_t)lane * tiles + blockIdx.x] : 0u;
        uint32_t incl = c;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += u;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        if (lane < (unsigned)NL) {
            uint32_t run = incl - c + kt;
            for (int ww = 0; ww < W; ww++) {
                s_off[lane][ww] = run;
                run += (uint32_t)__popc(s_bal[lane][ww]);
            }
            s_off[lane][W] = run;
        }
        if (lane == 0) s_total = tot;
        if (blockIdx.x == 0 && lane == 0) t.kmeta[kKmTotal] = tot;
    }
    if (valid && dl <= T) atomicMax(&s_maxT, T);
    __syncthreads();
    if ((int64_t)s_total > t.cap) {   // the build kernel sees the same total and stops
        if (blockIdx.x == 0 && tid == 0) set_err(err, kErrNodeCap);
        return;
    }
    uint32_t *info = reinterpret_cast<uint32_t *>(t.info);
    uint32_t *aux = reinterpret_cast<uint32_t *>(t.aux);
    float rs = 0.0f;
    if (valid) {
        const uint32_t sg = g.seg_of ? g.seg_of[a] : 0u;
        const float4 box = g.box[sg];
        rs = box.w;
        // the nodes a starts: cells along a's key path, from the root
        if (dl <= T) {
            const uint64_t key = key_at<D>(keys, a);
            float cor[3] = {box.x, box.y, box.z};
            float sz = box.w;
            for (uint32_t L = 0; L < dl; L++) {
                const float half = fmul(sz, 0.5f);
                const unsigned q = digit<D>(key, (int)L);
#pragma unroll
                for (int ax = 0; ax < D; ax++) cor[ax] = fadd(cor[ax], ((q >> ax) & 1u) ? half : 0.0f);
                sz = half;
            }
            for (uint32_t L = dl; L <= T; L++) {
                const uint32_t slot = s_off[L][w] + (uint32_t)__popc(s_bal[L][w] & lt);
                s_start[L][slot - s_off[L][0]] = (uint8_t)tid;
                t.cell[slot] = make_float4(cor[0], cor[1], D == 3 ? cor[2] : 0.0f, sz);
                info[4 * (size_t)slot + 0] =
                    L < T ? s_off[L + 1][w] + (uint32_t)__popc(s_bal[L + 1][w] & lt) : 0u;
                info[4 * (size_t)slot + 2] = a;
                const uint32_t parent =
                    L > 0 ? s_off[L - 1][w] + (uint32_t)__popc(s_bal[L - 1][w] & le) - 1u : kEmpty;
                aux[4 * (size_t)slot + 0] = L;
                aux[4 * (size_t)slot + 2] = parent;
                aux[4 * (size_t)slot + 3] = L == X ? 1u : 0u;
                if (L > 0) {
                    const uint32_t bit = 1u << digit<D>(key, (int)L - 1);
                    atomicOr(&t.pend[parent], bit);
                    // and in the tile's copy when the parent started in the tile
                    const uint32_t pl = parent - s_off[L - 1][0];
                    if (parent >= s_off[L - 1][0] && pl < (uint32_t)kKT)
                        atomicOr(&s_cm[L - 1][pl >> 2], bit << (8u * (pl & 3u)));
                }
                if (L == X) {   // exact-rebuild roots have disjoint ranges: fewer than n
                    atomicOr(&t.pend[slot], 1u << 31);
                    const uint32_t r = atomicAdd(&t.kmeta[kKmRoots], 1u);
                    if (r < n) t.kroots[r] = slot;
                }
                if (L < T) {
                    const float half = fmul(sz, 0.5f);
                    const unsigned q = digit<D>(key, (int)L);
#pragma unroll
                    for (int ax = 0; ax < D; ax++) cor[ax] = fadd(cor[ax], ((q >> ax) & 1u) ? half : 0.0f);
                    sz = half;
                }
            }
        }
        // the nodes holding a-1 that end at a (and, when they started in the
        // tile, their bits in s_loc)
        if (a > 0)
            for (uint32_t L = dl; L <= Tp; L++) {
                const uint32_t slot = s_off[L][w] + (uint32_t)__popc(s_bal[L][w] & lt) - 1u;
                info[4 * (size_t)slot + 3] = a;
                aux[4 * (size_t)slot + 1] = L - dl;
                const uint32_t j = slot - s_off[L][0];
                if (slot >= s_off[L][0]) atomicOr(&s_loc[L][j >> 5], 1u << (j & 31u));
            }
        // how many key nodes end at a (and at n): the walk layout's end counts
        t.endcnt[a] = a > 0 && dl <= Tp ? Tp - dl + 1u : 0u;
        if (a == n - 1) t.endcnt[n] = T + 1u;
        if (a == n - 1)   // the nodes that end at the end of the particle array
            for (uint32_t L = 0; L <= T; L++) {
                const uint32_t slot = s_off[L][w] + (uint32_t)__popc(s_bal[L][w] & le) - 1u;
                info[4 * (size_t)slot + 3] = n;
                aux[4 * (size_t)slot + 1] = L;
                const uint32_t j = slot - s_off[L][0];
                if (slot >= s_off[L][0]) atomicOr(&s_loc[L][j >> 5], 1u << (j & 31u));
            }
        // a leaf's mass (computeLeafMass): up to the first level-T boundary after a
        if (dl <= T && T == lam && T != X) {
            uint32_t e = a + 1u;
            while (e < w0 + kKT && s_dlb[e - w0] > T) e++;
            if (e == w0 + kKT)
                while (e < n && t.kdl[e] > T) e++;
            s_leaf[tid] = leaf_mass<D>(s, a, e);
        }
    }
    s_rs[tid] = rs;
    {
        const uint32_t ml = __reduce_max_sync(0xffffffffu, valid && dl <= T ? T + 1u : 0u);
        if (lane == 0 && ml) atomicMax(&t.kmeta[kKmLevels], ml);
    }
    __syncthreads();

    // ---- masses, bottom-up: every leaf, and every node whose particles all
    // lie in this tile and whose children are all done (not an exact-rebuild
    // root or above one).  A done node's walk entry is final and its aux.w is
    // 2; the build kernel combines the rest.  A node's children are the
    // contiguous level-(L+1) slots from its first child, in quadrant order. ----
    const uint32_t dl_next = w0 + kKT < n ? t.kdl[w0 + kKT] : 0u;
    for (int L = (int)s_maxT; L >= 0; --L) {
        const uint32_t first = s_off[L][0], K = s_off[L][W] - first;
        if (K == 0u) continue;   // no node of this level starts in the tile
        if (tid < K) {
            const uint32_t slot = first + tid;
            const uint32_t o = s_start[L][tid];   // tile index of the starting particle
            const uint32_t ww = o >> 5, ol = o & 31u;
            bool done = false;
            float4 cm = make_float4(0.f, 0.f, 0.f, 0.f);
            const uint32_t ox = s_x[o];
            if ((uint32_t)L != ox) {
                if ((uint32_t)L == s_lam[o]) {
                    cm = s_leaf[o];
                    done = true;
                } else {
                    // inside the tile: a particle of the tile ended it, or the
                    // next tile's first particle is a level-L boundary
                    const bool local = dl_next <= (uint32_t)L || ((s_loc[L][tid >> 5] >> (tid & 31u)) & 1u);
                    if (local) {
                        // all its children started in the tile: their bits are in s_cm
                        const uint32_t mask = (s_cm[L][tid >> 2] >> (8u * (tid & 3u))) & 0xFFu;
                        const uint32_t c0 = s_off[L + 1][ww] + (uint32_t)__popc(s_bal[L + 1][ww] & ((1u << ol) - 1u))
                                            - s_off[L + 1][0];   // first child, tile index
                        const int pb = (L + 1) & 1;
                        const uint32_t nch = (uint32_t)__popc(mask);
                        bool all = true;
                        for (uint32_t c = 0; c < nch; c++) all = all && s_done[pb][c0 + c];
                        if (all) {   // computeInternalMass: children x-major
                            float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
                            for (int kk = 0; kk < Q; kk++) {
                                unsigned q;
                                if (D == 2) q = ((kk >> 1) & 1) | ((kk & 1) << 1);
                                else q = ((kk >> 2) & 1) | (((kk >> 1) & 1) << 1) | ((kk & 1) << 2);
                                if (!((mask >> q) & 1u)) continue;
                                const float4 cw = s_walk[pb][c0 + __popc(mask & ((1u << q) - 1u))];
                                gm = fadd(gm, cw.w);
                                c[0] = fadd(c[0], fmul(cw.x, cw.w));
                                c[1] = fadd(c[1], fmul(cw.y, cw.w));
                                if (D == 3) c[2] = fadd(c[2], fmul(cw.z, cw.w));
                            }
                            if (gm > 0.0f) {
                                c[0] = fdiv(c[0], gm); c[1] = fdiv(c[1], gm);
                                if (D == 3) c[2] = fdiv(c[2], gm);
                            }
                            cm = make_float4(c[0], c[1], c[2], gm);
                            done = true;
                        }
                    }
                }
            }
            s_done[L & 1][tid] = done ? 1u : 0u;
            if (done) {
                s_walk[L & 1][tid] = cm;
                // size at level L: the root's halved L times (exact)
                const float szl = s_rs[o] * __int_as_float((127 - L) << 23);
                put_walk<D>(t, slot, cm, szl);
                aux[4 * (size_t)slot + 3] = 2u;
            }
        }
        __syncthreads();
    }
}

template <int D>
cudaError_t key_build(const State &s, const StepParams &p, const Segs &g, const uint64_t *keys,
                      Tree &t, uint32_t *err, int num_sms, cudaStream_t st) {
    constexpr int NL = KeyBits<D>::B + 1;
    const int n = p.n;
    cudaError_t e = launch_zero(t.kmeta, kKeyMetaWords, st);
    if (e != cudaSuccess) return e;
    const int blocks = (n + kKT - 1) / kKT;
    if ((e = launch_dep(k_key_levels<D>, blocks, kKT, st, s, p, g, keys, t)) != cudaSuccess) return e;
    if ((e = launch_dep(k_key_check<D>, num_sms * 4, kKT, st, s, p, g, keys, t)) != cudaSuccess) return e;
    const int tiles = (n + kKeyTile - 1) / kKeyTile;
    if ((e = launch_dep(k_key_count<D>, tiles, kKT, st, p, t, tiles)) != cudaSuccess) return e;
    if ((e = launch_dep(k_key_scan<D>, NL, 1024, st, t, tiles)) != cudaSuccess) return e;
    return launch_dep(k_key_emit<D>, tiles, kKT, st, s, p, g, keys, t, tiles, err);
}

}  // namespace

int64_t key_suspect_cap(int64_t n) { return n / 8 + 4096; }

cudaError_t launch_key_build(int dims, const State &s, const StepParams &p, const Segs &g,
                             const uint64_t *keys, Tree &t, uint32_t *err, int num_sms,
                             cudaStream_t st) {
    if (p.n < 1) return cudaSuccess;
    if ((int64_t)(p.n + kKeyTile - 1) / kKeyTile > (int64_t)t.ktile_cap) return cudaErrorInvalidValue;
    return dims == 2 ? key_build<2>(s, p, g, keys, t, err, num_sms, st)
                     : key_build<3>(s, p, g, keys, t, err, num_sms, st);
}

}  // namespace ge
