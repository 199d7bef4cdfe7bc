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
              kKmLevelTot = 8;

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
    constexpr int B = KeyBits<D>::B;
    __shared__ int8_t sd[kKT + 2 * kHalo + 1];
    const int n = p.n;
    const int64_t base = (int64_t)blockIdx.x * kKT;
    for (int q = threadIdx.x; q < kKT + 2 * kHalo + 1; q += kKT)
        sd[q] = (int8_t)delta_at<D>(g, keys, base - kHalo + q, n);
    // parent child bits and counts are accumulated into pend by the emit pass
    for (int64_t k = (int64_t)blockIdx.x * kKT + threadIdx.x; k < t.cap;
         k += (int64_t)gridDim.x * kKT)
        t.pend[k] = 0u;
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
    int l_gate = 127, l_min = 127;
    {
        float sz = box.w;
        for (int L = 0; L <= B; L++) {
            if (l_gate == 127 && sz <= p.size_gate) l_gate = L;
            if (sz <= p.min_size) { l_min = L; break; }
            sz = fmul(sz, 0.5f);
        }
    }
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
// false), by a whole warp (all lanes call it with the same arguments and
// get the same result): 32 probes per round narrow the range 33-fold.
template <typename F>
__device__ __forceinline__ uint32_t warp_lower_bound(uint32_t first, uint32_t last, F pred) {
    const unsigned lane = threadIdx.x & 31u;
    while (last - first > 32u) {
        const uint32_t len = last - first;
        const uint32_t q = first + (uint32_t)(((uint64_t)len * (lane + 1u)) / 33u);
        const unsigned t = __popc(__ballot_sync(0xffffffffu, pred(q)));   // probes still true
        const uint32_t nf = t ? __shfl_sync(0xffffffffu, q, t - 1) + 1u : first;
        const uint32_t nl = t < 32u ? __shfl_sync(0xffffffffu, q, t) + 1u : last;
        first = nf;
        last = nl;
    }
    const bool v = first + lane < last && pred(first + lane);
    return first + (uint32_t)__popc(__ballot_sync(0xffffffffu, v));
}

template <int D>
__global__ void __launch_bounds__(kKT)
k_key_check(State s, StepParams p, Segs g, const uint64_t *__restrict__ keys, Tree t) {
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
        // the node's range: the run of keys that agree with ki on L digits
        const uint32_t a =
            warp_lower_bound(lo, i, [&](uint32_t j) { return (key_at<D>(keys, j) >> shift) < pre; });
        const uint32_t e = warp_lower_bound(
            i + 1, hi, [&](uint32_t j) { return (key_at<D>(keys, j) >> shift) <= pre; });
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
        // the key boundaries: first particle of every digit value
        bool differ = false;
        for (unsigned q = 1; q < (unsigned)Q; q++) {
            const uint32_t kb = warp_lower_bound(
                a, e, [&](uint32_t j) { return digit<D>(key_at<D>(keys, j), L) < q; });
            differ |= kb != b[q];
        }
        if (differ)
            for (uint32_t j = a + lane; j < e; j += 32) atomicMin(&t.kxr[j], (uint32_t)L);
    }
}

// Node starts of every level, per tile (kKeyTile particles): ktile[L][tile]
template <int D>
__global__ void __launch_bounds__(kKT)
k_key_count(StepParams p, Tree t, int tiles) {
    constexpr int NL = KeyBits<D>::B + 1;
    __shared__ uint32_t sc[NL];
    if (threadIdx.x < NL) sc[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t a = blockIdx.x * kKeyTile + threadIdx.x;
    const bool valid = a < (uint32_t)p.n;
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
// the levels above, in the order of their first particles.  A warp walks the
// levels together; the ballot of the lanes that start a level-L node ranks
// them.  With excl = the level-L nodes started before particle a:
//   a starts (L, a)            -> slot excl
//   the level-L node holding a -> excl - 1 + (a starts it)
//   the node holding a-1 ends at a when a is a level-L boundary -> slot excl - 1
template <int D>
__global__ void __launch_bounds__(kKT)
k_key_emit(State s, StepParams p, Segs g, const uint64_t *__restrict__ keys, Tree t, int tiles,
           uint32_t *err) {
    constexpr int B = KeyBits<D>::B, NL = B + 1, W = kKT / 32, Q = 1 << D;
    __shared__ uint32_t s_w[NL][W];     // per warp: level-L starts; then their offsets
    __shared__ uint32_t s_total, s_maxT;
    __shared__ uint32_t s_slot[NL][kKT];   // slot of the level-L node each particle starts
    __shared__ float4 s_walk[2][kKT];       // mass and centre of mass by level parity
    __shared__ uint8_t s_done[2][kKT];
    __shared__ uint64_t s_key[kKT];
    __shared__ uint8_t s_dl[kKT];
    __shared__ uint32_t s_bb[W], s_bc[W];
    const uint32_t n = (uint32_t)p.n;
    const unsigned tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t a = blockIdx.x * kKeyTile + tid;
    const bool valid = a < n;
    const uint32_t dl = valid ? t.kdl[a] : 1u;   // a starts the nodes of levels dl .. T
    const uint32_t T = valid ? key_depth(t, a) : 0u;
    const uint32_t Tp = valid && a > 0 ? key_depth(t, a - 1) : 0u;
    const bool ends = valid && a > 0 && dl <= Tp;   // nodes holding a-1 end at a
#pragma unroll
    for (int L = 0; L < NL; L++) {
        const unsigned b = __ballot_sync(0xffffffffu, dl <= (uint32_t)L && (uint32_t)L <= T);
        if (lane == 0) s_w[L][w] = (uint32_t)__popc(b);
    }
    __syncthreads();
    if (tid < NL) {
        uint32_t base = 0, tot = 0;
        for (int L = 0; L < NL; L++) {
            const uint32_t c = t.kmeta[kKmLevelTot + L];
            if (L < (int)tid) base += c;
            tot += c;
        }
        uint32_t run = base + t.ktile[(size_t)tid * tiles + blockIdx.x];
        for (int ww = 0; ww < W; ww++) {
            const uint32_t c = s_w[tid][ww];
            s_w[tid][ww] = run;
            run += c;
        }
        if (tid == 0) s_total = tot;
        if (blockIdx.x == 0 && tid == 0) t.kmeta[kKmTotal] = tot;
    }
    __syncthreads();
    if ((int64_t)s_total > t.cap) {   // the build kernel sees the same total and stops
        if (blockIdx.x == 0 && tid == 0) set_err(err, kErrNodeCap);
        return;
    }
    uint32_t *info = reinterpret_cast<uint32_t *>(t.info);
    uint32_t *aux = reinterpret_cast<uint32_t *>(t.aux);
    const uint32_t X = valid ? __ldcg(&t.kxr[a]) : kEmpty;
    uint64_t key = 0;
    float cor[3] = {0.f, 0.f, 0.f}, sz = 0.f;
    if (valid && dl <= T) {
        key = key_at<D>(keys, a);
        const float4 box = g.box[g.seg_of ? g.seg_of[a] : 0u];
        cor[0] = box.x; cor[1] = box.y; cor[2] = box.z;
        sz = box.w;
    }
    const uint32_t top = valid ? max(T, ends ? Tp : 0u) : 0u;
    const float root_size = sz;
    uint32_t held = kEmpty;   // the level-(L-1) node holding a
    uint32_t maxl = 0;
    for (int L = 0; L < NL; L++) {
        if (!__any_sync(0xffffffffu, valid && (uint32_t)L <= top)) break;
        const bool st = dl <= (uint32_t)L && (uint32_t)L <= T;
        const unsigned b = __ballot_sync(0xffffffffu, st);
        const uint32_t excl = s_w[L][w] + (uint32_t)__popc(b & lt);
        if (ends && dl <= (uint32_t)L && (uint32_t)L <= Tp) {
            info[4 * (size_t)(excl - 1u) + 3] = a;
            aux[4 * (size_t)(excl - 1u) + 1] = (uint32_t)L - dl;
        }
        if (valid && st) {
            const uint32_t slot = excl;
            s_slot[L][tid] = slot;
            t.cell[slot] = make_float4(cor[0], cor[1], D == 3 ? cor[2] : 0.0f, sz);
            info[4 * (size_t)slot + 2] = a;
            if ((uint32_t)L == T) info[4 * (size_t)slot + 0] = 0u;
            if ((uint32_t)L > dl) info[4 * (size_t)held + 0] = slot;   // a's own parent
            aux[4 * (size_t)slot + 0] = (uint32_t)L;
            aux[4 * (size_t)slot + 2] = L > 0 ? held : kEmpty;
            aux[4 * (size_t)slot + 3] = (uint32_t)L == X ? 1u : 0u;
            if (L > 0) atomicOr(&t.pend[held], 1u << digit<D>(key, L - 1));
            if ((uint32_t)L == X) {   // exact-rebuild roots have disjoint ranges: fewer than n
                atomicOr(&t.pend[slot], 1u << 31);
                const uint32_t r = atomicAdd(&t.kmeta[kKmRoots], 1u);
                if (r < n) t.kroots[r] = slot;
            }
            maxl = max(maxl, (uint32_t)L);
        }
        const uint32_t hold = excl - 1u + (st ? 1u : 0u);   // the level-L node holding a
        if (valid && a == n - 1 && (uint32_t)L <= T) {       // nodes ending at the array's end
            info[4 * (size_t)hold + 3] = n;
            aux[4 * (size_t)hold + 1] = (uint32_t)L;
        }
        held = hold;
        if (valid && dl <= T && (uint32_t)L < T) {
            const float half = fmul(sz, 0.5f);
            const unsigned q = digit<D>(key, L);
#pragma unroll
            for (int ax = 0; ax < D; ax++) cor[ax] = fadd(cor[ax], ((q >> ax) & 1u) ? half : 0.0f);
            sz = half;
        }
    }
    for (int o = 16; o > 0; o >>= 1) maxl = max(maxl, __shfl_xor_sync(0xffffffffu, maxl, o));
    if (lane == 0) atomicMax(&t.kmeta[kKmLevels], maxl + 1u);

    // ---- masses, bottom-up: every leaf, and every node whose particles all
    // lie in this tile and whose children are all done (not an exact-rebuild
    // root or above one).  A done node's walk entry is final and its aux.w is
    // 2; the build kernel combines the rest.  Sums in the reference's order:
    // a leaf's particles in order, a node's children x-major. ----
    s_key[tid] = key;
    const uint32_t dlb = valid ? dl : 0u;   // past the array's end: a boundary at every level
    s_dl[tid] = (uint8_t)dlb;
    if (tid == 0) s_maxT = 0u;
    __syncthreads();
    if (valid && dl <= T) atomicMax(&s_maxT, T);
    const uint32_t w0 = blockIdx.x * kKeyTile;
    const uint32_t lam = valid ? (uint32_t)t.klam[a] : 0u;
    // a leaf's mass first (its range: up to the first level-T boundary after a)
    float4 leaf_cm = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid && dl <= T && T == lam && T != X) {
        uint32_t e = a + 1u;
        while (e < w0 + kKT && e < n && s_dl[e - w0] > T) e++;
        if (e == w0 + kKT)
            while (e < n && t.kdl[e] > T) e++;
        leaf_cm = leaf_mass<D>(s, a, e);
    }
    __syncthreads();
    // the next tile's first particle bounds every level at or below dl_next
    const uint32_t dl_next = w0 + kKT < n ? t.kdl[w0 + kKT] : 0u;
    for (int L = (int)s_maxT; L >= 0; --L) {
        const unsigned bb = __ballot_sync(0xffffffffu, dlb <= (uint32_t)L);
        const unsigned bc = __ballot_sync(0xffffffffu, valid && dl == (uint32_t)L + 1u);
        if (lane == 0) { s_bb[w] = bb; s_bc[w] = bc; }
        __syncthreads();
        if (valid && dl <= (uint32_t)L && (uint32_t)L <= T) {
            const uint32_t slot = s_slot[L][tid];
            bool done = false;
            float4 cm = make_float4(0.f, 0.f, 0.f, 0.f);
            if ((uint32_t)L != X) {
                // the node's end: the first level-L boundary after a (tile index)
                uint32_t ie = kKT;
                if ((uint32_t)L != lam)
                    for (uint32_t wi = (tid + 1u) >> 5; wi < (uint32_t)W; wi++) {
                        uint32_t bits = s_bb[wi];
                        if (wi == ((tid + 1u) >> 5)) bits &= ~((1u << ((tid + 1u) & 31u)) - 1u);
                        if (bits) { ie = wi * 32u + (uint32_t)(__ffs(bits) - 1); break; }
                    }
                if ((uint32_t)L == lam) {   // leaf (computeLeafMass, above)
                    cm = leaf_cm;
                    done = true;
                } else if (ie < (uint32_t)kKT || dl_next <= (uint32_t)L) {
                    // inside the tile: children start at a and at the level-(L+1)
                    // boundaries before the end
                    const int pb = (L + 1) & 1;
                    uint64_t lanes = 0;
                    uint32_t cmask = 0;
                    bool all = true;
                    auto take = [&](uint32_t j) {
                        const unsigned q = digit<D>(s_key[j], L);
                        cmask |= 1u << q;
                        lanes |= (uint64_t)j << (8 * q);
                        all = all && s_done[pb][j];
                    };
                    take(tid);
                    for (uint32_t wi = (tid + 1u) >> 5; wi < (uint32_t)W && wi * 32u < ie; wi++) {
                        uint32_t bits = s_bc[wi];
                        if (wi == ((tid + 1u) >> 5)) bits &= ~((1u << ((tid + 1u) & 31u)) - 1u);
                        if (ie < wi * 32u + 32u) bits &= (1u << (ie & 31u)) - 1u;
                        while (bits) {
                            take(wi * 32u + (uint32_t)(__ffs(bits) - 1));
                            bits &= bits - 1u;
                        }
                    }
                    if (all) {   // computeInternalMass: children x-major
                        float gm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
                        for (int kk = 0; kk < Q; kk++) {
                            unsigned q;
                            if (D == 2) q = ((kk >> 1) & 1) | ((kk & 1) << 1);
                            else q = ((kk >> 2) & 1) | (((kk >> 1) & 1) << 1) | ((kk & 1) << 2);
                            if (!((cmask >> q) & 1u)) continue;
                            const float4 cw = s_walk[pb][(lanes >> (8 * q)) & 0xFFu];
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
            s_done[L & 1][tid] = done ? 1u : 0u;
            if (done) {
                s_walk[L & 1][tid] = cm;
                float szl = root_size;
                for (int l = 0; l < L; l++) szl = fmul(szl, 0.5f);
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
    cudaError_t e = cudaMemsetAsync(t.kmeta, 0, sizeof(uint32_t) * kKeyMetaWords, st);
    if (e != cudaSuccess) return e;
    const int blocks = (n + kKT - 1) / kKT;
    k_key_levels<D><<<blocks, kKT, 0, st>>>(s, p, g, keys, t);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_key_check<D><<<num_sms * 4, kKT, 0, st>>>(s, p, g, keys, t);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int tiles = (n + kKeyTile - 1) / kKeyTile;
    k_key_count<D><<<tiles, kKT, 0, st>>>(p, t, tiles);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_key_scan<D><<<NL, 1024, 0, st>>>(t, tiles);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_key_emit<D><<<tiles, kKT, 0, st>>>(s, p, g, keys, t, tiles, err);
    return cudaGetLastError();
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
