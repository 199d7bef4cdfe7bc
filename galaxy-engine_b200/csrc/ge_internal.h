// ge_internal.h -- device buffer layout and kernel launchers shared by the
// C-ABI host code (ge_api.cu) and the kernel files.
#pragma once
#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

#include "ge_bh.h"

namespace ge {

// Launch that may begin while the previous kernel in the stream drains
// (programmatic dependent launch): its blocks are scheduled early and wait in
// dep_wait() for the previous kernel's completion, so only the launch latency
// overlaps.  The kernel must call dep_wait() before touching memory.
template <typename... KArgs, typename... Args>
cudaError_t launch_dep(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st,
                       Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Particle state, structure-of-arrays, in Morton order.  z/vz/az are unused
// in 2D.  pvx..pvz (prevVel) and pinned are optional (nullptr).
struct State {
    float *x, *y, *z;
    float *vx, *vy, *vz;
    float *ax, *ay, *az;
    float *m;
    uint32_t *id;
    float *pvx, *pvy, *pvz;
    uint8_t *pinned;
    // GE_PREC_MIXED: Kahan compensation terms of positions and velocities
    // (nullptr in the other modes)
    float *kx, *ky, *kz;
    float *kvx, *kvy, *kvz;
    float *temp;          // temperatures (nullptr unless heat exchange is on)
};

// Tree nodes, structure-of-arrays.
//   walk    float4  2D: {com.x, com.y, mass, size^2}   3D: {com.x, com.y, com.z, mass}
//   size2   float   3D only: size^2
//   info    uint4   {first_child, child_mask, start, end}; child_mask bit q set when
//                   child slot q is occupied; children are stored contiguously from
//                   first_child in increasing q; child_mask == 0 marks a leaf
//   cell    float4  {corner.x, corner.y, corner.z, size} (build only)
//   level   uint32  first node of each level (nodes are stored level by level)
//   aux     uint4   {level, number of proper ancestors whose range ends where this
//                   node's range ends, parent, walk entry (set by the layout)}
//   pend    uint32  children whose mass is not final yet (build only)
//
// Walk layout (written at the end of the build): one array of "sources" in
// depth-first pre-order in which every leaf is followed by its particles, so
// opening any source leads to the next entry (first child, or the leaf's
// first particle) and only the skip target has to be stored:
//   src     float4  2D node {com.x, com.y, mass, size^2}; particle {x, y, m, -1}
//                   3D node {com.x, com.y, com.z, mass};  particle {x, y, z, m}
//   link    2D uint32 skip; 3D uint2 {skip, size^2 bits} (particles: size^2 = -1,
//                   massless nodes: -2, both accepted by every opening test).  skip is where the walk
//                   goes after accepting the entry: the successor of the node's
//                   subtree, or the next entry for a particle.
//   slot_of uint32  entry index of each particle (for the self test)
// The walk starts at entry 0 (the root) and ends at node_count + n.  The
// positions need no top-down pass: with C(e) = #{nodes whose range ends at or
// before e}, node k sits at C(start_k) + level_k + start_k and its subtree's
// successor at C(end_k) + level_k - same_end_ancestors_k + end_k.
struct Tree {
    float4 *walk;
    float *size2;
    uint4 *info;
    float4 *cell;
    uint4 *aux;
    uint32_t *pend;
    uint2 *small;         // [small_cap] queued small subtrees {node slot, build id} (build only)
    uint32_t small_cap;
    uint32_t *endcnt;    // [n + 1] node-end histogram, scanned in place
    uint32_t *blocksum;   // [build grid] scan partials
    float4 *src;          // [n + cap + 1]
    void *link;           // [n + cap + 1] uint32 (2D) / uint2 (3D)
    uint32_t *slot_of;    // [n]
    uint2 *nrange;        // [cap] each node slot's {layout entry, subtree successor}
    uint32_t *wctr;       // [kWWCtrWords] warp walk: chunk counter, fallback count
    uint32_t *level;      // [kMaxLevels + 2]
    uint32_t *lvl_alloc;  // [kMaxLevels + 2] per-level child allocation counters
    uint32_t *meta;       // [8] {node_count, levels, bar_count, bar_gen, err, small,
                          //      phase-2 nodes, timeline entries}
    unsigned long long *tl;   // [kTimeline] build timeline (globaltimer ns)
    // GE_PREC_MIXED node moments (nullptr in the other modes):
    //   mom   double [cap * kMomWords]  {mass, com (D), second moments about the
    //                                   com (xx, xy, yy | xx, yy, zz, xy, xz, yz)}
    //   mq0   float4 per walk entry     2D {com_lo.x, com_lo.y, Ixx, Ixy}
    //                                   3D {com_lo.x, com_lo.y, com_lo.z, Ixx}
    //   mq1   float4 per walk entry     3D {Iyy, Izz, Ixy, Ixz}
    //   mq2   float  per walk entry     2D Iyy, 3D Iyz
    // (com = src com + com_lo as a double-float pair)
    double *mom;
    float4 *mq0, *mq1;
    float *mq2;
    // the same per node slot, for the group walk (nullptr when unused):
    //   gw    float4  2D {com_hi.x, com_hi.y, mass, b^2}  3D {com_hi.x, com_hi.y, com_hi.z, mass}
    //   gq0   float4  as mq0;  gq1 float4 3D as mq1
    //   gq2   float2  2D {Iyy, 0}   3D {Iyz, b^2}
    // (mass 0 marks a massless node)
    float4 *gw, *gq0, *gq1;
    float2 *gq2;
    uint32_t *wl;         // group walk: a work stack per resident warp
    uint32_t wl_warps;    // warps the work stacks are sized for
    uint2 *grp;           // group walk: particle range of each group [n + 1]
    // heat exchange (nullptr unless on): node temperature sums per slot, and
    // per walk entry the temperature the walk reads (a node's average, a
    // particle's own, both as before the walk)
    float *ntemp;
    float *tv;
    // key-prefix build (ge_kbuild.cu), per particle: kdl = 1 + the level at
    // which its key first differs from the previous particle's (0 at a
    // simulation's first particle), klam = its leaf level by the key runs
    // (levels + 1 when the keys cannot resolve it), kxr = the level of the
    // exact-rebuild root that holds it (kEmpty: none); ksus = suspect
    // {level, particle} pairs, kroots = exact-rebuild roots, ktile = per-tile
    // node counts of every level, kmeta = counters and level totals
    uint8_t *kdl, *klam;
    uint32_t *kxr;
    uint2 *ksus;
    uint32_t ksus_cap;
    uint32_t *kroots;
    // exact-rebuild roots too large for one warp to mark: {level, start, end}
    // (kbig, kKeyBigCap entries), each once (kbig_keys: a set of {start, level})
    uint4 *kbig;
    unsigned long long *kbig_keys;
    uint32_t *ktile;
    uint32_t ktile_cap;
    uint32_t *kmeta;
    uint32_t *kdone;      // leaves of exact rebuilds whose upward pass is deferred [n + 1]
    int64_t cap;
};

template <int D> struct MomWords;
template <> struct MomWords<2> { static constexpr int value = 6; };
template <> struct MomWords<3> { static constexpr int value = 10; };

// Independent simulations ("segments") stepped together: the particles of
// segment s occupy [off[s], off[s+1]) of the state arrays and never leave it;
// boxes, keys, the sort, the trees and the walks never mix segments.  With a
// single segment the arrays may be null (segment 0 = all particles).
struct Segs {
    int S;
    const uint32_t *off;        // [S + 1]
    const uint32_t *seg_of;     // [n] segment of each particle slot
    const uint32_t *tile_base;  // [S + 1] first sort tile of each segment
    const uint32_t *tile_seg;   // [tiles] segment of each sort tile
    int64_t tiles;              // sort tiles over all segments
    float4 *box;                // [S] root boxes {x, y, z, size}
    uint32_t *boxmm;            // [S * 6] order-preserving min/max words
    uint32_t *root_begin;       // [S] walk entry of each root
    uint32_t *root_end;         // [S] end of each root's walk
    const uint8_t *direct;      // [S] 1: the segment takes the direct sum and the
                                // walk skips it (nullptr: every segment walks)
};

__host__ __device__ __forceinline__ uint32_t seg_lo(const Segs &g, uint32_t s) {
    return g.off ? g.off[s] : 0u;
}
__host__ __device__ __forceinline__ uint32_t seg_hi(const Segs &g, uint32_t s, uint32_t n) {
    return g.off ? g.off[s + 1] : n;
}

// Scratch for keys and sort.
struct SortScratch {
    uint64_t *keys[2];     // 2D: (key << 28 | index) packed; 3D: keys
    uint32_t *vals[2];     // 3D: indices
    uint32_t *hist;        // [passes][S][radix] per-segment digit counts
    uint32_t *status;      // [passes][tiles][radix] decoupled look-back words
    uint32_t *tile_ctr;    // [8]
    int box_blocks;        // grid of the kick/box kernel
    // look-back polls of a radix pass before it gives up (0: kSpinLimit)
    uint32_t spin_limit;
    // test hook (ge_set_sort_wait_test): 1 = the first tile of every pass
    // keeps its digit counts to itself, so the look-back waits of the tiles
    // after it run out and the sort reports GE_ERR_TIMEOUT
    uint32_t withhold_first;
};

struct StepParams {
    int n;
    float dt, half_dt;
    float G, theta, theta2, eps2;
    uint32_t leaf_cap;
    float size_gate, min_size;
    int periodic;
    float domain[3], half_domain[3];
    int group_size;   // GE_PREC_MIXED: 0 = per-particle walk, else the group walk
    float heat_cond;  // heat exchange coefficient (used when State::temp is set)
    float direct_eps2;   // value the direct sum adds to r^2
    int i0;              // the per-particle walk: first particle (up to n), 0 by default
    int mixed;           // GE_PREC_MIXED: the moment pass rewrites the node entries
    int walk_kind;       // GE_PREC_FAST: 0 per-particle walk, 1 warp-cooperative walk
    int layout_extras;   // tree build: kLayoutEntry | kLayoutRange (the optional layout arrays)
};

// 2D walk entries {x, y, m, w}.  Plain layout: w = size^2 (-1 for a particle,
// -2 for a massless node), the subtree successor in link[].  Packed layout
// (tree meta word kMetaWalkPacked = 1): a node's w holds its level L (6 bits)
// and its successor (26 bits); its size is the simulation's root size rs
// halved L times (exact), so the plain layout's size^2 = fl(size_L^2) =
// fl(rs^2) * 4^-L: fl(rs^2) with 2L taken off its exponent, exact while both
// are normal floats (every rs below 1e19 and min_size >= 1e-18, checked by
// the build).  Massless nodes and particles carry the marker levels below
// (L <= 46 for real levels); link[] holds every successor in both layouts.
constexpr int kMetaWalkPacked = 13;
// optional walk-layout arrays a build writes: each node's entry in aux.w (the
// moment and node-temperature passes read it) and its entry range in nrange
// (the warp-cooperative walk reads it)
constexpr int kLayoutEntry = 1, kLayoutRange = 2;
constexpr int kMetaBigRoot = 14;   // tree meta word: some simulation's root size >= 1e19
constexpr int kMetaWords = 32;     // tree meta words allocated
// warp-cooperative walk counters (Tree::wctr, zeroed before each launch): the
// chunk counter and the count of chunks that fell back to the per-particle walk
constexpr int kWWCtrWords = 2;
__device__ __forceinline__ float packed_size2(uint32_t w_bits, uint32_t rs2_bits) {
    return __uint_as_float(rs2_bits - ((w_bits >> 2) & 0x3F000000u));   // exponent - 2L
}
constexpr uint32_t kPackSkipBits = 26, kPackMaxLevel = 46;
__host__ __device__ constexpr uint32_t pack_entry_word(uint32_t level, uint32_t skip) {
    return (level << kPackSkipBits) | skip;
}
// Level values above kPackMaxLevel mark the packed entries that every opening
// test accepts: a massless node (62; its successor follows) and a particle
// (63; its successor is the next entry).  One unsigned compare of the word
// tells them from the nodes, and every entry's successor is in its word.
constexpr uint32_t kPackMassless = 62, kPackParticle = 63;
__host__ __device__ __forceinline__ bool packed_accepts(uint32_t w_bits) {
    return w_bits >= (kPackMassless << kPackSkipBits);
}
__host__ __device__ __forceinline__ bool packed_particle(uint32_t w_bits) {
    return w_bits >= (kPackParticle << kPackSkipBits);
}

constexpr int kBBoxThreads = 256;
constexpr int kBoxItems = 8;       // particles per thread per block tile of the kick/box pass
constexpr int kSortTile = 4096;   // keys per look-back tile (512 threads x 8)
constexpr int kSortDigitWords = 7 * 512;   // hist / status words per segment / tile (3D keys)
constexpr int kTimeline = 256;    // build timeline entries
constexpr int kDirectTile = 128;  // particles per block of the direct sum

// the reference's particle records (ge_aos.cu): members of n records into
// the state (k_aos_in), and the updated members back into each particle's
// record before the frame's sort (k_aos_out, after sort and permute)
using AosLayout = ge_aos_layout;
cudaError_t launch_aos_in(int dims, const unsigned char *phys, const unsigned char *rend,
                          const AosLayout &L, int n, const State &s, cudaStream_t st);
cudaError_t launch_aos_out(int dims, unsigned char *phys, const AosLayout &L, int n,
                           const State &s, const SortScratch &ss, cudaStream_t st);

// --- launchers (each runs on `st`) ----------------------------------------
// integrateStart (kick + drift) fused with the per-segment bounding-box
// reduction; a second small kernel applies the reference's box formula per
// segment and seeds each segment's root node.
cudaError_t launch_kick_drift_bbox(int dims, const State &s, const StepParams &p, bool kick_drift,
                                   const Segs &g, SortScratch &ss, Tree &t, cudaStream_t st);
// sets every segment's min/max words to their identities (needed once after
// the words are allocated; the box kernel leaves them reset)
cudaError_t launch_reset_boxes(const Segs &g, cudaStream_t st);
// segment of every particle slot and of every sort tile, from the segment
// offsets off [S + 1] and first tiles tile_base [S + 1]
cudaError_t launch_seg_tables(const uint32_t *off, const uint32_t *tile_base, int S, int n,
                              int64_t tiles, uint32_t *seg_of, uint32_t *tile_seg,
                              cudaStream_t st);
// Morton keys from each segment's root box plus the per-segment digit
// histograms of every pass
// count 32-bit words set to zero by a kernel (launched like the step's others)
cudaError_t launch_zero(uint32_t *w, int64_t count, cudaStream_t st);
cudaError_t launch_keys(int dims, const State &s, int n, const Segs &g, SortScratch &ss,
                        cudaStream_t st);
// all radix passes (stable within each segment); leaves the sorted keys in
// ss.keys[0] (and vals[0])
cudaError_t launch_sort(int dims, int n, const Segs &g, SortScratch &ss, uint32_t *err,
                        cudaStream_t st);
// stable radix passes of 8-bit digits over bits [shift0, shift0 + 8 * passes)
// of the 64-bit words in words[0] (one range, no segments); digit histograms
// in hist [passes][256]; *result = the buffer that holds the sorted words
cudaError_t launch_radix_words(uint64_t *const words[2], int n, int shift0, int passes,
                               const uint32_t *hist, uint32_t *status, uint32_t *tile_ctr,
                               uint32_t *err, int *result, cudaStream_t st);
// SPH neighbour grid of particles [lo, lo + n) (ge_sph.cu); outputs are device
// arrays keys/index/cell_x/cell_y [n], offsets [table]
int sph_grid_passes(uint32_t table);
cudaError_t launch_sph_grid(const State &s, uint32_t lo, int n, float cell, uint32_t table,
                            SortScratch &ss, uint32_t *err, uint32_t *keys, uint32_t *index,
                            int32_t *cell_x, int32_t *cell_y, uint32_t *offsets, int num_sms,
                            cudaStream_t st);
// gather of the state into `out` by the sorted order
cudaError_t launch_permute(int dims, int n, const SortScratch &ss, const State &in,
                           const State &out, bool with_acc, cudaStream_t st);
// order (sorted slot -> previous index) copy-out for the stage API
cudaError_t launch_perm_out(int dims, int n, const SortScratch &ss, uint32_t *perm,
                            cudaStream_t st);
cudaError_t launch_keys_out(int dims, int n, const SortScratch &ss, uint64_t *keys,
                            cudaStream_t st);
// tree build + mass/centre of mass + walk layout (one cooperative launch);
// keyed: the key-prefix passes (launch_key_build) ran first, and this launch
// completes their tree (leaf sums, upward masses, exact rebuilds, layout)
int build_grid_blocks(int dims, int num_sms);
int64_t build_node_slack(int dims, int num_sms);
cudaError_t launch_build(int dims, const State &s, const StepParams &p, const Segs &g, Tree &t,
                         uint32_t *err, int num_sms, cudaStream_t st, bool keyed = false);
// key-prefix tree passes (ge_kbuild.cu) over the Morton-sorted particles and
// their sorted keys (2D: key << 28 | index words; 3D: keys)
constexpr int kKeyMaxCap = 32;   // leaf capacities the key-prefix build handles
constexpr int kKeyTile = 256;    // particles per tile of its node-count scan (one per thread)
constexpr int kKeyBigCap = 256;   // large exact-rebuild roots recorded per build
constexpr int kKeyBigHash = 1024; // slots of their set
constexpr int kKeyMetaWords = 96;
int64_t key_suspect_cap(int64_t n);
cudaError_t launch_key_build(int dims, const State &s, const StepParams &p, const Segs &g,
                             const uint64_t *keys, Tree &t, uint32_t *err, int num_sms,
                             cudaStream_t st);
// GE_PREC_MIXED group walk (ge_gwalk.cu): warps walk for groups of
// p.group_size consecutive particles of one simulation; counter = one word
int group_walk_warps(int dims, int num_sms);
// the group walk's potential pass: *epot = sum_i m_i u_i, phi_i = -G u_i
// (monopole + quadrupole of the softened kernel), groups of 32; no state
// is written
cudaError_t launch_group_potential(int dims, const State &s, const StepParams &p, const Segs &g,
                                   const Tree &t, uint32_t *counter, uint32_t *err, double *epot,
                                   cudaStream_t st);
uint32_t group_walk_stack_entries();
cudaError_t launch_group_walk(int dims, const State &s, const StepParams &p, const Segs &g,
                              const Tree &t, bool integrate_end, unsigned long long *inter_count,
                              uint32_t *counter, uint32_t *err, cudaStream_t st);
// O(N^2) direct sum of the segments listed by tiles[ntiles] ({segment,
// first particle}, kDirectTile particles each, inside one segment), fused
// with integrateEnd like the walk
cudaError_t launch_direct(int dims, int precision, const State &s, const StepParams &p,
                          const Segs &g, const uint2 *tiles, int64_t ntiles, bool integrate_end,
                          cudaStream_t st);
// tree walk; integrate_end fuses integrateEnd (v += a*dt/2).  With
// p.walk_kind == 1, GE_PREC_FAST with eps2 > 0 and without periodic wrap or
// heat exchange runs the warp-cooperative walk (ge_wwalk.cu); everything else
// the per-particle walk (ge_walk.cu)
cudaError_t launch_walk(int dims, int precision, const State &s, const StepParams &p,
                        const Segs &g, const Tree &t, bool integrate_end,
                        unsigned long long *inter_count, uint32_t *err, int num_sms,
                        cudaStream_t st);
// the warp-cooperative FAST walk of particles [p.i0, p.n) (ge_wwalk.cu)
cudaError_t launch_warp_walk(int dims, const State &s, const StepParams &p, const Segs &g,
                             const Tree &t, bool integrate_end, unsigned long long *inter_count,
                             uint32_t *err, int num_sms, cudaStream_t st);
cudaError_t launch_integrate_end(int dims, const State &s, const StepParams &p, cudaStream_t st);
// gravity field display: strength (and RGBA8 colour) of every cell
cudaError_t launch_field(const State &s, uint32_t lo, uint32_t hi, int amount_x, int amount_y,
                         float cell, float G, float soft2, int periodic, float dom_x, float dom_y,
                         const ge_field_params &fp, float *strength, uint32_t *rgba,
                         cudaStream_t st);
// trajectory preview: probes stepped against the walk layout of the last
// build, entries [begin, end) (one simulation's tree)
cudaError_t launch_predict(int dims, const Tree &t, const StepParams &p, const float4 *box,
                           uint32_t begin,
                           uint32_t end, float eps2, int nprobes, const float *pos,
                           const float *vel, const float *mass, int steps, float *path,
                           cudaStream_t st);
// heat exchange: node temperature sums bottom-up in the reference's order and
// the walk's temperature entries (after launch_build)
cudaError_t launch_node_temps(int dims, const State &s, const StepParams &p, Tree &t,
                              int num_sms, cudaStream_t st);
// GE_PREC_MIXED: FP64 mass, centre of mass and second moments of every node,
// bottom-up from the particles, written into the walk entries with the
// offset-corrected opening radius (after launch_build)
cudaError_t launch_moments(int dims, const State &s, const StepParams &p, Tree &t, uint32_t *err,
                           int num_sms, cudaStream_t st);
// FP64 diagnostics
// (each target sums over its own segment only; idx sorted ascending keeps a
// block's targets inside one or two segments)
cudaError_t launch_direct_f64(int dims, const State &s, int n, const Segs &g, const uint32_t *idx,
                              int nt, double G, double eps2, double *out, cudaStream_t st);
cudaError_t launch_sums_f64(int dims, const State &s, int n, double *out, cudaStream_t st);

}  // namespace ge
