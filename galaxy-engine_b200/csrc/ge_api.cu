// ge_api.cu -- host side of the C ABI (include/ge_bh.h): context, resident
// device state, the per-frame pipeline, the stage calls and the batch of
// independent simulations.
//
// One frame (GalaxyEngine/src/globalLogic.cpp:1155-1370 in 2D, :1584-1719 in 3D):
//   1. kick + drift fused with the bounding boxes         (integrateStart, boundingBox)
//   2. Morton keys + digit histograms                      (computeMortonKeys)
//   3. stable radix sort passes                            (sortParticlesByMortonKey)
//   4. gather of the state into Morton order
//   5. tree build with mass / centre of mass               (Quadtree / Octree)
//   6. tree walk with the second half kick fused           (calculateForceFromGrid, integrateEnd)
// All of it is enqueued on the context's stream; nothing returns to the host
// between stages.  A context holds S >= 1 independent simulations back to
// back in its arrays (segments, ge_internal.h); every stage runs once over
// all of them, so a batch of many small simulations costs one launch per
// stage instead of one per simulation.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

using namespace ge;

namespace gehost {

// Device allocations of one buffer set.  A dry list only adds up the bytes
// (ge_estimate_bytes): its pointers are placeholders that are never used.
struct AllocList {
    std::vector<void *> ptrs;
    size_t bytes = 0;
    bool dry = false;
};

// Device buffers sized for a particle capacity; replaced as a whole when the
// capacity grows (the particle state is copied across).
struct Buffers {
    int64_t cap_n = 0;
    State st[2]{};
    SortScratch ss{};
    Tree tree{};
    unsigned long long *d_inter = nullptr;
    bool prev = false;     // prevVel arrays allocated
    bool pinned = false;   // pin flag arrays allocated
    bool temp = false;     // temperatures and node temperature arrays allocated
    bool mixed = false;    // GE_PREC_MIXED Kahan terms and node moments allocated
    bool mixed_entry = false;   // ... the per-particle walk's entry arrays
    bool mixed_group = false;   // ... the group walk's slot arrays and work stacks
    AllocList allocs;
};

// Segment tables, sized for a segment, tile and particle capacity.
struct SegBuffers {
    int64_t seg_cap = 0, tile_cap = 0, n_cap = 0;
    uint32_t *off = nullptr, *tile_base = nullptr, *seg_of = nullptr, *tile_seg = nullptr;
    float4 *box = nullptr;
    uint32_t *boxmm = nullptr, *root_begin = nullptr, *root_end = nullptr;
    uint32_t *hist = nullptr, *status = nullptr;
    uint2 *dtiles = nullptr;    // direct sum: {segment, first particle} of each tile
    uint8_t *dflag = nullptr;   // direct sum: 1 for a segment that skips the walk
    int64_t dtile_cap = 0;
    AllocList allocs;
};

struct SimRec {
    int32_t handle;
    int64_t n;
    int64_t step0;   // context steps when the simulation was added
};

inline void free_all(AllocList &L) {
    if (!L.dry)
        for (void *q : L.ptrs) cudaFree(q);
    L.ptrs.clear();
    L.bytes = 0;
}

template <typename T>
cudaError_t dalloc(AllocList &L, T **p, size_t count) {
    const size_t bytes = sizeof(T) * (count ? count : 1);
    if (L.dry) {
        L.bytes += (bytes + 255) & ~size_t(255);
        *p = reinterpret_cast<T *>(uintptr_t(256));
        return cudaSuccess;
    }
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return e;
    L.ptrs.push_back(q);
    L.bytes += bytes;
    *p = (T *)q;
    return cudaSuccess;
}


}  // namespace gehost

using namespace gehost;

struct ge_ctx {
    ge_params p{};
    int dev = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    int64_t n = 0;                // particles over all simulations
    int cur = 0;                  // which of b.st[2] holds the state
    bool has_pinned = false;      // pin flags uploaded and in effect
    Buffers b;
    SegBuffers sb;
    Segs g{};
    std::vector<SimRec> sims;     // in slot order
    int64_t sims_reserved = 0;    // segment capacity asked for by ge_reserve
    int32_t next_handle = 1;
    int64_t total_steps = 0;
    int32_t pending_steps = 0;    // steps enqueued by ge_step_async, not yet waited for
    std::vector<uint32_t> h_off, h_tile_base;
    // direct sum (params.direct_below): its tiles, and whether some segment
    // takes the direct sum / the walk
    std::vector<uint2> h_dtiles;
    std::vector<uint8_t> h_dflag;
    bool any_direct = false, any_walk = true;
    uint32_t *d_err = nullptr;
    uint32_t *h_meta = nullptr;   // pinned copy of the tree meta words
    int64_t slots = 0;            // node slots of the last build (holes included)
    bool count_inter = false;
    bool tree_ranges = false;   // the last build wrote the layout ranges (warp walk)
    bool tree_valid = false;
    bool keys_valid = false;
    cudaEvent_t ev[8]{};
    // ge_frame_host: a second stream for the copies that overlap the step
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t xev[3]{};
    // ge_step: two consecutive steps captured as one CUDA graph (every
    // buffer role is back where it started after two), replayed while the
    // launches they hold would not change; two kept, by the bytes that
    // decide those launches (frame_signature)
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        std::vector<uint8_t> sig;
    } graphs[2];
    int next_graph = 0;
    bool graph_failed = false;    // capture or instantiation refused: plain launches
    bool framed = false;          // a frame was enqueued (one-time launch setup done)
    // ge_set_sort_wait_test: the sort's look-back poll cap and withheld tile,
    // kept here so that a reallocation of the buffers keeps them
    uint32_t sort_spin_limit = 0, sort_withhold = 0;
    // ge_frame_aos: device copies of the caller's records and the order output
    unsigned char *d_aos = nullptr, *d_aos_r = nullptr;
    size_t aos_bytes = 0, aos_r_bytes = 0;
    uint32_t *d_order = nullptr;
    int64_t order_cap = 0;
    ge_stats stats{};
    std::string err;
};

namespace {

int fail(ge_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(ge_ctx *c, cudaError_t e, const char *where) {
    if (e == cudaErrorMemoryAllocation)
        return fail(c, GE_ERR_OOM, std::string(where) + ": " + cudaGetErrorString(e));
    return fail(c, GE_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define GE_CHECK(ctx, call)                                      \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
    } while (0)

void drop_graphs(ge_ctx *c) {
    for (auto &g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
        g.sig.clear();
    }
}

void free_buffers(ge_ctx *c) {
    drop_graphs(c);
    free_all(c->b.allocs);
    free_all(c->sb.allocs);
    c->b = Buffers{};
    c->sb = SegBuffers{};
    c->g = Segs{};
    c->d_err = nullptr;
    c->has_pinned = false;
    c->n = 0;
    c->cur = 0;
    c->sims.clear();
    c->tree_valid = false;
    c->keys_valid = false;
}

StepParams step_params(const ge_ctx *c) {
    StepParams s{};
    s.n = (int)c->n;
    s.dt = c->p.dt;
    s.half_dt = c->p.dt * 0.5f;
    s.G = c->p.G;
    s.theta = c->p.theta;
    s.theta2 = c->p.theta * c->p.theta;
    s.eps2 = c->p.eps2;
    s.leaf_cap = c->p.leaf_cap;
    s.size_gate = c->p.size_gate;
    s.min_size = c->p.min_size;
    s.periodic = c->p.periodic ? 1 : 0;
    s.group_size = c->p.group_size;
    s.heat_cond = c->p.heat_cond;
    s.direct_eps2 = c->p.direct_eps2;
    s.mixed = c->p.precision == GE_PREC_MIXED ? 1 : 0;
    s.walk_kind = c->p.walk_kind;
    for (int a = 0; a < 3; a++) {
        s.domain[a] = c->p.domain[a];
        s.half_domain[a] = c->p.domain[a] * 0.5f;
    }
    return s;
}

int validate(ge_ctx *c, const ge_params *p) {
    if (!p) return fail(c, GE_ERR_ARG, "params is NULL");
    if (p->dims != 2 && p->dims != 3) return fail(c, GE_ERR_ARG, "dims must be 2 or 3");
    if (p->precision != GE_PREC_FAST && p->precision != GE_PREC_EXACT &&
        p->precision != GE_PREC_MIXED)
        return fail(c, GE_ERR_ARG, "unknown precision mode");
    if (!(p->theta >= 0.0f)) return fail(c, GE_ERR_ARG, "theta must be >= 0");
    if (!(p->eps2 >= 0.0f)) return fail(c, GE_ERR_ARG, "eps2 must be >= 0");
    if (p->leaf_cap < 1) return fail(c, GE_ERR_ARG, "leaf_cap must be >= 1");
    if (!(p->node_cap_factor >= 1.0f)) return fail(c, GE_ERR_ARG, "node_cap_factor must be >= 1");
    if (p->temp_enabled && p->precision == GE_PREC_MIXED)
        return fail(c, GE_ERR_UNSUPPORTED, "heat exchange runs in GE_PREC_EXACT and GE_PREC_FAST");
    if (p->direct_below < 0) return fail(c, GE_ERR_ARG, "direct_below must be >= 0");
    if (p->direct_below > 0 && p->precision == GE_PREC_MIXED)
        return fail(c, GE_ERR_UNSUPPORTED, "the direct sum runs in GE_PREC_EXACT and GE_PREC_FAST");
    if (p->direct_below > 0 && !(p->direct_eps2 > 0.0f && p->direct_eps2 < INFINITY))
        return fail(c, GE_ERR_ARG, "direct_eps2 must be positive and finite (the self term divides by it)");
    if (p->walk_kind != 0 && p->walk_kind != 1) return fail(c, GE_ERR_ARG, "walk_kind must be 0 or 1");
    if (p->group_size != 0 && p->group_size != 32 && p->group_size != 64 && p->group_size != 128)
        return fail(c, GE_ERR_ARG, "group_size must be 0, 32, 64 or 128");
    if (p->periodic && (!(p->domain[0] > 0) || !(p->domain[1] > 0) ||
                        (p->dims == 3 && !(p->domain[2] > 0))))
        return fail(c, GE_ERR_ARG, "periodic wrap needs a positive domain");
    return GE_OK;
}

// Allocates every per-particle and tree buffer of `nb` for cap particles.
int alloc_buffers(ge_ctx *c, Buffers &nb, int64_t cap, int64_t node_cap, bool prev, bool pinned,
                  bool temp = false) {
    const int D = c->p.dims;
    const size_t N = (size_t)cap;
    auto &L = nb.allocs;
    nb.cap_n = cap;
    nb.prev = prev;
    nb.pinned = pinned;
    for (int k = 0; k < 2; k++) {
        State &s = nb.st[k];
        GE_CHECK(c, dalloc(L, &s.x, N)); GE_CHECK(c, dalloc(L, &s.y, N));
        GE_CHECK(c, dalloc(L, &s.vx, N)); GE_CHECK(c, dalloc(L, &s.vy, N));
        GE_CHECK(c, dalloc(L, &s.ax, N)); GE_CHECK(c, dalloc(L, &s.ay, N));
        if (D == 3) {
            GE_CHECK(c, dalloc(L, &s.z, N)); GE_CHECK(c, dalloc(L, &s.vz, N));
            GE_CHECK(c, dalloc(L, &s.az, N));
        }
        GE_CHECK(c, dalloc(L, &s.m, N));
        GE_CHECK(c, dalloc(L, &s.id, N));
        if (prev) {
            GE_CHECK(c, dalloc(L, &s.pvx, N)); GE_CHECK(c, dalloc(L, &s.pvy, N));
            if (D == 3) GE_CHECK(c, dalloc(L, &s.pvz, N));
        }
        if (pinned) GE_CHECK(c, dalloc(L, &s.pinned, N));
        if (temp) {
            GE_CHECK(c, dalloc(L, &s.temp, N));
            if (!L.dry) GE_CHECK(c, cudaMemsetAsync(s.temp, 0, sizeof(float) * N, c->stream));
        }
    }
    SortScratch &ss = nb.ss;
    GE_CHECK(c, dalloc(L, &ss.keys[0], N)); GE_CHECK(c, dalloc(L, &ss.keys[1], N));
    if (D == 3) { GE_CHECK(c, dalloc(L, &ss.vals[0], N)); GE_CHECK(c, dalloc(L, &ss.vals[1], N)); }
    GE_CHECK(c, dalloc(L, &ss.tile_ctr, 8));
    Tree &t = nb.tree;
    t.cap = node_cap;
    GE_CHECK(c, dalloc(L, &t.walk, (size_t)node_cap));
    if (D == 3) GE_CHECK(c, dalloc(L, &t.size2, (size_t)node_cap));
    GE_CHECK(c, dalloc(L, &t.info, (size_t)node_cap));
    GE_CHECK(c, dalloc(L, &t.cell, (size_t)node_cap));
    GE_CHECK(c, dalloc(L, &t.aux, (size_t)node_cap));
    GE_CHECK(c, dalloc(L, &t.pend, (size_t)node_cap));
    GE_CHECK(c, dalloc(L, &t.small, N / 2 + 1));
    t.small_cap = (uint32_t)(N / 2 + 1);
    // entries carry the id of the build that queued them (ids start at 1)
    if (!L.dry) GE_CHECK(c, cudaMemsetAsync(t.small, 0, sizeof(uint2) * (N / 2 + 1), c->stream));
    GE_CHECK(c, dalloc(L, &t.endcnt, N + 1));
    const int bblocks = build_grid_blocks(D, c->num_sms);
    if (bblocks < 1) return fail(c, GE_ERR_CUDA, "tree build kernel cannot be made resident");
    GE_CHECK(c, dalloc(L, &t.blocksum, (size_t)bblocks));
    GE_CHECK(c, dalloc(L, &t.src, N + (size_t)node_cap + 1));
    if (D == 2) {
        uint32_t *l = nullptr;
        GE_CHECK(c, dalloc(L, &l, N + (size_t)node_cap + 1));
        t.link = l;
    } else {
        uint2 *l = nullptr;
        GE_CHECK(c, dalloc(L, &l, N + (size_t)node_cap + 1));
        t.link = l;
    }
    GE_CHECK(c, dalloc(L, &t.slot_of, N));
    GE_CHECK(c, dalloc(L, &t.nrange, (size_t)node_cap));
    GE_CHECK(c, dalloc(L, &t.wctr, kWWCtrWords));
    GE_CHECK(c, dalloc(L, &t.level, kMaxLevels + 2));
    GE_CHECK(c, dalloc(L, &t.lvl_alloc, kMaxLevels + 2));
    GE_CHECK(c, dalloc(L, &t.meta, kMetaWords));
    GE_CHECK(c, dalloc(L, &t.tl, kTimeline));
    // key-prefix build
    GE_CHECK(c, dalloc(L, &t.kdl, N));
    GE_CHECK(c, dalloc(L, &t.klam, N));
    GE_CHECK(c, dalloc(L, &t.kxr, N));
    t.ksus_cap = (uint32_t)key_suspect_cap((int64_t)N);
    GE_CHECK(c, dalloc(L, &t.ksus, (size_t)t.ksus_cap));
    GE_CHECK(c, dalloc(L, &t.kroots, N + 1));
    GE_CHECK(c, dalloc(L, &t.kbig, kKeyBigCap));
    GE_CHECK(c, dalloc(L, &t.kbig_keys, kKeyBigHash));
    t.ktile_cap = (uint32_t)(N / kKeyTile + 1);
    GE_CHECK(c, dalloc(L, &t.ktile, (size_t)t.ktile_cap * 22));
    GE_CHECK(c, dalloc(L, &t.kmeta, kKeyMetaWords));
    GE_CHECK(c, dalloc(L, &t.kdone, N + 1));
    if (temp) {
        GE_CHECK(c, dalloc(L, &t.ntemp, (size_t)node_cap));
        GE_CHECK(c, dalloc(L, &t.tv, N + (size_t)node_cap + 1));
    }
    nb.temp = temp;
    if (!L.dry) GE_CHECK(c, cudaMemsetAsync(t.meta, 0, kMetaWords * sizeof(uint32_t), c->stream));
    GE_CHECK(c, dalloc(L, &nb.d_inter, 1));
    return GE_OK;
}

// Whether the mixed mode walks in groups (a group size is set and the
// domain is not periodic) or particle by particle.
bool wants_group(const ge_params &p) { return p.group_size != 0 && !p.periodic; }

// GE_PREC_MIXED arrays: Kahan terms of both state buffers (zeroed), the node
// moments, and the node data of the walk the group size selects.
int alloc_mixed(ge_ctx *c, Buffers &nb) {
    const int D = c->p.dims;
    const size_t N = (size_t)nb.cap_n, E = N + (size_t)nb.tree.cap + 1;
    const size_t NC = (size_t)nb.tree.cap;
    auto &L = nb.allocs;
    Tree &t = nb.tree;
    if (!nb.mixed) {
        for (int k = 0; k < 2; k++) {
            State &s = nb.st[k];
            float **kp[6] = {&s.kx, &s.ky, &s.kz, &s.kvx, &s.kvy, &s.kvz};
            for (int a = 0; a < 6; a++) {
                if (D == 2 && (a == 2 || a == 5)) continue;
                GE_CHECK(c, dalloc(L, kp[a], N));
                if (!L.dry) GE_CHECK(c, cudaMemsetAsync(*kp[a], 0, sizeof(float) * N, c->stream));
            }
        }
        GE_CHECK(c, dalloc(L, &t.mom, NC * (D == 2 ? MomWords<2>::value : MomWords<3>::value)));
        nb.mixed = true;
    }
    if (!wants_group(c->p) && !nb.mixed_entry) {
        GE_CHECK(c, dalloc(L, &t.mq0, E));
        if (D == 3) GE_CHECK(c, dalloc(L, &t.mq1, E));
        GE_CHECK(c, dalloc(L, &t.mq2, E));
        nb.mixed_entry = true;
    }
    if (wants_group(c->p) && !nb.mixed_group) {
        GE_CHECK(c, dalloc(L, &t.gw, NC));
        GE_CHECK(c, dalloc(L, &t.gq0, NC));
        if (D == 3) GE_CHECK(c, dalloc(L, &t.gq1, NC));
        GE_CHECK(c, dalloc(L, &t.gq2, NC));
        // a work stack per resident warp, but no more warps than one per 16
        // particles of capacity (a group holds up to 128 particles)
        int warps = group_walk_warps(D, c->num_sms);
        if (warps < 1) return fail(c, GE_ERR_CUDA, "group walk kernel cannot be made resident");
        const int64_t need = ((nb.cap_n + 15) / 16 + 3) / 4 * 4;
        if (need < warps) warps = (int)need;
        GE_CHECK(c, dalloc(L, &t.wl, (size_t)warps * group_walk_stack_entries()));
        GE_CHECK(c, dalloc(L, &t.grp, N + 1));
        t.wl_warps = (uint32_t)warps;
        nb.mixed_group = true;
    }
    return GE_OK;
}

// The tree as a mixed-mode pass sees it: only the node arrays of the walk
// that runs.
Tree mixed_view(const ge_ctx *c) {
    Tree t = c->b.tree;
    if (!wants_group(c->p)) t.gw = t.gq0 = t.gq1 = nullptr, t.gq2 = nullptr;
    else t.mq0 = t.mq1 = nullptr, t.mq2 = nullptr;
    return t;
}

bool group_walk_on(const ge_ctx *c) {
    return c->p.precision == GE_PREC_MIXED && wants_group(c->p);
}

// Copies particles [soff, soff + cnt) of src to [doff, doff + cnt) of dst
// (device to device, on the context's stream).
int copy_range(ge_ctx *c, const State &dst, int64_t doff, const State &src, int64_t soff,
               int64_t cnt, bool prev, bool pinned) {
    if (cnt <= 0) return GE_OK;
    const bool d3 = c->p.dims == 3;
    const bool kah = dst.kx && src.kx;
    const size_t B = sizeof(float) * (size_t)cnt;
    float *const fd[] = {dst.x, dst.y, d3 ? dst.z : nullptr, dst.vx, dst.vy, d3 ? dst.vz : nullptr,
                         dst.ax, dst.ay, d3 ? dst.az : nullptr, dst.m,
                         prev ? dst.pvx : nullptr, prev ? dst.pvy : nullptr,
                         prev && d3 ? dst.pvz : nullptr,
                         kah ? dst.kx : nullptr, kah ? dst.ky : nullptr,
                         kah && d3 ? dst.kz : nullptr, kah ? dst.kvx : nullptr,
                         kah ? dst.kvy : nullptr, kah && d3 ? dst.kvz : nullptr};
    const float *const fs[] = {src.x, src.y, src.z, src.vx, src.vy, src.vz, src.ax, src.ay,
                               src.az, src.m, src.pvx, src.pvy, src.pvz,
                               src.kx, src.ky, src.kz, src.kvx, src.kvy, src.kvz};
    for (size_t k = 0; k < sizeof(fd) / sizeof(fd[0]); k++)
        if (fd[k])
            GE_CHECK(c, cudaMemcpyAsync(fd[k] + doff, fs[k] + soff, B, cudaMemcpyDeviceToDevice,
                                        c->stream));
    GE_CHECK(c, cudaMemcpyAsync(dst.id + doff, src.id + soff, sizeof(uint32_t) * (size_t)cnt,
                                cudaMemcpyDeviceToDevice, c->stream));
    if (pinned)
        GE_CHECK(c, cudaMemcpyAsync(dst.pinned + doff, src.pinned + soff, (size_t)cnt,
                                    cudaMemcpyDeviceToDevice, c->stream));
    if (dst.temp && src.temp)
        GE_CHECK(c, cudaMemcpyAsync(dst.temp + doff, src.temp + soff, B, cudaMemcpyDeviceToDevice,
                                    c->stream));
    return GE_OK;
}

int64_t node_cap_for(const ge_ctx *c, int64_t n, int64_t S, int64_t slack) {
    return (int64_t)(c->p.node_cap_factor * (double)n) + 1024 + slack + S;
}

// Makes the buffers hold n particles in S simulations.  With `keep` the
// current c->n particles survive a reallocation (they move to st[0]).
int ensure_capacity(ge_ctx *c, int64_t n, int64_t S, bool keep, bool exact = false) {
    const int D = c->p.dims;
    const int64_t slack = build_node_slack(D, c->num_sms);
    if (slack <= 0) return fail(c, GE_ERR_CUDA, "tree build kernel cannot be made resident");
    if (D == 2 && n >= (1ll << 28)) return fail(c, GE_ERR_ARG, "2D supports N < 2^28 per context");
    if (n >= (1ll << 31)) return fail(c, GE_ERR_ARG, "N must be < 2^31 per context");
    const bool want_prev = c->p.track_prev_vel != 0;
    Buffers &ob = c->b;
    if (n <= ob.cap_n && node_cap_for(c, n, S, slack) <= ob.tree.cap && ob.prev == want_prev)
        return GE_OK;
    // a live context grows by half again at least, so adding simulations one
    // by one reallocates O(log) times
    int64_t cap = n, scap = S;
    if (keep && ob.cap_n > 0 && !exact) {
        cap = std::max(n, ob.cap_n + ob.cap_n / 2);
        scap = S + S / 2;
        const int64_t lim = D == 2 ? (1ll << 28) - 1 : (1ll << 31) - 1;
        if (cap > lim) cap = lim;
    }
    const int64_t node_cap = node_cap_for(c, cap, scap, slack);
    if (node_cap >= (1ll << 32) - 1) return fail(c, GE_ERR_ARG, "node capacity exceeds 2^32");
    Buffers nb;
    int rc = alloc_buffers(c, nb, cap, node_cap, want_prev, ob.pinned, ob.temp);
    if (!rc && (ob.mixed || c->p.precision == GE_PREC_MIXED)) rc = alloc_mixed(c, nb);
    if (!rc && ((ob.mixed_entry && !nb.mixed_entry) || (ob.mixed_group && !nb.mixed_group))) {
        // keep every array set the old buffers had
        const ge_params keep = c->p;
        c->p.periodic = 0;
        c->p.group_size = ob.mixed_entry && !nb.mixed_entry ? 0 : 32;
        rc = alloc_mixed(c, nb);
        if (!rc && ob.mixed_group && !nb.mixed_group) {
            c->p.group_size = 32;
            rc = alloc_mixed(c, nb);
        }
        c->p = keep;
    }
    if (rc) {
        cudaStreamSynchronize(c->stream);
        free_all(nb.allocs);
        return rc;
    }
    if (keep && c->n > 0) {
        rc = copy_range(c, nb.st[0], 0, ob.st[c->cur], 0, c->n, ob.prev && want_prev, ob.pinned);
        if (rc) {
            cudaStreamSynchronize(c->stream);
            free_all(nb.allocs);
            return rc;
        }
    }
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    free_all(ob.allocs);
    c->b = std::move(nb);
    c->b.ss.spin_limit = c->sort_spin_limit;
    c->cur = 0;
    c->d_err = c->b.tree.meta + 4;
    c->tree_valid = false;
    c->keys_valid = false;
    return GE_OK;
}

// Segment tables for seg_cap simulations over n_cap particles.
int alloc_segs(ge_ctx *c, SegBuffers &nb, int64_t seg_cap, int64_t n_cap, int64_t tiles) {
    nb.seg_cap = std::max<int64_t>(seg_cap, 1);
    nb.n_cap = n_cap;
    nb.tile_cap = std::max<int64_t>(tiles, nb.n_cap / kSortTile + nb.seg_cap + 1);
    const size_t SC = (size_t)nb.seg_cap, TC = (size_t)nb.tile_cap;
    auto &L = nb.allocs;
    GE_CHECK(c, dalloc(L, &nb.off, SC + 1));
    GE_CHECK(c, dalloc(L, &nb.tile_base, SC + 1));
    GE_CHECK(c, dalloc(L, &nb.seg_of, (size_t)nb.n_cap));
    GE_CHECK(c, dalloc(L, &nb.tile_seg, TC));
    GE_CHECK(c, dalloc(L, &nb.box, SC));
    GE_CHECK(c, dalloc(L, &nb.boxmm, 6 * SC));
    GE_CHECK(c, dalloc(L, &nb.root_begin, SC));
    GE_CHECK(c, dalloc(L, &nb.root_end, SC));
    GE_CHECK(c, dalloc(L, &nb.hist, (size_t)kSortDigitWords * SC));
    GE_CHECK(c, dalloc(L, &nb.status, (size_t)kSortDigitWords * TC));
    nb.dtile_cap = nb.n_cap / kDirectTile + nb.seg_cap + 1;
    GE_CHECK(c, dalloc(L, &nb.dtiles, (size_t)nb.dtile_cap));
    GE_CHECK(c, dalloc(L, &nb.dflag, SC));
    if (!L.dry) {
        Segs all{};
        all.S = (int)nb.seg_cap;
        all.boxmm = nb.boxmm;
        GE_CHECK(c, launch_reset_boxes(all, c->stream));
    }
    return GE_OK;
}

// Which simulations take the direct sum (fewer than params.direct_below
// particles), the direct sum's tiles of kDirectTile particles over them, and
// the per-segment flag the walk skips them by (bound to c->g only when both
// kinds are present).
int direct_tables(ge_ctx *c) {
    const int64_t S = (int64_t)c->sims.size();
    c->h_dtiles.clear();
    c->h_dflag.assign((size_t)std::max<int64_t>(S, 1), 0u);
    c->any_direct = false;
    c->any_walk = S == 0;
    for (int64_t s = 0; s < S; s++) {
        const int64_t ns = c->sims[s].n;
        if (ns < (int64_t)c->p.direct_below) {
            c->h_dflag[s] = 1u;
            c->any_direct = true;
            for (int64_t o = 0; o < ns; o += kDirectTile)
                c->h_dtiles.push_back(make_uint2((uint32_t)s, c->h_off[s] + (uint32_t)o));
        } else {
            c->any_walk = true;
        }
    }
    c->g.direct = nullptr;
    if (!c->any_direct) return GE_OK;
    SegBuffers &sb = c->sb;
    if ((int64_t)c->h_dtiles.size() > sb.dtile_cap || S > sb.seg_cap)
        return fail(c, GE_ERR_STATE, "direct-sum tables exceed their capacity");
    GE_CHECK(c, cudaMemcpyAsync(sb.dtiles, c->h_dtiles.data(), sizeof(uint2) * c->h_dtiles.size(),
                                cudaMemcpyHostToDevice, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(sb.dflag, c->h_dflag.data(), (size_t)S, cudaMemcpyHostToDevice,
                                c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));   // the host tables are reused
    if (c->any_walk) c->g.direct = sb.dflag;
    return GE_OK;
}

// Rebuilds the segment tables from c->sims (after any change of the
// simulations or of the capacity) and binds them to the sort scratch.
int sync_segments(ge_ctx *c) {
    const int64_t S = (int64_t)c->sims.size();
    c->h_off.assign((size_t)S + 1, 0u);
    c->h_tile_base.assign((size_t)S + 1, 0u);
    for (int64_t s = 0; s < S; s++) {
        c->h_off[s + 1] = c->h_off[s] + (uint32_t)c->sims[s].n;
        c->h_tile_base[s + 1] =
            c->h_tile_base[s] + (uint32_t)((c->sims[s].n + kSortTile - 1) / kSortTile);
    }
    const int64_t tiles = c->h_tile_base[S];
    SegBuffers &sb = c->sb;
    if (S > sb.seg_cap || tiles > sb.tile_cap || c->b.cap_n > sb.n_cap) {
        SegBuffers nb;
        const int64_t scap = std::max<int64_t>(std::max<int64_t>(S, c->sims_reserved),
                                               sb.seg_cap + sb.seg_cap / 2);
        int rc = alloc_segs(c, nb, scap, c->b.cap_n, tiles);
        if (rc) {
            cudaStreamSynchronize(c->stream);
            free_all(nb.allocs);
            return rc;
        }
        GE_CHECK(c, cudaStreamSynchronize(c->stream));
        free_all(sb.allocs);
        sb = std::move(nb);
    }
    Segs &g = c->g;
    g = Segs{};
    g.S = (int)S;
    g.tiles = tiles;
    g.box = sb.box;
    g.boxmm = sb.boxmm;
    g.root_begin = sb.root_begin;
    g.root_end = sb.root_end;
    if (S > 1) {
        GE_CHECK(c, cudaMemcpyAsync(sb.off, c->h_off.data(), sizeof(uint32_t) * (S + 1),
                                    cudaMemcpyHostToDevice, c->stream));
        GE_CHECK(c, cudaMemcpyAsync(sb.tile_base, c->h_tile_base.data(), sizeof(uint32_t) * (S + 1),
                                    cudaMemcpyHostToDevice, c->stream));
        GE_CHECK(c, launch_seg_tables(sb.off, sb.tile_base, (int)S, (int)c->n, tiles, sb.seg_of,
                                      sb.tile_seg, c->stream));
        GE_CHECK(c, cudaStreamSynchronize(c->stream));   // the host tables are reused
        g.off = sb.off;
        g.seg_of = sb.seg_of;
        g.tile_base = sb.tile_base;
        g.tile_seg = sb.tile_seg;
    }
    c->b.ss.hist = sb.hist;
    c->b.ss.status = sb.status;
    int64_t bb = (c->n + kBBoxThreads * kBoxItems - 1) / (kBBoxThreads * kBoxItems);
    if (bb > (int64_t)c->num_sms * 4) bb = (int64_t)c->num_sms * 4;
    if (bb < 1) bb = 1;
    c->b.ss.box_blocks = (int)bb;
    c->tree_valid = false;
    c->keys_valid = false;
    return direct_tables(c);
}

// Reads back the error word and tree size; clears the error word.
int check_device(ge_ctx *c) {
    GE_CHECK(c, cudaMemcpyAsync(c->h_meta, c->b.tree.meta, 10 * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    const uint32_t e = c->h_meta[4];
    c->stats.nodes = c->h_meta[0];
    c->stats.depth = (int32_t)c->h_meta[1];
    c->slots = c->h_meta[9];
    if (e) {
        GE_CHECK(c, cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), c->stream));
        GE_CHECK(c, cudaStreamSynchronize(c->stream));
        c->tree_valid = false;
        if (e & kErrNodeCap)
            return fail(c, GE_ERR_CAPACITY, "tree node capacity exceeded; raise node_cap_factor");
        if (e & kErrDepth) return fail(c, GE_ERR_CAPACITY, "tree deeper than the level limit");
        if (e & kErrStack) return fail(c, GE_ERR_CAPACITY, "walk stack capacity exceeded");
        if (e & kErrSpin) return fail(c, GE_ERR_TIMEOUT, "a bounded device wait gave up");
        return fail(c, GE_ERR_CUDA, "device error word set");
    }
    return GE_OK;
}

// The state as the kernels see it: pin flags only when uploaded, Kahan terms
// only in the mixed mode (the walk sees temperatures only with heat exchange
// on, enqueue_walk).
State view(ge_ctx *c, int which) {
    State s = c->b.st[which];
    if (!c->has_pinned) s.pinned = nullptr;
    if (c->p.precision != GE_PREC_MIXED) s.kx = s.ky = s.kz = s.kvx = s.kvy = s.kvz = nullptr;
    return s;   // temperatures travel with the particles whenever they exist
}

State cur_state(ge_ctx *c) { return view(c, c->cur); }
State other_state(ge_ctx *c) { return view(c, c->cur ^ 1); }

int enqueue_bbox(ge_ctx *c, bool kick) {
    StepParams p = step_params(c);
    State s = cur_state(c);
    GE_CHECK(c, launch_kick_drift_bbox(c->p.dims, s, p, kick, c->g, c->b.ss, c->b.tree, c->stream));
    return GE_OK;
}

int enqueue_keys(ge_ctx *c) {
    GE_CHECK(c, launch_keys(c->p.dims, cur_state(c), (int)c->n, c->g, c->b.ss, c->stream));
    return GE_OK;
}

int enqueue_sort(ge_ctx *c) {
    GE_CHECK(c, launch_sort(c->p.dims, (int)c->n, c->g, c->b.ss, c->d_err, c->stream));
    return GE_OK;
}

int enqueue_permute(ge_ctx *c, bool with_acc) {
    GE_CHECK(c, launch_permute(c->p.dims, (int)c->n, c->b.ss, cur_state(c), other_state(c),
                               with_acc, c->stream));
    c->cur ^= 1;
    return GE_OK;
}

// fresh_keys: the sort's keys (c->b.ss.keys[0]) belong to the current
// particle order and positions (a sort and permute ran since the particles
// last moved), so the tree can be built from them (ge_kbuild.cu)
int enqueue_build(ge_ctx *c, bool fresh_keys = false) {
    StepParams p = step_params(c);
    // the optional layout arrays this build's readers need
    const bool temps = c->p.temp_enabled && c->b.temp;
    p.layout_extras = (c->p.precision == GE_PREC_MIXED || temps ? kLayoutEntry : 0) |
                      (c->p.walk_kind == 1 ? kLayoutRange : 0);
    c->tree_ranges = c->p.walk_kind == 1;
    const bool keyed = fresh_keys && c->p.leaf_cap >= 1 && c->p.leaf_cap <= (uint32_t)kKeyMaxCap;
    if (keyed)
        GE_CHECK(c, launch_key_build(c->p.dims, cur_state(c), p, c->g, c->b.ss.keys[0], c->b.tree,
                                     c->d_err, c->num_sms, c->stream));
    GE_CHECK(c, launch_build(c->p.dims, cur_state(c), p, c->g, c->b.tree, c->d_err, c->num_sms,
                             c->stream, keyed));
    if (c->p.precision == GE_PREC_MIXED) {
        Tree t = mixed_view(c);
        GE_CHECK(c, launch_moments(c->p.dims, cur_state(c), p, t, c->d_err, c->num_sms,
                                   c->stream));
    }
    if (temps)
        GE_CHECK(c, launch_node_temps(c->p.dims, cur_state(c), p, c->b.tree, c->num_sms,
                                      c->stream));
    return GE_OK;
}

// The mixed-precision arrays, when the mode (or its walk) was switched on
// after the upload.
int ensure_mode(ge_ctx *c) {
    if (c->p.precision != GE_PREC_MIXED) return GE_OK;
    const bool have = c->b.mixed && (wants_group(c->p) ? c->b.mixed_group : c->b.mixed_entry);
    if (have) return GE_OK;
    int rc = alloc_mixed(c, c->b);
    if (rc) return rc;
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int enqueue_walk(ge_ctx *c, bool integrate_end) {
    StepParams p = step_params(c);
    // a tree built without the layout ranges takes the per-particle walk
    if (!c->tree_ranges) p.walk_kind = 0;
    unsigned long long *cnt = nullptr;
    if (c->count_inter) {
        GE_CHECK(c, cudaMemsetAsync(c->b.d_inter, 0, sizeof(unsigned long long), c->stream));
        cnt = c->b.d_inter;
    }
    if (group_walk_on(c)) {
        GE_CHECK(c, launch_group_walk(c->p.dims, cur_state(c), p, c->g, mixed_view(c),
                                      integrate_end, cnt, c->b.tree.meta + 10, c->d_err,
                                      c->stream));
        return GE_OK;
    }
    State s = cur_state(c);
    if (c->any_direct)
        GE_CHECK(c, launch_direct(c->p.dims, c->p.precision, s, p, c->g, c->sb.dtiles,
                                  (int64_t)c->h_dtiles.size(), integrate_end, c->stream));
    if (!c->any_walk) return GE_OK;
    if (!c->p.temp_enabled) s.temp = nullptr;
    GE_CHECK(c, launch_walk(c->p.dims, c->p.precision, s, p, c->g, mixed_view(c), integrate_end,
                            cnt, c->d_err, c->num_sms, c->stream));
    return GE_OK;
}

int enqueue_frame(ge_ctx *c, cudaEvent_t *ev) {
    int rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[0], c->stream));
    if ((rc = enqueue_bbox(c, true))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[1], c->stream));
    if ((rc = enqueue_keys(c))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[2], c->stream));
    if ((rc = enqueue_sort(c))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[3], c->stream));
    if ((rc = enqueue_permute(c, false))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[4], c->stream));
    if ((rc = enqueue_build(c, true))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[5], c->stream));
    if ((rc = enqueue_walk(c, true))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[6], c->stream));
    return GE_OK;
}

int require_state(ge_ctx *c) {
    if (!c) return GE_ERR_ARG;
    if (c->n <= 0) return fail(c, GE_ERR_STATE, "no particles uploaded");
    return ensure_mode(c);
}

int check_host_arrays(ge_ctx *c, int64_t n, const float *x, const float *y, const float *z,
                      const float *vx, const float *vy, const float *vz, const float *m) {
    if (n < 1) return fail(c, GE_ERR_ARG, "n must be >= 1");
    if (!x || !y || !vx || !vy || !m || (c->p.dims == 3 && (!z || !vz)))
        return fail(c, GE_ERR_ARG, "positions, velocities and masses are required");
    return GE_OK;
}

// Host arrays into particles [off, off + n) of the current state.
int put_host(ge_ctx *c, int64_t off, int64_t n, const float *x, const float *y, const float *z,
             const float *vx, const float *vy, const float *vz, const float *m,
             const uint32_t *id, const float *ax, const float *ay, const float *az) {
    const int D = c->p.dims;
    const State &s = c->b.st[c->cur];
    const size_t B = sizeof(float) * (size_t)n;
    cudaStream_t st = c->stream;
    GE_CHECK(c, cudaMemcpyAsync(s.x + off, x, B, cudaMemcpyHostToDevice, st));
    GE_CHECK(c, cudaMemcpyAsync(s.y + off, y, B, cudaMemcpyHostToDevice, st));
    GE_CHECK(c, cudaMemcpyAsync(s.vx + off, vx, B, cudaMemcpyHostToDevice, st));
    GE_CHECK(c, cudaMemcpyAsync(s.vy + off, vy, B, cudaMemcpyHostToDevice, st));
    GE_CHECK(c, cudaMemcpyAsync(s.m + off, m, B, cudaMemcpyHostToDevice, st));
    if (D == 3) {
        GE_CHECK(c, cudaMemcpyAsync(s.z + off, z, B, cudaMemcpyHostToDevice, st));
        GE_CHECK(c, cudaMemcpyAsync(s.vz + off, vz, B, cudaMemcpyHostToDevice, st));
    }
    if (ax) GE_CHECK(c, cudaMemcpyAsync(s.ax + off, ax, B, cudaMemcpyHostToDevice, st));
    else GE_CHECK(c, cudaMemsetAsync(s.ax + off, 0, B, st));
    if (ay) GE_CHECK(c, cudaMemcpyAsync(s.ay + off, ay, B, cudaMemcpyHostToDevice, st));
    else GE_CHECK(c, cudaMemsetAsync(s.ay + off, 0, B, st));
    if (D == 3) {
        if (az) GE_CHECK(c, cudaMemcpyAsync(s.az + off, az, B, cudaMemcpyHostToDevice, st));
        else GE_CHECK(c, cudaMemsetAsync(s.az + off, 0, B, st));
    }
    if (id) {
        GE_CHECK(c, cudaMemcpyAsync(s.id + off, id, sizeof(uint32_t) * (size_t)n,
                                    cudaMemcpyHostToDevice, st));
        GE_CHECK(c, cudaStreamSynchronize(st));
    } else {
        std::vector<uint32_t> iota((size_t)n);
        for (int64_t i = 0; i < n; i++) iota[(size_t)i] = (uint32_t)i;
        GE_CHECK(c, cudaMemcpyAsync(s.id + off, iota.data(), sizeof(uint32_t) * (size_t)n,
                                    cudaMemcpyHostToDevice, st));
        GE_CHECK(c, cudaStreamSynchronize(st));
    }
    if (c->b.prev) {
        GE_CHECK(c, cudaMemcpyAsync(s.pvx + off, s.vx + off, B, cudaMemcpyDeviceToDevice, st));
        GE_CHECK(c, cudaMemcpyAsync(s.pvy + off, s.vy + off, B, cudaMemcpyDeviceToDevice, st));
        if (D == 3)
            GE_CHECK(c, cudaMemcpyAsync(s.pvz + off, s.vz + off, B, cudaMemcpyDeviceToDevice, st));
    }
    if (c->b.pinned) GE_CHECK(c, cudaMemsetAsync(s.pinned + off, 0, (size_t)n, st));
    if (s.temp) GE_CHECK(c, cudaMemsetAsync(s.temp + off, 0, B, st));
    if (s.kx) {
        float *kp[6] = {s.kx, s.ky, s.kz, s.kvx, s.kvy, s.kvz};
        for (float *q : kp)
            if (q) GE_CHECK(c, cudaMemsetAsync(q + off, 0, B, st));
    }
    return GE_OK;
}

// Particles [off, off + n) of the current state into host arrays.
int get_host(ge_ctx *c, int64_t off, int64_t n, float *x, float *y, float *z, float *vx,
             float *vy, float *vz, float *ax, float *ay, float *az, float *m, uint32_t *id) {
    const State &s = c->b.st[c->cur];
    const size_t B = sizeof(float) * (size_t)n;
    const bool d3 = c->p.dims == 3;
    struct { void *h; const void *d; size_t b; } cp[] = {
        {x, s.x + off, B}, {y, s.y + off, B}, {d3 ? z : nullptr, d3 ? s.z + off : nullptr, B},
        {vx, s.vx + off, B}, {vy, s.vy + off, B}, {d3 ? vz : nullptr, d3 ? s.vz + off : nullptr, B},
        {ax, s.ax + off, B}, {ay, s.ay + off, B}, {d3 ? az : nullptr, d3 ? s.az + off : nullptr, B},
        {m, s.m + off, B}, {id, s.id + off, sizeof(uint32_t) * (size_t)n}};
    for (auto &q : cp)
        if (q.h) GE_CHECK(c, cudaMemcpyAsync(q.h, q.d, q.b, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

// ge_frame_host on a context that holds the same single simulation as its
// last frame: the same upload, step and download, but the masses and ids go
// up beside the kick, box, keys and sort (they are needed from the
// permutation on), and the positions, masses and ids come back beside the
// build and the walk (they are final once permuted); only the velocities and
// accelerations wait for the walk.  Everything ends synchronised, as the
// serial path does.
int frame_overlapped(ge_ctx *c, int64_t n, const float *x, const float *y, const float *z,
                     const float *vx, const float *vy, const float *vz, const float *ax,
                     const float *ay, const float *az, const float *m, const uint32_t *id,
                     float *ox, float *oy, float *oz, float *ovx, float *ovy, float *ovz,
                     float *oax, float *oay, float *oaz, float *om, uint32_t *oid) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!c->copy_stream) {
        GE_CHECK(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        for (auto &e : c->xev) GE_CHECK(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaStream_t s0 = c->stream, s1 = c->copy_stream;
    const int D = c->p.dims;
    const size_t B = sizeof(float) * (size_t)n;
    // as ge_upload: pin flags cleared, the simulation restarts its count
    c->has_pinned = false;
    c->sims.assign(1, SimRec{c->next_handle++, n, c->total_steps});
    c->tree_valid = false;
    c->keys_valid = false;
    GE_CHECK(c, cudaEventRecord(c->xev[0], s0));   // the copy stream starts after earlier work
    GE_CHECK(c, cudaStreamWaitEvent(s1, c->xev[0], 0));
    {
        const State &s = c->b.st[c->cur];
        GE_CHECK(c, cudaMemcpyAsync(s.x, x, B, cudaMemcpyHostToDevice, s0));
        GE_CHECK(c, cudaMemcpyAsync(s.y, y, B, cudaMemcpyHostToDevice, s0));
        GE_CHECK(c, cudaMemcpyAsync(s.vx, vx, B, cudaMemcpyHostToDevice, s0));
        GE_CHECK(c, cudaMemcpyAsync(s.vy, vy, B, cudaMemcpyHostToDevice, s0));
        if (D == 3) {
            GE_CHECK(c, cudaMemcpyAsync(s.z, z, B, cudaMemcpyHostToDevice, s0));
            GE_CHECK(c, cudaMemcpyAsync(s.vz, vz, B, cudaMemcpyHostToDevice, s0));
        }
        const float *acc[3] = {ax, ay, az};
        float *dacc[3] = {s.ax, s.ay, s.az};
        for (int a = 0; a < D; a++) {
            if (acc[a]) GE_CHECK(c, cudaMemcpyAsync(dacc[a], acc[a], B, cudaMemcpyHostToDevice, s0));
            else GE_CHECK(c, cudaMemsetAsync(dacc[a], 0, B, s0));
        }
        if (c->b.prev) {
            GE_CHECK(c, cudaMemcpyAsync(s.pvx, s.vx, B, cudaMemcpyDeviceToDevice, s0));
            GE_CHECK(c, cudaMemcpyAsync(s.pvy, s.vy, B, cudaMemcpyDeviceToDevice, s0));
            if (D == 3) GE_CHECK(c, cudaMemcpyAsync(s.pvz, s.vz, B, cudaMemcpyDeviceToDevice, s0));
        }
        if (c->b.pinned) GE_CHECK(c, cudaMemsetAsync(s.pinned, 0, (size_t)n, s0));
        if (s.temp) GE_CHECK(c, cudaMemsetAsync(s.temp, 0, B, s0));
        if (s.kx) {
            float *kp[6] = {s.kx, s.ky, s.kz, s.kvx, s.kvy, s.kvz};
            for (float *q : kp)
                if (q) GE_CHECK(c, cudaMemsetAsync(q, 0, B, s0));
        }
        GE_CHECK(c, cudaMemcpyAsync(s.m, m, B, cudaMemcpyHostToDevice, s1));
        GE_CHECK(c, cudaMemcpyAsync(s.id, id, sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice, s1));
        GE_CHECK(c, cudaEventRecord(c->xev[1], s1));
    }
    GE_CHECK(c, cudaEventRecord(c->ev[6], s0));
    if ((rc = enqueue_bbox(c, true)) || (rc = enqueue_keys(c)) || (rc = enqueue_sort(c))) return rc;
    GE_CHECK(c, cudaStreamWaitEvent(s0, c->xev[1], 0));
    if ((rc = enqueue_permute(c, false))) return rc;
    GE_CHECK(c, cudaEventRecord(c->xev[2], s0));
    GE_CHECK(c, cudaStreamWaitEvent(s1, c->xev[2], 0));
    {
        const State &s = c->b.st[c->cur];   // permuted
        GE_CHECK(c, cudaMemcpyAsync(ox, s.x, B, cudaMemcpyDeviceToHost, s1));
        GE_CHECK(c, cudaMemcpyAsync(oy, s.y, B, cudaMemcpyDeviceToHost, s1));
        if (D == 3 && oz) GE_CHECK(c, cudaMemcpyAsync(oz, s.z, B, cudaMemcpyDeviceToHost, s1));
        if (om) GE_CHECK(c, cudaMemcpyAsync(om, s.m, B, cudaMemcpyDeviceToHost, s1));
        if (oid) GE_CHECK(c, cudaMemcpyAsync(oid, s.id, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToHost, s1));
    }
    if ((rc = enqueue_build(c, true))) return rc;
    {
        const State &s = c->b.st[c->cur];
        float *h[6] = {ovx, ovy, ovz, oax, oay, oaz};
        const float *dv[6] = {s.vx, s.vy, s.vz, s.ax, s.ay, s.az};
        auto back = [&](int64_t lo, int64_t hi, cudaStream_t on) -> cudaError_t {
            for (int q = 0; q < 6; q++)
                if (h[q] && (D == 3 || (q % 3) != 2)) {
                    const cudaError_t e = cudaMemcpyAsync(h[q] + lo, dv[q] + lo,
                                                          sizeof(float) * (size_t)(hi - lo),
                                                          cudaMemcpyDeviceToHost, on);
                    if (e != cudaSuccess) return e;
                }
            return cudaSuccess;
        };
        if (group_walk_on(c) || c->any_direct || c->count_inter) {
            if ((rc = enqueue_walk(c, true))) return rc;
            GE_CHECK(c, back(0, n, s0));
        } else {
            // the per-particle walk in particle ranges: each range's velocities and
            // accelerations go back while the next range walks
            constexpr int kParts = 4;
            StepParams p = step_params(c);
            State ws = cur_state(c);
            if (!c->p.temp_enabled) ws.temp = nullptr;
            for (int part = 0; part < kParts; part++) {
                const int64_t lo = (n * part / kParts) & ~int64_t(255);
                const int64_t hi = part + 1 == kParts ? n : (n * (part + 1) / kParts) & ~int64_t(255);
                if (hi <= lo) continue;
                p.i0 = (int)lo;
                p.n = (int)hi;
                GE_CHECK(c, launch_walk(c->p.dims, c->p.precision, ws, p, c->g, mixed_view(c), true,
                                        nullptr, c->d_err, c->num_sms, s0));
                GE_CHECK(c, cudaEventRecord(c->xev[2], s0));
                GE_CHECK(c, cudaStreamWaitEvent(s1, c->xev[2], 0));
                GE_CHECK(c, back(lo, hi, s1));
            }
        }
    }
    GE_CHECK(c, cudaEventRecord(c->ev[7], s0));
    GE_CHECK(c, cudaStreamSynchronize(s1));
    // as ge_step_wait for one step (check_device synchronises the compute stream)
    rc = check_device(c);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]);
    c->stats.ms_last_step = ms;
    c->stats.steps += 1;
    c->total_steps += 1;
    c->tree_valid = rc == GE_OK;
    if (rc == GE_OK && c->count_inter) {
        unsigned long long v = 0;
        GE_CHECK(c, cudaMemcpy(&v, c->b.d_inter, sizeof(v), cudaMemcpyDeviceToHost));
        c->stats.interactions = v;
    }
    return rc;
}

int frame_overlapped(ge_ctx *c, int64_t n, float *x, float *y, float *z, float *vx, float *vy,
                     float *vz, float *ax, float *ay, float *az, float *m, uint32_t *id) {
    return frame_overlapped(c, n, x, y, z, vx, vy, vz, ax, ay, az, m, id, x, y, z, vx, vy, vz, ax,
                            ay, az, m, id);
}

// Temperature arrays (both state buffers, zeroed) and the node temperature
// arrays, when the context has none yet.
int ensure_temp(ge_ctx *c) {
    if (c->b.temp) return GE_OK;
    auto &L = c->b.allocs;
    const size_t N = (size_t)c->b.cap_n;
    for (int k = 0; k < 2; k++) {
        GE_CHECK(c, dalloc(L, &c->b.st[k].temp, N));
        GE_CHECK(c, cudaMemsetAsync(c->b.st[k].temp, 0, sizeof(float) * N, c->stream));
    }
    GE_CHECK(c, dalloc(L, &c->b.tree.ntemp, (size_t)c->b.tree.cap));
    GE_CHECK(c, dalloc(L, &c->b.tree.tv, N + (size_t)c->b.tree.cap + 1));
    c->b.temp = true;
    return GE_OK;
}

// Pin flag arrays (both state buffers), when the context has none yet.
int ensure_pinned(ge_ctx *c) {
    if (c->b.pinned) return GE_OK;
    for (int k = 0; k < 2; k++)
        GE_CHECK(c, dalloc(c->b.allocs, &c->b.st[k].pinned, (size_t)c->b.cap_n));
    c->b.pinned = true;
    return GE_OK;
}

// A device buffer of at least `bytes`, grown (and its contents dropped) when
// too small.
int ensure_bytes(ge_ctx *c, unsigned char **buf, size_t *have, size_t bytes) {
    if (*have >= bytes && *buf) return GE_OK;
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *have = 0;
    GE_CHECK(c, cudaMalloc((void **)buf, bytes));
    *have = bytes;
    return GE_OK;
}

int find_sim(ge_ctx *c, int32_t handle) {
    for (size_t k = 0; k < c->sims.size(); k++)
        if (c->sims[k].handle == handle) return (int)k;
    return -1;
}

}  // namespace

extern "C" {

int ge_abi_version(void) { return GE_ABI_VERSION; }

void ge_params_default(ge_params *p, int dims) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->dims = dims == 3 ? 3 : 2;
    p->precision = GE_PREC_FAST;
    p->G = 6.674e-11f;          // parameters.h:114
    p->theta = 0.8f;            // parameters.h:117
    p->eps2 = p->dims == 2 ? 1.5f * 1.5f : 1.5f;   // softening 1.5 (parameters.h:116)
    p->dt = 0.045f;             // fixedDeltaTime (parameters.h:129)
    p->leaf_cap = 4;
    p->size_gate = 2.0f;
    p->min_size = 1e-6f;
    p->node_cap_factor = p->dims == 2 ? 4.0f : 8.0f;   // quadtree.cpp:94, :278
    p->domain[0] = p->dims == 2 ? 3840.0f : 1300.0f;   // parameters.h:97-99
    p->domain[1] = p->dims == 2 ? 2160.0f : 1300.0f;
    p->domain[2] = 1300.0f;
    p->group_size = 32;
    p->heat_cond = 0.045f;      // globalHeatConductivity (parameters.h:120)
    p->direct_eps2 = 1.5f;      // softening, added un-squared by naiveGravity
}

int ge_create(const ge_params *p, ge_ctx **out) {
    if (!out) return GE_ERR_ARG;
    *out = nullptr;
    ge_ctx *c = new ge_ctx();
    int rc = validate(c, p);
    if (rc) { delete c; return rc; }
    c->p = *p;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        delete c;
        return GE_ERR_NO_DEVICE;
    }
    cudaGetDevice(&c->dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c->dev) != cudaSuccess || prop.major < 10) {
        delete c;
        return GE_ERR_NO_DEVICE;
    }
    c->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return GE_ERR_CUDA;
    }
    for (auto &e : c->ev) cudaEventCreate(&e);
    if (cudaMallocHost(&c->h_meta, 16 * sizeof(uint32_t)) != cudaSuccess) {
        ge_destroy(c);
        return GE_ERR_CUDA;
    }
    *out = c;
    return GE_OK;
}

int ge_batch_create(const ge_params *p, ge_ctx **out) { return ge_create(p, out); }

int ge_destroy(ge_ctx *c) {
    if (!c) return GE_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_buffers(c);
    for (auto &e : c->ev) if (e) cudaEventDestroy(e);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    for (auto &e : c->xev) if (e) cudaEventDestroy(e);
    if (c->h_meta) cudaFreeHost(c->h_meta);
    if (c->d_aos) cudaFree(c->d_aos);
    if (c->d_aos_r) cudaFree(c->d_aos_r);
    if (c->d_order) cudaFree(c->d_order);
    if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return GE_OK;
}

const char *ge_last_error(const ge_ctx *c) { return c ? c->err.c_str() : "null context"; }

int ge_set_params(ge_ctx *c, const ge_params *p) {
    if (!c) return GE_ERR_ARG;
    int rc = validate(c, p);
    if (rc) return rc;
    if (p->dims != c->p.dims && c->b.cap_n) {
        GE_CHECK(c, cudaStreamSynchronize(c->stream));
        free_buffers(c);
    }
    const bool realloc = c->b.cap_n && (p->node_cap_factor != c->p.node_cap_factor ||
                                        (p->track_prev_vel != 0) != c->b.prev);
    if (realloc) return fail(c, GE_ERR_STATE, "node_cap_factor / track_prev_vel change needs a new upload");
    const bool to_mixed = p->precision == GE_PREC_MIXED && c->p.precision != GE_PREC_MIXED;
    const bool new_direct = p->direct_below != c->p.direct_below;
    c->p = *p;
    if (new_direct && c->sb.seg_cap) {
        rc = direct_tables(c);
        if (rc) return rc;
    }
    if (to_mixed && c->b.mixed) {
        // the compensation terms were not carried in the other modes: restart them
        for (int k = 0; k < 2; k++) {
            const State &s = c->b.st[k];
            float *kp[6] = {s.kx, s.ky, s.kz, s.kvx, s.kvy, s.kvz};
            for (float *q : kp)
                if (q) GE_CHECK(c, cudaMemsetAsync(q, 0, sizeof(float) * (size_t)c->b.cap_n, c->stream));
        }
    }
    c->tree_valid = false;
    return GE_OK;
}

int ge_set_stream(ge_ctx *c, void *s) {
    if (!c) return GE_ERR_ARG;
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    if (c->own_stream) cudaStreamDestroy(c->stream);
    if (s) {
        c->stream = (cudaStream_t)s;
        c->own_stream = false;
    } else {
        GE_CHECK(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    return GE_OK;
}

int ge_sync(ge_ctx *c) {
    if (!c) return GE_ERR_ARG;
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int ge_get_stats(ge_ctx *c, ge_stats *out) {
    if (!c || !out) return GE_ERR_ARG;
    c->stats.n = c->n;
    *out = c->stats;
    return GE_OK;
}

int ge_set_sort_wait_test(ge_ctx *c, uint32_t spin_limit, int32_t withhold) {
    if (!c) return GE_ERR_ARG;
    if (withhold != 0 && withhold != 1) return fail(c, GE_ERR_ARG, "withhold must be 0 or 1");
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    c->sort_spin_limit = spin_limit;
    c->sort_withhold = (uint32_t)withhold;
    c->b.ss.spin_limit = spin_limit;
    return GE_OK;
}

int ge_set_count_interactions(ge_ctx *c, int32_t enable) {
    if (!c) return GE_ERR_ARG;
    c->count_inter = enable != 0;
    return GE_OK;
}

int ge_upload(ge_ctx *c, int64_t n, const float *x, const float *y, const float *z,
              const float *vx, const float *vy, const float *vz, const float *m,
              const uint32_t *id, const float *ax, const float *ay, const float *az) {
    if (!c) return GE_ERR_ARG;
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    int rc = check_host_arrays(c, n, x, y, z, vx, vy, vz, m);
    if (rc) return rc;
    if ((rc = ensure_capacity(c, n, 1, false))) return rc;
    c->cur = 0;
    c->has_pinned = false;
    if ((rc = put_host(c, 0, n, x, y, z, vx, vy, vz, m, id, ax, ay, az))) return rc;
    c->n = n;
    c->sims.assign(1, SimRec{c->next_handle++, n, c->total_steps});
    return sync_segments(c);
}

int ge_upload_pinned(ge_ctx *c, const uint8_t *pinned) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!pinned) {
        c->has_pinned = false;
        return GE_OK;
    }
    if ((rc = ensure_pinned(c))) return rc;
    GE_CHECK(c, cudaMemcpyAsync(c->b.st[c->cur].pinned, pinned, (size_t)c->n,
                                cudaMemcpyHostToDevice, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    c->has_pinned = true;
    return GE_OK;
}

int ge_upload_temp(ge_ctx *c, const float *temp) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!temp) return fail(c, GE_ERR_ARG, "temp is NULL");
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    if ((rc = ensure_temp(c))) return rc;
    GE_CHECK(c, cudaMemcpyAsync(c->b.st[c->cur].temp, temp, sizeof(float) * (size_t)c->n,
                                cudaMemcpyHostToDevice, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    c->tree_valid = false;
    return GE_OK;
}

int ge_download_temp(ge_ctx *c, float *temp) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!temp) return fail(c, GE_ERR_ARG, "temp is NULL");
    if (!c->b.temp) return fail(c, GE_ERR_STATE, "no temperatures uploaded");
    GE_CHECK(c, cudaMemcpyAsync(temp, c->b.st[c->cur].temp, sizeof(float) * (size_t)c->n,
                                cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int ge_download(ge_ctx *c, float *x, float *y, float *z, float *vx, float *vy, float *vz,
                float *ax, float *ay, float *az, float *m, uint32_t *id) {
    int rc = require_state(c);
    if (rc) return rc;
    return get_host(c, 0, c->n, x, y, z, vx, vy, vz, ax, ay, az, m, id);
}

void ge_aos_layout_default(ge_aos_layout *l, int dims) {
    if (!l) return;
    // member offsets of the reference's records (include/Particles/particle.h):
    // ParticlePhysics 128 B, ParticlePhysics3D 160 B, ParticleRendering[3D] 60 B
    if (dims == 3) *l = ge_aos_layout{160, 0, 12, 24, 48, 96, 148, 136, 60, 56};
    else *l = ge_aos_layout{128, 0, 8, 16, 32, 64, 116, 104, 60, 56};
}

int ge_frame_aos(ge_ctx *c, int64_t n, void *phys, const void *rend, const ge_aos_layout *L,
                 uint32_t *order) {
    if (!c) return GE_ERR_ARG;
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    if (n < 1 || !phys || !L) return fail(c, GE_ERR_ARG, "records and layout are required");
    const int D = c->p.dims;
    const int vec = 4 * D;
    auto member_ok = [&](int32_t off, int bytes) {
        return off >= 0 && off % 4 == 0 && (int64_t)off + bytes <= L->stride;
    };
    if (L->stride < 4 || L->stride % 4 != 0 || !member_ok(L->off_pos, vec) ||
        !member_ok(L->off_vel, vec) || !member_ok(L->off_acc, vec) || !member_ok(L->off_mass, 4) ||
        !member_ok(L->off_id, 4) || (L->off_prev_vel != -1 && !member_ok(L->off_prev_vel, vec)) ||
        (L->off_temp != -1 && !member_ok(L->off_temp, 4)))
        return fail(c, GE_ERR_ARG, "record layout: offsets must be 4-byte aligned members inside the stride");
    const bool pins = rend && L->r_off_pinned >= 0;
    if (pins && !(L->r_stride >= 1 && L->r_off_pinned < L->r_stride))
        return fail(c, GE_ERR_ARG, "record layout: isPinned outside the rendering record");
    const bool temps = c->p.temp_enabled && L->off_temp >= 0;
    const bool prevs = c->p.track_prev_vel && L->off_prev_vel >= 0;
    // (the members could also be read and written in place when the records
    // are page-locked, over PCIe from the kernels: measured 2.5x slower than
    // these copies at 1M particles -- scattered 32-byte reads of 128-byte
    // records -- so every record array goes through one device copy)
    unsigned char *phys_map = nullptr, *rend_map = nullptr;
    int rc;
    if ((rc = ensure_capacity(c, n, 1, false))) return rc;
    if (!phys_map && (rc = ensure_bytes(c, &c->d_aos, &c->aos_bytes, (size_t)n * L->stride)))
        return rc;
    if (pins && !rend_map &&
        (rc = ensure_bytes(c, &c->d_aos_r, &c->aos_r_bytes, (size_t)n * L->r_stride)))
        return rc;
    if (order && c->order_cap < n) {
        GE_CHECK(c, cudaStreamSynchronize(c->stream));
        if (c->d_order) cudaFree(c->d_order);
        c->d_order = nullptr;
        c->order_cap = 0;
        GE_CHECK(c, cudaMalloc((void **)&c->d_order, sizeof(uint32_t) * (size_t)n));
        c->order_cap = n;
    }
    if (pins && (rc = ensure_pinned(c))) return rc;
    if (temps && (rc = ensure_temp(c))) return rc;
    if ((rc = ensure_mode(c))) return rc;
    // as ge_upload: one simulation, restarting its step count
    c->cur = 0;
    c->has_pinned = pins;
    c->n = n;
    c->sims.assign(1, SimRec{c->next_handle++, n, c->total_steps});
    c->tree_valid = false;
    c->keys_valid = false;
    if ((rc = sync_segments(c))) return rc;
    cudaStream_t st = c->stream;
    unsigned char *dphys = phys_map ? phys_map : c->d_aos;
    const unsigned char *drend = pins ? (rend_map ? rend_map : c->d_aos_r) : nullptr;
    if (!phys_map)
        GE_CHECK(c, cudaMemcpyAsync(c->d_aos, phys, (size_t)n * L->stride, cudaMemcpyHostToDevice,
                                    st));
    if (pins && !rend_map)
        GE_CHECK(c, cudaMemcpyAsync(c->d_aos_r, rend, (size_t)n * L->r_stride,
                                    cudaMemcpyHostToDevice, st));
    State s = c->b.st[c->cur];
    if (!pins) s.pinned = nullptr;
    if (!temps) s.temp = nullptr;
    if (!c->b.prev) s.pvx = s.pvy = s.pvz = nullptr;
    GE_CHECK(c, launch_aos_in(D, dphys, drend, *L, (int)n, s, st));
    {   // the mixed mode's compensation terms start at zero, as after ge_upload
        const State &sb = c->b.st[c->cur];
        float *kp[6] = {sb.kx, sb.ky, sb.kz, sb.kvx, sb.kvy, sb.kvz};
        for (float *q : kp)
            if (q) GE_CHECK(c, cudaMemsetAsync(q, 0, sizeof(float) * (size_t)n, st));
    }
    GE_CHECK(c, cudaEventRecord(c->ev[6], st));
    if ((rc = enqueue_frame(c, nullptr))) return rc;
    GE_CHECK(c, cudaEventRecord(c->ev[7], st));
    State o = c->b.st[c->cur];
    if (!temps) o.temp = nullptr;
    if (!prevs) o.pvx = o.pvy = o.pvz = nullptr;
    GE_CHECK(c, launch_aos_out(D, dphys, *L, (int)n, o, c->b.ss, st));
    if (!phys_map) {
        // the byte span of each record that the frame changed, one pitched copy
        int32_t lo = std::min(L->off_pos, std::min(L->off_vel, L->off_acc));
        int32_t hi = std::max(L->off_pos, std::max(L->off_vel, L->off_acc)) + vec;
        if (prevs) { lo = std::min(lo, L->off_prev_vel); hi = std::max(hi, L->off_prev_vel + vec); }
        if (temps) { lo = std::min(lo, L->off_temp); hi = std::max(hi, L->off_temp + 4); }
        GE_CHECK(c, cudaMemcpy2DAsync((unsigned char *)phys + lo, (size_t)L->stride, c->d_aos + lo,
                                      (size_t)L->stride, (size_t)(hi - lo), (size_t)n,
                                      cudaMemcpyDeviceToHost, st));
    }
    if (order) {
        GE_CHECK(c, launch_perm_out(D, (int)n, c->b.ss, c->d_order, st));
        GE_CHECK(c, cudaMemcpyAsync(order, c->d_order, sizeof(uint32_t) * (size_t)n,
                                    cudaMemcpyDeviceToHost, st));
    }
    rc = check_device(c);   // synchronises the stream
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]);
    c->stats.ms_last_step = ms;
    c->stats.steps += 1;
    c->total_steps += 1;
    c->tree_valid = rc == GE_OK;
    return rc;
}

int ge_download_state(ge_ctx *c, const ge_state_arrays *h) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!h) return fail(c, GE_ERR_ARG, "state arrays are NULL");
    if ((rc = get_host(c, 0, c->n, h->x, h->y, h->z, h->vx, h->vy, h->vz, h->ax, h->ay, h->az,
                       h->m, h->id)))
        return rc;
    const State &s = c->b.st[c->cur];
    const bool d3 = c->p.dims == 3;
    const size_t B = sizeof(float) * (size_t)c->n;
    struct { float *h; const float *d; } cp[] = {
        {h->kx, c->b.mixed ? s.kx : nullptr}, {h->ky, c->b.mixed ? s.ky : nullptr},
        {d3 ? h->kz : nullptr, c->b.mixed ? s.kz : nullptr},
        {h->kvx, c->b.mixed ? s.kvx : nullptr}, {h->kvy, c->b.mixed ? s.kvy : nullptr},
        {d3 ? h->kvz : nullptr, c->b.mixed ? s.kvz : nullptr},
        {h->pvx, c->b.prev ? s.pvx : nullptr}, {h->pvy, c->b.prev ? s.pvy : nullptr},
        {d3 ? h->pvz : nullptr, c->b.prev ? s.pvz : nullptr},
        {h->temp, c->b.temp ? s.temp : nullptr}};
    for (auto &q : cp) {
        if (!q.h) continue;
        if (q.d) GE_CHECK(c, cudaMemcpyAsync(q.h, q.d, B, cudaMemcpyDeviceToHost, c->stream));
        else std::memset(q.h, 0, B);
    }
    if (h->pinned) {
        if (c->has_pinned)
            GE_CHECK(c, cudaMemcpyAsync(h->pinned, s.pinned, (size_t)c->n, cudaMemcpyDeviceToHost,
                                        c->stream));
        else std::memset(h->pinned, 0, (size_t)c->n);
    }
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int ge_upload_state(ge_ctx *c, int64_t n, const ge_state_arrays *h) {
    if (!c) return GE_ERR_ARG;
    if (!h) return fail(c, GE_ERR_ARG, "state arrays are NULL");
    const bool d3 = c->p.dims == 3;
    const bool comp = h->kx || h->ky || h->kvx || h->kvy || (d3 && (h->kz || h->kvz));
    if (comp && c->p.precision != GE_PREC_MIXED)
        return fail(c, GE_ERR_STATE, "compensation terms exist in GE_PREC_MIXED only");
    int rc = ge_upload(c, n, h->x, h->y, h->z, h->vx, h->vy, h->vz, h->m, h->id, h->ax, h->ay,
                       h->az);
    if (rc) return rc;
    if ((rc = require_state(c))) return rc;   // the mixed mode's arrays
    const State &s = c->b.st[c->cur];
    const size_t B = sizeof(float) * (size_t)n;
    struct { const float *h; float *d; } cp[] = {
        {h->kx, s.kx}, {h->ky, s.ky}, {d3 ? h->kz : nullptr, s.kz},
        {h->kvx, s.kvx}, {h->kvy, s.kvy}, {d3 ? h->kvz : nullptr, s.kvz},
        {h->pvx, c->b.prev ? s.pvx : nullptr}, {h->pvy, c->b.prev ? s.pvy : nullptr},
        {d3 ? h->pvz : nullptr, c->b.prev ? s.pvz : nullptr}};
    for (auto &q : cp)
        if (q.h && q.d) GE_CHECK(c, cudaMemcpyAsync(q.d, q.h, B, cudaMemcpyHostToDevice, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    if (h->pinned && (rc = ge_upload_pinned(c, h->pinned))) return rc;
    if (h->temp && (rc = ge_upload_temp(c, h->temp))) return rc;
    return GE_OK;
}

int ge_download_prev_vel(ge_ctx *c, float *pvx, float *pvy, float *pvz) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!c->b.prev) return fail(c, GE_ERR_STATE, "track_prev_vel is off");
    const State &s = c->b.st[c->cur];
    const size_t B = sizeof(float) * (size_t)c->n;
    if (pvx) GE_CHECK(c, cudaMemcpyAsync(pvx, s.pvx, B, cudaMemcpyDeviceToHost, c->stream));
    if (pvy) GE_CHECK(c, cudaMemcpyAsync(pvy, s.pvy, B, cudaMemcpyDeviceToHost, c->stream));
    if (pvz && c->p.dims == 3)
        GE_CHECK(c, cudaMemcpyAsync(pvz, s.pvz, B, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

// The bytes that decide what enqueue_frame launches and with which
// arguments: parameters, counts, buffer roles and every device pointer the
// kernels take.  A graph whose bytes match launches exactly what
// enqueue_frame would.
std::vector<uint8_t> frame_signature(const ge_ctx *c) {
    std::vector<uint8_t> v;
    v.reserve(1024);
    auto put = [&](const void *q, size_t nb) {
        const uint8_t *b = static_cast<const uint8_t *>(q);
        v.insert(v.end(), b, b + nb);
    };
    put(&c->p, sizeof c->p);
    put(&c->n, sizeof c->n);
    put(&c->cur, sizeof c->cur);
    const uint8_t flags[8] = {c->has_pinned, c->any_direct, c->any_walk, c->count_inter,
                              c->b.prev, c->b.pinned, c->b.temp, c->b.mixed};
    put(flags, sizeof flags);
    put(&c->b.st[0], sizeof(State));
    put(&c->b.st[1], sizeof(State));
    put(&c->b.ss, sizeof(SortScratch));
    put(&c->b.tree, sizeof(Tree));
    put(&c->b.d_inter, sizeof c->b.d_inter);
    put(&c->g, sizeof(Segs));
    put(&c->sb.dtiles, sizeof c->sb.dtiles);
    const size_t nd = c->h_dtiles.size();
    put(&nd, sizeof nd);
    put(&c->stream, sizeof c->stream);
    put(&c->d_err, sizeof c->d_err);
    put(&c->num_sms, sizeof c->num_sms);
    return v;
}

// Capture two steps into graph slot `slot` (nothing runs; the host-side
// buffer roles, flipped twice, end where they began).  On any refusal the
// context falls back to plain launches for good.
void capture_two_frames(ge_ctx *c, int slot, std::vector<uint8_t> sig) {
    ge_ctx::StepGraph &sg = c->graphs[slot];
    if (sg.exec) cudaGraphExecDestroy(sg.exec);
    sg.exec = nullptr;
    sg.sig.clear();
    const int cur0 = c->cur;
    const SortScratch ss0 = c->b.ss;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        (void)cudaGetLastError();
        c->graph_failed = true;
        return;
    }
    int rc = enqueue_frame(c, nullptr);
    if (!rc) rc = enqueue_frame(c, nullptr);
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    const bool same = c->cur == cur0 && std::memcmp(&c->b.ss, &ss0, sizeof ss0) == 0;
    c->cur = cur0;
    c->b.ss = ss0;
    if (rc || e != cudaSuccess || !graph || !same ||
        cudaGraphInstantiate(&sg.exec, graph, 0) != cudaSuccess) {
        (void)cudaGetLastError();
        sg.exec = nullptr;
        c->graph_failed = true;
        c->err.clear();
    } else {
        sg.sig = std::move(sig);
    }
    if (graph) cudaGraphDestroy(graph);
}

int ge_step_async(ge_ctx *c, int32_t nsteps) {
    int rc = require_state(c);
    if (rc) return rc;
    if (nsteps < 0) return fail(c, GE_ERR_ARG, "nsteps must be >= 0");
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    if (nsteps == 0) return GE_OK;
    GE_CHECK(c, cudaEventRecord(c->ev[6], c->stream));
    int k = 0;
    if (!c->framed) {   // the first frame plainly: one-time launch setup outside a capture
        if ((rc = enqueue_frame(c, nullptr))) return rc;
        c->framed = true;
        k = 1;
    }
    if (nsteps - k >= 2 && !c->p.no_graph && !c->graph_failed) {
        std::vector<uint8_t> sig = frame_signature(c);
        int slot = -1;
        for (int q = 0; q < 2; q++)
            if (c->graphs[q].exec && c->graphs[q].sig == sig) slot = q;
        if (slot < 0) {
            slot = c->next_graph;
            c->next_graph ^= 1;
            capture_two_frames(c, slot, std::move(sig));
        }
        if (c->graphs[slot].exec)
            for (; k + 2 <= nsteps; k += 2)
                GE_CHECK(c, cudaGraphLaunch(c->graphs[slot].exec, c->stream));
    }
    for (; k < nsteps; k++)
        if ((rc = enqueue_frame(c, nullptr))) return rc;
    GE_CHECK(c, cudaEventRecord(c->ev[7], c->stream));
    c->pending_steps = nsteps;
    c->tree_valid = false;
    return GE_OK;
}

int ge_step_wait(ge_ctx *c) {
    if (!c) return GE_ERR_ARG;
    const int32_t nsteps = c->pending_steps;
    if (!nsteps) return GE_OK;
    c->pending_steps = 0;
    int rc = check_device(c);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]);
    c->stats.ms_last_step = ms / (float)nsteps;
    c->stats.steps += nsteps;
    c->total_steps += nsteps;
    c->tree_valid = rc == GE_OK;
    if (rc == GE_OK && c->count_inter) {
        unsigned long long v = 0;
        GE_CHECK(c, cudaMemcpy(&v, c->b.d_inter, sizeof(v), cudaMemcpyDeviceToHost));
        c->stats.interactions = v;
    }
    return rc;
}

int ge_step(ge_ctx *c, int32_t nsteps) {
    int rc = ge_step_async(c, nsteps);
    if (rc) return rc;
    return ge_step_wait(c);
}

int ge_batch_step(ge_ctx *c, int32_t nsteps) { return ge_step(c, nsteps); }

int ge_autotune(ge_ctx *c, int32_t reps, ge_tune_result *out) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!out || reps < 1) return fail(c, GE_ERR_ARG, "bad autotune arguments");
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    if (c->p.precision != GE_PREC_MIXED || c->p.periodic)
        return fail(c, GE_ERR_STATE, "autotuning needs the mixed mode's group walk");
    std::memset(out, 0, sizeof(*out));
    const ge_params keep = c->p;
    static const int32_t kGroups[3] = {32, 64, 128}, kLeaves[4] = {1, 4, 8, 16};
    // the tree is built over the Morton order of the current positions
    if ((rc = enqueue_bbox(c, false)) || (rc = enqueue_keys(c)) || (rc = enqueue_sort(c)) ||
        (rc = enqueue_permute(c, true)))
        return rc;
    float best = 3.0e38f;
    int bi = -1;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 4; b++) {
            c->p.group_size = kGroups[a];
            c->p.leaf_cap = (uint32_t)kLeaves[b];
            float tmin = 3.0e38f;
            for (int r = 0; r < reps + 1; r++) {   // the first pass is a warm-up
                GE_CHECK(c, cudaEventRecord(c->ev[0], c->stream));
                if ((rc = enqueue_bbox(c, false)) || (rc = enqueue_build(c, true)) ||
                    (rc = enqueue_walk(c, false))) {
                    c->p = keep;
                    return rc;
                }
                GE_CHECK(c, cudaEventRecord(c->ev[1], c->stream));
                if ((rc = check_device(c))) {
                    c->p = keep;
                    return rc;
                }
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
                if (r > 0) tmin = std::min(tmin, ms);
            }
            out->ms[a * 4 + b] = tmin;
            out->tried++;
            if (tmin < best) { best = tmin; bi = a * 4 + b; }
        }
    c->p = keep;
    c->p.group_size = kGroups[bi / 4];
    c->p.leaf_cap = (uint32_t)kLeaves[bi % 4];
    out->group_size = c->p.group_size;
    out->leaf_cap = (int32_t)c->p.leaf_cap;
    // accelerations of the current positions under the chosen configuration
    if ((rc = enqueue_bbox(c, false)) || (rc = enqueue_build(c, true)) ||
        (rc = enqueue_walk(c, false)))
        return rc;
    rc = check_device(c);
    c->tree_valid = rc == GE_OK;
    return rc;
}

int ge_profile_step(ge_ctx *c) {
    int rc = require_state(c);
    if (rc) return rc;
    if ((rc = enqueue_frame(c, c->ev))) return rc;
    if ((rc = check_device(c))) return rc;
    for (int k = 0; k < 6; k++)
        cudaEventElapsedTime(&c->stats.stage_ms[k], c->ev[k], c->ev[k + 1]);
    cudaEventElapsedTime(&c->stats.stage_ms[6], c->ev[0], c->ev[6]);
    c->stats.steps += 1;
    c->total_steps += 1;
    c->tree_valid = true;
    return GE_OK;
}

int ge_frame_host(ge_ctx *c, int64_t n, float *x, float *y, float *z, float *vx, float *vy,
                  float *vz, float *ax, float *ay, float *az, float *m, uint32_t *id) {
    if (!c) return GE_ERR_ARG;
    const bool d3 = c->p.dims == 3;
    // the same one simulation as the last frame: copies overlap the step
    if (c->n == n && n > 0 && c->sims.size() == 1 && !c->pending_steps && id && x && y && vx &&
        vy && m && (!d3 || (z && vz)))
        return frame_overlapped(c, n, x, y, z, vx, vy, vz, ax, ay, az, m, id);
    int rc = ge_upload(c, n, x, y, z, vx, vy, vz, m, id, ax, ay, az);
    if (rc) return rc;
    if ((rc = ge_step(c, 1))) return rc;
    return ge_download(c, x, y, z, vx, vy, vz, ax, ay, az, m, id);
}

int ge_integrate_start(ge_ctx *c) {
    int rc = require_state(c);
    if (rc) return rc;
    if ((rc = enqueue_bbox(c, true))) return rc;
    c->tree_valid = false;
    c->keys_valid = false;
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int ge_bounding_box(ge_ctx *c, float *out) {
    int rc = require_state(c);
    if (rc) return rc;
    if ((rc = enqueue_bbox(c, false))) return rc;
    float4 bb;
    GE_CHECK(c, cudaMemcpyAsync(&bb, c->g.box, sizeof(bb), cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    float v[4] = {bb.x, bb.y, bb.z, bb.w};
    if (c->p.dims == 2) { v[2] = bb.w; v[3] = 0.0f; }
    std::memcpy(c->stats.bbox, v, sizeof(v));
    if (out) std::memcpy(out, v, sizeof(float) * (c->p.dims == 2 ? 3 : 4));
    return GE_OK;
}

int ge_compute_morton_keys(ge_ctx *c, uint64_t *keys_out) {
    int rc = require_state(c);
    if (rc) return rc;
    if ((rc = enqueue_bbox(c, false))) return rc;
    if ((rc = enqueue_keys(c))) return rc;
    c->keys_valid = true;
    if (keys_out) {
        uint64_t *tmp = nullptr;
        GE_CHECK(c, cudaMallocAsync((void **)&tmp, sizeof(uint64_t) * (size_t)c->n, c->stream));
        // keys of the current order: the packed words hold them above bit 28 in 2D
        GE_CHECK(c, launch_keys_out(c->p.dims, (int)c->n, c->b.ss, tmp, c->stream));
        GE_CHECK(c, cudaMemcpyAsync(keys_out, tmp, sizeof(uint64_t) * (size_t)c->n,
                                    cudaMemcpyDeviceToHost, c->stream));
        GE_CHECK(c, cudaFreeAsync(tmp, c->stream));
    }
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int ge_sort_by_morton_key(ge_ctx *c, uint32_t *perm_out) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!c->keys_valid) return fail(c, GE_ERR_STATE, "compute the Morton keys first");
    // the wait test's withheld tile applies to this stage call only (a whole
    // frame would go on to build on an unsorted order)
    c->b.ss.withhold_first = c->sort_withhold;
    rc = enqueue_sort(c);
    c->b.ss.withhold_first = 0u;
    if (rc) return rc;
    if ((rc = enqueue_permute(c, true))) return rc;
    c->keys_valid = false;
    c->tree_valid = false;
    if (perm_out) {
        uint32_t *tmp = nullptr;
        GE_CHECK(c, cudaMallocAsync((void **)&tmp, sizeof(uint32_t) * (size_t)c->n, c->stream));
        GE_CHECK(c, launch_perm_out(c->p.dims, (int)c->n, c->b.ss, tmp, c->stream));
        GE_CHECK(c, cudaMemcpyAsync(perm_out, tmp, sizeof(uint32_t) * (size_t)c->n,
                                    cudaMemcpyDeviceToHost, c->stream));
        GE_CHECK(c, cudaFreeAsync(tmp, c->stream));
    }
    return check_device(c);
}

int ge_build_tree(ge_ctx *c) {
    int rc = require_state(c);
    if (rc) return rc;
    if ((rc = enqueue_bbox(c, false))) return rc;   // seeds the root cells
    if ((rc = enqueue_build(c))) return rc;
    rc = check_device(c);
    c->tree_valid = rc == GE_OK;
    return rc;
}

int ge_compute_forces(ge_ctx *c) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!c->tree_valid) return fail(c, GE_ERR_STATE, "build the tree first");
    if ((rc = enqueue_walk(c, false))) return rc;
    rc = check_device(c);
    if (rc == GE_OK && c->count_inter) {
        unsigned long long v = 0;
        GE_CHECK(c, cudaMemcpy(&v, c->b.d_inter, sizeof(v), cudaMemcpyDeviceToHost));
        c->stats.interactions = v;
    }
    return rc;
}

int ge_integrate_end(ge_ctx *c) {
    int rc = require_state(c);
    if (rc) return rc;
    StepParams p = step_params(c);
    GE_CHECK(c, launch_integrate_end(c->p.dims, cur_state(c), p, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int ge_direct_sum_f64(ge_ctx *c, int64_t nt, const uint32_t *idx, double *ax, double *ay,
                      double *az) {
    int rc = require_state(c);
    if (rc) return rc;
    if (nt < 0 || (nt > 0 && (!idx || !ax || !ay))) return fail(c, GE_ERR_ARG, "bad sample");
    if (nt == 0) return GE_OK;
    for (int64_t k = 0; k < nt; k++)
        if ((int64_t)idx[k] >= c->n) return fail(c, GE_ERR_ARG, "sample index out of range");
    const int D = c->p.dims;
    // targets in ascending slot order, so each block's targets share a segment
    std::vector<int64_t> ord((size_t)nt);
    for (int64_t k = 0; k < nt; k++) ord[(size_t)k] = k;
    std::stable_sort(ord.begin(), ord.end(),
                     [&](int64_t a, int64_t b) { return idx[a] < idx[b]; });
    std::vector<uint32_t> sidx((size_t)nt);
    for (int64_t k = 0; k < nt; k++) sidx[(size_t)k] = idx[ord[(size_t)k]];
    uint32_t *d_idx = nullptr;
    double *d_out = nullptr;
    GE_CHECK(c, cudaMallocAsync((void **)&d_idx, sizeof(uint32_t) * nt, c->stream));
    GE_CHECK(c, cudaMallocAsync((void **)&d_out, sizeof(double) * nt * D, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(d_idx, sidx.data(), sizeof(uint32_t) * nt, cudaMemcpyHostToDevice,
                                c->stream));
    GE_CHECK(c, launch_direct_f64(D, cur_state(c), (int)c->n, c->g, d_idx, (int)nt,
                                  (double)c->p.G, (double)c->p.eps2, d_out, c->stream));
    std::vector<double> h((size_t)(nt * D));
    GE_CHECK(c, cudaMemcpyAsync(h.data(), d_out, sizeof(double) * nt * D, cudaMemcpyDeviceToHost,
                                c->stream));
    GE_CHECK(c, cudaFreeAsync(d_idx, c->stream));
    GE_CHECK(c, cudaFreeAsync(d_out, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    for (int64_t r = 0; r < nt; r++) {
        const int64_t k = ord[(size_t)r];
        ax[k] = h[(size_t)(r * D)];
        ay[k] = h[(size_t)(r * D + 1)];
        if (D == 3 && az) az[k] = h[(size_t)(r * D + 2)];
    }
    return GE_OK;
}

int ge_predict_trajectory(ge_ctx *c, int32_t sim, int32_t nprobes, const float *pos,
                          const float *vel, const float *mass, float eps2, int32_t steps,
                          float *path) {
    int rc = require_state(c);
    if (rc) return rc;
    if (nprobes < 0 || steps < 0 || (nprobes > 0 && (!pos || !vel || !mass || !path)))
        return fail(c, GE_ERR_ARG, "bad probes");
    if (nprobes == 0 || steps == 0) return GE_OK;
    if (c->p.precision == GE_PREC_MIXED)
        return fail(c, GE_ERR_UNSUPPORTED, "trajectory preview needs GE_PREC_EXACT or GE_PREC_FAST");
    if (!c->tree_valid) return fail(c, GE_ERR_STATE, "no tree: step or build first");
    int r = 0;
    if (sim != 0 && (r = find_sim(c, sim)) < 0) return fail(c, GE_ERR_ARG, "no such simulation");
    const int D = c->p.dims;
    uint32_t be[2];
    GE_CHECK(c, cudaMemcpyAsync(&be[0], c->g.root_begin + r, sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(&be[1], c->g.root_end + r, sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, c->stream));
    float *d = nullptr;
    const size_t np = (size_t)nprobes, pn = np * (size_t)steps * D;
    GE_CHECK(c, cudaMallocAsync((void **)&d, sizeof(float) * (np * (2 * D + 1) + pn), c->stream));
    float *dpos = d, *dvel = d + np * D, *dm = d + 2 * np * D, *dpath = d + np * (2 * D + 1);
    GE_CHECK(c, cudaMemcpyAsync(dpos, pos, sizeof(float) * np * D, cudaMemcpyHostToDevice, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(dvel, vel, sizeof(float) * np * D, cudaMemcpyHostToDevice, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(dm, mass, sizeof(float) * np, cudaMemcpyHostToDevice, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    StepParams p = step_params(c);
    GE_CHECK(c, launch_predict(D, c->b.tree, p, c->g.box + r, be[0], be[1], eps2, nprobes, dpos,
                               dvel, dm, steps, dpath, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(path, dpath, sizeof(float) * pn, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaFreeAsync(d, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

void ge_field_params_default(ge_field_params *fp) {
    if (!fp) return;
    std::memset(fp, 0, sizeof(*fp));
    fp->res = 150;            // field.h:20
    fp->softness = 0.85f;     // field.h:30
    fp->threshold = 1000.0f;  // field.h:26
    fp->stretch = 90.0f;      // field.h:433
    fp->exposure = 3.0f;      // field.h:437
    // colorVisuals.pColor {0, 40, 68} and sColor {155, 80, 40} (particleColorVisuals.h:25-26)
    const float lo[3] = {0.0f, 40.0f, 68.0f}, hi[3] = {155.0f, 80.0f, 40.0f};
    for (int a = 0; a < 3; a++) {
        fp->color_low[a] = lo[a] / 255.0f;
        fp->color_high[a] = hi[a] / 255.0f;
    }
}

int ge_gravity_field(ge_ctx *c, int32_t sim, const ge_field_params *fp, int64_t cap,
                     float *strength, uint8_t *rgba, int32_t *amount_x, int32_t *amount_y) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!fp || fp->res < 1 || !(fp->threshold > 0.0f)) return fail(c, GE_ERR_ARG, "bad field parameters");
    if (c->p.dims != 2) return fail(c, GE_ERR_UNSUPPORTED, "the field view is 2D");
    if (!(c->p.domain[0] > 0.0f) || !(c->p.domain[1] > 0.0f))
        return fail(c, GE_ERR_ARG, "the field view needs a positive domain");
    int r = 0;
    if (sim != 0 && (r = find_sim(c, sim)) < 0) return fail(c, GE_ERR_ARG, "no such simulation");
    // Field::initializeCells (field.h:59-80)
    const float dx = c->p.domain[0], dy = c->p.domain[1];
    const float cell = (dx >= dy ? dy : dx) / (float)fp->res;
    const int ax = (int)(dx / cell), ay = (int)(dy / cell);
    if (amount_x) *amount_x = ax;
    if (amount_y) *amount_y = ay;
    const int64_t cells = (int64_t)ax * ay;
    if (cells > cap) return fail(c, GE_ERR_CAPACITY, "field arrays smaller than the cell count");
    if (cells < 1) return GE_OK;
    float *d = nullptr;
    GE_CHECK(c, cudaMallocAsync((void **)&d, sizeof(float) * 2 * (size_t)cells, c->stream));
    float *ds = d;
    uint32_t *dc = reinterpret_cast<uint32_t *>(d + cells);
    const uint32_t lo = c->h_off[(size_t)r], hi = c->h_off[(size_t)r + 1];
    GE_CHECK(c, launch_field(cur_state(c), lo, hi, ax, ay, cell, c->p.G, fp->softness * fp->softness,
                             c->p.periodic, dx, dy, *fp, ds, rgba ? dc : nullptr, c->stream));
    if (strength)
        GE_CHECK(c, cudaMemcpyAsync(strength, ds, sizeof(float) * (size_t)cells,
                                    cudaMemcpyDeviceToHost, c->stream));
    if (rgba)
        GE_CHECK(c, cudaMemcpyAsync(rgba, dc, 4 * (size_t)cells, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaFreeAsync(d, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int ge_sph_grid(ge_ctx *c, int32_t sim, float cell_size, uint32_t table_size, int64_t cap,
                uint32_t *keys, uint32_t *index, int32_t *cell_x, int32_t *cell_y,
                uint32_t *offsets) {
    int rc = require_state(c);
    if (rc) return rc;
    if (c->p.dims != 2) return fail(c, GE_ERR_UNSUPPORTED, "the SPH grid is 2D");
    if (!(cell_size > 0.0f && cell_size < INFINITY))
        return fail(c, GE_ERR_ARG, "cell_size must be positive and finite");
    if (table_size < 1u || table_size > (1u << 24))
        return fail(c, GE_ERR_ARG, "table_size must be in [1, 2^24]");
    if (!keys || !index || !cell_x || !cell_y || !offsets)
        return fail(c, GE_ERR_ARG, "every output array is required");
    int r = 0;
    if (sim != 0 && (r = find_sim(c, sim)) < 0) return fail(c, GE_ERR_ARG, "no such simulation");
    const uint32_t lo = c->h_off[(size_t)r], hi = c->h_off[(size_t)r + 1];
    const int64_t n = (int64_t)hi - lo;
    if (n > cap) return fail(c, GE_ERR_CAPACITY, "output arrays smaller than the simulation");
    if (n >= (int64_t(1) << 28)) return fail(c, GE_ERR_CAPACITY, "more than 2^28 particles");
    if (n < 1) return GE_OK;
    const size_t words = 4 * (size_t)n + table_size;
    uint32_t *d = nullptr;
    GE_CHECK(c, cudaMallocAsync((void **)&d, sizeof(uint32_t) * words, c->stream));
    uint32_t *dk = d, *di = d + n, *dofs = d + 4 * n;
    int32_t *dx = reinterpret_cast<int32_t *>(d + 2 * n), *dy = reinterpret_cast<int32_t *>(d + 3 * n);
    c->keys_valid = false;   // the Morton sort scratch is reused
    GE_CHECK(c, launch_sph_grid(cur_state(c), lo, (int)n, cell_size, table_size, c->b.ss, c->d_err,
                                dk, di, dx, dy, dofs, c->num_sms, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(keys, dk, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(index, di, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(cell_x, dx, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(cell_y, dy, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(offsets, dofs, 4 * (size_t)table_size, cudaMemcpyDeviceToHost,
                                c->stream));
    GE_CHECK(c, cudaFreeAsync(d, c->stream));
    return check_device(c);
}

int ge_build_timeline(ge_ctx *c, int32_t cap, uint64_t *ns, int32_t *count) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!count || (cap > 0 && !ns)) return fail(c, GE_ERR_ARG, "bad timeline buffers");
    uint32_t m[8];
    GE_CHECK(c, cudaMemcpyAsync(m, c->b.tree.meta, sizeof(m), cudaMemcpyDeviceToHost, c->stream));
    unsigned long long tl[kTimeline];
    GE_CHECK(c, cudaMemcpyAsync(tl, c->b.tree.tl, sizeof(tl), cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    const int32_t k = (int32_t)(m[7] < (uint32_t)kTimeline ? m[7] : kTimeline);
    *count = k;
    for (int32_t i = 0; i < k && i < cap; i++) ns[i] = (uint64_t)(tl[i] - tl[0]);
    return GE_OK;
}

int ge_energy_f64(ge_ctx *c, double *out) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!out) return fail(c, GE_ERR_ARG, "out is NULL");
    if (!group_walk_on(c))
        return fail(c, GE_ERR_UNSUPPORTED, "the energy pass needs the mixed mode's group walk");
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    if (!c->tree_valid) {
        if ((rc = enqueue_bbox(c, false)) || (rc = enqueue_keys(c)) || (rc = enqueue_sort(c)) ||
            (rc = enqueue_permute(c, true)) || (rc = enqueue_bbox(c, false)) ||
            (rc = enqueue_build(c, true)))
            return rc;
        if ((rc = check_device(c))) return rc;
        c->tree_valid = true;
    }
    double *d = nullptr;
    GE_CHECK(c, cudaMallocAsync((void **)&d, sizeof(double) * 6, c->stream));
    StepParams p = step_params(c);
    GE_CHECK(c, launch_group_potential(c->p.dims, cur_state(c), p, c->g, mixed_view(c),
                                       c->b.tree.meta + 10, c->d_err, d, c->stream));
    GE_CHECK(c, launch_sums_f64(c->p.dims, cur_state(c), (int)c->n, d + 1, c->stream));
    double h[6];
    GE_CHECK(c, cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaFreeAsync(d, c->stream));
    if ((rc = check_device(c))) return rc;
    out[0] = h[1];
    out[1] = -0.5 * (double)c->p.G * h[0];
    out[2] = out[0] + out[1];
    return GE_OK;
}

int ge_sums_f64(ge_ctx *c, double *out) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!out) return fail(c, GE_ERR_ARG, "out is NULL");
    double *d = nullptr;
    GE_CHECK(c, cudaMallocAsync((void **)&d, sizeof(double) * 5, c->stream));
    GE_CHECK(c, launch_sums_f64(c->p.dims, cur_state(c), (int)c->n, d, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(out, d, sizeof(double) * 5, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaFreeAsync(d, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

// --- capacity and memory ------------------------------------------------

int ge_reserve(ge_ctx *c, int64_t n, int64_t sims) {
    if (!c) return GE_ERR_ARG;
    if (n < 1 || sims < 1) return fail(c, GE_ERR_ARG, "n and sims must be >= 1");
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    c->sims_reserved = std::max<int64_t>(c->sims_reserved, sims);
    int rc = ensure_capacity(c, std::max<int64_t>(n, c->n), std::max<int64_t>(sims, (int64_t)c->sims.size()),
                             true, true);
    if (rc) return rc;
    if ((rc = ensure_mode(c))) return rc;
    return sync_segments(c);
}

int ge_memory_bytes(ge_ctx *c, int64_t *bytes) {
    if (!c || !bytes) return GE_ERR_ARG;
    *bytes = (int64_t)(c->b.allocs.bytes + c->sb.allocs.bytes);
    return GE_OK;
}

int ge_estimate_bytes(const ge_params *p, int64_t n, int64_t sims, int64_t *bytes) {
    if (!bytes) return GE_ERR_ARG;
    ge_ctx tmp;
    int rc = validate(&tmp, p);
    if (rc) return rc;
    if (n < 1 || sims < 1) return GE_ERR_ARG;
    tmp.p = *p;
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return GE_ERR_NO_DEVICE;
    tmp.num_sms = prop.multiProcessorCount;
    const int64_t slack = build_node_slack(p->dims, tmp.num_sms);
    if (slack <= 0) return GE_ERR_CUDA;
    Buffers nb;
    nb.allocs.dry = true;
    rc = alloc_buffers(&tmp, nb, n, node_cap_for(&tmp, n, sims, slack), p->track_prev_vel != 0,
                       false);
    if (!rc && p->precision == GE_PREC_MIXED) rc = alloc_mixed(&tmp, nb);
    SegBuffers sb;
    sb.allocs.dry = true;
    if (!rc) rc = alloc_segs(&tmp, sb, sims, n, n / kSortTile + sims + 1);
    if (rc) return rc;
    *bytes = (int64_t)(nb.allocs.bytes + sb.allocs.bytes);
    return GE_OK;
}

// --- batched simulations ------------------------------------------------

int ge_batch_add_sim(ge_ctx *c, int64_t n, const float *x, const float *y, const float *z,
                     const float *vx, const float *vy, const float *vz, const float *m,
                     const uint32_t *id, int32_t *sim) {
    if (!c) return GE_ERR_ARG;
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    int rc = check_host_arrays(c, n, x, y, z, vx, vy, vz, m);
    if (rc) return rc;
    if (c->next_handle == INT32_MAX) return fail(c, GE_ERR_CAPACITY, "simulation handles exhausted");
    const int64_t old_n = c->n;
    if ((rc = ensure_capacity(c, old_n + n, (int64_t)c->sims.size() + 1, true))) return rc;
    if ((rc = put_host(c, old_n, n, x, y, z, vx, vy, vz, m, id, nullptr, nullptr, nullptr)))
        return rc;
    const int32_t h = c->next_handle++;
    c->sims.push_back(SimRec{h, n, c->total_steps});
    c->n = old_n + n;
    if ((rc = sync_segments(c))) {
        c->sims.pop_back();
        c->n = old_n;
        sync_segments(c);
        return rc;
    }
    if (sim) *sim = h;
    return GE_OK;
}

int ge_batch_remove_sims(ge_ctx *c, int32_t count, const int32_t *sims) {
    if (!c || count < 0 || (count && !sims)) return GE_ERR_ARG;
    if (c->pending_steps) return fail(c, GE_ERR_STATE, "ge_step_wait first");
    std::vector<char> drop(c->sims.size(), 0);
    for (int32_t k = 0; k < count; k++) {
        const int r = find_sim(c, sims[k]);
        if (r < 0) return fail(c, GE_ERR_ARG, "no such simulation");
        drop[(size_t)r] = 1;
    }
    size_t first_drop = 0;
    while (first_drop < drop.size() && !drop[first_drop]) first_drop++;
    bool suffix = true;
    for (size_t r = first_drop; r < drop.size(); r++) suffix = suffix && drop[r];
    if (suffix) {   // only the last simulations go: nothing moves
        c->n = c->h_off[first_drop];
        c->sims.resize(first_drop);
        return sync_segments(c);
    }
    // the kept simulations move down, in order, through the other state
    // buffer (no copy overlaps itself); runs of kept simulations move as one
    const State &src = c->b.st[c->cur];
    const State &dst = c->b.st[c->cur ^ 1];
    std::vector<SimRec> kept;
    int64_t out = 0;
    size_t r = 0;
    bool moved = false;
    while (r < c->sims.size()) {
        if (drop[r]) { r++; moved = true; continue; }
        const size_t r0 = r;
        while (r < c->sims.size() && !drop[r]) kept.push_back(c->sims[r++]);
        const int64_t lo = c->h_off[r0], hi = c->h_off[r];
        int rc = copy_range(c, dst, out, src, lo, hi - lo, c->b.prev, c->b.pinned);
        if (rc) return rc;
        out += hi - lo;
    }
    if (moved) c->cur ^= 1;
    c->sims.swap(kept);
    c->n = out;
    return sync_segments(c);
}

int ge_batch_remove_sim(ge_ctx *c, int32_t sim) { return ge_batch_remove_sims(c, 1, &sim); }

int ge_batch_list(ge_ctx *c, int32_t cap, int32_t *sims, int32_t *count) {
    if (!c || !count) return GE_ERR_ARG;
    *count = (int32_t)c->sims.size();
    if (sims)
        for (int32_t k = 0; k < cap && k < *count; k++) sims[k] = c->sims[(size_t)k].handle;
    return GE_OK;
}

int ge_batch_query(ge_ctx *c, int32_t sim, int64_t *n, int64_t *offset, int64_t *steps) {
    if (!c) return GE_ERR_ARG;
    const int r = find_sim(c, sim);
    if (r < 0) return fail(c, GE_ERR_ARG, "no such simulation");
    if (n) *n = c->sims[(size_t)r].n;
    if (offset) *offset = c->h_off[(size_t)r];
    if (steps) *steps = c->total_steps - c->sims[(size_t)r].step0;
    return GE_OK;
}

int ge_batch_download_sim(ge_ctx *c, int32_t sim, float *x, float *y, float *z, float *vx,
                          float *vy, float *vz, float *ax, float *ay, float *az, float *m,
                          uint32_t *id) {
    if (!c) return GE_ERR_ARG;
    const int r = find_sim(c, sim);
    if (r < 0) return fail(c, GE_ERR_ARG, "no such simulation");
    return get_host(c, c->h_off[(size_t)r], c->sims[(size_t)r].n, x, y, z, vx, vy, vz, ax, ay, az,
                    m, id);
}

int ge_export_tree(ge_ctx *c, int64_t cap, int64_t *count, float *pos, float *size, float *com,
                   float *mass, uint32_t *start, uint32_t *end, uint32_t *next,
                   uint32_t *child) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!c->tree_valid) return fail(c, GE_ERR_STATE, "no valid tree");
    if ((rc = check_device(c))) return rc;
    const int D = c->p.dims, Q = 1 << D;
    const int64_t nn = c->stats.nodes;
    if (count) *count = nn;
    if (nn > cap) return fail(c, GE_ERR_CAPACITY, "export capacity smaller than the node count");
    // nodes sit in the first `slots` entries, with unused (hole) slots among them
    const int64_t ns = c->slots > nn ? c->slots : nn;
    std::vector<float4> w((size_t)ns), cell((size_t)ns);
    std::vector<uint4> inf((size_t)ns);
    const Tree &t = c->b.tree;
    GE_CHECK(c, cudaMemcpy(w.data(), t.walk, sizeof(float4) * ns, cudaMemcpyDeviceToHost));
    GE_CHECK(c, cudaMemcpy(cell.data(), t.cell, sizeof(float4) * ns, cudaMemcpyDeviceToHost));
    GE_CHECK(c, cudaMemcpy(inf.data(), t.info, sizeof(uint4) * ns, cudaMemcpyDeviceToHost));
    // depth-first pre-order numbering, children in slot order (the reference's
    // emission order, quadtree.cpp:67-87), the simulations' roots (slots
    // 0..S-1) one after another; next = number of descendants
    std::vector<uint32_t> order;
    order.reserve((size_t)nn);
    std::vector<uint32_t> stack;
    for (int r = c->g.S - 1; r >= 0; --r) stack.push_back((uint32_t)r);
    std::vector<uint32_t> newid((size_t)ns, kEmpty);
    while (!stack.empty()) {
        uint32_t k = stack.back();
        stack.pop_back();
        if ((int64_t)order.size() >= nn || k >= (uint32_t)ns)
            return fail(c, GE_ERR_STATE, "tree is not consistent");
        newid[k] = (uint32_t)order.size();
        order.push_back(k);
        const uint32_t mask = inf[k].y;
        const int nc = __builtin_popcount(mask);
        for (int cidx = nc - 1; cidx >= 0; --cidx) stack.push_back(inf[k].x + (uint32_t)cidx);
    }
    if ((int64_t)order.size() != nn) return fail(c, GE_ERR_STATE, "tree is not connected");
    std::vector<uint32_t> desc((size_t)ns, 0);
    for (int64_t r = nn - 1; r >= 0; --r) {
        const uint32_t k = order[(size_t)r];
        const uint32_t mask = inf[k].y;
        uint32_t s = 0;
        const int nc = __builtin_popcount(mask);
        for (int cidx = 0; cidx < nc; cidx++) s += 1 + desc[inf[k].x + (uint32_t)cidx];
        desc[k] = s;
    }
    for (int64_t r = 0; r < nn; r++) {
        const uint32_t k = order[(size_t)r];
        const float4 cw = w[k], cc = cell[k];
        const uint4 ci = inf[k];
        if (pos) { pos[r * D] = cc.x; pos[r * D + 1] = cc.y; if (D == 3) pos[r * D + 2] = cc.z; }
        if (size) size[r] = cc.w;
        if (com) { com[r * D] = cw.x; com[r * D + 1] = cw.y; if (D == 3) com[r * D + 2] = cw.z; }
        if (mass) mass[r] = D == 2 ? cw.z : cw.w;
        if (start) start[r] = ci.z;
        if (end) end[r] = ci.w;
        if (next) next[r] = desc[k];
        if (child) {
            int cidx = 0;
            for (int q = 0; q < Q; q++) {
                if ((ci.y >> q) & 1u) child[r * Q + q] = newid[ci.x + (uint32_t)(cidx++)];
                else child[r * Q + q] = kEmpty;
            }
        }
    }
    return GE_OK;
}

}  // extern "C"
