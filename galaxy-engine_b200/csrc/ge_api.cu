// ge_api.cu -- host side of the C ABI (include/ge_bh.h): context, resident
// device state, the per-frame pipeline and the stage calls.
//
// One frame (GalaxyEngine/src/globalLogic.cpp:1155-1370 in 2D, :1584-1719 in 3D):
//   1. kick + drift fused with the bounding box          (integrateStart, boundingBox)
//   2. Morton keys + digit histograms                      (computeMortonKeys)
//   3. stable radix sort passes                            (sortParticlesByMortonKey)
//   4. gather of the state into Morton order
//   5. tree build with mass / centre of mass               (Quadtree / Octree)
//   6. tree walk with the second half kick fused           (calculateForceFromGrid, integrateEnd)
// All of it is enqueued on the context's stream; nothing returns to the host
// between stages.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ge_bh.h"
#include "ge_device.cuh"
#include "ge_internal.h"

using namespace ge;

struct ge_ctx {
    ge_params p{};
    int dev = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    int64_t n = 0, cap_n = 0;
    State st[2]{};
    int cur = 0;
    bool has_pinned = false;
    bool has_prev = false;
    SortScratch ss{};
    Tree tree{};
    uint32_t *d_err = nullptr;
    unsigned long long *d_inter = nullptr;
    uint32_t *h_meta = nullptr;   // pinned copy of the tree meta words
    int64_t slots = 0;            // node slots of the last build (holes included)
    bool count_inter = false;
    bool tree_valid = false;
    bool keys_valid = false;
    cudaEvent_t ev[8]{};
    ge_stats stats{};
    std::string err;
    std::vector<void *> allocs;
};

namespace {

int fail(ge_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(ge_ctx *c, cudaError_t e, const char *where) {
    return fail(c, GE_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define GE_CHECK(ctx, call)                                      \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
    } while (0)

template <typename T>
cudaError_t dalloc(ge_ctx *c, T **p, size_t count) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * (count ? count : 1));
    if (e != cudaSuccess) return e;
    c->allocs.push_back(q);
    *p = (T *)q;
    return cudaSuccess;
}

void free_buffers(ge_ctx *c) {
    for (void *q : c->allocs) cudaFree(q);
    c->allocs.clear();
    c->st[0] = State{};
    c->st[1] = State{};
    c->ss = SortScratch{};
    c->tree = Tree{};
    c->d_err = nullptr;
    c->d_inter = nullptr;
    c->cap_n = 0;
    c->has_pinned = false;
    c->has_prev = false;
}

StepParams step_params(const ge_ctx *c) {
    StepParams s{};
    s.n = (int)c->n;
    s.dt = c->p.dt;
    s.half_dt = c->p.dt * 0.5f;
    s.G = c->p.G;
    s.theta2 = c->p.theta * c->p.theta;
    s.eps2 = c->p.eps2;
    s.leaf_cap = c->p.leaf_cap;
    s.size_gate = c->p.size_gate;
    s.min_size = c->p.min_size;
    s.periodic = c->p.periodic ? 1 : 0;
    for (int a = 0; a < 3; a++) {
        s.domain[a] = c->p.domain[a];
        s.half_domain[a] = c->p.domain[a] * 0.5f;
    }
    return s;
}

int validate(ge_ctx *c, const ge_params *p) {
    if (!p) return fail(c, GE_ERR_ARG, "params is NULL");
    if (p->dims != 2 && p->dims != 3) return fail(c, GE_ERR_ARG, "dims must be 2 or 3");
    if (p->precision != GE_PREC_FAST && p->precision != GE_PREC_EXACT)
        return fail(c, GE_ERR_UNSUPPORTED, "precision mode not supported by this build");
    if (!(p->theta >= 0.0f)) return fail(c, GE_ERR_ARG, "theta must be >= 0");
    if (!(p->eps2 >= 0.0f)) return fail(c, GE_ERR_ARG, "eps2 must be >= 0");
    if (p->leaf_cap < 1) return fail(c, GE_ERR_ARG, "leaf_cap must be >= 1");
    if (!(p->node_cap_factor >= 1.0f)) return fail(c, GE_ERR_ARG, "node_cap_factor must be >= 1");
    if (p->periodic && (!(p->domain[0] > 0) || !(p->domain[1] > 0) ||
                        (p->dims == 3 && !(p->domain[2] > 0))))
        return fail(c, GE_ERR_ARG, "periodic wrap needs a positive domain");
    return GE_OK;
}

// (Re)allocate every device buffer for n particles.
int ensure_capacity(ge_ctx *c, int64_t n) {
    const int D = c->p.dims;
    const int64_t slack = build_node_slack(D, c->num_sms);
    if (slack <= 0) return fail(c, GE_ERR_CUDA, "tree build kernel cannot be made resident");
    const int64_t node_cap = (int64_t)(c->p.node_cap_factor * (double)n) + 1024 + slack;
    if (n <= c->cap_n && node_cap <= c->tree.cap && c->has_prev == (bool)c->p.track_prev_vel)
        return GE_OK;
    if (D == 2 && n >= (1ll << 28)) return fail(c, GE_ERR_ARG, "2D supports N < 2^28");
    if (node_cap >= (1ll << 32) - 1) return fail(c, GE_ERR_ARG, "node capacity exceeds 2^32");
    free_buffers(c);
    const size_t N = (size_t)n;
    for (int b = 0; b < 2; b++) {
        State &s = c->st[b];
        GE_CHECK(c, dalloc(c, &s.x, N)); GE_CHECK(c, dalloc(c, &s.y, N));
        GE_CHECK(c, dalloc(c, &s.vx, N)); GE_CHECK(c, dalloc(c, &s.vy, N));
        GE_CHECK(c, dalloc(c, &s.ax, N)); GE_CHECK(c, dalloc(c, &s.ay, N));
        if (D == 3) {
            GE_CHECK(c, dalloc(c, &s.z, N)); GE_CHECK(c, dalloc(c, &s.vz, N));
            GE_CHECK(c, dalloc(c, &s.az, N));
        }
        GE_CHECK(c, dalloc(c, &s.m, N));
        GE_CHECK(c, dalloc(c, &s.id, N));
        if (c->p.track_prev_vel) {
            GE_CHECK(c, dalloc(c, &s.pvx, N)); GE_CHECK(c, dalloc(c, &s.pvy, N));
            if (D == 3) GE_CHECK(c, dalloc(c, &s.pvz, N));
        }
    }
    c->has_prev = c->p.track_prev_vel != 0;
    SortScratch &ss = c->ss;
    GE_CHECK(c, dalloc(c, &ss.keys[0], N)); GE_CHECK(c, dalloc(c, &ss.keys[1], N));
    if (D == 3) { GE_CHECK(c, dalloc(c, &ss.vals[0], N)); GE_CHECK(c, dalloc(c, &ss.vals[1], N)); }
    ss.tiles = (n + kSortTile - 1) / kSortTile;
    GE_CHECK(c, dalloc(c, &ss.hist, 8 * 256));
    GE_CHECK(c, dalloc(c, &ss.status, (size_t)8 * ss.tiles * 256));
    GE_CHECK(c, dalloc(c, &ss.tile_ctr, 8));
    int bb = (int)((n + kBBoxThreads - 1) / kBBoxThreads);
    if (bb > c->num_sms * 4) bb = c->num_sms * 4;
    if (bb < 1) bb = 1;
    ss.bbox_blocks = bb;
    GE_CHECK(c, dalloc(c, &ss.bbox_part, 2 * (size_t)bb));
    GE_CHECK(c, dalloc(c, &ss.bbox_ctr, 1));
    GE_CHECK(c, dalloc(c, &ss.bbox, 1));
    GE_CHECK(c, cudaMemset(ss.bbox_ctr, 0, sizeof(uint32_t)));
    Tree &t = c->tree;
    t.cap = node_cap;
    GE_CHECK(c, dalloc(c, &t.walk, (size_t)node_cap));
    if (D == 3) GE_CHECK(c, dalloc(c, &t.size2, (size_t)node_cap));
    GE_CHECK(c, dalloc(c, &t.info, (size_t)node_cap));
    GE_CHECK(c, dalloc(c, &t.cell, (size_t)node_cap));
    GE_CHECK(c, dalloc(c, &t.aux, (size_t)node_cap));
    GE_CHECK(c, dalloc(c, &t.pend, (size_t)node_cap));
    GE_CHECK(c, dalloc(c, &t.small, N / 2 + 1));
    GE_CHECK(c, dalloc(c, &t.endcnt, N + 1));
    const int bblocks = build_grid_blocks(D, c->num_sms);
    if (bblocks < 1) return fail(c, GE_ERR_CUDA, "tree build kernel cannot be made resident");
    GE_CHECK(c, dalloc(c, &t.blocksum, (size_t)bblocks));
    GE_CHECK(c, dalloc(c, &t.src, N + (size_t)node_cap + 1));
    if (D == 2) {
        uint32_t *l = nullptr;
        GE_CHECK(c, dalloc(c, &l, N + (size_t)node_cap + 1));
        t.link = l;
    } else {
        uint2 *l = nullptr;
        GE_CHECK(c, dalloc(c, &l, N + (size_t)node_cap + 1));
        t.link = l;
    }
    GE_CHECK(c, dalloc(c, &t.slot_of, N));
    GE_CHECK(c, dalloc(c, &t.level, kMaxLevels + 2));
    GE_CHECK(c, dalloc(c, &t.lvl_alloc, kMaxLevels + 2));
    GE_CHECK(c, dalloc(c, &t.meta, 16));
    GE_CHECK(c, dalloc(c, &t.tl, kTimeline));
    GE_CHECK(c, cudaMemset(t.meta, 0, 16 * sizeof(uint32_t)));
    c->d_err = t.meta + 4;
    GE_CHECK(c, dalloc(c, &c->d_inter, 1));
    c->cap_n = n;
    c->tree_valid = false;
    c->keys_valid = false;
    return GE_OK;
}

// Reads back the error word and tree size; clears the error word.
int check_device(ge_ctx *c) {
    GE_CHECK(c, cudaMemcpyAsync(c->h_meta, c->tree.meta, 10 * sizeof(uint32_t),
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

State cur_state(ge_ctx *c) {
    State s = c->st[c->cur];
    if (!c->has_pinned) s.pinned = nullptr;
    return s;
}

int enqueue_bbox(ge_ctx *c, bool kick) {
    StepParams p = step_params(c);
    State s = cur_state(c);
    GE_CHECK(c, launch_kick_drift_bbox(c->p.dims, s, p, kick, c->ss, c->tree, c->d_err, c->stream));
    return GE_OK;
}

int enqueue_keys(ge_ctx *c) {
    GE_CHECK(c, launch_keys(c->p.dims, cur_state(c), (int)c->n, c->ss, c->stream));
    return GE_OK;
}

int enqueue_sort_permute(ge_ctx *c, bool with_acc) {
    GE_CHECK(c, launch_sort(c->p.dims, (int)c->n, c->ss, c->d_err, c->stream));
    State in = cur_state(c);
    State out = c->st[c->cur ^ 1];
    if (!c->has_pinned) out.pinned = nullptr;
    GE_CHECK(c, launch_permute(c->p.dims, (int)c->n, c->ss, in, out, with_acc, c->stream));
    c->cur ^= 1;
    return GE_OK;
}

int enqueue_build(ge_ctx *c) {
    StepParams p = step_params(c);
    GE_CHECK(c, launch_build(c->p.dims, cur_state(c), p, c->tree, c->d_err, c->num_sms, c->stream));
    return GE_OK;
}

int enqueue_walk(ge_ctx *c, bool integrate_end) {
    StepParams p = step_params(c);
    unsigned long long *cnt = nullptr;
    if (c->count_inter) {
        GE_CHECK(c, cudaMemsetAsync(c->d_inter, 0, sizeof(unsigned long long), c->stream));
        cnt = c->d_inter;
    }
    GE_CHECK(c, launch_walk(c->p.dims, c->p.precision, cur_state(c), p, c->tree, integrate_end,
                            cnt, c->d_err, c->stream));
    return GE_OK;
}

int enqueue_frame(ge_ctx *c, cudaEvent_t *ev) {
    int rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[0], c->stream));
    if ((rc = enqueue_bbox(c, true))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[1], c->stream));
    if ((rc = enqueue_keys(c))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[2], c->stream));
    GE_CHECK(c, launch_sort(c->p.dims, (int)c->n, c->ss, c->d_err, c->stream));
    if (ev) GE_CHECK(c, cudaEventRecord(ev[3], c->stream));
    {
        State in = cur_state(c);
        State out = c->st[c->cur ^ 1];
        if (!c->has_pinned) out.pinned = nullptr;
        GE_CHECK(c, launch_permute(c->p.dims, (int)c->n, c->ss, in, out, false, c->stream));
        c->cur ^= 1;
    }
    if (ev) GE_CHECK(c, cudaEventRecord(ev[4], c->stream));
    if ((rc = enqueue_build(c))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[5], c->stream));
    if ((rc = enqueue_walk(c, true))) return rc;
    if (ev) GE_CHECK(c, cudaEventRecord(ev[6], c->stream));
    return GE_OK;
}

int require_state(ge_ctx *c) {
    if (!c) return GE_ERR_ARG;
    if (c->n <= 0) return fail(c, GE_ERR_STATE, "no particles uploaded");
    return GE_OK;
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

int ge_destroy(ge_ctx *c) {
    if (!c) return GE_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_buffers(c);
    for (auto &e : c->ev) if (e) cudaEventDestroy(e);
    if (c->h_meta) cudaFreeHost(c->h_meta);
    if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return GE_OK;
}

const char *ge_last_error(const ge_ctx *c) { return c ? c->err.c_str() : "null context"; }

int ge_set_params(ge_ctx *c, const ge_params *p) {
    if (!c) return GE_ERR_ARG;
    int rc = validate(c, p);
    if (rc) return rc;
    if (p->dims != c->p.dims && c->cap_n) {
        GE_CHECK(c, cudaStreamSynchronize(c->stream));
        free_buffers(c);
        c->n = 0;
    }
    const bool realloc = c->cap_n && (p->node_cap_factor != c->p.node_cap_factor ||
                                      (p->track_prev_vel != 0) != c->has_prev);
    if (realloc) return fail(c, GE_ERR_STATE, "node_cap_factor / track_prev_vel change needs a new upload");
    c->p = *p;
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

int ge_set_count_interactions(ge_ctx *c, int32_t enable) {
    if (!c) return GE_ERR_ARG;
    c->count_inter = enable != 0;
    return GE_OK;
}

int ge_upload(ge_ctx *c, int64_t n, const float *x, const float *y, const float *z,
              const float *vx, const float *vy, const float *vz, const float *m,
              const uint32_t *id, const float *ax, const float *ay, const float *az) {
    if (!c) return GE_ERR_ARG;
    const int D = c->p.dims;
    if (n < 1) return fail(c, GE_ERR_ARG, "n must be >= 1");
    if (!x || !y || !vx || !vy || !m || (D == 3 && (!z || !vz)))
        return fail(c, GE_ERR_ARG, "positions, velocities and masses are required");
    int rc = ensure_capacity(c, n);
    if (rc) return rc;
    c->n = n;
    c->cur = 0;
    c->has_pinned = false;
    State &s = c->st[0];
    const size_t B = sizeof(float) * (size_t)n;
    cudaStream_t st = c->stream;
    GE_CHECK(c, cudaMemcpyAsync(s.x, x, B, cudaMemcpyHostToDevice, st));
    GE_CHECK(c, cudaMemcpyAsync(s.y, y, B, cudaMemcpyHostToDevice, st));
    GE_CHECK(c, cudaMemcpyAsync(s.vx, vx, B, cudaMemcpyHostToDevice, st));
    GE_CHECK(c, cudaMemcpyAsync(s.vy, vy, B, cudaMemcpyHostToDevice, st));
    GE_CHECK(c, cudaMemcpyAsync(s.m, m, B, cudaMemcpyHostToDevice, st));
    if (D == 3) {
        GE_CHECK(c, cudaMemcpyAsync(s.z, z, B, cudaMemcpyHostToDevice, st));
        GE_CHECK(c, cudaMemcpyAsync(s.vz, vz, B, cudaMemcpyHostToDevice, st));
    }
    if (ax) GE_CHECK(c, cudaMemcpyAsync(s.ax, ax, B, cudaMemcpyHostToDevice, st));
    else GE_CHECK(c, cudaMemsetAsync(s.ax, 0, B, st));
    if (ay) GE_CHECK(c, cudaMemcpyAsync(s.ay, ay, B, cudaMemcpyHostToDevice, st));
    else GE_CHECK(c, cudaMemsetAsync(s.ay, 0, B, st));
    if (D == 3) {
        if (az) GE_CHECK(c, cudaMemcpyAsync(s.az, az, B, cudaMemcpyHostToDevice, st));
        else GE_CHECK(c, cudaMemsetAsync(s.az, 0, B, st));
    }
    if (id) {
        GE_CHECK(c, cudaMemcpyAsync(s.id, id, sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
    } else {
        std::vector<uint32_t> iota((size_t)n);
        for (int64_t i = 0; i < n; i++) iota[(size_t)i] = (uint32_t)i;
        GE_CHECK(c, cudaMemcpyAsync(s.id, iota.data(), sizeof(uint32_t) * (size_t)n,
                                    cudaMemcpyHostToDevice, st));
        GE_CHECK(c, cudaStreamSynchronize(st));
    }
    if (c->has_prev) {
        GE_CHECK(c, cudaMemcpyAsync(s.pvx, s.vx, B, cudaMemcpyDeviceToDevice, st));
        GE_CHECK(c, cudaMemcpyAsync(s.pvy, s.vy, B, cudaMemcpyDeviceToDevice, st));
        if (D == 3) GE_CHECK(c, cudaMemcpyAsync(s.pvz, s.vz, B, cudaMemcpyDeviceToDevice, st));
    }
    c->tree_valid = false;
    c->keys_valid = false;
    return GE_OK;
}

int ge_upload_pinned(ge_ctx *c, const uint8_t *pinned) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!pinned) {
        c->has_pinned = false;
        return GE_OK;
    }
    if (!c->st[0].pinned) {
        GE_CHECK(c, dalloc(c, &c->st[0].pinned, (size_t)c->cap_n));
        GE_CHECK(c, dalloc(c, &c->st[1].pinned, (size_t)c->cap_n));
    }
    GE_CHECK(c, cudaMemcpyAsync(c->st[c->cur].pinned, pinned, (size_t)c->n, cudaMemcpyHostToDevice,
                                c->stream));
    c->has_pinned = true;
    return GE_OK;
}

int ge_download(ge_ctx *c, float *x, float *y, float *z, float *vx, float *vy, float *vz,
                float *ax, float *ay, float *az, float *m, uint32_t *id) {
    int rc = require_state(c);
    if (rc) return rc;
    const State &s = c->st[c->cur];
    const size_t B = sizeof(float) * (size_t)c->n;
    cudaStream_t st = c->stream;
    const bool d3 = c->p.dims == 3;
    struct { void *h; const void *d; size_t b; } cp[] = {
        {x, s.x, B}, {y, s.y, B}, {d3 ? z : nullptr, s.z, B}, {vx, s.vx, B}, {vy, s.vy, B},
        {d3 ? vz : nullptr, s.vz, B}, {ax, s.ax, B}, {ay, s.ay, B}, {d3 ? az : nullptr, s.az, B},
        {m, s.m, B}, {id, s.id, sizeof(uint32_t) * (size_t)c->n}};
    for (auto &q : cp)
        if (q.h) GE_CHECK(c, cudaMemcpyAsync(q.h, q.d, q.b, cudaMemcpyDeviceToHost, st));
    GE_CHECK(c, cudaStreamSynchronize(st));
    return GE_OK;
}

int ge_download_prev_vel(ge_ctx *c, float *pvx, float *pvy, float *pvz) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!c->has_prev) return fail(c, GE_ERR_STATE, "track_prev_vel is off");
    const State &s = c->st[c->cur];
    const size_t B = sizeof(float) * (size_t)c->n;
    if (pvx) GE_CHECK(c, cudaMemcpyAsync(pvx, s.pvx, B, cudaMemcpyDeviceToHost, c->stream));
    if (pvy) GE_CHECK(c, cudaMemcpyAsync(pvy, s.pvy, B, cudaMemcpyDeviceToHost, c->stream));
    if (pvz && c->p.dims == 3)
        GE_CHECK(c, cudaMemcpyAsync(pvz, s.pvz, B, cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    return GE_OK;
}

int ge_step(ge_ctx *c, int32_t nsteps) {
    int rc = require_state(c);
    if (rc) return rc;
    if (nsteps < 0) return fail(c, GE_ERR_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return GE_OK;
    GE_CHECK(c, cudaEventRecord(c->ev[6], c->stream));
    for (int k = 0; k < nsteps; k++)
        if ((rc = enqueue_frame(c, nullptr))) return rc;
    GE_CHECK(c, cudaEventRecord(c->ev[7], c->stream));
    rc = check_device(c);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]);
    c->stats.ms_last_step = ms / (float)nsteps;
    c->stats.steps += nsteps;
    c->tree_valid = rc == GE_OK;
    if (rc == GE_OK && c->count_inter) {
        unsigned long long v = 0;
        GE_CHECK(c, cudaMemcpy(&v, c->d_inter, sizeof(v), cudaMemcpyDeviceToHost));
        c->stats.interactions = v;
    }
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
    c->tree_valid = true;
    return GE_OK;
}

int ge_frame_host(ge_ctx *c, int64_t n, float *x, float *y, float *z, float *vx, float *vy,
                  float *vz, float *ax, float *ay, float *az, float *m, uint32_t *id) {
    if (!c) return GE_ERR_ARG;
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
    GE_CHECK(c, cudaMemcpyAsync(&bb, c->ss.bbox, sizeof(bb), cudaMemcpyDeviceToHost, c->stream));
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
        GE_CHECK(c, launch_keys_out(c->p.dims, (int)c->n, c->ss, tmp, c->stream));
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
    if ((rc = enqueue_sort_permute(c, true))) return rc;
    c->keys_valid = false;
    c->tree_valid = false;
    if (perm_out) {
        uint32_t *tmp = nullptr;
        GE_CHECK(c, cudaMallocAsync((void **)&tmp, sizeof(uint32_t) * (size_t)c->n, c->stream));
        GE_CHECK(c, launch_perm_out(c->p.dims, (int)c->n, c->ss, tmp, c->stream));
        GE_CHECK(c, cudaMemcpyAsync(perm_out, tmp, sizeof(uint32_t) * (size_t)c->n,
                                    cudaMemcpyDeviceToHost, c->stream));
        GE_CHECK(c, cudaFreeAsync(tmp, c->stream));
    }
    return check_device(c);
}

int ge_build_tree(ge_ctx *c) {
    int rc = require_state(c);
    if (rc) return rc;
    if ((rc = enqueue_bbox(c, false))) return rc;   // seeds the root cell
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
        GE_CHECK(c, cudaMemcpy(&v, c->d_inter, sizeof(v), cudaMemcpyDeviceToHost));
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
    uint32_t *d_idx = nullptr;
    double *d_out = nullptr;
    GE_CHECK(c, cudaMallocAsync((void **)&d_idx, sizeof(uint32_t) * nt, c->stream));
    GE_CHECK(c, cudaMallocAsync((void **)&d_out, sizeof(double) * nt * D, c->stream));
    GE_CHECK(c, cudaMemcpyAsync(d_idx, idx, sizeof(uint32_t) * nt, cudaMemcpyHostToDevice, c->stream));
    GE_CHECK(c, launch_direct_f64(D, cur_state(c), (int)c->n, d_idx, (int)nt, (double)c->p.G,
                                  (double)c->p.eps2, d_out, c->stream));
    std::vector<double> h((size_t)(nt * D));
    GE_CHECK(c, cudaMemcpyAsync(h.data(), d_out, sizeof(double) * nt * D, cudaMemcpyDeviceToHost,
                                c->stream));
    GE_CHECK(c, cudaFreeAsync(d_idx, c->stream));
    GE_CHECK(c, cudaFreeAsync(d_out, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    for (int64_t k = 0; k < nt; k++) {
        ax[k] = h[(size_t)(k * D)];
        ay[k] = h[(size_t)(k * D + 1)];
        if (D == 3 && az) az[k] = h[(size_t)(k * D + 2)];
    }
    return GE_OK;
}

int ge_build_timeline(ge_ctx *c, int32_t cap, uint64_t *ns, int32_t *count) {
    int rc = require_state(c);
    if (rc) return rc;
    if (!count || (cap > 0 && !ns)) return fail(c, GE_ERR_ARG, "bad timeline buffers");
    uint32_t m[8];
    GE_CHECK(c, cudaMemcpyAsync(m, c->tree.meta, sizeof(m), cudaMemcpyDeviceToHost, c->stream));
    unsigned long long tl[kTimeline];
    GE_CHECK(c, cudaMemcpyAsync(tl, c->tree.tl, sizeof(tl), cudaMemcpyDeviceToHost, c->stream));
    GE_CHECK(c, cudaStreamSynchronize(c->stream));
    const int32_t k = (int32_t)(m[7] < (uint32_t)kTimeline ? m[7] : kTimeline);
    *count = k;
    for (int32_t i = 0; i < k && i < cap; i++) ns[i] = (uint64_t)(tl[i] - tl[0]);
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
    GE_CHECK(c, cudaMemcpy(w.data(), c->tree.walk, sizeof(float4) * ns, cudaMemcpyDeviceToHost));
    GE_CHECK(c, cudaMemcpy(cell.data(), c->tree.cell, sizeof(float4) * ns, cudaMemcpyDeviceToHost));
    GE_CHECK(c, cudaMemcpy(inf.data(), c->tree.info, sizeof(uint4) * ns, cudaMemcpyDeviceToHost));
    // depth-first pre-order numbering, children in slot order (the reference's
    // emission order, quadtree.cpp:67-87); next = number of descendants
    std::vector<uint32_t> order;
    order.reserve((size_t)nn);
    std::vector<uint32_t> stack{0u};
    std::vector<uint32_t> newid((size_t)ns, kEmpty);
    while (!stack.empty()) {
        uint32_t k = stack.back();
        stack.pop_back();
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
