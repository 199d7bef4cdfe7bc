// ge_server.cu -- serving loop: continuous batching of independent
// simulations under a device-memory budget (C ABI in include/ge_bh.h).
//
// No counterpart in the reference, which steps one particle system per
// process.  A server owns two batch contexts ("pools", 2D and 3D), each sized
// once at creation from its share of the HBM budget (ge_estimate_bytes /
// ge_reserve), so admission never allocates and the pools never exceed the
// budget.  Requests (a simulation and a step count) are queued by
// ge_server_submit from any host thread.  Each pool's loop -- on its own
// worker thread (ge_server_start), or both pools per ge_server_poll --
// repeats:
//   1. admit: queued requests join their pool, first come first served, as
//      long as the pool's particle and simulation capacity allow (a request
//      that does not fit waits for running ones to finish; later requests of
//      the same pool wait behind it);
//   2. step: one step of all of the pool's running simulations
//      (ge_step_async on the pool's stream, then ge_step_wait); the pools step
//      independently, each at its own rate, and their kernels overlap on the
//      device;
//   3. retire: simulations that reached their step count are copied to host
//      memory and removed from their pool in one compaction.
// A simulation's result does not depend on what else runs in its pool
// (segments never mix), so every result equals the same request run alone.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "ge_bh.h"

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

struct Request {
    int64_t id = 0;
    int dims = 2;
    int64_t n = 0;
    int32_t steps = 0;
    int32_t steps_done = 0;
    int32_t state = GE_REQ_QUEUED;
    int32_t sim = 0;            // handle in its pool while running
    std::vector<float> in;      // x, y, (z), vx, vy, (vz), m
    std::vector<float> out;     // x, y, (z), vx, vy, (vz), ax, ay, (az), m
    std::vector<uint32_t> out_id;
    double t_submit = 0, t_admit = 0, t_done = 0;
};

struct Pool {
    ge_ctx *ctx = nullptr;
    int dims = 2;
    int64_t cap_n = 0;          // particles admitted at once
    int64_t used_n = 0;
    int32_t max_sims = 0;
    std::deque<int64_t> queue;  // waiting requests, first come first served
    std::vector<int64_t> running;
    // the pool's loop
    std::thread worker;
    bool stepping = false;
    Clock::time_point t_step;
    int64_t iterations = 0;
    double busy_s = 0.0, admit_s = 0.0, retire_s = 0.0;
    int64_t particle_steps = 0;
    std::vector<double> step_ms;
};

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

struct ge_server {
    ge_server_config cfg{};
    int dev = 0;
    Pool pool[2];
    std::mutex mu;
    std::condition_variable cv;       // submissions and completions
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    int64_t next_id = 1;
    bool running_thread = false;
    bool stop = false;
    Clock::time_point t0 = Clock::now();
    // statistics
    int64_t submitted = 0, completed = 0, failed = 0, particle_steps = 0;
    std::vector<double> latency_s;
    std::vector<double> queue_wait_s;
    std::string err;
    int loop_error = GE_OK;
};

namespace {

int sfail(ge_server *s, int code, const std::string &msg) {
    if (s) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->err = msg;
    }
    return code;
}

// Particles of a pool for `share` bytes: the largest n whose reservation
// (ge_estimate_bytes with max_sims simulations) fits.
int size_pool(const ge_params *p, int64_t share, int32_t max_sims, int64_t *cap) {
    int64_t lo = 0, hi = p->dims == 2 ? (1ll << 28) - 1 : (1ll << 31) - 1;
    int64_t b = 0;
    int rc = ge_estimate_bytes(p, 1, max_sims, &b);
    if (rc) return rc;
    if (b > share) { *cap = 0; return GE_OK; }
    lo = 1;
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo + 1) / 2;
        if ((rc = ge_estimate_bytes(p, mid, max_sims, &b))) return rc;
        if (b <= share) lo = mid;
        else hi = mid - 1;
    }
    *cap = lo;
    return GE_OK;
}

// 1. admit queued requests of pool k that fit (caller holds no lock)
int admit(ge_server *s, int k) {
    Pool &P = s->pool[k];
    if (!P.ctx) return GE_OK;
    const Clock::time_point ta = Clock::now();
    struct AddTime {   // time spent adding simulations, on every way out
        ge_server *s;
        Pool &P;
        Clock::time_point t;
        ~AddTime() {
            std::lock_guard<std::mutex> lk(s->mu);
            P.admit_s += seconds_since(t);
        }
    } add_time{s, P, ta};
    while (true) {
        Request *r = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (P.queue.empty()) break;
            Request *h = s->reqs[P.queue.front()].get();
            if (P.used_n + h->n > P.cap_n || (int32_t)P.running.size() >= P.max_sims) break;
            P.queue.pop_front();
            r = h;
        }
        const int64_t n = r->n;
        const float *b = r->in.data();
        const bool d3 = P.dims == 3;
        const float *x = b, *y = b + n, *z = d3 ? b + 2 * n : nullptr;
        const float *vx = b + (d3 ? 3 : 2) * n, *vy = vx + n, *vz = d3 ? vy + n : nullptr;
        const float *m = b + (d3 ? 6 : 4) * n;
        int32_t h = 0;
        const int rc = ge_batch_add_sim(P.ctx, n, x, y, z, vx, vy, vz, m, nullptr, &h);
        std::lock_guard<std::mutex> lk(s->mu);
        if (rc) {
            r->state = GE_REQ_FAILED;
            s->failed++;
            s->err = ge_last_error(P.ctx);
            s->cv.notify_all();
            continue;
        }
        r->sim = h;
        r->state = GE_REQ_RUNNING;
        r->t_admit = seconds_since(s->t0);
        s->queue_wait_s.push_back(r->t_admit - r->t_submit);
        r->in.clear();
        r->in.shrink_to_fit();
        P.used_n += n;
        P.running.push_back(r->id);
    }
    return GE_OK;
}

// 2. one step of every running simulation of pool k, in two halves so that
// several pools can be in flight on their own streams
int start_step(ge_server *s, int k) {
    Pool &P = s->pool[k];
    if (!P.ctx || P.running.empty()) return GE_OK;
    P.t_step = Clock::now();
    P.stepping = true;
    const int rc = ge_step_async(P.ctx, 1);
    if (rc) {
        P.stepping = false;
        return sfail(s, rc, ge_last_error(P.ctx));
    }
    return GE_OK;
}

// finish the step of pool k, then 3. retire its finished simulations
int finish_step(ge_server *s, int k, int32_t *stepped) {
    Pool &P = s->pool[k];
    if (!P.stepping) return GE_OK;
    P.stepping = false;
    int rc = ge_step_wait(P.ctx);
    if (rc) return sfail(s, rc, ge_last_error(P.ctx));
    const double dt = seconds_since(P.t_step);
    const int64_t ps = P.used_n;
    const Clock::time_point tr = Clock::now();
    *stepped = 1;
    std::vector<int32_t> gone;
    std::vector<int64_t> keep, done;
    std::vector<Request *> fin;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (int64_t id : P.running) {
            Request *r = s->reqs[id].get();
            r->steps_done++;
            if (r->steps_done < r->steps) keep.push_back(id);
            else { fin.push_back(r); done.push_back(id); }
        }
    }
    for (Request *r : fin) {   // running requests are only touched by their pool's loop
        const int64_t n = r->n;
        const int q = P.dims;
        r->out.resize((size_t)n * (3 * q + 1));
        r->out_id.resize((size_t)n);
        float *o = r->out.data();
        float *x = o, *y = o + n, *z = q == 3 ? o + 2 * n : nullptr;
        float *vx = o + q * n, *vy = vx + n, *vz = q == 3 ? vy + n : nullptr;
        float *ax = o + 2 * q * n, *ay = ax + n, *az = q == 3 ? ay + n : nullptr;
        float *m = o + 3 * q * n;
        rc = ge_batch_download_sim(P.ctx, r->sim, x, y, z, vx, vy, vz, ax, ay, az, m,
                                   r->out_id.data());
        if (rc) return sfail(s, rc, ge_last_error(P.ctx));
        gone.push_back(r->sim);
    }
    if (!gone.empty()) {
        rc = ge_batch_remove_sims(P.ctx, (int32_t)gone.size(), gone.data());
        if (rc) return sfail(s, rc, ge_last_error(P.ctx));
    }
    std::lock_guard<std::mutex> lk(s->mu);
    for (int64_t id : done) {
        Request *r = s->reqs[id].get();
        r->state = GE_REQ_DONE;
        r->t_done = seconds_since(s->t0);
        P.used_n -= r->n;
        s->completed++;
        s->latency_s.push_back(r->t_done - r->t_submit);
    }
    P.running.swap(keep);
    P.iterations++;
    s->particle_steps += ps;
    P.particle_steps += ps;
    P.busy_s += dt;
    P.retire_s += seconds_since(tr);
    if (P.step_ms.size() < (1u << 22)) P.step_ms.push_back(dt * 1e3);
    s->cv.notify_all();
    return GE_OK;
}

// One loop iteration of each pool on the calling thread: both pools' steps
// are in flight together.
int iterate_all(ge_server *s, int32_t *stepped) {
    int rc;
    for (int k = 0; k < 2; k++)
        if ((rc = admit(s, k))) return rc;
    for (int k = 0; k < 2; k++)
        if ((rc = start_step(s, k))) return rc;
    for (int k = 0; k < 2; k++)
        if ((rc = finish_step(s, k, stepped))) return rc;
    return GE_OK;
}

// The loop of one pool on its own thread.
void worker_main(ge_server *s, int k) {
    cudaSetDevice(s->dev);
    Pool &P = s->pool[k];
    while (true) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop) break;
        }
        int32_t stepped = 0;
        int rc = admit(s, k);
        if (!rc) rc = start_step(s, k);
        if (!rc) rc = finish_step(s, k, &stepped);
        std::unique_lock<std::mutex> lk(s->mu);
        if (rc) {
            s->loop_error = rc;
            s->cv.notify_all();
            break;
        }
        // nothing running in this pool: sleep until a submission (or stop)
        if (!stepped && P.queue.empty() && !s->stop) s->cv.wait_for(lk, std::chrono::milliseconds(20));
    }
}

}  // namespace

extern "C" {

int ge_server_create(const ge_server_config *cfg, ge_server **out) {
    if (!cfg || !out) return GE_ERR_ARG;
    *out = nullptr;
    if (cfg->hbm_budget_bytes <= 0 || cfg->max_sims < 1 || !(cfg->frac_2d >= 0.0) ||
        !(cfg->frac_2d <= 1.0))
        return GE_ERR_ARG;
    if (cfg->params[0].dims != 2 || cfg->params[1].dims != 3) return GE_ERR_ARG;
    auto s = std::make_unique<ge_server>();
    s->cfg = *cfg;
    if (cudaGetDevice(&s->dev) != cudaSuccess) return GE_ERR_NO_DEVICE;
    auto cleanup = [&](int rc) {
        for (Pool &Q : s->pool)
            if (Q.ctx) ge_destroy(Q.ctx);
        return rc;
    };
    const int64_t share[2] = {(int64_t)((double)cfg->hbm_budget_bytes * cfg->frac_2d),
                              cfg->hbm_budget_bytes -
                                  (int64_t)((double)cfg->hbm_budget_bytes * cfg->frac_2d)};
    for (int k = 0; k < 2; k++) {
        Pool &P = s->pool[k];
        P.dims = k == 0 ? 2 : 3;
        P.max_sims = cfg->max_sims;
        if (share[k] <= 0) continue;
        int64_t cap = 0;
        int rc = size_pool(&cfg->params[k], share[k], cfg->max_sims, &cap);
        if (rc) return cleanup(rc);
        if (cap < 1) continue;
        if ((rc = ge_create(&cfg->params[k], &P.ctx))) return cleanup(rc);
        if ((rc = ge_reserve(P.ctx, cap, cfg->max_sims))) return cleanup(rc);
        P.cap_n = cap;
    }
    *out = s.release();
    return GE_OK;
}

int ge_server_destroy(ge_server *s) {
    if (!s) return GE_OK;
    ge_server_stop(s);
    for (Pool &P : s->pool)
        if (P.ctx) ge_destroy(P.ctx);
    delete s;
    return GE_OK;
}

const char *ge_server_last_error(const ge_server *s) { return s ? s->err.c_str() : "null server"; }

int ge_server_submit(ge_server *s, int32_t dims, int64_t n, const float *x, const float *y,
                     const float *z, const float *vx, const float *vy, const float *vz,
                     const float *m, int32_t steps, int64_t *request) {
    if (!s || !request) return GE_ERR_ARG;
    if ((dims != 2 && dims != 3) || n < 1 || steps < 1) return sfail(s, GE_ERR_ARG, "bad request");
    if (!x || !y || !vx || !vy || !m || (dims == 3 && (!z || !vz)))
        return sfail(s, GE_ERR_ARG, "positions, velocities and masses are required");
    Pool &P = s->pool[dims == 3 ? 1 : 0];
    if (!P.ctx || n > P.cap_n)
        return sfail(s, GE_ERR_CAPACITY, "request larger than its pool's share of the budget");
    auto r = std::make_unique<Request>();
    r->dims = dims;
    r->n = n;
    r->steps = steps;
    const int q = dims;
    r->in.resize((size_t)n * (2 * q + 1));
    float *b = r->in.data();
    const size_t B = sizeof(float) * (size_t)n;
    std::memcpy(b, x, B);
    std::memcpy(b + n, y, B);
    if (q == 3) std::memcpy(b + 2 * n, z, B);
    std::memcpy(b + q * n, vx, B);
    std::memcpy(b + (q + 1) * n, vy, B);
    if (q == 3) std::memcpy(b + 5 * n, vz, B);
    std::memcpy(b + 2 * q * n, m, B);
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    r->t_submit = seconds_since(s->t0);
    *request = r->id;
    P.queue.push_back(r->id);
    s->reqs[r->id] = std::move(r);
    s->submitted++;
    s->cv.notify_all();
    return GE_OK;
}

int ge_server_start(ge_server *s) {
    if (!s) return GE_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->running_thread) return GE_OK;
    s->stop = false;
    s->running_thread = true;
    for (int k = 0; k < 2; k++)
        if (s->pool[k].ctx) s->pool[k].worker = std::thread(worker_main, s, k);
    return GE_OK;
}

int ge_server_stop(ge_server *s) {
    if (!s) return GE_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->running_thread) return s->loop_error;
        s->stop = true;
        s->cv.notify_all();
    }
    for (Pool &P : s->pool)
        if (P.worker.joinable()) P.worker.join();
    std::lock_guard<std::mutex> lk(s->mu);
    s->running_thread = false;
    return s->loop_error;
}

int ge_server_poll(ge_server *s, int32_t *stepped) {
    if (!s) return GE_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->running_thread) return GE_ERR_STATE;
    }
    int32_t st = 0;
    const int rc = iterate_all(s, &st);
    if (stepped) *stepped = st;
    return rc;
}

int ge_server_wait(ge_server *s, int64_t request, double timeout_s) {
    if (!s) return GE_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                             std::chrono::duration<double>(timeout_s));
    while (true) {
        auto it = s->reqs.find(request);
        if (it == s->reqs.end()) return GE_ERR_ARG;
        const int32_t st = it->second->state;
        if (st == GE_REQ_DONE) return GE_OK;
        if (st == GE_REQ_FAILED) return GE_ERR_STATE;
        if (s->loop_error) return s->loop_error;
        if (!s->running_thread) return GE_ERR_STATE;   // nobody would finish it
        if (s->cv.wait_until(lk, deadline) == std::cv_status::timeout) return GE_ERR_TIMEOUT;
    }
}

int ge_server_status(ge_server *s, int64_t request, int32_t *state, int32_t *steps_done,
                     double *latency_s) {
    if (!s) return GE_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request);
    if (it == s->reqs.end()) return GE_ERR_ARG;
    const Request &r = *it->second;
    if (state) *state = r.state;
    if (steps_done) *steps_done = r.steps_done;
    if (latency_s) *latency_s = r.state == GE_REQ_DONE ? r.t_done - r.t_submit : -1.0;
    return GE_OK;
}

int ge_server_take(ge_server *s, int64_t request, float *x, float *y, float *z, float *vx,
                   float *vy, float *vz, float *ax, float *ay, float *az, float *m,
                   uint32_t *id) {
    if (!s) return GE_ERR_ARG;
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(request);
        if (it == s->reqs.end()) return GE_ERR_ARG;
        if (it->second->state != GE_REQ_DONE) return GE_ERR_STATE;
        r = std::move(it->second);
        s->reqs.erase(it);
    }
    const int64_t n = r->n;
    const int q = r->dims;
    const float *o = r->out.data();
    const size_t B = sizeof(float) * (size_t)n;
    float *dst[] = {x, y, q == 3 ? z : nullptr, vx, vy, q == 3 ? vz : nullptr,
                    ax, ay, q == 3 ? az : nullptr, m};
    const float *src[] = {o, o + n, q == 3 ? o + 2 * n : nullptr,
                          o + q * n, o + (q + 1) * n, q == 3 ? o + 5 * n : nullptr,
                          o + 2 * q * n, o + (2 * q + 1) * n, q == 3 ? o + 8 * n : nullptr,
                          o + 3 * q * n};
    for (size_t k = 0; k < sizeof(dst) / sizeof(dst[0]); k++)
        if (dst[k] && src[k]) std::memcpy(dst[k], src[k], B);
    if (id) std::memcpy(id, r->out_id.data(), sizeof(uint32_t) * (size_t)n);
    return GE_OK;
}

int ge_server_get_stats(ge_server *s, ge_server_stats *out) {
    if (!s || !out) return GE_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->queued = (int64_t)(s->pool[0].queue.size() + s->pool[1].queue.size());
    out->running = (int64_t)(s->pool[0].running.size() + s->pool[1].running.size());
    out->particle_steps = s->particle_steps;
    std::vector<double> all;
    for (int k = 0; k < 2; k++) {
        const Pool &P = s->pool[k];
        out->iterations += P.iterations;
        out->busy_s += P.busy_s;
        out->pool_iterations[k] = P.iterations;
        out->pool_step_ms_p50[k] = percentile(P.step_ms, 0.50);
        out->pool_step_ms_p99[k] = percentile(P.step_ms, 0.99);
        out->pool_busy_s[k] = P.busy_s;
        out->pool_admit_s[k] = P.admit_s;
        out->pool_retire_s[k] = P.retire_s;
        out->pool_particle_steps[k] = P.particle_steps;
        all.insert(all.end(), P.step_ms.begin(), P.step_ms.end());
    }
    out->queue_wait_s_p50 = percentile(s->queue_wait_s, 0.50);
    out->queue_wait_s_p99 = percentile(s->queue_wait_s, 0.99);
    out->step_ms_p50 = percentile(all, 0.50);
    out->step_ms_p99 = percentile(all, 0.99);
    out->latency_s_p50 = percentile(s->latency_s, 0.50);
    out->latency_s_p99 = percentile(s->latency_s, 0.99);
    for (int k = 0; k < 2; k++) {
        int64_t b = 0;
        if (s->pool[k].ctx) ge_memory_bytes(s->pool[k].ctx, &b);
        out->pool_bytes[k] = b;
        out->pool_capacity[k] = s->pool[k].cap_n;
    }
    return GE_OK;
}

}  // extern "C"
