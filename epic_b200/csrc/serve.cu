// Served ensembles (include/epic_serve.h): a pool of worker threads, one per
// slot, each running one simulation at a time on its own context and CUDA
// stream; admission of the first queued request (in arrival order, or the
// smallest estimated work first) that fits the free slots and the HBM budget; idle
// contexts kept per configuration and reused, so that a steady stream of
// requests allocates (and frees, which synchronises the whole device) no
// device memory.
#include "ctx.hpp"
#include "../../include/epic_serve.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <set>
#include <mutex>
#include <thread>
#include <vector>

namespace epic {

// Device bytes of a context created with cfg (the allocations of
// epic_gpu_create plus the step's stream-ordered scratch), with a margin.
static double estimate_bytes(const epic_cfg& g) {
    const double nx = g.nx, ny = g.ny, nz = g.nz;
    const double ncell = nx * ny * nz;
    double cap = g.capacity > 0 ? (double)g.capacity : 2.0 * ncell * std::max(1, g.n_per_cell) + 1024.0;
    const double fsz = nx * ny * (nz + 3);
    const double store = (g.precision == EPIC_PRECISION_MIXED ? PARCEL_BYTES_MIXED : PARCEL_BYTES_PLAIN) * cap;
    double b = store * (g.keep_order ? 1.0 : 2.0);
    b += fsz * 8.0 * (21 + 14 + 16 + 12) + fsz * 8.0;   // fields, work, gather records, tables, counts
    b += cap * 32.0;                                     // sort keys / merge and split scratch
    return 1.15 * b + 64.0 * (1 << 20);
}

struct Job {
    int64_t id;
    epic_request req;
    double t_submit;
    double bytes;
    double work;   // estimated parcel-steps: cells x parcels per cell x steps
};

struct PooledCtx {
    epic_cfg cfg;
    epic_ctx* ctx;
    double bytes;
};

}  // namespace epic

using namespace epic;

struct epic_server {
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job> queue;
    std::map<int64_t, epic_result> results;   // finished, not yet waited for
    std::set<int64_t> pending;                 // submitted, not yet finished
    std::vector<PooledCtx> idle;
    std::vector<std::thread> workers;
    int device = 0;
    double budget = 0.0, in_use = 0.0;   // bytes: running requests + idle contexts
    int64_t next_id = 1, running = 0, n_collected = 0;
    int policy = EPIC_SRV_ARRIVAL;
    bool stop = false;
    std::chrono::steady_clock::time_point t0;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

// Field by field (the struct has padding, which callers need not clear).
static bool same_cfg(const epic_cfg& a, const epic_cfg& b) {
    auto eq3 = [](const double* x, const double* y) { return x[0] == y[0] && x[1] == y[1] && x[2] == y[2]; };
    return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && eq3(a.lower, b.lower) && eq3(a.extent, b.extent) &&
           a.size_factor == b.size_factor && a.grow_factor == b.grow_factor && a.shrink_factor == b.shrink_factor &&
           a.n_per_cell == b.n_per_cell && a.lambda_max == b.lambda_max && a.min_vratio == b.min_vratio &&
           a.correction_iters == b.correction_iters && a.gradient_pref == b.gradient_pref &&
           a.max_compression == b.max_compression && a.t_initial == b.t_initial && a.t_limit == b.t_limit &&
           a.alpha == b.alpha && a.precise_stop == b.precise_stop && a.use_fixed_dt == b.use_fixed_dt &&
           a.fixed_dt == b.fixed_dt && a.rk_order == b.rk_order && a.gravity == b.gravity && a.L_v == b.L_v &&
           a.c_p == b.c_p && a.theta_0 == b.theta_0 && a.q_0 == b.q_0 && a.height_c == b.height_c &&
           a.ang_vel == b.ang_vel && a.lat_degrees == b.lat_degrees &&
           a.l_planetary_vorticity == b.l_planetary_vorticity && a.bndry_zeta_zero[0] == b.bndry_zeta_zero[0] &&
           a.bndry_zeta_zero[1] == b.bndry_zeta_zero[1] && a.capacity == b.capacity && a.precision == b.precision &&
           a.keep_order == b.keep_order && a.damping_vorticity_prefactor == b.damping_vorticity_prefactor &&
           a.damping_scalars_prefactor == b.damping_scalars_prefactor && a.damping_vorticity == b.damping_vorticity &&
           a.damping_surface_vorticity == b.damping_surface_vorticity && a.damping_scalars == b.damping_scalars &&
           a.damping_surface_scalars == b.damping_surface_scalars && a.labels == b.labels &&
           a.label_seed == b.label_seed;
}

// Take an idle context of this configuration out of the pool (nullptr if none).
static epic_ctx* pool_take(epic_server* s, const epic_cfg& cfg, double* bytes) {
    for (size_t k = 0; k < s->idle.size(); ++k)
        if (same_cfg(s->idle[k].cfg, cfg)) {
            epic_ctx* c = s->idle[k].ctx;
            *bytes = s->idle[k].bytes;
            s->idle.erase(s->idle.begin() + k);
            return c;
        }
    return nullptr;
}

static void run_job(epic_server* s, const Job& job, int slot, epic_ctx* ctx, epic_result& r) {
    int rc = EPIC_OK;
    const bool fresh = ctx == nullptr;
    if (!ctx) rc = epic_gpu_create(&job.req.cfg, &ctx);
    double t = job.req.cfg.t_initial;
    epic_step_info info{};
    int64_t psteps = 0;
    if (rc == EPIC_OK) rc = epic_gpu_init_state(ctx, &job.req.init);
    // a new context tunes its launch shapes once if asked; pooled ones keep theirs
    if (rc == EPIC_OK && fresh && job.req.tune) rc = epic_gpu_autotune(ctx, nullptr);
    if (rc == EPIC_OK) rc = epic_gpu_init_correction(ctx);
    for (int k = 0; rc == EPIC_OK && k < job.req.steps; ++k) {
        int64_t n0 = 0;
        epic_gpu_num_parcels(ctx, &n0);
        rc = epic_gpu_step(ctx, &t, &info);
        psteps += n0;
    }
    r.status = rc;
    r.slot = slot;
    if (rc != EPIC_OK) {
        const char* m = ctx ? epic_gpu_last_error(ctx) : "context creation failed";
        std::snprintf(r.message, sizeof(r.message), "%s", m ? m : "");
    }
    r.parcel_steps = psteps;
    r.n_parcels = info.n_parcels;
    r.t_final = t;
    r.ke = info.parcel_stats[1];
    r.enstrophy = info.parcel_stats[12];
    std::lock_guard<std::mutex> lk(s->mu);
    r.t_done = s->now();
    if (rc == EPIC_OK) {
        s->idle.push_back({job.req.cfg, ctx, job.bytes});   // keeps its share of in_use
    } else {
        if (ctx) epic_gpu_destroy(ctx);
        s->in_use -= job.bytes;
    }
    --s->running;
    s->results[job.id] = r;
    s->pending.erase(job.id);
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

static void worker(epic_server* s, int slot) {
    cudaSetDevice(s->device);
    for (;;) {
        Job job;
        epic_ctx* ctx = nullptr;
        double pooled_bytes = 0.0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->queue.empty()) {
                    if (s->stop) return;
                    s->cv_work.wait(lk);
                    continue;
                }
                // the first queued request (in arrival order) that can start now:
                // a pooled context of its configuration, or room in the budget
                // (after freeing idle contexts of other configurations)
                size_t pick = s->queue.size();
                std::vector<size_t> order(s->queue.size());
                for (size_t q = 0; q < order.size(); ++q) order[q] = q;
                if (s->policy == EPIC_SRV_SHORTEST_FIRST)
                    std::stable_sort(order.begin(), order.end(),
                                     [&](size_t a, size_t b) { return s->queue[a].work < s->queue[b].work; });
                for (size_t oq = 0; oq < order.size() && pick == s->queue.size(); ++oq) {
                    const size_t q = order[oq];
                    Job& cand = s->queue[q];
                    ctx = pool_take(s, cand.req.cfg, &pooled_bytes);
                    if (ctx) { pick = q; break; }                    // its memory is already counted
                    double idle_bytes = 0.0;
                    for (auto& p : s->idle) idle_bytes += p.bytes;
                    if (s->in_use - idle_bytes + cand.bytes <= s->budget) {
                        while (s->in_use + cand.bytes > s->budget && !s->idle.empty()) {
                            PooledCtx p = s->idle.back();
                            s->idle.pop_back();
                            s->in_use -= p.bytes;
                            epic_gpu_destroy(p.ctx);
                        }
                        pick = q;
                    }
                }
                // nothing fits while nothing runs: the head starts anyway (it
                // passed the budget check at submission)
                if (pick == s->queue.size() && s->running == 0) {
                    while (!s->idle.empty()) {
                        PooledCtx p = s->idle.back();
                        s->idle.pop_back();
                        s->in_use -= p.bytes;
                        epic_gpu_destroy(p.ctx);
                    }
                    pick = 0;
                }
                if (pick < s->queue.size()) {
                    job = s->queue[pick];
                    s->queue.erase(s->queue.begin() + (long)pick);
                    break;
                }
                s->cv_work.wait(lk);                                  // wait for a running job to finish
            }
            if (ctx) job.bytes = pooled_bytes;
            else s->in_use += job.bytes;
            ++s->running;
        }
        epic_result r{};
        r.id = job.id;
        r.t_submit = job.t_submit;
        r.device_bytes = job.bytes;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r.t_start = s->now();
        }
        run_job(s, job, slot, ctx, r);
    }
}

extern "C" int epic_srv_create(int32_t max_slots, double hbm_fraction, epic_server** out) {
    if (!out || max_slots < 1 || max_slots > 64 || !(hbm_fraction > 0.0 && hbm_fraction <= 1.0))
        return EPIC_ERR_ARG;
    auto* s = new epic_server();
    s->t0 = std::chrono::steady_clock::now();
    if (cudaGetDevice(&s->device) != cudaSuccess) { delete s; return EPIC_ERR_CUDA; }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { delete s; return EPIC_ERR_CUDA; }
    s->budget = hbm_fraction * (double)free_b;
    try {
        for (int k = 0; k < max_slots; ++k) s->workers.emplace_back(worker, s, k);
    } catch (const std::exception&) {
        // a thread could not be started: stop the ones that were
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
            s->cv_work.notify_all();
        }
        for (auto& w : s->workers) w.join();
        delete s;
        return EPIC_ERR_CUDA;
    }
    *out = s;
    return EPIC_OK;
}

static int submit_locked(epic_server* s, const epic_request* req, int64_t* id);

extern "C" int epic_srv_submit(epic_server* s, const epic_request* req, int64_t* id) {
    if (!s || !req || !id || req->steps < 0) return EPIC_ERR_ARG;
    try {
        return submit_locked(s, req, id);
    } catch (const std::exception&) {   // host memory for the queue or the results
        return EPIC_ERR_CUDA;
    }
}

static int submit_locked(epic_server* s, const epic_request* req, int64_t* id) {
    std::lock_guard<std::mutex> lk(s->mu);
    Job j;
    j.id = s->next_id++;
    j.req = *req;
    j.t_submit = s->now();
    j.bytes = estimate_bytes(req->cfg);
    j.work = (double)req->cfg.nx * req->cfg.ny * req->cfg.nz * std::max(1, (int)req->init.n_per_cell) *
             (double)req->steps;
    *id = j.id;
    if (j.bytes > s->budget) {
        epic_result r{};
        r.id = j.id;
        r.status = EPIC_ERR_CAPACITY;
        r.slot = -1;
        r.t_submit = r.t_start = r.t_done = j.t_submit;
        r.device_bytes = j.bytes;
        std::snprintf(r.message, sizeof(r.message), "request needs %.3g bytes, server budget %.3g", j.bytes, s->budget);
        s->results[j.id] = r;
        s->cv_done.notify_all();
        return EPIC_OK;
    }
    s->queue.push_back(j);
    s->pending.insert(j.id);
    s->cv_work.notify_all();
    return EPIC_OK;
}

extern "C" int epic_srv_wait(epic_server* s, int64_t id, epic_result* out) {
    if (!s || !out || id < 1) return EPIC_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (id >= s->next_id || (!s->results.count(id) && !s->pending.count(id))) return EPIC_ERR_ARG;   // unknown or collected
    s->cv_done.wait(lk, [&] { return s->results.count(id) != 0; });
    *out = s->results[id];
    s->results.erase(id);   // handed over: the server keeps no finished results
    ++s->n_collected;
    return EPIC_OK;
}

extern "C" int epic_srv_counts(epic_server* s, int64_t* queued, int64_t* running, int64_t* done) {
    if (!s) return EPIC_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = (int64_t)s->queue.size();
    if (running) *running = s->running;
    if (done) *done = (int64_t)s->results.size() + s->n_collected;
    return EPIC_OK;
}

extern "C" int epic_srv_set_policy(epic_server* s, int32_t policy) {
    if (!s || (policy != EPIC_SRV_ARRIVAL && policy != EPIC_SRV_SHORTEST_FIRST)) return EPIC_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->policy = policy;
    return EPIC_OK;
}

extern "C" void epic_srv_destroy(epic_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    for (auto& w : s->workers) w.join();
    for (auto& p : s->idle) epic_gpu_destroy(p.ctx);
    delete s;
}
