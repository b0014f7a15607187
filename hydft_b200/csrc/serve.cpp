// Serving: solve requests on one GPU with continuous batching.
//
// A request is one model (params, optional initial state, a number of RK3
// steps).  Requests wait in arrival order until their device footprint fits
// the server's HBM budget and a slot is free; a setup thread then builds the
// model (HNC c(k) cached across requests with the same inputs), sets the
// state and dt, and hands it to the scheduler thread.  The scheduler keeps
// every admitted model's state resident and launches its captured step
// graph in chunks on the model's own stream, so the chunks of all admitted
// requests overlap on the device; requests that arrive while others run are
// admitted as memory frees up.  When a request has run its steps, its
// scalars (and, if asked, its final fields) are copied to the host and its
// device memory is released by the setup thread, off the scheduler's path
// (freeing device memory waits for the whole device).
//
// The reference has no serving layer; each request runs the driver loop of
// src/hydft.f90:41-51 for its model.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hydft_gpu.h"
#include "handle.hpp"

using namespace hydft;

namespace {

using Clock = std::chrono::steady_clock;

struct CachedStructure {
    std::vector<double> k, c;
    double u_ex = 0, du_dgamma = 0;
    int has_energy = 0;
};

std::string hnc_key(const hydft_params &p)
{
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s|%.17g|%.17g|%.17g|%.17g|%.17g|%d|%.17g|%.17g|%.17g|%d|%s|%s", p.kind, p.gamma,
                  p.kappa, p.rs, p.theta, p.mass, p.hnc_nr, p.hnc_rmax, p.hnc_tol, p.hnc_mix, p.hnc_maxiter,
                  p.structure, p.structure_kind);
    return buf;
}

struct Req {
    int64_t id = 0;
    hydft_params p{};
    std::vector<double> n, mom, pi;
    bool has_state = false;
    int nsteps = 0;
    bool keep_state = false;
    int state = HYDFT_REQ_QUEUED;
    double bytes = 0;
    double t_submit = 0, t_admit = 0, t_start = 0, t_done = 0;
    hydft_gpu *h = nullptr;
    int remaining = 0;
    bool inflight = false;
    cudaEvent_t ev = nullptr;
    int rc = 0;
    std::string err;
    std::vector<double> out_n, out_mom, out_pi;
    double info[HYDFT_SERVE_INFO_LEN] = {0};
    // the request is deleted once both its device memory is released and
    // its result has been collected, whichever comes last
    bool released = false, collected = false, collecting = false;
};

}  // namespace

struct hydft_server {
    int device = 0;
    double budget = 0, used = 0;
    int max_slots = 1, chunk = 1;
    std::mutex mu;
    std::condition_variable cv_setup, cv_sched, cv_done;
    std::deque<Req *> queue;   // submitted, waiting for admission
    std::deque<Req *> ready;   // set up, not yet seen by the scheduler
    std::deque<Req *> spent;   // finished, device memory still to release
    std::map<int64_t, std::unique_ptr<Req>> reqs;
    std::map<std::string, CachedStructure> cache;   // setup thread only
    int64_t next_id = 1;
    int holding = 0;           // admitted requests holding device memory
    int max_holding = 0;
    int64_t completed = 0;
    bool stop = false;
    Clock::time_point t0;
    std::thread setup_thread, sched_thread;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void release(hydft_server *s, Req *r)
{
    if (r->h) {
        cudaSetDevice(s->device);
        hydft_gpu_destroy(r->h);
        r->h = nullptr;
    }
    if (r->ev) {
        cudaEventDestroy(r->ev);
        r->ev = nullptr;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->used -= r->bytes;
    s->holding--;
    r->released = true;
    if (r->collected) s->reqs.erase(r->id);
}

// model, state and dt of an admitted request (setup thread)
int build(hydft_server *s, Req *r)
{
    cudaSetDevice(s->device);
    hydft_structure st{};
    const hydft_structure *sp = nullptr;
    const std::string key = hnc_key(r->p);
    const bool hnc = std::string(r->p.structure) == "hnc";
    auto it = s->cache.find(key);
    if (hnc && it != s->cache.end()) {
        st.n = (int)it->second.k.size();
        st.k = it->second.k.data();
        st.c = it->second.c.data();
        st.u_ex = it->second.u_ex;
        st.du_dgamma = it->second.du_dgamma;
        st.has_energy = it->second.has_energy;
        sp = &st;
    }
    int rc = hydft_gpu_create(&r->p, sp, s->device, &r->h);
    if (rc) {
        r->err = hydft_gpu_create_error();
        return rc;
    }
    if (hnc && it == s->cache.end() && r->h->mh.has_st) {
        CachedStructure c;
        c.k = r->h->mh.st_k;
        c.c = r->h->mh.st_c;
        c.u_ex = r->h->mh.u_ex;
        c.du_dgamma = r->h->mh.du_dgamma;
        c.has_energy = r->h->mh.has_energy ? 1 : 0;
        s->cache[key] = std::move(c);
    }
    if (r->has_state) {
        // Pi starts at zero when the request gives none (as model_t%init leaves it)
        if (r->pi.empty() && r->h->s->setup().evolve) r->pi.assign(6 * r->n.size(), 0.0);
        rc = hydft_gpu_set_state(r->h, r->n.data(), r->mom.data(), r->pi.empty() ? nullptr : r->pi.data());
    } else if (std::string(r->p.ic) != "uniform") {
        rc = hydft_gpu_set_initial_condition(r->h, r->p.ic, r->p.ic_amplitude, r->p.ic_mode, r->p.ic_width,
                                             r->p.ic_seed);
    }
    if (!rc && !(r->p.dt > 0.0)) {
        double dt = 0.0;
        rc = hydft_gpu_compute_dt(r->h, &dt);
    }
    if (rc) {
        r->err = hydft_gpu_last_error(r->h);
        return rc;
    }
    if (cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming) != cudaSuccess) {
        r->err = "event creation failed";
        return HYDFT_ERR_CUDA;
    }
    // the input copies are no longer needed
    std::vector<double>().swap(r->n);
    std::vector<double>().swap(r->mom);
    std::vector<double>().swap(r->pi);
    r->remaining = r->nsteps;
    return HYDFT_OK;
}

void finish(hydft_server *s, Req *r, int rc)
{
    std::lock_guard<std::mutex> lk(s->mu);
    r->rc = rc;
    r->t_done = s->now();
    r->state = rc ? HYDFT_REQ_FAILED : HYDFT_REQ_DONE;
    r->info[10] = r->t_submit;
    r->info[11] = r->t_admit;
    r->info[12] = r->t_start;
    r->info[13] = r->t_done;
    r->info[14] = r->bytes;
    s->completed++;
    s->cv_done.notify_all();
}

void setup_loop(hydft_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        Req *r = nullptr, *dead = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_setup.wait(lk, [&] {
                if (s->stop || !s->spent.empty()) return true;
                if (s->queue.empty() || s->holding >= s->max_slots) return false;
                return s->used + s->queue.front()->bytes <= s->budget;
            });
            if (!s->spent.empty()) {
                dead = s->spent.front();
                s->spent.pop_front();
            } else if (s->stop) {
                return;
            } else {
                r = s->queue.front();
                s->queue.pop_front();
                s->used += r->bytes;
                s->holding++;
                s->max_holding = std::max(s->max_holding, s->holding);
                r->state = HYDFT_REQ_SETUP;
                r->t_admit = s->now();
            }
        }
        if (dead) {
            release(s, dead);
            s->cv_setup.notify_one();
            continue;
        }
        const int rc = build(s, r);
        if (rc) {
            release(s, r);
            finish(s, r, rc);
            continue;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->state = HYDFT_REQ_RUNNING;
            s->ready.push_back(r);
        }
        s->cv_sched.notify_one();
    }
}

// final scalars (and fields) of a request that has run all its steps
int collect(Req *r)
{
    hydft_gpu *h = r->h;
    double t, dt, mass, mom[3], ekin, fe, nmin, nmax;
    int64_t step;
    int rc = hydft_gpu_get_time(h, &t, &dt, &step);
    if (!rc && r->keep_state) {
        const size_t nc = (size_t)r->p.nx * r->p.ny * r->p.nz;
        r->out_n.resize(nc);
        r->out_mom.resize(3 * nc);
        if (h->s->setup().evolve) r->out_pi.resize(6 * nc);
        rc = hydft_gpu_get_state(h, r->out_n.data(), r->out_mom.data(), r->out_pi.empty() ? nullptr : r->out_pi.data());
    }
    if (!rc) rc = hydft_gpu_budgets(h, &mass, mom, &ekin, &fe, &nmin, &nmax);
    if (rc) {
        r->err = hydft_gpu_last_error(h);
        return rc;
    }
    const double v[10] = {t, dt, (double)step, mass, mom[0], mom[1], mom[2], ekin, nmin, nmax};
    std::memcpy(r->info, v, sizeof v);
    r->info[15] = (double)h->s->launches;
    return HYDFT_OK;
}

void sched_loop(hydft_server *s)
{
    cudaSetDevice(s->device);
    std::vector<Req *> active;
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            while (!s->ready.empty()) {
                active.push_back(s->ready.front());
                s->ready.pop_front();
            }
            if (s->stop) break;
        }
        bool did = false;
        for (size_t i = 0; i < active.size();) {
            Req *r = active[i];
            int rc = HYDFT_OK;
            bool done = false;
            if (r->inflight) {
                if (cudaEventQuery(r->ev) == cudaErrorNotReady) {
                    ++i;
                    continue;
                }
                r->inflight = false;
                rc = r->h->s->poll_status();
                if (rc) r->err = r->h->s->err;
                done = rc != 0;
                did = true;
            }
            if (!done && r->remaining > 0) {
                if (r->t_start == 0.0) r->t_start = s->now();
                const int k = std::min(s->chunk, r->remaining);
                rc = r->h->s->launch_steps(k);
                if (rc) {
                    r->err = r->h->s->err;
                    done = true;
                } else {
                    r->remaining -= k;
                    cudaEventRecord(r->ev, static_cast<cudaStream_t>(r->h->s->stream()));
                    r->inflight = true;
                }
                did = true;
            } else if (!done) {
                rc = collect(r);
                done = true;
                did = true;
            }
            if (done) {
                finish(s, r, rc);
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    s->spent.push_back(r);
                }
                s->cv_setup.notify_one();
                active.erase(active.begin() + i);
                continue;
            }
            ++i;
        }
        if (!did) {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_sched.wait_for(lk, std::chrono::microseconds(100), [&] { return s->stop || !s->ready.empty(); });
        }
    }
    // shutting down: wait for in-flight chunks and hand everything back
    for (Req *r : active) {
        if (r->ev) cudaEventSynchronize(r->ev);
        std::lock_guard<std::mutex> lk(s->mu);
        s->spent.push_back(r);
    }
}

}  // namespace

extern "C" {

int hydft_serve_create(int device, double hbm_budget_bytes, int max_slots, int chunk_steps, hydft_server **out)
{
    if (!out || max_slots < 1 || chunk_steps < 1 || hbm_budget_bytes < 0) return HYDFT_ERR_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        set_thread_error("no CUDA device available (the solver has no CPU path)");
        return HYDFT_ERR_CUDA;
    }
    cudaSetDevice(device);
    auto s = std::make_unique<hydft_server>();
    s->device = device;
    s->max_slots = max_slots;
    s->chunk = chunk_steps;
    if (hbm_budget_bytes > 0) {
        s->budget = hbm_budget_bytes;
    } else {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        s->budget = 0.8 * (double)fr;
    }
    s->t0 = Clock::now();
    hydft_server *sp = s.get();
    s->setup_thread = std::thread(setup_loop, sp);
    s->sched_thread = std::thread(sched_loop, sp);
    *out = s.release();
    return HYDFT_OK;
}

int hydft_serve_submit(hydft_server *s, const hydft_params *p, const double *n, const double *mom, const double *pi,
                       int nsteps, int keep_state, int64_t *id)
{
    if (!s || !p || !id || nsteps < 0) return HYDFT_ERR_BAD_ARG;
    auto r = std::make_unique<Req>();
    r->p = *p;
    const double bytes = footprint_bytes(p);
    if (bytes < 0) {
        set_thread_error("serve: invalid grid");
        return HYDFT_ERR_BAD_ARG;
    }
    if (bytes > s->budget) {
        set_thread_error("serve: the request needs " + std::to_string((long long)bytes) +
                         " bytes of device memory, more than the server's budget of " +
                         std::to_string((long long)s->budget));
        return HYDFT_ERR_OOM;
    }
    r->bytes = bytes;
    r->nsteps = nsteps;
    r->keep_state = keep_state != 0;
    if (n) {
        const size_t nc = (size_t)p->nx * p->ny * p->nz;
        r->has_state = true;
        r->n.assign(n, n + nc);
        r->mom.assign(3 * nc, 0.0);
        if (mom) std::copy(mom, mom + 3 * nc, r->mom.begin());
        if (pi) r->pi.assign(pi, pi + 6 * nc);
    }
    Req *raw = r.get();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        raw->id = s->next_id++;
        raw->t_submit = s->now();
        *id = raw->id;
        s->queue.push_back(raw);
        s->reqs[raw->id] = std::move(r);
    }
    s->cv_setup.notify_one();
    return HYDFT_OK;
}

int hydft_serve_wait(hydft_server *s, int64_t id, double timeout_s, int *state)
{
    if (!s) return HYDFT_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return HYDFT_ERR_BAD_ARG;
    Req *r = it->second.get();
    auto fin = [&] { return r->state == HYDFT_REQ_DONE || r->state == HYDFT_REQ_FAILED; };
    if (timeout_s < 0)
        s->cv_done.wait(lk, fin);
    else
        s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), fin);
    if (state) *state = r->state;
    return HYDFT_OK;
}

int hydft_serve_result(hydft_server *s, int64_t id, double *n, double *mom, double *pi, double *info)
{
    if (!s) return HYDFT_ERR_BAD_ARG;
    Req *r = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end() || it->second->collecting) return HYDFT_ERR_BAD_ARG;
        r = it->second.get();
        if (r->state != HYDFT_REQ_DONE && r->state != HYDFT_REQ_FAILED) return HYDFT_ERR_BAD_ARG;
        r->collecting = true;
    }
    // a finished request's results no longer change, and it is not deleted
    // before it is marked collected below
    if (info) std::memcpy(info, r->info, sizeof r->info);
    const int rc = r->rc;
    if (rc) {
        set_thread_error("request " + std::to_string((long long)id) + ": " + r->err);
    } else {
        if (n && !r->out_n.empty()) std::copy(r->out_n.begin(), r->out_n.end(), n);
        if (mom && !r->out_mom.empty()) std::copy(r->out_mom.begin(), r->out_mom.end(), mom);
        if (pi && !r->out_pi.empty()) std::copy(r->out_pi.begin(), r->out_pi.end(), pi);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    r->collected = true;
    if (r->released) s->reqs.erase(id);
    return rc;
}

int hydft_serve_stats(hydft_server *s, double *stats)
{
    if (!s || !stats) return HYDFT_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    stats[0] = (double)s->queue.size();
    stats[1] = (double)s->holding;
    stats[2] = (double)s->completed;
    stats[3] = (double)s->max_holding;
    stats[4] = s->used;
    stats[5] = s->budget;
    return HYDFT_OK;
}

void hydft_serve_destroy(hydft_server *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_sched.notify_all();
    if (s->sched_thread.joinable()) s->sched_thread.join();
    s->cv_setup.notify_all();
    if (s->setup_thread.joinable()) s->setup_thread.join();
    // models still held (set up but never scheduled, or handed back at stop)
    for (Req *r : s->ready) s->spent.push_back(r);
    s->ready.clear();
    for (Req *r : s->spent) release(s, r);
    s->spent.clear();
    delete s;
}

}  // extern "C"
