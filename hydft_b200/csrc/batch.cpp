// Ensembles: many independent simulations (different grids, Gamma, kappa,
// closures) advanced together by one CUDA graph launch per step.
//
// Each member is a full hydft_gpu handle with its own device state, work
// buffers and stream.  The ensemble captures one RK3 step of every member
// into a single graph: a fork event on the ensemble's root stream, each
// member's step kernels on its own stream, and a join back to the root, so
// the members are independent branches that the GPU runs concurrently (a
// 32^3 member alone cannot fill 148 SMs; hundreds of them side by side
// can).  Replaying the graph advances every member by one step with one
// launch.  The reference runs one model_t per process (src/hydft.f90:41-51,
// the loop every member follows); this grouping has no counterpart there.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hydft_gpu.h"
#include "handle.hpp"

using namespace hydft;

// Members whose steps record the same launches (kernel kinds and shapes)
// step together: each launch of the step runs once for the whole group, on
// the group's stream, with the members' arguments (packs) as kernel
// parameters.
struct EnsembleGroup {
    std::vector<int> members;
    std::vector<LaunchRec> recs;     // the first member's launches (kinds and shapes)
    std::vector<std::vector<unsigned char>> packs;   // per launch: the members' packs back to back
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
};

struct hydft_batch {
    std::vector<hydft_gpu *> m;
    int device = 0;
    cudaStream_t root = nullptr;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t gexec = nullptr;
    std::vector<int64_t> gens;           // member graph generations at capture
    std::vector<int64_t> step_launches;  // kernels of one member step, as the member alone would launch them
    std::vector<EnsembleGroup> groups;
    std::vector<int> solo;               // members stepping on their own stream (no ensemble form)
    int64_t graph_kernels = 0;           // kernels per graph launch
    int64_t launches = 0;                // kernels launched by this ensemble's graph so far
    unsigned *hstat = nullptr;           // pinned status words, one per member
    int failed = -1;
    std::string err;
};

namespace {

struct CachedStructure {
    std::vector<double> k, c;
    double u_ex = 0, du_dgamma = 0;
    int has_energy = 0;
};

// members whose HNC inputs agree share one solve
std::string hnc_key(const hydft_params &p)
{
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s|%.17g|%.17g|%.17g|%.17g|%.17g|%d|%.17g|%.17g|%.17g|%d|%s|%s", p.kind, p.gamma,
                  p.kappa, p.rs, p.theta, p.mass, p.hnc_nr, p.hnc_rmax, p.hnc_tol, p.hnc_mix, p.hnc_maxiter,
                  p.structure, p.structure_kind);
    return buf;
}

int fail(hydft_batch *b, int rc, const std::string &msg)
{
    b->err = msg;
    return rc;
}

void destroy_member(hydft_gpu *h)
{
    if (!h) return;
    if (h->s) {
        cudaSetDevice(h->device);
        delete h->s;
    }
    delete h;
}

void drop_groups(hydft_batch *b)
{
    for (auto &g : b->groups) {
        if (g.done) cudaEventDestroy(g.done);
        if (g.st) cudaStreamDestroy(g.st);
    }
    b->groups.clear();
    b->solo.clear();
}

void drop_graph(hydft_batch *b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
}

// the launch kinds and shapes of a recorded step, as a grouping key
std::string step_signature(const std::vector<LaunchRec> &recs)
{
    std::string k;
    char buf[160];
    for (const LaunchRec &r : recs) {
        std::snprintf(buf, sizeof buf, "%p:%u,%u,%u:%u,%u,%u:%zu:%zu;", r.kind, r.grid.x, r.grid.y, r.grid.z, r.block.x,
                      r.block.y, r.block.z, r.smem, r.pack.size());
        k += buf;
    }
    return k;
}

// Records every member's step, groups members with the same launches and
// gathers their packs; members without an ensemble form step alone.
int build_groups(hydft_batch *b)
{
    drop_groups(b);
    const size_t n = b->m.size();
    std::vector<std::vector<LaunchRec>> recs(n);
    std::map<std::string, size_t> key_to_group;
    for (size_t i = 0; i < n; ++i) {
        const int rc = b->m[i]->s->record_step(recs[i]);
        if (rc == HYDFT_ERR_UNSUPPORTED) {
            b->solo.push_back((int)i);
            continue;
        }
        if (rc) return fail(b, rc, "member " + std::to_string(i) + ": " + b->m[i]->s->err);
        const std::string key = step_signature(recs[i]);
        auto it = key_to_group.find(key);
        if (it == key_to_group.end()) {
            key_to_group[key] = b->groups.size();
            b->groups.emplace_back();
            b->groups.back().recs = recs[i];
            it = key_to_group.find(key);
        }
        b->groups[it->second].members.push_back((int)i);
    }
    // per launch per group: the members' packs back to back
    for (auto &g : b->groups) {
        g.packs.resize(g.recs.size());
        for (size_t r = 0; r < g.recs.size(); ++r) {
            const size_t sz = g.recs[r].pack.size();
            g.packs[r].assign(sz * g.members.size(), 0);
            for (size_t j = 0; j < g.members.size(); ++j)
                std::memcpy(g.packs[r].data() + j * sz, recs[g.members[j]][r].pack.data(), sz);
        }
    }
    for (auto &g : b->groups) {
        if (cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming) != cudaSuccess)
            return fail(b, HYDFT_ERR_CUDA, "ensemble: group stream or event creation failed");
        for (const LaunchRec &r : g.recs) {
            cudaError_t e = r.prepare(r.smem);
            if (e != cudaSuccess) return fail(b, HYDFT_ERR_CUDA, std::string("ensemble: ") + cudaGetErrorString(e));
        }
        for (int i : g.members) b->step_launches[i] = (int64_t)recs[i].size();
    }
    return HYDFT_OK;
}

// one graph: fork -> each group's launches on its stream, and each member
// without an ensemble form on its own stream -> join
int capture(hydft_batch *b)
{
    drop_graph(b);
    const size_t n = b->m.size();
    for (size_t i = 0; i < n; ++i)
        if (int rc = b->m[i]->s->prepare()) return fail(b, rc, "member " + std::to_string(i) + ": " + b->m[i]->s->err);
    if (int rc = build_groups(b)) return rc;
    std::vector<int64_t> before(n);
    for (size_t i = 0; i < n; ++i) before[i] = b->m[i]->s->launches;
    cudaError_t e = cudaStreamBeginCapture(b->root, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(b, HYDFT_ERR_CUDA, std::string("begin capture: ") + cudaGetErrorString(e));
    cudaEventRecord(b->fork, b->root);
    int64_t kernels = 0;
    for (auto &g : b->groups) {
        cudaStreamWaitEvent(g.st, b->fork, 0);
        for (size_t r = 0; r < g.recs.size(); ++r) {
            const LaunchRec &lr = g.recs[r];
            lr.launch(g.packs[r].data(), (unsigned)g.members.size(), lr.grid, lr.block, lr.smem, g.st);
            const cudaError_t le = cudaGetLastError();
            if (le != cudaSuccess) {
                cudaGraph_t dead = nullptr;
                cudaStreamEndCapture(b->root, &dead);
                if (dead) cudaGraphDestroy(dead);
                char buf[256];
                std::snprintf(buf, sizeof buf, "ensemble launch %zu (%s) of %zu members, grid %u x %u x %u, block %u, "
                              "%zu bytes shared: ", r, lr.name, g.members.size(), lr.grid.x, lr.grid.y, lr.grid.z,
                              lr.block.x, lr.smem);
                return fail(b, HYDFT_ERR_CUDA, buf + std::string(cudaGetErrorString(le)));
            }
        }
        for (const LaunchRec &lr : g.recs)
            kernels += (int64_t)((g.members.size() + lr.per_launch - 1) / lr.per_launch);
        cudaEventRecord(g.done, g.st);
        cudaStreamWaitEvent(b->root, g.done, 0);
    }
    for (int i : b->solo) {
        cudaStream_t s = static_cast<cudaStream_t>(b->m[i]->s->stream());
        cudaStreamWaitEvent(s, b->fork, 0);
        b->m[i]->s->enqueue_steps(1);
        cudaEventRecord(b->join[i], s);
        cudaStreamWaitEvent(b->root, b->join[i], 0);
    }
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->root, &g);
    if (e != cudaSuccess) return fail(b, HYDFT_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(b, HYDFT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    for (int i : b->solo) {
        b->step_launches[i] = b->m[i]->s->launches - before[i];
        b->m[i]->s->launches = before[i];
        kernels += b->step_launches[i];
    }
    for (size_t i = 0; i < n; ++i) b->gens[i] = b->m[i]->s->graph_gen;
    b->graph_kernels = kernels;
    return HYDFT_OK;
}

}  // namespace

extern "C" {

int hydft_batch_create(int n, const hydft_params *params, const hydft_structure *structures, int device,
                       hydft_batch **out)
{
    if (n < 1 || !params || !out) return HYDFT_ERR_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        set_thread_error("no CUDA device available (the solver has no CPU path)");
        return HYDFT_ERR_CUDA;
    }
    cudaSetDevice(device);
    auto b = std::make_unique<hydft_batch>();
    b->device = device;
    // Members are built on several host threads (the setup kernels run on
    // each thread's own default stream, so the HNC solves of different
    // members overlap on the device).  Members whose HNC inputs agree share
    // one solve: one member per distinct input is built first, the others
    // then take its structure table.
    std::vector<hydft_gpu *> hs(n, nullptr);
    std::vector<int> rcs(n, 0);
    std::vector<std::string> errs(n);
    std::vector<std::string> keys(n);
    std::map<std::string, int> first;   // key -> the member that solves it
    std::vector<int> wave1, wave2;
    for (int i = 0; i < n; ++i) {
        keys[i] = hnc_key(params[i]);
        const bool given = structures && structures[i].n > 0;
        const bool hnc = std::string(params[i].structure) == "hnc";
        if (!given && hnc) {
            auto it = first.find(keys[i]);
            if (it == first.end()) {
                first[keys[i]] = i;
                wave1.push_back(i);
            } else {
                wave2.push_back(i);
            }
        } else {
            wave1.push_back(i);
        }
    }
    std::map<std::string, CachedStructure> cache;
    auto build = [&](int i, const hydft_structure *sp) {
        cudaSetDevice(device);
        rcs[i] = hydft_gpu_create(&params[i], sp, device, &hs[i]);
        if (rcs[i]) errs[i] = hydft_gpu_create_error();
    };
    auto run_wave = [&](const std::vector<int> &wave, bool cached) {
        const int nth = std::max(1, std::min<int>((int)wave.size(), std::min(16u, std::max(1u, std::thread::hardware_concurrency()))));
        std::atomic<int> next{0};
        auto worker = [&]() {
            for (int w; (w = next.fetch_add(1)) < (int)wave.size();) {
                const int i = wave[w];
                hydft_structure st{};
                const hydft_structure *sp = nullptr;
                if (structures && structures[i].n > 0) {
                    sp = &structures[i];
                } else if (cached) {
                    const CachedStructure &c = cache.at(keys[i]);
                    st.n = (int)c.k.size();
                    st.k = c.k.data();
                    st.c = c.c.data();
                    st.u_ex = c.u_ex;
                    st.du_dgamma = c.du_dgamma;
                    st.has_energy = c.has_energy;
                    sp = &st;
                }
                build(i, sp);
            }
        };
        std::vector<std::thread> ths;
        for (int k = 0; k < nth; ++k) ths.emplace_back(worker);
        for (auto &th : ths) th.join();
    };
    auto cleanup = [&]() {
        for (auto *h : hs) destroy_member(h);
    };
    auto first_error = [&]() -> int {
        for (int i = 0; i < n; ++i)
            if (rcs[i]) {
                cleanup();
                set_thread_error("member " + std::to_string(i) + ": " + errs[i]);
                return rcs[i];
            }
        return 0;
    };
    run_wave(wave1, false);
    if (int rc = first_error()) return rc;
    for (auto &kv : first) {
        const hydft_gpu *h = hs[kv.second];
        if (!h->mh.has_st) continue;
        CachedStructure c;
        c.k = h->mh.st_k;
        c.c = h->mh.st_c;
        c.u_ex = h->mh.u_ex;
        c.du_dgamma = h->mh.du_dgamma;
        c.has_energy = h->mh.has_energy ? 1 : 0;
        cache[kv.first] = std::move(c);
    }
    // a key whose first member found no table: the others solve themselves
    std::vector<int> cached2, solve2;
    for (int i : wave2) (cache.count(keys[i]) ? cached2 : solve2).push_back(i);
    run_wave(cached2, true);
    run_wave(solve2, false);
    if (int rc = first_error()) return rc;
    for (int i = 0; i < n; ++i) {
        hs[i]->owned_by_batch = true;
        b->m.push_back(hs[i]);
    }
    auto cleanup_members = [&]() {
        for (auto *h : b->m) destroy_member(h);
        b->m.clear();
    };
    cudaSetDevice(device);
    if (cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&b->hstat, sizeof(unsigned) * n) != cudaSuccess) {
        cleanup_members();
        set_thread_error("ensemble: stream, event or pinned buffer creation failed");
        return HYDFT_ERR_CUDA;
    }
    b->join.resize(n);
    for (int i = 0; i < n; ++i)
        if (cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) != cudaSuccess) {
            cleanup_members();
            set_thread_error("ensemble: event creation failed");
            return HYDFT_ERR_CUDA;
        }
    b->gens.assign(n, -1);
    b->step_launches.assign(n, 0);
    *out = b.release();
    return HYDFT_OK;
}

void hydft_batch_destroy(hydft_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->root) cudaStreamSynchronize(b->root);
    drop_graph(b);
    drop_groups(b);
    for (auto *h : b->m) destroy_member(h);
    for (auto e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->done) cudaEventDestroy(b->done);
    if (b->root) cudaStreamDestroy(b->root);
    if (b->hstat) cudaFreeHost(b->hstat);
    delete b;
}

int hydft_batch_size(const hydft_batch *b) { return b ? (int)b->m.size() : 0; }

int hydft_batch_member(hydft_batch *b, int i, hydft_gpu **member)
{
    if (!b || !member || i < 0 || i >= (int)b->m.size()) return HYDFT_ERR_BAD_ARG;
    *member = b->m[i];
    return HYDFT_OK;
}

const char *hydft_batch_last_error(const hydft_batch *b) { return b ? b->err.c_str() : ""; }

int hydft_batch_failed_member(const hydft_batch *b) { return b ? b->failed : -1; }

int hydft_batch_advance(hydft_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return HYDFT_ERR_BAD_ARG;
    if (nsteps == 0) return HYDFT_OK;
    cudaSetDevice(b->device);
    const size_t n = b->m.size();
    b->failed = -1;
    for (size_t i = 0; i < n; ++i) {
        double t, dt;
        int64_t s;
        b->m[i]->s->get_time(&t, &dt, &s);
        if (!(dt > 0.0)) {
            b->failed = (int)i;
            return fail(b, HYDFT_ERR_BAD_ARG, "member " + std::to_string(i) + ": dt is not set (call compute_dt)");
        }
    }
    bool stale = !b->gexec;
    for (size_t i = 0; i < n && !stale; ++i) stale = b->gens[i] != b->m[i]->s->graph_gen;
    if (stale)
        if (int rc = capture(b)) return rc;
    // the graph starts after whatever the members' own streams hold
    for (size_t i = 0; i < n; ++i) {
        cudaStream_t s = static_cast<cudaStream_t>(b->m[i]->s->stream());
        cudaEventRecord(b->join[i], s);
        cudaStreamWaitEvent(b->root, b->join[i], 0);
    }
    for (int k = 0; k < nsteps; ++k) {
        cudaError_t e = cudaGraphLaunch(b->gexec, b->root);
        if (e != cudaSuccess) return fail(b, HYDFT_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
    }
    b->launches += b->graph_kernels * nsteps;
    for (size_t i = 0; i < n; ++i) {
        b->m[i]->s->launches += b->step_launches[i] * nsteps;
        cudaMemcpyAsync(b->hstat + i, b->m[i]->s->status_word(), sizeof(unsigned), cudaMemcpyDeviceToHost, b->root);
    }
    // later work on the members' streams follows the graph
    cudaEventRecord(b->done, b->root);
    for (size_t i = 0; i < n; ++i)
        cudaStreamWaitEvent(static_cast<cudaStream_t>(b->m[i]->s->stream()), b->done, 0);
    cudaError_t e = cudaStreamSynchronize(b->root);
    if (e != cudaSuccess) return fail(b, HYDFT_ERR_CUDA, std::string("ensemble step: ") + cudaGetErrorString(e));
    for (size_t i = 0; i < n; ++i) {
        // time and step count live on the device and advanced with the graph
        b->m[i]->s->mark_advanced();
        if (b->hstat[i]) {
            const int rc = b->m[i]->s->take_status(b->hstat[i]);
            if (rc) {
                b->failed = (int)i;
                return fail(b, rc, "member " + std::to_string(i) + ": " + b->m[i]->s->err);
            }
        }
    }
    return HYDFT_OK;
}

int64_t hydft_batch_launch_count(const hydft_batch *b) { return b ? b->launches : 0; }

int hydft_batch_grouped(const hydft_batch *b, int *groups, int *members)
{
    if (!b) return HYDFT_ERR_BAD_ARG;
    int nm = 0;
    for (const auto &g : b->groups) nm += (int)g.members.size();
    if (groups) *groups = (int)b->groups.size();
    if (members) *members = nm;
    return HYDFT_OK;
}

void *hydft_batch_stream(const hydft_batch *b) { return b ? (void *)b->root : nullptr; }

}  // extern "C"
