// mgp_batch.cu -- many independent solves at once: a batch of resident
// hierarchies solved concurrently, and a request server that admits solves
// as slots and device memory free up (continuous batching).
//
// Neither has a counterpart in the Fortran library, which solves one problem
// per call.  Both run the single-problem solver unchanged: concurrency comes
// from host workers that each own a CUDA stream, so the latency-bound kernels
// of different problems (the small levels, the single-CTA coarse cycle)
// overlap on the device.  A problem's kernels, their order and its
// reductions do not depend on what else runs, so every result is identical
// alone and in the mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mgp2d.h"
#include "mgp_kernels.cuh"

namespace mgp {
int record_error(int code, const char* msg);
int solver_create_on(const mgp_box* valid, const mgp_geo* geo, const mgp_bdry* bc, int kind, int flags,
                     int maxdepth_user, cudaStream_t st, mgp_solver** out);
size_t solver_device_bytes(const mgp_solver* s);
size_t solver_pool_cached_bytes();
struct Lockstep;
Lockstep* lockstep_new();
void lockstep_free(Lockstep* ls);
bool lockstep_ok(const std::vector<mgp_solver*>& ss, int numcycles, int nd, int nu);
int lockstep_vcycle(const std::vector<mgp_solver*>& ss, Lockstep* ls, mgp_array* phi, mgp_array* rhs,
                    const mgp_bdry* bc, int homog, double tol, int maxiters, int nd, int nu, int nb, int zerophi,
                    mgp_report* reports, cudaStream_t st, int pairs);
}  // namespace mgp

using namespace mgp;

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device bytes a hierarchy of nx x ny cells takes, before it exists: FP64
// fields ~21 per cell over all levels (geometry, inverse diagonal,
// corrections, residuals, the BiCGStab vectors), FP32 copies ~14, with
// MGP_FLAG_GMRES the 2m + 1 = 257 stored fields of GMRES(128), plus padding
// and the small buffers.
size_t estimate_bytes(const mgp_box* v, int flags) {
    const double n = (double)v->nx * (double)v->ny;
    const double per = 8.0 * 21.0 + ((flags & MGP_FLAG_MIXED) ? 4.0 * 14.0 : 0.0) +
                       ((flags & MGP_FLAG_GMRES) ? 8.0 * 257.0 : 0.0);
    return (size_t)(n * per) + ((size_t)8 << 20);
}

}  // namespace

// ===========================================================================
// Batch
// ===========================================================================
struct mgp_batch {
    int dev = 0;
    int nstreams = 1;
    int flags = 0;
    std::vector<mgp_solver*> solvers;
    std::vector<cudaStream_t> streams;
    std::vector<Lockstep*> lockstep;   // MGP_FLAG_LOCKSTEP: each group's phase-by-phase engine buffers
    // lockstep tuning (mgp_batch_set_tuning): groups (0: the default) and two sweeps per launch on small levels
    int lock_groups = 0;
    int lock_pairs = 0;
};

namespace {

// The lockstep path over up to kLockstepGroups groups of problems, each with
// its own stream, host thread and job tables, so that one group's coarse
// cycles (a CTA per problem, latency-bound) overlap another group's sweeps.
// Problems go to groups round-robin in decreasing order of cells, which
// balances the groups' work; a problem's kernels and their order are those
// of its group alone, so its bits do not depend on the grouping.
constexpr int kLockstepGroups = 4;

int batch_lockstep(mgp_batch* b, mgp_array* phi, mgp_array* rhs, const mgp_bdry* bc, int homog, double tol,
                   int maxiters, int nd, int nu, int nb, int zerophi, mgp_report* reports) {
    const int n = (int)b->solvers.size();
    const int want = b->lock_groups > 0 ? b->lock_groups : kLockstepGroups;
    const int ng = std::max(1, std::min({want, b->nstreams, n}));
    while ((int)b->lockstep.size() < ng) b->lockstep.push_back(lockstep_new());
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const mgp_solver* sx = b->solvers[x];
        const mgp_solver* sy = b->solvers[y];
        return solver_device_bytes(sx) > solver_device_bytes(sy);
    });
    std::vector<std::vector<int>> groups(ng);
    for (int k = 0; k < n; ++k) groups[k % ng].push_back(order[k]);
    std::vector<int> status(ng, MGP_OK);
    std::vector<std::string> msg(ng);
    auto run = [&](int g) {
        cudaSetDevice(b->dev);
        const std::vector<int>& ids = groups[g];
        std::vector<mgp_solver*> ss;
        std::vector<mgp_array> ph, rh;
        std::vector<mgp_bdry> bb;
        std::vector<mgp_report> rp;
        for (int i : ids) {
            ss.push_back(b->solvers[i]);
            ph.push_back(phi[i]);
            rh.push_back(rhs[i]);
            bb.push_back(bc[i]);
            mgp_report r{};
            if (reports) r.relres = reports[i].relres;
            rp.push_back(r);
        }
        status[g] = lockstep_vcycle(ss, b->lockstep[g], ph.data(), rh.data(), bb.data(), homog, tol, maxiters, nd, nu,
                                    nb, zerophi, rp.data(), b->streams[g], b->lock_pairs);
        if (status[g]) msg[g] = mgp_last_error();
        if (reports)
            for (size_t k = 0; k < ids.size(); ++k) reports[ids[k]] = rp[k];
    };
    std::vector<std::thread> pool;
    for (int g = 1; g < ng; ++g) pool.emplace_back(run, g);
    run(0);
    for (auto& t : pool) t.join();
    for (int g = 0; g < ng; ++g)
        if (status[g]) {
            record_error(status[g], msg[g].c_str());
            return status[g];
        }
    return MGP_OK;
}

}  // namespace

extern "C" {

int mgp_batch_create(int nprob, const mgp_box* valid, const mgp_geo* geo, const mgp_bdry* bc, int kind, int flags,
                     int maxdepth_user, int nstreams, mgp_batch** out) {
    if (!out || nprob <= 0 || !valid || !geo || !bc) return record_error(MGP_EINVAL, "batch_create: bad argument");
    *out = nullptr;
    mgp_batch* b = new mgp_batch();
    if (cudaGetDevice(&b->dev) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return record_error(MGP_ECUDA, "batch_create: no CUDA device");
    }
    b->nstreams = std::max(1, std::min(nstreams, nprob));
    b->flags = flags;
    for (int k = 0; k < b->nstreams; ++k) {
        cudaStream_t st;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            mgp_batch_destroy(b);
            return record_error(MGP_ECUDA, "batch_create: stream creation failed");
        }
        b->streams.push_back(st);
    }
    for (int i = 0; i < nprob; ++i) {
        mgp_solver* s = nullptr;
        const int rc = mgp_solver_create(&valid[i], &geo[i], &bc[i], kind, flags, maxdepth_user, &s);
        if (rc) {
            mgp_batch_destroy(b);
            return rc;
        }
        b->solvers.push_back(s);
    }
    *out = b;
    return MGP_OK;
}

int mgp_batch_destroy(mgp_batch* b) {
    if (!b) return MGP_OK;
    for (Lockstep* ls : b->lockstep) lockstep_free(ls);
    for (mgp_solver* s : b->solvers) mgp_solver_destroy(s);
    for (cudaStream_t st : b->streams) cudaStreamDestroy(st);
    delete b;
    return MGP_OK;
}

int mgp_batch_set_tuning(mgp_batch* b, int groups, int pairs) {
    if (!b || groups < 0 || groups > b->nstreams || pairs < 0 || pairs > 1)
        return record_error(MGP_EINVAL, "batch_set_tuning: bad argument");
    b->lock_groups = groups;
    b->lock_pairs = pairs;
    return MGP_OK;
}

int mgp_batch_get_tuning(const mgp_batch* b, int* groups, int* pairs) {
    if (!b || !groups || !pairs) return record_error(MGP_EINVAL, "batch_get_tuning: null argument");
    *groups = b->lock_groups > 0 ? b->lock_groups : std::min({kLockstepGroups, b->nstreams, (int)b->solvers.size()});
    *pairs = b->lock_pairs;
    return MGP_OK;
}

int mgp_batch_size(const mgp_batch* b, int* nprob) {
    if (!b || !nprob) return record_error(MGP_EINVAL, "batch_size: null argument");
    *nprob = (int)b->solvers.size();
    return MGP_OK;
}

int mgp_batch_vcycle(mgp_batch* b, mgp_array* phi, mgp_array* rhs, const mgp_bdry* bc, int homog, double tol,
                     int maxiters, int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
                     mgp_report* reports) {
    if (!b || !phi || !rhs || !bc) return record_error(MGP_EINVAL, "batch_vcycle: null argument");
    const int n = (int)b->solvers.size();
    if ((b->flags & MGP_FLAG_LOCKSTEP) && lockstep_ok(b->solvers, numcycles, smooth_down, smooth_up))
        return batch_lockstep(b, phi, rhs, bc, homog, tol, maxiters, smooth_down, smooth_up, smooth_bottom, zerophi,
                              reports);
    std::atomic<int> next{0};
    std::vector<int> status(n, MGP_OK);
    std::vector<std::string> msg(n);
    auto work = [&](int w) {
        cudaSetDevice(b->dev);
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            mgp_solver_set_stream(b->solvers[i], b->streams[w]);
            status[i] = mgp_solver_vcycle(b->solvers[i], &phi[i], &rhs[i], &bc[i], homog, tol, maxiters, numcycles,
                                          smooth_down, smooth_up, smooth_bottom, zerophi, 0,
                                          reports ? &reports[i] : nullptr);
            if (status[i]) msg[i] = mgp_last_error();
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < b->nstreams; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto& t : pool) t.join();
    for (int i = 0; i < n; ++i)
        if (status[i]) {
            record_error(status[i], msg[i].c_str());
            return status[i];
        }
    return MGP_OK;
}

}  // extern "C"

// ===========================================================================
// Server
// ===========================================================================
namespace {

struct Request {
    long long ticket = 0;
    unsigned long long key = 0;
    mgp_box valid{};
    mgp_geo geo{};
    mgp_bdry bc{};
    mgp_array phi{}, rhs{};
    int homog = 0, maxiters = 0, numcycles = 1, nd = 8, nu = 8, nb = 8, zerophi = 0;
    double tol = 0.0;
    std::vector<double> relres;
    mgp_report rep{};
    int status = MGP_OK;
    std::string err;
    bool done = false;
    double t_submit = 0.0, t_start = 0.0, t_end = 0.0;
};

struct Entry {   // a resident hierarchy kept for its key
    unsigned long long key;
    mgp_box valid;
    mgp_solver* s;
    size_t bytes;
    bool busy;
    double last_use;
};

}  // namespace

struct mgp_server {
    int dev = 0;
    int flags = 0;
    size_t budget = 0;
    size_t used = 0;   // bytes of hierarchies alive (running or cached)
    int running = 0;   // requests taken off the queue and not yet finished
    int holding = 0;   // of them, those whose hierarchy is admitted (its bytes count in `used`)
    bool stop = false;
    long long next_ticket = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_mem;
    std::deque<Request*> queue;
    std::map<long long, Request*> reqs;
    std::list<Entry> cache;
    std::vector<std::thread> workers;
};

namespace {

bool same_box(const mgp_box& a, const mgp_box& b) {
    return a.ilo == b.ilo && a.ihi == b.ihi && a.jlo == b.jlo && a.jhi == b.jhi && a.dx == b.dx && a.dy == b.dy;
}

// Frees the least recently used idle cached hierarchy; false if there is none.
// Called with the lock held.
bool evict_one(mgp_server* S, std::vector<mgp_solver*>& doomed) {
    auto victim = S->cache.end();
    for (auto it = S->cache.begin(); it != S->cache.end(); ++it)
        if (!it->busy && (victim == S->cache.end() || it->last_use < victim->last_use)) victim = it;
    if (victim == S->cache.end()) return false;
    S->used -= victim->bytes;
    doomed.push_back(victim->s);
    S->cache.erase(victim);
    return true;
}

void serve(mgp_server* S) {
    cudaSetDevice(S->dev);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            S->cv_work.wait(lock, [&] { return S->stop || !S->queue.empty(); });
            if (S->queue.empty()) break;   // stopping
            r = S->queue.front();
            S->queue.pop_front();
            ++S->running;
        }
        r->t_start = now_s();
        mgp_solver* sv = nullptr;
        size_t bytes = 0;
        bool cached = false;
        int rc = MGP_OK;
        std::vector<mgp_solver*> doomed;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            if (r->key) {
                for (auto& e : S->cache)
                    if (e.key == r->key && !e.busy && same_box(e.valid, r->valid)) {
                        e.busy = true;
                        sv = e.s;
                        bytes = e.bytes;
                        cached = true;
                        break;
                    }
            }
            if (!sv) {   // admission by device memory
                bytes = estimate_bytes(&r->valid, S->flags);
                if (bytes > S->budget) {   // could never fit, even with every other hierarchy gone
                    rc = record_error(MGP_ENOMEM, "server: the request's hierarchy is larger than the memory budget");
                } else {
                    // wait for memory only while some admitted request will
                    // release some; a worker waiting here holds none itself
                    while (S->used + bytes > S->budget && !S->stop) {
                        if (evict_one(S, doomed)) continue;
                        if (S->holding == 0) break;   // nothing left to free: the accounting is all there is
                        S->cv_mem.wait(lock);
                    }
                    if (S->stop) rc = record_error(MGP_EINVAL, "server: stopped before the request was admitted");
                }
                if (!rc) {
                    S->used += bytes;
                    ++S->holding;
                }
            } else {
                ++S->holding;
            }
        }
        const bool held = !rc;
        for (mgp_solver* d : doomed) mgp_solver_destroy(d);
        if (!sv && !rc) {
            rc = solver_create_on(&r->valid, &r->geo, &r->bc, MGP_KIND_MG, S->flags, -1, st, &sv);
            const size_t actual = rc ? 0 : solver_device_bytes(sv);
            std::lock_guard<std::mutex> lock(S->mu);
            S->used = S->used - bytes + actual;
            bytes = actual;
        }
        if (!rc) {
            mgp_solver_set_stream(sv, st);
            rc = mgp_solver_vcycle(sv, &r->phi, &r->rhs, &r->bc, r->homog, r->tol, r->maxiters, r->numcycles, r->nd,
                                   r->nu, r->nb, r->zerophi, 0, &r->rep);
        }
        if (rc) r->err = mgp_last_error();
        r->t_end = now_s();
        mgp_solver* drop = nullptr;
        {
            std::lock_guard<std::mutex> lock(S->mu);
            if (sv && r->key && !rc) {
                if (cached) {
                    for (auto& e : S->cache)
                        if (e.s == sv) {
                            e.busy = false;
                            e.last_use = r->t_end;
                        }
                } else {
                    S->cache.push_back(Entry{r->key, r->valid, sv, bytes, false, r->t_end});
                }
            } else if (sv) {
                if (cached) S->cache.remove_if([&](const Entry& e) { return e.s == sv; });
                S->used -= bytes;
                drop = sv;
            }
            r->status = rc;
            r->done = true;
            --S->running;
            if (held) --S->holding;
        }
        if (drop) mgp_solver_destroy(drop);
        S->cv_done.notify_all();
        S->cv_mem.notify_all();
    }
    if (st) cudaStreamDestroy(st);
}

}  // namespace

extern "C" {

int mgp_server_create(int nworkers, size_t mem_budget, int flags, mgp_server** out) {
    if (!out || nworkers <= 0) return record_error(MGP_EINVAL, "server_create: bad argument");
    *out = nullptr;
    mgp_server* S = new mgp_server();
    if (cudaGetDevice(&S->dev) != cudaSuccess) {
        cudaGetLastError();
        delete S;
        return record_error(MGP_ECUDA, "server_create: no CUDA device");
    }
    S->flags = flags;
    if (mem_budget == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            cudaGetLastError();
            delete S;
            return record_error(MGP_ECUDA, "server_create: cudaMemGetInfo failed");
        }
        fr += solver_pool_cached_bytes();   // freed solver memory the pool keeps serves new solvers too
        mem_budget = fr / 10 * 9;
    }
    S->budget = mem_budget;
    for (int w = 0; w < nworkers; ++w) S->workers.emplace_back(serve, S);
    *out = S;
    return MGP_OK;
}

int mgp_server_submit(mgp_server* S, unsigned long long key, const mgp_box* valid, const mgp_geo* geo,
                      const mgp_bdry* bc, mgp_array* phi, mgp_array* rhs, int homog, double tol, int maxiters,
                      int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
                      long long* ticket) {
    if (!S || !valid || !geo || !bc || !phi || !rhs || !ticket || maxiters < 0)
        return record_error(MGP_EINVAL, "server_submit: bad argument");
    Request* r = new Request();
    r->key = key;
    r->valid = *valid;
    r->geo = *geo;
    r->bc = *bc;
    r->phi = *phi;
    r->rhs = *rhs;
    r->homog = homog;
    r->tol = tol;
    r->maxiters = maxiters;
    r->numcycles = numcycles;
    r->nd = smooth_down;
    r->nu = smooth_up;
    r->nb = smooth_bottom;
    r->zerophi = zerophi;
    r->relres.assign((size_t)maxiters + 1, 0.0);
    r->rep.relres = r->relres.data();
    r->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lock(S->mu);
        if (S->stop) {
            delete r;
            return record_error(MGP_EINVAL, "server_submit: server is stopping");
        }
        r->ticket = S->next_ticket++;
        S->reqs[r->ticket] = r;
        S->queue.push_back(r);
    }
    *ticket = r->ticket;
    S->cv_work.notify_one();
    return MGP_OK;
}

int mgp_server_wait(mgp_server* S, long long ticket, mgp_report* report, double* latency_s, double* queue_s) {
    if (!S) return record_error(MGP_EINVAL, "server_wait: null server");
    Request* r = nullptr;
    {
        std::unique_lock<std::mutex> lock(S->mu);
        auto it = S->reqs.find(ticket);
        if (it == S->reqs.end()) return record_error(MGP_EINVAL, "server_wait: unknown ticket");
        r = it->second;
        S->cv_done.wait(lock, [&] { return r->done; });
        S->reqs.erase(it);
    }
    if (report) {
        double* dst = report->relres;
        *report = r->rep;
        report->relres = dst;
        if (dst)
            for (int k = 0; k <= r->rep.iterations && k <= r->maxiters; ++k) dst[k] = r->relres[k];
    }
    if (latency_s) *latency_s = r->t_end - r->t_submit;
    if (queue_s) *queue_s = r->t_start - r->t_submit;
    const int rc = r->status;
    if (rc) record_error(rc, r->err.c_str());
    delete r;
    return rc;
}

int mgp_server_destroy(mgp_server* S) {
    if (!S) return MGP_OK;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    S->cv_mem.notify_all();
    for (auto& t : S->workers) t.join();
    for (auto& e : S->cache) mgp_solver_destroy(e.s);
    for (auto& kv : S->reqs) delete kv.second;
    delete S;
    return MGP_OK;
}

}  // extern "C"
