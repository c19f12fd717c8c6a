// Serving loop: solve requests of different scenes, sizes and right-hand-side counts as they
// arrive, several co-resident on one GPU.
//
// Each request is copied at submission and queued first-in first-out.  Worker threads (as many as
// requests may run at once) take the head of the queue when its device footprint fits beside the
// requests already running (admission by HBM footprint); a request larger than the whole budget is
// refused.  A running request owns its own handle, CUDA stream, operator tables and Krylov state,
// so co-resident solves overlap on the GPU and each result is the one the request would get alone
// (no state or reduction is shared between requests).  A request with several right-hand sides
// solves them as one block (foggy_solve_block), so they share every operator application.
// Results stay with the server until released.  The reference has no serving layer; the solve each request runs is
// lib_mie_ms_solver_run (FoggySim/src/lib/mie_theory/lib_mie_ms_solver_interface.f90:143-154).
#include <algorithm>
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

#include <cuda_runtime.h>

#include "foggy_internal.h"

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    foggy_params prm{};
    int N = 0, NP = 0, nw = 0, per_wave = 0;
    std::vector<double> centres, mref, radius, theta, phi, jones, g, phase, d0;
    std::vector<int32_t> pidx, nr;
    int64_t footprint = 0;
    int state = FOGGY_REQ_QUEUED;
    int32_t status = FOGGY_OK;
    int nrhs = 1;
    std::vector<double> x, cs;   // nrhs solutions (reference layout) and cross-sections
    foggy_stats stats{};
    double t_submit = 0, t_start = 0, t_end = 0;
    std::string error;
};

bool terminal(int state) { return state >= FOGGY_REQ_DONE; }

}  // namespace

struct foggy_server_s {
    int device = 0;
    int64_t budget = 0;
    int64_t in_flight = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> queue;
    std::map<int64_t, std::shared_ptr<Request>> reqs;
    std::vector<std::thread> workers;
    bool stopping = false;
    int64_t next_id = 1;
    std::string last_error;
};

namespace {

// the solve of one admitted request, on its own handle
void run_request(foggy_server_s* S, Request& r) {
    foggy_handle h = nullptr;
    foggy_params prm = r.prm;
    prm.device_memory_budget = r.footprint;
    auto done = [&](int32_t rc) {
        if (rc != FOGGY_OK && r.error.empty()) r.error = foggy_last_error(h);
        if (h) foggy_destroy(h);
        return rc;
    };
    int32_t rc = foggy_create(&prm, S->device, &h);
    if (rc != FOGGY_OK) {
        r.error = foggy_last_error(nullptr);
        r.status = rc;
        return;
    }
    rc = foggy_set_spheres(h, r.N, r.centres.data(), r.pidx.data(), r.NP, r.mref.data(), r.radius.data(), r.nr.data());
    if (rc == FOGGY_OK)
        rc = foggy_set_plane_waves(h, r.nw, r.theta.data(), r.phi.data(), r.jones.data(), r.g.data(), r.phase.data(),
                                   r.d0.data());
    if (rc != FOGGY_OK) {
        r.status = done(rc);
        return;
    }
    const int64_t len = foggy_vector_length(h);
    r.nrhs = r.per_wave ? r.nw : 1;
    r.x.assign((size_t)(2 * len * r.nrhs), 0.0);
    r.cs.assign((size_t)(3 * r.nrhs), 0.0);
    if (r.per_wave && r.nw > 1) {
        // the request's right-hand sides share every operator application
        rc = foggy_solve_block(h, r.nw, nullptr, r.x.data(), FOGGY_MEM_HOST, &r.stats, r.cs.data(), nullptr, nullptr);
    } else if (r.per_wave) {
        rc = foggy_solve_rhs(h, r.nw, nullptr, r.x.data(), FOGGY_MEM_HOST, &r.stats, r.cs.data());
    } else {
        rc = foggy_solve(h, nullptr, r.x.data(), FOGGY_MEM_HOST, &r.stats);
        if (rc == FOGGY_OK) rc = foggy_cross_sections(h, r.x.data(), FOGGY_MEM_HOST, r.cs.data());
    }
    r.status = done(rc);
}

void worker(foggy_server_s* S) {
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            for (;;) {
                if (S->stopping) return;
                if (!S->queue.empty()) {
                    auto it = S->reqs.find(S->queue.front());
                    Request& q = *it->second;
                    if (q.footprint > S->budget) {   // never fits: refuse, keep the queue moving
                        S->queue.pop_front();
                        q.state = FOGGY_REQ_REFUSED;
                        q.status = FOGGY_ERR_NOMEM;
                        q.error = "request needs " + std::to_string(q.footprint) + " device bytes, the server has " +
                                  std::to_string(S->budget);
                        q.t_end = now_ms();
                        S->cv_done.notify_all();
                        continue;
                    }
                    if (S->in_flight + q.footprint <= S->budget) {
                        S->queue.pop_front();
                        S->in_flight += q.footprint;
                        q.state = FOGGY_REQ_RUNNING;
                        q.t_start = now_ms();
                        r = it->second;
                        break;
                    }
                }
                // nothing to do, or the head waits for memory held by running requests
                S->cv_work.wait(lk);
            }
        }
        run_request(S, *r);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->in_flight -= r->footprint;
            r->t_end = now_ms();
            r->state = r->status == FOGGY_OK ? FOGGY_REQ_DONE : FOGGY_REQ_FAILED;
        }
        S->cv_work.notify_all();
        S->cv_done.notify_all();
    }
}

template <class T>
std::vector<T> copy_of(const T* p, size_t n) {
    return p ? std::vector<T>(p, p + n) : std::vector<T>(n, T(0));
}

}  // namespace

extern "C" {

int32_t foggy_server_start(int32_t device, int32_t max_concurrent, int64_t memory_budget, foggy_server* out) {
    if (!out || max_concurrent < 1 || max_concurrent > 64) return FOGGY_ERR_ARGUMENT;
    auto* S = new (std::nothrow) foggy_server_s();
    if (!S) return FOGGY_ERR_NOMEM;
    S->device = device;
    if (memory_budget <= 0) {
        size_t fr = 0, tot = 0;
        if (cudaSetDevice(device) == cudaSuccess && cudaMemGetInfo(&fr, &tot) == cudaSuccess)
            memory_budget = (int64_t)(0.85 * (double)fr);
        else
            memory_budget = 0;   // no device: every request fails when it runs
    }
    S->budget = memory_budget;
    for (int i = 0; i < max_concurrent; ++i) S->workers.emplace_back(worker, S);
    *out = S;
    return FOGGY_OK;
}

int32_t foggy_server_submit(foggy_server S, const foggy_request* q, int64_t* id) {
    if (!S || !q || !id || !q->params) return FOGGY_ERR_ARGUMENT;
    if (q->n_spheres < 1 || q->n_param < 1 || q->nw < 1 || !q->centres || !q->param_index || !q->refractive_index ||
        !q->radius || !q->n_range || !q->theta || !q->phi || !q->jones || !q->g)
        return FOGGY_ERR_ARGUMENT;
    for (int j = 0; j < q->n_spheres; ++j)
        if (q->param_index[j] < 0 || q->param_index[j] >= q->n_param) return FOGGY_ERR_ARGUMENT;
    auto r = std::make_shared<Request>();
    r->prm = *q->params;
    r->N = q->n_spheres;
    r->NP = q->n_param;
    r->nw = q->nw;
    r->per_wave = q->rhs_per_wave ? 1 : 0;
    r->centres = copy_of(q->centres, 3 * (size_t)q->n_spheres);
    r->pidx = copy_of(q->param_index, (size_t)q->n_spheres);
    r->mref = copy_of(q->refractive_index, 2 * (size_t)q->n_param);
    r->radius = copy_of(q->radius, (size_t)q->n_param);
    r->nr = copy_of(q->n_range, 2 * (size_t)q->n_param);
    r->theta = copy_of(q->theta, (size_t)q->nw);
    r->phi = copy_of(q->phi, (size_t)q->nw);
    r->jones = copy_of(q->jones, 4 * (size_t)q->nw);
    r->g = copy_of(q->g, (size_t)q->nw);
    r->phase = copy_of(q->phase, (size_t)q->nw);
    r->d0 = copy_of(q->d_0_i, 3 * (size_t)q->nw);
    // pair tables when they take at most an equal share of the budget beside the solve itself
    int64_t tb = 0;
    const int64_t base = foggy::estimate_solve_bytes(r->prm, r->N, r->pidx.data(), r->NP, r->nr.data(), 0, &tb);
    const int share = (int)std::max<size_t>(1, S->workers.size());
    bool tables = r->prm.pair_tables == 1 || (r->prm.pair_tables == 0 && base + tb <= S->budget / share);
    r->prm.pair_tables = tables ? 1 : -1;
    r->footprint = base + (tables ? tb : 0) +
                   (r->per_wave && r->nw > 1
                        ? foggy::estimate_block_bytes(r->prm, r->N, r->pidx.data(), r->NP, r->nr.data(), r->nw)
                        : 0);
    r->prm.matvec_mode = FOGGY_MATVEC_DIRECT;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) return FOGGY_ERR_STATE;
        r->id = S->next_id++;
        r->t_submit = now_ms();
        S->reqs[r->id] = r;
        S->queue.push_back(r->id);
        *id = r->id;
    }
    S->cv_work.notify_all();
    return FOGGY_OK;
}

int32_t foggy_server_poll(foggy_server S, int64_t id, int32_t wait_ms, foggy_request_info* info, double* x,
                          int64_t x_len, double* cross_sections) {
    if (!S || !info) return FOGGY_ERR_ARGUMENT;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return FOGGY_ERR_ARGUMENT;
    std::shared_ptr<Request> r = it->second;
    if (wait_ms != 0 && !terminal(r->state)) {
        auto pred = [&] { return terminal(r->state); };
        if (wait_ms < 0)
            S->cv_done.wait(lk, pred);
        else
            S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), pred);
    }
    std::memset(info, 0, sizeof(*info));
    info->state = r->state;
    info->footprint = r->footprint;
    const double t_now = now_ms();
    info->ms_queued = ((r->t_start > 0) ? r->t_start : (terminal(r->state) ? r->t_end : t_now)) - r->t_submit;
    info->ms_solve = (r->t_start > 0) ? ((r->t_end > 0 ? r->t_end : t_now) - r->t_start) : 0.0;
    info->ms_latency = (terminal(r->state) ? r->t_end : t_now) - r->t_submit;
    // the worker writes the results without the lock while the request runs and publishes them
    // by setting a terminal state under it, so they are read only from then on
    if (!terminal(r->state)) return FOGGY_OK;
    info->status = r->status;
    info->nrhs = r->nrhs;
    info->x_len = (int64_t)r->x.size();
    info->stats = r->stats;
    std::strncpy(info->error, r->error.c_str(), sizeof(info->error) - 1);
    if (r->state == FOGGY_REQ_DONE) {
        if (x) {
            if (x_len < (int64_t)r->x.size()) return FOGGY_ERR_ARGUMENT;
            std::memcpy(x, r->x.data(), r->x.size() * sizeof(double));
        }
        if (cross_sections) std::memcpy(cross_sections, r->cs.data(), r->cs.size() * sizeof(double));
    }
    return FOGGY_OK;
}

int32_t foggy_server_cancel(foggy_server S, int64_t id) {
    if (!S) return FOGGY_ERR_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->reqs.find(id);
        if (it == S->reqs.end()) return FOGGY_ERR_ARGUMENT;
        Request& r = *it->second;
        if (r.state != FOGGY_REQ_QUEUED) return FOGGY_ERR_STATE;   // running or finished
        S->queue.erase(std::find(S->queue.begin(), S->queue.end(), id));
        r.state = FOGGY_REQ_CANCELLED;
        r.status = FOGGY_ERR_STATE;
        r.t_end = now_ms();
    }
    S->cv_work.notify_all();
    S->cv_done.notify_all();
    return FOGGY_OK;
}

int32_t foggy_server_release(foggy_server S, int64_t id) {
    if (!S) return FOGGY_ERR_ARGUMENT;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return FOGGY_ERR_ARGUMENT;
    if (!terminal(it->second->state)) return FOGGY_ERR_STATE;
    S->reqs.erase(it);
    return FOGGY_OK;
}

int32_t foggy_server_stop(foggy_server S) {
    if (!S) return FOGGY_ERR_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        // queued requests never start; running ones finish
        for (int64_t id : S->queue) {
            Request& r = *S->reqs[id];
            r.state = FOGGY_REQ_CANCELLED;
            r.status = FOGGY_ERR_STATE;
        }
        S->queue.clear();
    }
    S->cv_work.notify_all();
    S->cv_done.notify_all();
    for (auto& t : S->workers) t.join();
    delete S;
    return FOGGY_OK;
}

}  // extern "C"
