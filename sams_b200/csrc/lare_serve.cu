// lare_serve.cu -- continuous batching of LARE3D solves under an HBM budget.
//
// Requests (a full solve: parameters, boundary conditions, initial state and
// a step count) arrive at any time.  A scheduler thread owns one Batch and
// loops:
//   1. admit queued requests in arrival order while their device footprint
//      fits the budget and, when a cap is set, the interior cells of the
//      running solves stay under it (allocate, upload the initial state);
//   2. advance every running solve by one step: solves whose step runs the
//      single-solve path's fused kernels (Solver::fused_path: z lines long
//      enough to fill their tiles) each launch their own step graph on their
//      own stream, and all other solves advance together by one batched
//      step (one graph launch; re-recorded when that set changes), on one
//      more stream, so the steps of all running solves overlap on the GPU;
//   3. retire solves that reached their step count: copy the state to the
//      host, free the device memory, stamp the completion time.
// Either path gives a solve the same bits (both equal the reference's), so
// where a solve runs changes its speed, not its result.
// State stays resident on the device from admission to retirement, and a
// request that arrives while others run is admitted as soon as memory frees
// up, so its steps overlap theirs on the device.  A solve whose CFL timestep
// goes non-finite is retired as failed without stopping the others.
#include "sams_lare.h"
#include "lare_batch.cuh"
#include "lare_solver.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

void sams_capi_set_last_error(const std::string &msg);

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    sams_lare_params p{};
    sams_lare_bcs bcs{};
    const double *ic[SAMS_NFIELDS] = {};
    double *out[9] = {};
    std::vector<std::vector<double>> staged;  // results kept by the server when out == NULL
    int64_t nsteps = 0;
    int64_t done = 0;
    long long cells = 0;
    int slot = -1;                          // batch slot (batched solves)
    std::unique_ptr<sams::Solver> solo;     // own solver (fused-path solves)
    bool fused = false;
    int status = SAMS_SERVE_QUEUED;
    bool cancel = false;  // set by sams_lare_serve_cancel while running
    long long bytes = 0;
    Clock::time_point t_submit, t_admit, t_done;
};

const int kStateFields[9] = {SAMS_F_RHO, SAMS_F_ENERGY_ELECTRON, SAMS_F_ENERGY_ION, SAMS_F_VX, SAMS_F_VY,
                             SAMS_F_VZ, SAMS_F_BX, SAMS_F_BY, SAMS_F_BZ};

}  // namespace

struct sams_lare_server {
    sams::Batch batch;
    int device = 0;
    long long budget = 0;
    long long in_use = 0;
    long long max_cells = 0;       // cap on running interior cells (0 = none)
    long long cells_in_use = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false;
    int64_t next_id = 1;
    std::deque<Request *> queue;
    std::vector<Request *> running;
    std::map<int64_t, std::unique_ptr<Request>> all;
    std::vector<double> latencies;  // completed requests, seconds
    double cell_updates = 0.0;
    int64_t failed = 0, completed = 0;
    Clock::time_point t_start;
    std::string worker_error;

    void loop();
    bool admit_locked();
    int admit_one(Request *r);
    void drop(Request *r);
    void retire(Request *r, bool ok);
};

// Allocate r's solve (its own solver or a batch slot) and upload its
// initial state.
int sams_lare_server::admit_one(Request *r)
{
    int rc;
    if (r->fused) {
        r->solo.reset(new (std::nothrow) sams::Solver());
        if (!r->solo) return SAMS_ERR_NOMEM;
        rc = r->solo->init(r->p, r->bcs, device);
        for (int f = 0; rc == SAMS_OK && f < SAMS_NFIELDS; ++f)
            if (r->ic[f]) rc = r->solo->upload(f, r->ic[f], cudaMemcpyDefault);
        if (rc == SAMS_OK) rc = r->solo->sync();
        if (rc != SAMS_OK) {
            worker_error = r->solo->err;
            r->solo.reset();
        }
        return rc;
    }
    int slot = -1;
    rc = batch.add(r->p, r->bcs, &slot);
    for (int f = 0; rc == SAMS_OK && f < SAMS_NFIELDS; ++f)
        if (r->ic[f]) rc = batch.upload(slot, f, r->ic[f], cudaMemcpyDefault);
    if (rc == SAMS_OK) rc = batch.sync();
    if (rc != SAMS_OK) {
        if (slot >= 0) batch.remove(slot);
        worker_error = batch.err;
        return rc;
    }
    r->slot = slot;
    return SAMS_OK;
}

// Free r's device memory (its solver or its batch slot).
void sams_lare_server::drop(Request *r)
{
    if (r->solo) r->solo.reset();
    else if (r->slot >= 0) batch.remove(r->slot);
    r->slot = -1;
}

bool sams_lare_server::admit_locked()
{
    bool any = false;
    while (!queue.empty()) {
        Request *r = queue.front();
        if (in_use + r->bytes > budget && !running.empty()) break;  // wait for memory
        // wait for work to drain: a smaller running set finishes each solve
        // sooner once the set already keeps the GPU busy
        if (max_cells > 0 && cells_in_use + r->cells > max_cells && !running.empty()) break;
        if (in_use + r->bytes > budget && running.empty() && r->bytes > budget) {
            // can never fit
            queue.pop_front();
            r->status = SAMS_SERVE_FAILED;
            r->t_done = Clock::now();
            ++failed;
            continue;
        }
        queue.pop_front();
        if (admit_one(r) != SAMS_OK) {
            r->status = SAMS_SERVE_FAILED;
            r->t_done = Clock::now();
            ++failed;
            continue;
        }
        r->status = SAMS_SERVE_RUNNING;
        r->t_admit = Clock::now();
        in_use += r->bytes;
        cells_in_use += r->cells;
        running.push_back(r);
        any = true;
    }
    return any;
}

void sams_lare_server::retire(Request *r, bool ok)
{
    if (ok) {
        for (int q = 0; q < 9; ++q) {
            double *dst = r->out[q];
            if (!dst) {
                const long long n = (r->p.nx + 5) * (r->p.ny + 5) * (r->p.nz + 5);
                r->staged.emplace_back((size_t)n);
                dst = r->staged.back().data();
            }
            const int rc = r->solo ? r->solo->download(kStateFields[q], dst, cudaMemcpyDefault)
                                   : batch.download(r->slot, kStateFields[q], dst, cudaMemcpyDefault);
            if (rc != SAMS_OK) ok = false;
        }
    }
    drop(r);
    r->t_done = Clock::now();
    std::lock_guard<std::mutex> lk(mu);
    in_use -= r->bytes;
    cells_in_use -= r->cells;
    r->status = ok ? SAMS_SERVE_DONE : SAMS_SERVE_FAILED;
    if (ok) {
        ++completed;
        latencies.push_back(std::chrono::duration<double>(r->t_done - r->t_submit).count());
    } else {
        ++failed;
    }
    cv.notify_all();
}

void sams_lare_server::loop()
{
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return stop || !queue.empty() || !running.empty(); });
            if (stop) return;
            // running solves cancelled since the last step leave before it
            std::vector<Request *> keep;
            for (Request *r : running) {
                if (!r->cancel) {
                    keep.push_back(r);
                    continue;
                }
                drop(r);
                in_use -= r->bytes;
                cells_in_use -= r->cells;
                r->status = SAMS_SERVE_CANCELLED;
                r->t_done = Clock::now();
            }
            if (keep.size() != running.size()) {
                running.swap(keep);
                cv.notify_all();
            }
            admit_locked();
        }
        if (running.empty()) continue;
        // one step for every running solve: each fused-path solve launches
        // its own step graph on its own stream, the others one batched step
        std::vector<Request *> lost;  // solves whose step could not run
        bool any_batched = false;
        for (Request *r : running) {
            if (!r->solo) any_batched = true;
            else if (r->solo->step_graph(1) != SAMS_OK) lost.push_back(r);
        }
        bool batch_ok = !any_batched || (batch.step_graph(1) == SAMS_OK && batch.sync() == SAMS_OK);
        if (!batch_ok) worker_error = batch.err;
        for (Request *r : running)
            if (r->solo && std::find(lost.begin(), lost.end(), r) == lost.end() &&
                cudaStreamSynchronize(r->solo->stream()) != cudaSuccess)
                lost.push_back(r);
        std::vector<Request *> keep;
        for (Request *r : running) {
            if ((!r->solo && !batch_ok) || std::find(lost.begin(), lost.end(), r) != lost.end()) {
                if (r->solo) worker_error = r->solo->err;
                drop(r);
                std::lock_guard<std::mutex> lk(mu);
                in_use -= r->bytes;
                cells_in_use -= r->cells;
                r->status = SAMS_SERVE_FAILED;
                r->t_done = Clock::now();
                ++failed;
                cv.notify_all();
                continue;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                r->done += 1;
                cell_updates += (double)r->p.nx * (double)r->p.ny * (double)r->p.nz;
            }
            bool finished = r->done >= r->nsteps;
            bool bad = false;
            if (finished || (r->done & 63) == 0) {
                sams::Scalars sc;
                const int rc = r->solo ? r->solo->scalars(sc) : batch.scalars(r->slot, sc);
                if (rc != SAMS_OK || sc.status) bad = true;
            }
            if (bad) retire(r, false);
            else if (finished) retire(r, true);
            else keep.push_back(r);
        }
        std::lock_guard<std::mutex> lk(mu);
        running.swap(keep);
    }
}

static double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    double pos = q * (double)(v.size() - 1);
    size_t lo = (size_t)pos;
    size_t hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

extern "C" {

int sams_lare_serve_create(int device, int64_t budget_bytes, sams_lare_server **out)
{
    if (!out || budget_bytes <= 0) {
        sams_capi_set_last_error("sams_lare_serve_create: null argument or non-positive budget");
        return SAMS_ERR_INVALID;
    }
    *out = nullptr;
    auto *s = new (std::nothrow) sams_lare_server();
    if (!s) return SAMS_ERR_NOMEM;
    int rc = s->batch.init(device);
    if (rc != SAMS_OK) {
        sams_capi_set_last_error(s->batch.err);
        delete s;
        return rc;
    }
    s->budget = budget_bytes;
    s->device = device;
    s->t_start = Clock::now();
    s->worker = std::thread([s, device] {
        cudaSetDevice(device);
        s->loop();
    });
    *out = s;
    return SAMS_OK;
}

int sams_lare_serve_submit(sams_lare_server *s, const sams_lare_params *p, const sams_lare_bcs *bcs,
                           const double *const ic[SAMS_NFIELDS], int64_t nsteps, double *const out[9],
                           int64_t *ticket)
{
    if (!s || !p || !bcs || !ic || nsteps < 1 || !ticket) {
        sams_capi_set_last_error("sams_lare_serve_submit: invalid argument");
        return SAMS_ERR_INVALID;
    }
    if (p->geometry < 0 || p->geometry > 2) {
        sams_capi_set_last_error("sams_lare_serve_submit: geometry must be 0, 1 or 2");
        return SAMS_ERR_UNSUPPORTED;
    }
    auto r = std::make_unique<Request>();
    r->p = *p;
    r->bcs = *bcs;
    for (int f = 0; f < SAMS_NFIELDS; ++f) r->ic[f] = ic[f];
    for (int q = 0; q < 9; ++q) r->out[q] = out ? out[q] : nullptr;
    r->nsteps = nsteps;
    r->fused = sams::Solver::fused_path(*p);
    r->bytes = r->fused ? sams::Solver::bytes_for(*p) : sams::Batch::bytes_for(*p);
    r->cells = (long long)(p->nx * p->ny * p->nz);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->bytes > s->budget) {
        sams_capi_set_last_error("sams_lare_serve_submit: the solve alone exceeds the memory budget");
        return SAMS_ERR_BUDGET;
    }
    r->id = s->next_id++;
    *ticket = r->id;
    s->queue.push_back(r.get());
    s->all.emplace(r->id, std::move(r));
    s->cv.notify_all();
    return SAMS_OK;
}

int sams_lare_serve_solve_bytes(const sams_lare_params *p, int64_t *bytes)
{
    if (!p || !bytes) return SAMS_ERR_INVALID;
    *bytes = (int64_t)(sams::Solver::fused_path(*p) ? sams::Solver::bytes_for(*p) : sams::Batch::bytes_for(*p));
    return SAMS_OK;
}

int sams_lare_serve_set_max_cells(sams_lare_server *s, int64_t max_cells)
{
    if (!s || max_cells < 0) {
        sams_capi_set_last_error("sams_lare_serve_set_max_cells: null server or negative cap");
        return SAMS_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->max_cells = (long long)max_cells;
    s->cv.notify_all();
    return SAMS_OK;
}

int sams_lare_serve_poll(sams_lare_server *s, int64_t ticket, int *status, double *latency_s)
{
    if (!s || !status) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) {
        sams_capi_set_last_error("sams_lare_serve_poll: unknown ticket");
        return SAMS_ERR_INVALID;
    }
    Request *r = it->second.get();
    *status = r->status;
    if (latency_s)
        *latency_s = (r->status == SAMS_SERVE_DONE || r->status == SAMS_SERVE_FAILED ||
                      r->status == SAMS_SERVE_CANCELLED)
                         ? std::chrono::duration<double>(r->t_done - r->t_submit).count()
                         : std::chrono::duration<double>(Clock::now() - r->t_submit).count();
    return SAMS_OK;
}

int sams_lare_serve_fetch(sams_lare_server *s, int64_t ticket, int state_index, double *host_box)
{
    if (!s || !host_box || state_index < 0 || state_index > 8) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end() || it->second->status != SAMS_SERVE_DONE || it->second->staged.size() != 9) {
        sams_capi_set_last_error("sams_lare_serve_fetch: no staged result for this ticket");
        return SAMS_ERR_INVALID;
    }
    const auto &v = it->second->staged[state_index];
    std::copy(v.begin(), v.end(), host_box);
    return SAMS_OK;
}

int sams_lare_serve_cancel(sams_lare_server *s, int64_t ticket)
{
    if (!s) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) {
        sams_capi_set_last_error("sams_lare_serve_cancel: unknown ticket");
        return SAMS_ERR_INVALID;
    }
    Request *r = it->second.get();
    if (r->status == SAMS_SERVE_QUEUED) {
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
        r->status = SAMS_SERVE_CANCELLED;
        r->t_done = Clock::now();
        s->cv.notify_all();
        return SAMS_OK;
    }
    if (r->status == SAMS_SERVE_RUNNING) {
        r->cancel = true;  // the scheduler retires it before its next step
        s->cv.notify_all();
        return SAMS_OK;
    }
    sams_capi_set_last_error("sams_lare_serve_cancel: request already finished");
    return SAMS_ERR_INVALID;
}

int sams_lare_serve_release(sams_lare_server *s, int64_t ticket)
{
    if (!s) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return SAMS_ERR_INVALID;
    if (it->second->status != SAMS_SERVE_DONE && it->second->status != SAMS_SERVE_FAILED &&
        it->second->status != SAMS_SERVE_CANCELLED) {
        sams_capi_set_last_error("sams_lare_serve_release: request still queued or running");
        return SAMS_ERR_INVALID;
    }
    s->all.erase(it);
    return SAMS_OK;
}

int sams_lare_serve_drain(sams_lare_server *s, double timeout_s)
{
    if (!s) return SAMS_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                             [&] { return s->queue.empty() && s->running.empty(); });
    if (!ok) {
        sams_capi_set_last_error("sams_lare_serve_drain: requests still pending at the timeout");
        return SAMS_ERR_TIMEOUT;
    }
    return SAMS_OK;
}

int sams_lare_serve_get_stats(sams_lare_server *s, sams_lare_serve_stats *st)
{
    if (!s || !st) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    st->submitted = s->next_id - 1;
    st->completed = s->completed;
    st->failed = s->failed;
    st->queued = (int64_t)s->queue.size();
    st->running = (int64_t)s->running.size();
    st->p50_latency_s = percentile(s->latencies, 0.50);
    st->p99_latency_s = percentile(s->latencies, 0.99);
    double sum = 0.0;
    for (double x : s->latencies) sum += x;
    st->mean_latency_s = s->latencies.empty() ? 0.0 : sum / (double)s->latencies.size();
    st->cell_updates = s->cell_updates;
    st->wall_s = std::chrono::duration<double>(Clock::now() - s->t_start).count();
    st->cell_updates_per_s = st->wall_s > 0 ? st->cell_updates / st->wall_s : 0.0;
    st->device_bytes_in_use = s->in_use;
    double pending = 0.0;
    int64_t qbytes = 0;
    for (const Request *r : s->queue) {
        pending += (double)r->cells * (double)r->nsteps;
        qbytes += r->bytes;
    }
    for (const Request *r : s->running) pending += (double)r->cells * (double)(r->nsteps - r->done);
    st->pending_cell_updates = pending;
    st->queued_bytes = qbytes;
    return SAMS_OK;
}

int sams_lare_serve_destroy(sams_lare_server *s)
{
    if (!s) return SAMS_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    delete s;
    return SAMS_OK;
}

}  // extern "C"
