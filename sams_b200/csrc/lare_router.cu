// lare_router.cu -- serving LARE3D solves on several GPUs.
//
// Solves are independent (no data crosses between them), so serving on N
// GPUs needs no collective: one continuous-batching server per device (each
// with its own scheduler thread, stream and memory budget, lare_serve.cu)
// and a host router that places every submitted solve on one of them.  The
// placement reads each server's outstanding work (interior cells x steps
// still to run) and committed device bytes (admitted + queued) at submit
// time; submits are serialised so each placement sees the previous one.
#include "sams_lare.h"

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <vector>

void sams_capi_set_last_error(const std::string &msg);

namespace {

struct Placement {
    int server = -1;
    int64_t ticket = 0;
};

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct sams_lare_router {
    std::vector<sams_lare_server *> servers;
    std::vector<int64_t> budget;
    std::mutex mu;
    int64_t next_id = 1;
    std::map<int64_t, Placement> placed;
    std::vector<double> released;  // latencies of completed requests already released, seconds
};

extern "C" {

int sams_lare_route_pick(int n, const double *pending, const int64_t *committed, const int64_t *budget,
                         int64_t request_bytes, int *index)
{
    if (n < 1 || !pending || !committed || !budget || !index || request_bytes < 0) {
        sams_capi_set_last_error("sams_lare_route_pick: invalid argument");
        return SAMS_ERR_INVALID;
    }
    int best = -1;
    bool best_fits = false;
    for (int q = 0; q < n; ++q) {
        if (request_bytes > budget[q]) continue;  // can never run there
        const bool fits = committed[q] + request_bytes <= budget[q];
        bool better;
        if (best < 0) better = true;
        else if (fits != best_fits) better = fits;
        else if (pending[q] != pending[best]) better = pending[q] < pending[best];
        else better = committed[q] < committed[best];
        if (better) {
            best = q;
            best_fits = fits;
        }
    }
    if (best < 0) {
        sams_capi_set_last_error("sams_lare_route_pick: the solve exceeds every server's budget");
        return SAMS_ERR_BUDGET;
    }
    *index = best;
    return SAMS_OK;
}

int sams_lare_router_create(const int *devices, int ndevices, int64_t budget_bytes_per_device,
                            sams_lare_router **out)
{
    if (!devices || ndevices < 1 || !out || budget_bytes_per_device <= 0) {
        sams_capi_set_last_error("sams_lare_router_create: invalid argument");
        return SAMS_ERR_INVALID;
    }
    *out = nullptr;
    auto *r = new (std::nothrow) sams_lare_router();
    if (!r) return SAMS_ERR_NOMEM;
    for (int q = 0; q < ndevices; ++q) {
        sams_lare_server *s = nullptr;
        int rc = sams_lare_serve_create(devices[q], budget_bytes_per_device, &s);
        if (rc != SAMS_OK) {
            for (auto *t : r->servers) sams_lare_serve_destroy(t);
            delete r;
            return rc;
        }
        r->servers.push_back(s);
        r->budget.push_back(budget_bytes_per_device);
    }
    *out = r;
    return SAMS_OK;
}

int sams_lare_router_submit(sams_lare_router *r, const sams_lare_params *p, const sams_lare_bcs *bcs,
                            const double *const ic[SAMS_NFIELDS], int64_t nsteps, double *const out[9],
                            int64_t *ticket)
{
    if (!r || !p || !ticket) {
        sams_capi_set_last_error("sams_lare_router_submit: invalid argument");
        return SAMS_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(r->mu);
    const int n = (int)r->servers.size();
    std::vector<double> pending(n);
    std::vector<int64_t> committed(n);
    for (int q = 0; q < n; ++q) {
        sams_lare_serve_stats st{};
        int rc = sams_lare_serve_get_stats(r->servers[q], &st);
        if (rc != SAMS_OK) return rc;
        pending[q] = st.pending_cell_updates;
        committed[q] = st.device_bytes_in_use + st.queued_bytes;
    }
    int64_t bytes = 0;
    int rc = sams_lare_serve_solve_bytes(p, &bytes);
    if (rc != SAMS_OK) return rc;
    int pick = -1;
    rc = sams_lare_route_pick(n, pending.data(), committed.data(), r->budget.data(), bytes, &pick);
    if (rc != SAMS_OK) return rc;
    Placement pl;
    pl.server = pick;
    rc = sams_lare_serve_submit(r->servers[pick], p, bcs, ic, nsteps, out, &pl.ticket);
    if (rc != SAMS_OK) return rc;
    *ticket = r->next_id++;
    r->placed.emplace(*ticket, pl);
    return SAMS_OK;
}

static int find_placement(sams_lare_router *r, int64_t ticket, Placement *pl, const char *who)
{
    auto it = r->placed.find(ticket);
    if (it == r->placed.end()) {
        sams_capi_set_last_error(std::string(who) + ": unknown ticket");
        return SAMS_ERR_INVALID;
    }
    *pl = it->second;
    return SAMS_OK;
}

int sams_lare_router_placement(sams_lare_router *r, int64_t ticket, int *index)
{
    if (!r || !index) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->mu);
    Placement pl;
    int rc = find_placement(r, ticket, &pl, "sams_lare_router_placement");
    if (rc == SAMS_OK) *index = pl.server;
    return rc;
}

int sams_lare_router_set_max_cells(sams_lare_router *r, int64_t max_cells)
{
    if (!r) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->mu);
    for (auto *s : r->servers) {
        int rc = sams_lare_serve_set_max_cells(s, max_cells);
        if (rc != SAMS_OK) return rc;
    }
    return SAMS_OK;
}

int sams_lare_router_poll(sams_lare_router *r, int64_t ticket, int *status, double *latency_s)
{
    if (!r || !status) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->mu);
    Placement pl;
    int rc = find_placement(r, ticket, &pl, "sams_lare_router_poll");
    if (rc != SAMS_OK) return rc;
    return sams_lare_serve_poll(r->servers[pl.server], pl.ticket, status, latency_s);
}

int sams_lare_router_fetch(sams_lare_router *r, int64_t ticket, int state_index, double *host_box)
{
    if (!r) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->mu);
    Placement pl;
    int rc = find_placement(r, ticket, &pl, "sams_lare_router_fetch");
    if (rc != SAMS_OK) return rc;
    return sams_lare_serve_fetch(r->servers[pl.server], pl.ticket, state_index, host_box);
}

int sams_lare_router_cancel(sams_lare_router *r, int64_t ticket)
{
    if (!r) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->mu);
    Placement pl;
    int rc = find_placement(r, ticket, &pl, "sams_lare_router_cancel");
    if (rc != SAMS_OK) return rc;
    return sams_lare_serve_cancel(r->servers[pl.server], pl.ticket);
}

int sams_lare_router_release(sams_lare_router *r, int64_t ticket)
{
    if (!r) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->mu);
    Placement pl;
    int rc = find_placement(r, ticket, &pl, "sams_lare_router_release");
    if (rc != SAMS_OK) return rc;
    int status = 0;
    double lat = 0.0;
    const bool done = sams_lare_serve_poll(r->servers[pl.server], pl.ticket, &status, &lat) == SAMS_OK &&
                      status == SAMS_SERVE_DONE;
    rc = sams_lare_serve_release(r->servers[pl.server], pl.ticket);
    if (rc == SAMS_OK) {
        if (done) r->released.push_back(lat);
        r->placed.erase(ticket);
    }
    return rc;
}

int sams_lare_router_drain(sams_lare_router *r, double timeout_s)
{
    if (!r) return SAMS_ERR_INVALID;
    const double t_end = now_s() + timeout_s;
    for (auto *s : r->servers) {
        int rc = sams_lare_serve_drain(s, std::max(0.0, t_end - now_s()));
        if (rc != SAMS_OK) return rc;
    }
    return SAMS_OK;
}

int sams_lare_router_server_stats(sams_lare_router *r, int index, sams_lare_serve_stats *st)
{
    if (!r || !st || index < 0 || index >= (int)r->servers.size()) {
        sams_capi_set_last_error("sams_lare_router_server_stats: invalid argument");
        return SAMS_ERR_INVALID;
    }
    return sams_lare_serve_get_stats(r->servers[index], st);
}

int sams_lare_router_get_stats(sams_lare_router *r, sams_lare_serve_stats *st)
{
    if (!r || !st) return SAMS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(r->mu);
    sams_lare_serve_stats t{};
    std::vector<double> lat;
    double wall = 0.0;
    for (auto *s : r->servers) {
        sams_lare_serve_stats q{};
        int rc = sams_lare_serve_get_stats(s, &q);
        if (rc != SAMS_OK) return rc;
        t.submitted += q.submitted;
        t.completed += q.completed;
        t.failed += q.failed;
        t.queued += q.queued;
        t.running += q.running;
        t.cell_updates += q.cell_updates;
        t.device_bytes_in_use += q.device_bytes_in_use;
        t.pending_cell_updates += q.pending_cell_updates;
        t.queued_bytes += q.queued_bytes;
        wall = std::max(wall, q.wall_s);
    }
    // latencies of every completed request: released ones and those still held
    lat = r->released;
    for (auto &kv : r->placed) {
        int status = 0;
        double l = 0.0;
        if (sams_lare_serve_poll(r->servers[kv.second.server], kv.second.ticket, &status, &l) == SAMS_OK &&
            status == SAMS_SERVE_DONE)
            lat.push_back(l);
    }
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {
        if (lat.empty()) return 0.0;
        double pos = q * (double)(lat.size() - 1);
        size_t lo = (size_t)pos, hi = std::min(lo + 1, lat.size() - 1);
        return lat[lo] + (lat[hi] - lat[lo]) * (pos - (double)lo);
    };
    t.p50_latency_s = pct(0.50);
    t.p99_latency_s = pct(0.99);
    double sum = 0.0;
    for (double x : lat) sum += x;
    t.mean_latency_s = lat.empty() ? 0.0 : sum / (double)lat.size();
    t.wall_s = wall;
    t.cell_updates_per_s = wall > 0 ? t.cell_updates / wall : 0.0;
    *st = t;
    return SAMS_OK;
}

int sams_lare_router_destroy(sams_lare_router *r)
{
    if (!r) return SAMS_ERR_INVALID;
    for (auto *s : r->servers) sams_lare_serve_destroy(s);
    delete r;
    return SAMS_OK;
}

}  // extern "C"
