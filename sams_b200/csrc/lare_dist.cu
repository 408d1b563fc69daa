// lare_dist.cu -- one LARE3D solve split along x over several GPUs.
//
// The reference decomposes a solve over MPI ranks and refreshes the ghost
// layers between ranks with MPIManager::haloExchange
// (include/harness/mpiManager.h:1246-1277) wherever a boundary fill runs.
// Here each x slab is a Solver on its own device (or several slabs share
// one) with the whole grid's axes from its offset on, driven by its own host
// thread.  At every boundary fill of the step the x ghost planes are pulled
// from the neighbouring slabs' interiors by peer copies into the receiver's
// own buffers (no remote loads in kernels, no collective), then y and z are
// filled locally in the single-solve order; the CFL minimum is completed over
// all slabs before dt is formed.  The exchanged planes are the ones the
// single-solve x fill writes, from the same global points:
//   cell-centred fields: ghosts -1, 0 and n+1, n+2;
//   face/node fields:    ghosts -2, -1 and n+1, n+2, and at the grid's
//                        periodic lower edge also 0 (from global n; the
//                        upper half-cell index n keeps its value).
// A half-cell plane on a slab edge inside the grid is computed by both
// slabs from the same inputs and is not exchanged.  So each slab holds, at
// every point it reads, the value the undivided solve holds there.
#include "sams_lare.h"
#include "lare_solver.cuh"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

void sams_capi_set_last_error(const std::string &msg);

namespace sams {
namespace {

constexpr int kMaxParts = 64;
constexpr int kMinSlabCells = 3;  // every ghost plane comes from one neighbour's interior

// Reusable barrier for the slab threads (C++17 has none).
class Barrier {
public:
    explicit Barrier(int n) : n_(n) {}
    void wait()
    {
        std::unique_lock<std::mutex> lk(mu_);
        const long long gen = gen_;
        if (++count_ == n_) {
            count_ = 0;
            ++gen_;
            cv_.notify_all();
            return;
        }
        cv_.wait(lk, [&] { return gen_ != gen; });
    }

private:
    std::mutex mu_;
    std::condition_variable cv_;
    int n_, count_ = 0;
    long long gen_ = 0;
};

// min of this slab's and the gathered candidate minima into this slab's
// running minimum (the bit patterns of positive doubles order like the values)
__global__ void k_dt_merge(Scalars *sc, const unsigned long long *others, int n)
{
    unsigned long long m = sc->dtmin_bits;
    for (int q = 0; q < n; ++q) m = others[q] < m ? others[q] : m;
    sc->dtmin_bits = m;
}

}  // namespace

struct DistSolver final : Halo {
    int parts = 0;
    long long nx = 0;
    sams_lare_params p{};
    std::vector<long long> off;  // off[q]: global index of slab q's cell 0; off[parts] = nx
    std::vector<std::unique_ptr<Solver>> slab;
    std::vector<cudaEvent_t> ev_ready, ev_pulled;
    std::vector<unsigned long long *> dt_in;  // per slab: the other slabs' minima (device)
    std::unique_ptr<Barrier> bar;
    std::vector<int> errs;
    std::string err;

    int index_of(const Solver &s) const
    {
        for (int q = 0; q < parts; ++q)
            if (slab[q].get() == &s) return q;
        return -1;
    }
    long long n_of(int q) const { return off[q + 1] - off[q]; }

    // ---- Halo ----
    void fill_x(Solver &s, unsigned mask) override;
    void reduce_dt(Solver &s) override;

    int run_steps(long long nsteps);
    ~DistSolver() override;
};

void DistSolver::fill_x(Solver &s, unsigned mask)
{
    const int q = index_of(s);
    const int lq = (q + parts - 1) % parts, rq = (q + 1) % parts;
    const cudaStream_t st = s.stream();
    const BcTable &bc = s.bc_table();
    const Geom &g = s.geom();
    const size_t plane = (size_t)g.sx * sizeof(double);
    cudaEventRecord(ev_ready[q], st);
    bar->wait();  // every slab's producing kernels are enqueued before its ready event
    cudaStreamWaitEvent(st, ev_ready[lq], 0);
    cudaStreamWaitEvent(st, ev_ready[rq], 0);
    const bool first = q == 0, last = q == parts - 1;
    unsigned local_low = 0, local_high = 0;  // fields whose grid-edge condition is not periodic
    for (int f = 0; f < SAMS_NFIELDS; ++f) {
        if (!(mask & (1u << f))) continue;
        const bool half = sams_lare_field_stagger[f][0] != 0;
        double *mine = s.field_ptr(f);
        // lower ghosts
        if (!first || bc.kind[f][0][0] == SAMS_BC_PERIODIC) {
            const Solver &nb = *slab[lq];
            const int nn = (int)n_of(lq);
            // half: -2..-1 (and 0 at the grid's periodic edge); cell: -1..0
            const int lo = half ? -2 : -1, hi = (half && !first) ? -1 : 0;
            const double *src = nb.field_ptr(f) + (size_t)(lo + nn + 2) * g.sx;
            cudaMemcpyPeerAsync(mine + (size_t)(lo + 2) * g.sx, s.device(), src, nb.device(), plane * (hi - lo + 1), st);
        } else if (bc.kind[f][0][0] != SAMS_BC_NONE) {
            local_low |= 1u << f;
        }
        // upper ghosts n+1..n+2 from the next slab's 1..2
        if (!last || bc.kind[f][0][1] == SAMS_BC_PERIODIC) {
            const Solver &nb = *slab[rq];
            const int n = g.nx;
            const double *src = nb.field_ptr(f) + (size_t)(1 + 2) * g.sx;
            cudaMemcpyPeerAsync(mine + (size_t)(n + 1 + 2) * g.sx, s.device(), src, nb.device(), plane * 2, st);
        } else if (bc.kind[f][0][1] != SAMS_BC_NONE) {
            local_high |= 1u << f;
        }
    }
    cudaEventRecord(ev_pulled[q], st);
    bar->wait();
    // the neighbours must have read these planes before this slab writes them again
    cudaStreamWaitEvent(st, ev_pulled[lq], 0);
    cudaStreamWaitEvent(st, ev_pulled[rq], 0);
    if (local_low) s.bc_fill_edge(local_low, 0, 0);
    if (local_high) s.bc_fill_edge(local_high, 0, 1);
}

void DistSolver::reduce_dt(Solver &s)
{
    const int q = index_of(s);
    const cudaStream_t st = s.stream();
    cudaEventRecord(ev_ready[q], st);
    bar->wait();
    int k = 0;
    for (int r = 0; r < parts; ++r) {
        if (r == q) continue;
        cudaStreamWaitEvent(st, ev_ready[r], 0);
        const char *src = reinterpret_cast<const char *>(slab[r]->scalars_ptr()) + offsetof(Scalars, dtmin_bits);
        cudaMemcpyPeerAsync(dt_in[q] + k, s.device(), src, slab[r]->device(), sizeof(unsigned long long), st);
        ++k;
    }
    k_dt_merge<<<1, 1, 0, st>>>(s.scalars_ptr(), dt_in[q], k);
    cudaEventRecord(ev_pulled[q], st);
    bar->wait();
    // no slab resets its minimum (in the dt finalisation) before all have read it
    for (int r = 0; r < parts; ++r)
        if (r != q) cudaStreamWaitEvent(st, ev_pulled[r], 0);
}

int DistSolver::run_steps(long long nsteps)
{
    std::fill(errs.begin(), errs.end(), SAMS_OK);
    std::vector<std::thread> th;
    for (int q = 0; q < parts; ++q)
        th.emplace_back([this, q, nsteps] {
            Solver &s = *slab[q];
            cudaSetDevice(s.device());
            // every thread enqueues every step (and so meets every barrier)
            // whatever happens; errors are read afterwards
            for (long long k = 0; k < nsteps; ++k) s.enqueue_step();
            const cudaError_t e = cudaGetLastError();
            errs[q] = e == cudaSuccess ? s.sync() : SAMS_ERR_CUDA;
            if (e != cudaSuccess) s.err = std::string("step launch: ") + cudaGetErrorString(e);
        });
    for (auto &t : th) t.join();
    for (int q = 0; q < parts; ++q)
        if (errs[q] != SAMS_OK) {
            err = "slab " + std::to_string(q) + ": " + slab[q]->err;
            return errs[q];
        }
    return SAMS_OK;
}

DistSolver::~DistSolver()
{
    for (int q = 0; q < parts; ++q) {
        if (q < (int)slab.size() && slab[q]) cudaSetDevice(slab[q]->device());
        if (q < (int)ev_ready.size() && ev_ready[q]) cudaEventDestroy(ev_ready[q]);
        if (q < (int)ev_pulled.size() && ev_pulled[q]) cudaEventDestroy(ev_pulled[q]);
        if (q < (int)dt_in.size() && dt_in[q]) cudaFree(dt_in[q]);
    }
}

}  // namespace sams

struct sams_lare_dist {
    sams::DistSolver d;
};

extern "C" {

int sams_lare_dist_partition(int64_t nx, int nparts, int64_t *offsets)
{
    if (nparts < 1 || nparts > sams::kMaxParts || !offsets || nx < (int64_t)nparts * sams::kMinSlabCells) {
        sams_capi_set_last_error("sams_lare_dist_partition: need 1..64 slabs of at least 3 cells each");
        return SAMS_ERR_INVALID;
    }
    offsets[0] = 0;
    for (int q = 0; q < nparts; ++q) offsets[q + 1] = offsets[q] + nx / nparts + (q < nx % nparts ? 1 : 0);
    return SAMS_OK;
}

int sams_lare_dist_create(const sams_lare_params *params, const sams_lare_bcs *bcs, const int *devices, int nparts,
                          sams_lare_dist **out)
{
    if (!params || !bcs || !devices || !out || nparts < 2) {
        sams_capi_set_last_error("sams_lare_dist_create: invalid argument (at least two slabs)");
        return SAMS_ERR_INVALID;
    }
    *out = nullptr;
    std::vector<int64_t> off((size_t)nparts + 1);
    int rc = sams_lare_dist_partition(params->nx, nparts, off.data());
    if (rc != SAMS_OK) return rc;
    auto h = std::make_unique<sams_lare_dist>();
    sams::DistSolver &d = h->d;
    d.parts = nparts;
    d.nx = params->nx;
    d.p = *params;
    d.off.assign(off.begin(), off.end());
    d.bar = std::make_unique<sams::Barrier>(nparts);
    d.errs.assign(nparts, SAMS_OK);
    d.ev_ready.assign(nparts, nullptr);
    d.ev_pulled.assign(nparts, nullptr);
    d.dt_in.assign(nparts, nullptr);
    for (int q = 0; q < nparts; ++q) {
        sams_lare_params pq = *params;
        pq.nx = off[q + 1] - off[q];
        sams::XSlab xs;
        xs.off = off[q];
        xs.nx_global = params->nx;
        auto s = std::make_unique<sams::Solver>();
        rc = s->init_slab(pq, *bcs, devices[q], xs);
        if (rc != SAMS_OK) {
            sams_capi_set_last_error("sams_lare_dist_create: slab " + std::to_string(q) + ": " + s->err);
            return rc;
        }
        s->set_halo(&d);
        d.slab.push_back(std::move(s));
        cudaSetDevice(devices[q]);
        if (cudaEventCreateWithFlags(&d.ev_ready[q], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&d.ev_pulled[q], cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc(&d.dt_in[q], sizeof(unsigned long long) * (size_t)nparts) != cudaSuccess) {
            sams_capi_set_last_error("sams_lare_dist_create: event or buffer allocation failed");
            return SAMS_ERR_CUDA;
        }
    }
    // peer copies between devices work without peer access; enable it where
    // the hardware offers it so they go straight over NVLink
    for (int a = 0; a < nparts; ++a)
        for (int b = 0; b < nparts; ++b) {
            if (devices[a] == devices[b]) continue;
            int ok = 0;
            if (cudaDeviceCanAccessPeer(&ok, devices[a], devices[b]) == cudaSuccess && ok) {
                cudaSetDevice(devices[a]);
                if (cudaDeviceEnablePeerAccess(devices[b], 0) != cudaSuccess) cudaGetLastError();
            }
        }
    *out = h.release();
    return SAMS_OK;
}

int sams_lare_dist_slab(sams_lare_dist *h, int part, int64_t *first_cell, int64_t *ncells)
{
    if (!h || part < 0 || part >= h->d.parts || !first_cell || !ncells) return SAMS_ERR_INVALID;
    *first_cell = h->d.off[part] + 1;
    *ncells = h->d.n_of(part);
    return SAMS_OK;
}

// A slab's box holds global x planes off-2 .. off+n+2; the whole grid's box
// is planes -2 .. nx+2, each (ny+5)(nz+5) doubles, z fastest.
int sams_lare_dist_upload_field(sams_lare_dist *h, int field, const double *host_box)
{
    if (!h || !host_box || field < 0 || field >= SAMS_NFIELDS) return SAMS_ERR_INVALID;
    sams::DistSolver &d = h->d;
    const size_t plane = (size_t)(d.p.ny + 5) * (size_t)(d.p.nz + 5);
    for (int q = 0; q < d.parts; ++q) {
        // global plane off-2 sits at index off of the grid's box
        int rc = d.slab[q]->upload(field, host_box + (size_t)d.off[q] * plane, cudaMemcpyHostToDevice);
        if (rc == SAMS_OK) rc = d.slab[q]->sync();
        if (rc != SAMS_OK) {
            sams_capi_set_last_error(d.slab[q]->err);
            return rc;
        }
    }
    return SAMS_OK;
}

int sams_lare_dist_download_field(sams_lare_dist *h, int field, double *host_box)
{
    if (!h || !host_box || field < 0 || field >= SAMS_NFIELDS) return SAMS_ERR_INVALID;
    sams::DistSolver &d = h->d;
    const size_t plane = (size_t)(d.p.ny + 5) * (size_t)(d.p.nz + 5);
    std::vector<double> tmp;
    for (int q = 0; q < d.parts; ++q) {
        const long long n = d.n_of(q);
        tmp.resize((size_t)(n + 5) * plane);
        int rc = d.slab[q]->download(field, tmp.data(), cudaMemcpyDeviceToHost);
        if (rc != SAMS_OK) {
            sams_capi_set_last_error(d.slab[q]->err);
            return rc;
        }
        // slab q supplies global planes off+1 .. off+n, the first slab also
        // -2 .. off (its lower ghosts and half-cell plane 0), the last also
        // the grid's upper ghosts
        const long long g0 = q == 0 ? -2 : d.off[q] + 1;
        const long long g1 = q == d.parts - 1 ? d.off[q] + n + 2 : d.off[q] + n;
        const long long l0 = g0 - d.off[q];
        std::memcpy(host_box + (size_t)(g0 + 2) * plane, tmp.data() + (size_t)(l0 + 2) * plane,
                    (size_t)(g1 - g0 + 1) * plane * sizeof(double));
    }
    return SAMS_OK;
}

int sams_lare_dist_step(sams_lare_dist *h, int64_t nsteps)
{
    if (!h || nsteps < 0) return SAMS_ERR_INVALID;
    int rc = h->d.run_steps(nsteps);
    if (rc != SAMS_OK) sams_capi_set_last_error(h->d.err);
    return rc;
}

int sams_lare_dist_get_state(sams_lare_dist *h, double *dt, double *time, int64_t *step)
{
    if (!h) return SAMS_ERR_INVALID;
    sams::Scalars s;
    int rc = h->d.slab[0]->scalars(s);
    if (rc != SAMS_OK) {
        sams_capi_set_last_error(h->d.slab[0]->err);
        return rc;
    }
    if (dt) *dt = s.dt;
    if (time) *time = s.time;
    if (step) *step = s.step;
    return SAMS_OK;
}

int sams_lare_dist_destroy(sams_lare_dist *h)
{
    if (!h) return SAMS_ERR_INVALID;
    delete h;
    return SAMS_OK;
}

}  // extern "C"
