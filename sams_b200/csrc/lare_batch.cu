// lare_batch.cu -- batched LARE3D solves (see lare_batch.cuh).
//
// The per-point work is the same sams::ops code as the single-solve path;
// what changes is the launcher: a persistent grid strides over a worklist of
// tiles from every live solve, loading each tile's solve context (pointers,
// geometry, parameters) into shared memory.  Boundary fills walk a flattened
// index over the ghost shells of all solves.  One batched step is the same
// phase sequence as Solver::enqueue_step, each phase a single launch for the
// whole batch.
#include "lare_batch.cuh"
#include "lare_ops.cuh"
#include "lare_bc.cuh"
#include "lare_geom_host.h"

#include <algorithm>
#include <cstring>

namespace sams {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ void load_ctx(Ctx &dst, const Ctx *src)
{
    const int nw = (int)(sizeof(Ctx) / sizeof(int));
    const int *s = reinterpret_cast<const int *>(src);
    int *d = reinterpret_cast<int *>(&dst);
    for (int w = threadIdx.x; w < nw; w += blockDim.x) d[w] = s[w];
}

// GEO: some solve of the batch is curvilinear (the Cartesian instantiation,
// used when none is, carries no metric factors).
template <class Op, bool GEO, bool P2>
__global__ void __launch_bounds__(kT, (MinBlocksBatch<Op, P2>::value))
    kb_op(const Ctx *__restrict__ ctxs, const Tile *__restrict__ tiles, int ntiles, int arg, int tile_i,
          int resistive_only)
{
    __shared__ Ctx c;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        // threads walk the op's own (j, k) range (no idle lanes on the ghost
        // planes of thin solves); the tiles cover the whole box plane, so
        // every op's range is inside them, and a tile past the op's range
        // is skipped before its context is staged (uniform over the block)
        const Ctx *src = ctxs + tl.inst;
        const int resistive = src->p.resistive;
        if (resistive_only && !resistive) continue;
        const int a = arg >= 0 ? arg : resistive;
        int lo[3], hi[3];
        Op::bounds(src->g, a, lo, hi);
        const int nk = hi[2] - lo[2] + 1;
        if (tl.p0 >= (hi[1] - lo[1] + 1) * nk || tl.i0 > hi[0] || tl.i0 + tile_i - 1 < lo[0]) continue;
        __syncthreads();
        load_ctx(c, src);
        __syncthreads();
        const int p = tl.p0 + (int)threadIdx.x;
        if (p >= (hi[1] - lo[1] + 1) * nk) continue;
        const int j = lo[1] + p / nk, k = lo[2] + p % nk;
        const int ia = max(tl.i0, lo[0]), ib = min(tl.i0 + tile_i - 1, hi[0]);
        for (int i = ia; i <= ib; ++i) Op::template run<GEO, P2>(c, a, i, j, k);
    }
}

template <bool GEO, bool P2>
__global__ void __launch_bounds__(kT, 4)  // the split work at 4 blocks per SM, as k_visc_split
    kb_visc(const Ctx *__restrict__ ctxs, const Tile *__restrict__ tiles, int ntiles, int tile_i)
{
    __shared__ Ctx c;
    __shared__ double wmin[kT / 32];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        int lo[3], hi[3];
        ops::Visc::bounds(ctxs[tl.inst].g, 0, lo, hi);
        const int nk = hi[2] - lo[2] + 1;
        if (tl.p0 >= (hi[1] - lo[1] + 1) * nk || tl.i0 > hi[0] || tl.i0 + tile_i - 1 < lo[0]) continue;
        __syncthreads();
        load_ctx(c, ctxs + tl.inst);
        __syncthreads();
        // two threads per cell, as the single-solve k_visc_split: warps 0-3
        // run the heating and forces, warps 4-7 the viscous pressure and CFL
        // candidate, each over the tile's points in two rounds of 128
        const int half = (int)threadIdx.x >> 7;
        double best = DBL_MAX;
        bool bad = false;
        for (int r = 0; r < 2; ++r) {
            const int p = tl.p0 + r * (kT / 2) + ((int)threadIdx.x & (kT / 2 - 1));
            if (p >= (hi[1] - lo[1] + 1) * nk) continue;
            const int j = lo[1] + p / nk, k = lo[2] + p % nk;
            const int ia = max(tl.i0, lo[0]), ib = min(tl.i0 + tile_i - 1, hi[0]);
            for (int i = ia; i <= ib; ++i) {
                if (half == 0)
                    ops::Visc::template heat_forces<GEO, P2>(c, i, j, k, bad);
                else if (i <= c.g.nx && j <= c.g.ny && k <= c.g.nz)
                    best = dev::pmin(best, ops::Visc::template cfl<GEO, P2>(c, i, j, k, bad));
            }
        }
        if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&c.sc->status, 1);
        for (int off = 16; off > 0; off >>= 1) best = dev::pmin(best, __shfl_xor_sync(0xffffffffu, best, off));
        if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = best;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = wmin[0];
            for (int w = 1; w < kT / 32; ++w) m = dev::pmin(m, wmin[w]);
            if (m < DBL_MAX) atomicMin(&c.sc->dtmin_bits, (unsigned long long)__double_as_longlong(m));
        }
    }
}

// The z sweep's S6, S7 and S8 as one kernel over whole z lines (the
// single-solve k_zsweep): each tile is a run of lines of one solve,
// kThreads / (nz + 4) of them, starting at line p0 of (i, j) in
// 0..nx x 0..ny.
template <bool GEO>
__global__ void __launch_bounds__(ops::kZLineThreads, 4)
    kb_zsweep(const Ctx *__restrict__ ctxs, const Tile *__restrict__ tiles, int ntiles)
{
    __shared__ Ctx c;
    extern __shared__ double zsm[];
    constexpr int kZT = ops::kZLineThreads;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        __syncthreads();
        load_ctx(c, ctxs + tl.inst);
        __syncthreads();
        const Geom &g = c.g;
        const int W = g.nz + 4, lines = kZT / W, S = lines * W;
        const int line = (int)threadIdx.x / W, k = (int)threadIdx.x % W - 2;
        const long long q = (long long)tl.p0 + line;
        const bool on = line < lines && q < (long long)(g.nx + 1) * (g.ny + 1);
        const int i = on ? (int)(q / (g.ny + 1)) : 0, j = on ? (int)(q % (g.ny + 1)) : 0;
        using F = ops::SweepFused<2>;
        static_assert(!F::kSharedFluxSlots, "the z passes of stage B run without a barrier between them");
        const ops::LineStore st{zsm, S, line * W + k + 2};
        const ops::SweepOut w = ops::sweep_in_place(c);
        if (on) F::stage_a<GEO>(c, i, j, k, st, w, true);
        __syncthreads();
        if (on && k >= 1 && k <= g.nz) F::stage_b_energy(c, i, j, k, st, w);
        if (on && k >= -1 && k <= g.nz) F::stage_b_mom<GEO>(c, i, j, k, st);  // its own slots: no barrier between
        __syncthreads();
        if (on && k >= 0 && k <= g.nz) F::stage_c(c, i, j, k, st, w);
    }
}

// Per-solve CFL finalisation (the single-solve k_dt_finalize, one thread per
// live solve).
__global__ void kb_dt_finalize(const Ctx *__restrict__ ctxs, const int *__restrict__ live, int nlive)
{
    const int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= nlive) return;
    const Ctx &c = ctxs[live[li]];
    Scalars *sc = c.sc;
    double m = __longlong_as_double((long long)sc->dtmin_bits);
    double dt = c.p.dt_multiplier * m;
    sc->dtr = dt;
    dt = dt < DBL_MAX ? dt : DBL_MAX;
    sc->dt = dt;
    if (c.p.resistive) {
        int nsub = (int)(dt / sc->dtr) + 1;
        sc->nsub = nsub;
        sc->dt_sub = dt / (double)nsub;
    }
    sc->dtmin_bits = (unsigned long long)__double_as_longlong(DBL_MAX);
    if (!(m < DBL_MAX) || !(dt > 0.0) || !(dt < DBL_MAX)) sc->status = 1;
    sc->time += dt;
    sc->step += 1;
}

__device__ __forceinline__ int locate(const long long *off, int n, long long g)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}


// Composite periodic fill (see k_bc_periodic in lare_solver.cu) for every
// live solve whose fields in `mask` are all-periodic.  The flat index walks
// the ghost shell of each solve's whole box (-2..n+2 outside the interior
// 1..n: x slabs, then y slabs inside x, then z slabs inside x and y); a
// point is decomposed once and then copied for every field whose own range
// holds it.  The set of points each field receives and their sources are
// those of the per-field fill.
__global__ void kb_bc_periodic(const Ctx *__restrict__ ctxs, const int *__restrict__ live,
                               const unsigned *__restrict__ pfields, const long long *__restrict__ off, int nlive,
                               long long total, unsigned mask, int resistive_only)
{
    for (long long gi = (long long)blockIdx.x * blockDim.x + threadIdx.x; gi < total;
         gi += (long long)gridDim.x * blockDim.x) {
        const int li = locate(off, nlive, gi);
        if ((mask & ~pfields[li]) != 0) continue;
        const Ctx &c = ctxs[live[li]];
        if (resistive_only && !c.p.resistive) continue;
        const Geom &g = c.g;
        const int n0 = g.nx, n1 = g.ny, n2 = g.nz;
        const int E1 = n1 + 5, E2 = n2 + 5;
        int t = (int)(gi - off[li]);
        int q0, q1, q2;
        const int A = 5 * E1 * E2, B = n0 * 5 * E2;
        if (t < A) {
            const int gx = t / (E1 * E2), r = t - gx * (E1 * E2);
            q0 = gx < 3 ? gx - 2 : n0 + gx - 2;
            q1 = r / E2 - 2;
            q2 = r - (q1 + 2) * E2 - 2;
        } else if ((t -= A) < B) {
            const int i = t / (5 * E2), r = t - i * (5 * E2);
            const int gy = r / E2;
            q0 = 1 + i;
            q1 = gy < 3 ? gy - 2 : n1 + gy - 2;
            q2 = r - gy * E2 - 2;
        } else {
            t -= B;
            const int i = t / (n1 * 5), r = t - i * (n1 * 5);
            const int j = r / 5, gz = r - j * 5;
            q0 = 1 + i;
            q1 = 1 + j;
            q2 = gz < 3 ? gz - 2 : n2 + gz - 2;
        }
        const int s0 = q0 <= 0 ? q0 + n0 : (q0 > n0 ? q0 - n0 : q0);
        const int s1 = q1 <= 0 ? q1 + n1 : (q1 > n1 ? q1 - n1 : q1);
        const int s2 = q2 <= 0 ? q2 + n2 : (q2 > n2 ? q2 - n2 : q2);
        const long long dst = box_off(g, q0, q1, q2), src = box_off(g, s0, s1, s2);
        for (int f = 0; f < SAMS_NFIELDS; ++f) {
            if (!(mask & (1u << f))) continue;
            // centred dimensions start at -1
            if ((q0 < -1 && !field_half(f, 0)) || (q1 < -1 && !field_half(f, 1)) || (q2 < -1 && !field_half(f, 2)))
                continue;
            double *a = c.f[f];
            a[dst] = a[src];
        }
    }
}

// One (dimension, edge) of the fields in `mask` for every live solve (those
// handled by the composite fill are skipped when skip_periodic is set); the
// point formula and the ordering rule of small dimensions are lare_bc.cuh's.
__global__ void kb_bc_edge(const Ctx *__restrict__ ctxs, const BcTable *__restrict__ bcs, const int *__restrict__ live,
                           const unsigned *__restrict__ pfields, const long long *__restrict__ off, int nlive,
                           long long total, unsigned mask, int d, int e, int skip_periodic, int resistive_only)
{
    for (long long gi = (long long)blockIdx.x * blockDim.x + threadIdx.x; gi < total;
         gi += (long long)gridDim.x * blockDim.x) {
        const int li = locate(off, nlive, gi);
        if (skip_periodic && (mask & ~pfields[li]) == 0) continue;
        const int inst = live[li];
        const Ctx &c = ctxs[inst];
        if (resistive_only && !c.p.resistive) continue;
        const BcTable &bt = bcs[inst];
        const long long t = gi - off[li];
        const Geom &g = c.g;
        for (int f = 0; f < SAMS_NFIELDS; ++f) {
            if (!(mask & (1u << f))) continue;
            const int kind = bt.kind[f][d][e];
            if (kind == SAMS_BC_NONE) continue;
            const BcEdge sl = bc_edge_slab(g, f, d, e);
            const int e1 = sl.hi[1] - sl.lo[1] + 1, e2 = sl.hi[2] - sl.lo[2] + 1;
            if (t >= (long long)(sl.hi[0] - sl.lo[0] + 1) * e1 * e2) continue;
            int q[3];
            q[0] = sl.lo[0] + (int)(t / ((long long)e1 * e2));
            q[1] = sl.lo[1] + (int)((t / e2) % e1);
            q[2] = sl.lo[2] + (int)(t % e2);
            bc_edge_apply(c.f[f], g, sl, bt, f, d, e, q);
        }
    }
}

void axes_host(double lo, double hi, long long n, std::vector<double> &db, std::vector<double> &dc)
{
    std::vector<double> b(n + 5), c(n + 5);
    double d = (hi - lo) / (double)n;
    for (long long i = -2; i <= n + 2; ++i) b[i + 2] = lo + d * (double)i;
    for (long long i = -1; i <= n + 2; ++i) c[i + 2] = 0.5 * (b[i + 2] + b[i + 1]);
    db.assign(n + 6, 0.0);
    dc.assign(n + 6, 0.0);
    for (long long i = -1; i <= n + 2; ++i) db[i + 2] = b[i + 2] - b[i + 1];
    db[0] = db[1];
    for (long long i = 0; i <= n + 2; ++i) dc[i + 2] = c[i + 2] - c[i + 1];
    dc[1] = dc[2];
}

Geom batch_geom(const sams_lare_params &p)
{
    Geom g{};
    g.nx = (int)p.nx;
    g.ny = (int)p.ny;
    g.nz = (int)p.nz;
    if (p.nz >= 32) {  // long rows: pad to 8 doubles with interior k = 1 on a 32-byte boundary
        g.zoff = 3;
        g.sy = (int)(((p.nz + 6) + 7) / 8 * 8);
    } else {            // short rows (e.g. nz = 4): dense
        g.zoff = 2;
        g.sy = (int)(p.nz + 5);
    }
    g.sx = (int)((p.ny + 5) * g.sy);
    g.nelem = (p.nx + 5) * (long long)g.sx;
    return g;
}

long long ceil_div(long long a, long long b) { return (a + b - 1) / b; }

}  // namespace

// ---------------------------------------------------------------------------

Batch::~Batch()
{
    cudaSetDevice(device_);
    drop_graphs();
    for (auto &s : slots_) free_slot(s);
    cudaFree(d_ctx_);  // one buffer holds every device table
    if (own_stream_) cudaStreamDestroy(own_stream_);
}

int Batch::check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return SAMS_OK;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? SAMS_ERR_NOMEM : SAMS_ERR_CUDA;
}

void Batch::drop_graphs()
{
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
}

void Batch::free_slot(BatchSlot &s)
{
    if (s.arena) cudaFree(s.arena);
    if (s.axes) cudaFree(s.axes);
    if (s.sc) cudaFree(s.sc);
    s = BatchSlot{};
}

int Batch::init(int device)
{
    device_ = device;
    int rc;
    if ((rc = check(cudaSetDevice(device), "cudaSetDevice"))) return rc;
    if ((rc = check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "cudaStreamCreate"))) return rc;
    stream_ = own_stream_;
    cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device);
    return SAMS_OK;
}

int Batch::set_stream(cudaStream_t s)
{
    stream_ = s ? s : own_stream_;
    drop_graphs();
    return SAMS_OK;
}

long long Batch::bytes_for(const sams_lare_params &p)
{
    Geom g = batch_geom(p);
    return (long long)(SAMS_NFIELDS + NSCRATCH + (p.rke ? 1 : 0)) * g.nelem * 8 + 8 * 2 * (p.nx + p.ny + p.nz + 18) + 256 +
           (p.geometry ? 8LL * (long long)geom_table_size(p) : 0LL);
}

int Batch::add(const sams_lare_params &p, const sams_lare_bcs &bcs, int *id)
{
    if (p.nx < 1 || p.ny < 1 || p.nz < 1 || p.nx > 60000 || p.ny > 60000 || p.nz > 60000) {
        err = "grid sizes must be in 1..60000";
        return SAMS_ERR_INVALID;
    }
    if (p.geometry < 0 || p.geometry > 2) { err = "geometry must be 0 (Cartesian), 1 (cylindrical) or 2 (spherical)"; return SAMS_ERR_UNSUPPORTED; }
    if (!(p.x_max > p.x_min) || !(p.y_max > p.y_min) || !(p.z_max > p.z_min)) { err = "empty domain"; return SAMS_ERR_INVALID; }
    {
        // tile planes and ghost shells are indexed with 32-bit integers
        const long long e1 = p.ny + 5, e2 = p.nz + 5;
        const long long shell = 5 * e1 * e2 + p.nx * 5 * e2 + p.nx * p.ny * 5;
        const long long rows = (p.nz >= 32 ? ((p.nz + 6) + 7) / 8 * 8 : e2) * e1 * (p.nx + 5);
        if (rows > INT32_MAX || shell > INT32_MAX) {
            err = "one array or the ghost shell of this solve exceeds 2^31 points";
            return SAMS_ERR_UNSUPPORTED;
        }
    }
    int rc;
    if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
    BatchSlot s;
    s.p = p;
    {
        const long long n[3] = {p.nx, p.ny, p.nz};
        if (!bc_table_from(s.bc, bcs, n, &err)) return SAMS_ERR_INVALID;
    }
    for (int f = 0; f < SAMS_NFIELDS; ++f) {
        bool per = true;
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 2; ++e) per = per && bcs.kind[f][d][e] == SAMS_BC_PERIODIC;
        // the one-pass periodic gather needs every source inside the domain
        if (per && std::min(p.nx, std::min(p.ny, p.nz)) >= kBcSequentialBelow) s.periodic_groups |= 1u << f;
    }
    Geom g = batch_geom(p);
    const size_t abytes = (size_t)(SAMS_NFIELDS + NSCRATCH + (p.rke ? 1 : 0)) * (size_t)g.nelem * sizeof(double);
    if ((rc = check(cudaMalloc(&s.arena, abytes), "cudaMalloc(solve)"))) return rc;
    cudaMemsetAsync(s.arena, 0, abytes, stream_);
    std::vector<double> dxb, dyb, dzb, dxc, dyc, dzc;
    axes_host(p.x_min, p.x_max, p.nx, dxb, dxc);
    axes_host(p.y_min, p.y_max, p.ny, dyb, dyc);
    axes_host(p.z_min, p.z_max, p.nz, dzb, dzc);
    std::vector<double> packed;
    for (auto *v : {&dxb, &dyb, &dzb, &dxc, &dyc, &dzc}) packed.insert(packed.end(), v->begin(), v->end());
    const size_t geo_off = packed.size();
    if (p.geometry) {  // metric factors after the spacings
        std::vector<double> t = geom_tables(p);
        packed.insert(packed.end(), t.begin(), t.end());
    }
    if ((rc = check(cudaMalloc(&s.axes, packed.size() * sizeof(double)), "cudaMalloc(axes)"))) { free_slot(s); return rc; }
    if ((rc = check(cudaMemcpy(s.axes, packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice), "axes"))) {
        free_slot(s);
        return rc;
    }
    if ((rc = check(cudaMalloc(&s.sc, sizeof(Scalars)), "cudaMalloc(scalars)"))) { free_slot(s); return rc; }
    Scalars s0{};
    s0.dtmin_bits = 0x7FEFFFFFFFFFFFFFull;
    if ((rc = check(cudaMemcpy(s.sc, &s0, sizeof(s0), cudaMemcpyHostToDevice), "scalars"))) { free_slot(s); return rc; }
    Ctx &c = s.ctx;
    c.g = g;
    for (int f = 0; f < SAMS_NFIELDS; ++f) c.f[f] = s.arena + (size_t)f * g.nelem;
    for (int q = 0; q < NSCRATCH; ++q) c.s[q] = s.arena + (size_t)(SAMS_NFIELDS + q) * g.nelem;
    c.dke = p.rke ? s.arena + (size_t)(SAMS_NFIELDS + NSCRATCH) * g.nelem : nullptr;
    size_t o = 0;
    const double **slots[6] = {&c.ax.dxb, &c.ax.dyb, &c.ax.dzb, &c.ax.dxc, &c.ax.dyc, &c.ax.dzc};
    const size_t lens[6] = {dxb.size(), dyb.size(), dzb.size(), dxc.size(), dyc.size(), dzc.size()};
    for (int a = 0; a < 6; ++a) {
        *slots[a] = s.axes + o;
        o += lens[a];
    }
    c.gf = GeomF{};
    if (p.geometry) geom_bind(c.gf, s.axes + geo_off, p);
    c.p.geometry = (int)p.geometry;
    c.p.pow2 = p.geometry == 0 && pow2_grid(dxb, dyb, dzb, dxc, dyc, dzc, p.mu0, &c.rc) ? 1 : 0;
    c.p.gamma = p.gas_gamma;
    c.p.mu0 = p.mu0;
    c.p.visc1 = p.visc1;
    c.p.visc2_norm = 0.25 * (p.gas_gamma + 1.0) * p.visc2;
    c.p.dt_multiplier = p.dt_multiplier;
    c.p.eta_bg = p.eta_background;
    c.p.eta0 = p.eta0;
    c.p.j_max = p.j_max;
    c.p.resistive = p.resistive_mhd ? 1 : 0;
    c.p.rke = p.rke ? 1 : 0;
    c.sc = s.sc;
    s.bytes = (long long)abytes + (long long)(packed.size() * sizeof(double)) + (long long)sizeof(Scalars);
    s.live = true;
    int slot = -1;
    for (size_t q = 0; q < slots_.size(); ++q)
        if (!slots_[q].live) { slot = (int)q; break; }
    if (slot < 0) {
        slot = (int)slots_.size();
        slots_.push_back(BatchSlot{});
    }
    slots_[slot] = s;
    *id = slot;
    dirty_ = true;
    drop_graphs();
    return check(cudaStreamSynchronize(stream_), "add sync");
}

int Batch::remove(int id)
{
    if (id < 0 || id >= (int)slots_.size() || !slots_[id].live) { err = "no such solve"; return SAMS_ERR_INVALID; }
    int rc;
    if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
    if ((rc = check(cudaStreamSynchronize(stream_), "remove sync"))) return rc;
    free_slot(slots_[id]);
    dirty_ = true;
    drop_graphs();
    return SAMS_OK;
}

int Batch::upload(int id, int field, const double *src, cudaMemcpyKind kind)
{
    if (id < 0 || id >= (int)slots_.size() || !slots_[id].live || field < 0 || field >= SAMS_NFIELDS || !src) {
        err = "invalid solve, field or buffer";
        return SAMS_ERR_INVALID;
    }
    const Geom &g = slots_[id].ctx.g;
    const size_t w = (size_t)(g.nz + 5) * sizeof(double);
    const size_t rows = (size_t)(g.nx + 5) * (size_t)(g.ny + 5);
    double *dst = slots_[id].ctx.f[field] + (g.zoff - 2);
    return check(cudaMemcpy2DAsync(dst, (size_t)g.sy * sizeof(double), src, w, w, rows, kind, stream_), "upload");
}

int Batch::download_async(int id, int field, double *dst)
{
    if (id < 0 || id >= (int)slots_.size() || !slots_[id].live || field < 0 || field >= SAMS_NFIELDS || !dst) {
        err = "invalid solve, field or buffer";
        return SAMS_ERR_INVALID;
    }
    const Geom &g = slots_[id].ctx.g;
    const size_t w = (size_t)(g.nz + 5) * sizeof(double);
    const size_t rows = (size_t)(g.nx + 5) * (size_t)(g.ny + 5);
    const double *src = slots_[id].ctx.f[field] + (g.zoff - 2);
    return check(cudaMemcpy2DAsync(dst, w, src, (size_t)g.sy * sizeof(double), w, rows, cudaMemcpyDefault, stream_),
                 "download");
}

int Batch::download(int id, int field, double *dst, cudaMemcpyKind kind)
{
    (void)kind;
    int rc = download_async(id, field, dst);
    if (rc) return rc;
    return check(cudaStreamSynchronize(stream_), "download sync");
}

int Batch::rebuild()
{
    std::vector<Ctx> ctx(slots_.size());
    std::vector<BcTable> bcs(slots_.size());
    std::vector<int> live;
    std::vector<unsigned> pf;
    std::vector<long long> shell_off, slab_off[3];
    std::vector<Tile> tiles;
    long long shell = 0, slab[3] = {0, 0, 0};
    has_resistive_ = 0;
    has_rke_ = 0;
    has_geo_ = 0;
    all_pow2_ = 1;
    for (size_t q = 0; q < slots_.size(); ++q) {
        ctx[q] = slots_[q].ctx;
        bcs[q] = slots_[q].bc;
        if (!slots_[q].live) continue;
        live.push_back((int)q);
        pf.push_back(slots_[q].periodic_groups);
        const Geom &g = slots_[q].ctx.g;
        has_resistive_ |= slots_[q].ctx.p.resistive;
        has_rke_ |= slots_[q].ctx.p.rke;
        has_geo_ |= slots_[q].ctx.p.geometry != 0;
        all_pow2_ &= slots_[q].ctx.p.pow2;
        shell_off.push_back(shell);
        const long long e0 = g.nx + 5, e1 = g.ny + 5, e2 = g.nz + 5;
        shell += 5 * e1 * e2 + (long long)g.nx * 5 * e2 + (long long)g.nx * g.ny * 5;
        slab_off[0].push_back(slab[0]);
        slab_off[1].push_back(slab[1]);
        slab_off[2].push_back(slab[2]);
        slab[0] += 3 * e1 * e2;
        slab[1] += 3 * e0 * e2;
        slab[2] += 3 * e0 * e1;
        const int plane = (int)(e1 * e2);
        for (int i0 = -2; i0 <= g.nx + 2; i0 += tile_i_)
            for (int p0 = 0; p0 < plane; p0 += kT) tiles.push_back(Tile{(int)q, i0, p0, 0});
    }
    nlive_ = (int)live.size();
    ntiles_ = (int)tiles.size();
    // z-line tiles of the fused z sweep, after the plane tiles; used when no
    // solve needs the raw momentum fluxes (rke) and every z line fits a block
    constexpr int kZT = ops::kZLineThreads;
    zfuse_ = nlive_ > 0 && !has_rke_;
    for (int q : live)
        if (slots_[q].ctx.g.nz + 4 > kZT) zfuse_ = false;
    if (zfuse_)
        for (int q : live) {
            const Geom &g = slots_[q].ctx.g;
            const int lpb = kZT / (g.nz + 4);
            const long long nl = (long long)(g.nx + 1) * (g.ny + 1);
            for (long long first = 0; first < nl; first += lpb) tiles.push_back(Tile{q, 0, (int)first, 0});
        }
    nztiles_ = (int)tiles.size() - ntiles_;
    shell_total_ = shell;
    for (int d = 0; d < 3; ++d) slab_total_[d] = slab[d];
    // one device buffer for all tables
    const size_t nslot = slots_.size() ? slots_.size() : 1;
    const size_t need = nslot * sizeof(Ctx) + nslot * sizeof(BcTable) + std::max<size_t>(tiles.size(), 1) * sizeof(Tile) +
                        (size_t)std::max(nlive_, 1) * (sizeof(int) + sizeof(unsigned) + 4 * sizeof(long long)) + 1024;
    int rc;
    if (need > table_cap_bytes_) {
        cudaFree(d_ctx_);
        d_ctx_ = nullptr;
        size_t cap = need * 2;
        if ((rc = check(cudaMalloc((void **)&d_ctx_, cap), "cudaMalloc(batch tables)"))) return rc;
        table_cap_bytes_ = cap;
    }
    char *base = reinterpret_cast<char *>(d_ctx_);
    size_t o = nslot * sizeof(Ctx);
    d_bc_ = reinterpret_cast<BcTable *>(base + o);
    BcTable *d_bc = d_bc_;
    o += nslot * sizeof(BcTable);
    o = (o + 15) / 16 * 16;
    d_tiles_ = reinterpret_cast<Tile *>(base + o);
    o += std::max<size_t>(tiles.size(), 1) * sizeof(Tile);
    o = (o + 15) / 16 * 16;
    d_live_ = reinterpret_cast<int *>(base + o);
    o += (size_t)std::max(nlive_, 1) * sizeof(int);
    o = (o + 15) / 16 * 16;
    d_pf_ = reinterpret_cast<unsigned *>(base + o);
    unsigned *d_pf = d_pf_;
    o += (size_t)std::max(nlive_, 1) * sizeof(unsigned);
    o = (o + 15) / 16 * 16;
    d_shell_off_ = reinterpret_cast<long long *>(base + o);
    o += (size_t)std::max(nlive_, 1) * sizeof(long long);
    d_slab_off_ = reinterpret_cast<long long *>(base + o);
    (void)d_bc;
    (void)d_pf;
    auto cp = [&](void *dst, const void *src, size_t n) {
        return n ? check(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, stream_), "batch tables") : SAMS_OK;
    };
    if ((rc = cp(d_ctx_, ctx.data(), ctx.size() * sizeof(Ctx)))) return rc;
    if ((rc = cp(d_bc, bcs.data(), bcs.size() * sizeof(BcTable)))) return rc;
    if ((rc = cp(d_tiles_, tiles.data(), tiles.size() * sizeof(Tile)))) return rc;
    if ((rc = cp(d_live_, live.data(), live.size() * sizeof(int)))) return rc;
    if ((rc = cp(d_pf, pf.data(), pf.size() * sizeof(unsigned)))) return rc;
    if ((rc = cp(d_shell_off_, shell_off.data(), shell_off.size() * sizeof(long long)))) return rc;
    for (int d = 0; d < 3; ++d)
        if ((rc = cp(d_slab_off_ + (size_t)d * std::max(nlive_, 1), slab_off[d].data(),
                     slab_off[d].size() * sizeof(long long))))
            return rc;
    dirty_ = false;
    // keep the host-side copies alive until the async copies are done
    return check(cudaStreamSynchronize(stream_), "batch tables sync");
}

template <class Op>
void Batch::launch(int arg, bool resistive_only)
{
    if (ntiles_ == 0) return;
    const int grid = std::min(ntiles_, sm_count_ * blocks_per_sm_);
    const int ro = resistive_only ? 1 : 0;
    if (has_geo_)
        kb_op<Op, true, false><<<grid, kT, 0, stream_>>>(d_ctx_, d_tiles_, ntiles_, arg, tile_i_, ro);
    else if (all_pow2_)
        kb_op<Op, false, true><<<grid, kT, 0, stream_>>>(d_ctx_, d_tiles_, ntiles_, arg, tile_i_, ro);
    else
        kb_op<Op, false, false><<<grid, kT, 0, stream_>>>(d_ctx_, d_tiles_, ntiles_, arg, tile_i_, ro);
}

void Batch::launch_zsweep()
{
    if (nztiles_ == 0) return;
    constexpr int kZT = ops::kZLineThreads;
    const int grid = std::min(nztiles_, sm_count_ * 4);
    const size_t smem = (size_t)ops::SweepFused<2>::NARR * kZT * sizeof(double);
    if (has_geo_)
        kb_zsweep<true><<<grid, kZT, smem, stream_>>>(d_ctx_, d_tiles_ + ntiles_, nztiles_);
    else
        kb_zsweep<false><<<grid, kZT, smem, stream_>>>(d_ctx_, d_tiles_ + ntiles_, nztiles_);
}

void Batch::launch_visc()
{
    if (ntiles_ == 0) return;
    const int grid = std::min(ntiles_, sm_count_ * blocks_per_sm_);
    if (has_geo_)
        kb_visc<true, false><<<grid, kT, 0, stream_>>>(d_ctx_, d_tiles_, ntiles_, tile_i_);
    else if (all_pow2_)
        kb_visc<false, true><<<grid, kT, 0, stream_>>>(d_ctx_, d_tiles_, ntiles_, tile_i_);
    else
        kb_visc<false, false><<<grid, kT, 0, stream_>>>(d_ctx_, d_tiles_, ntiles_, tile_i_);
}

void Batch::bc_fill(unsigned mask, bool resistive_only)
{
    if (nlive_ == 0) return;
    const BcTable *d_bc = d_bc_;
    const unsigned *d_pf = d_pf_;
    const int grid = (int)std::min<long long>(ceil_div(shell_total_, kT), (long long)sm_count_ * 8);
    kb_bc_periodic<<<grid, kT, 0, stream_>>>(d_ctx_, d_live_, d_pf, d_shell_off_, nlive_, shell_total_, mask,
                                             resistive_only ? 1 : 0);
    bool any_general = false;
    for (auto &s : slots_)
        if (s.live && (mask & ~s.periodic_groups)) any_general = true;
    if (!any_general) return;
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 2; ++e) {
            const int g2 = (int)std::min<long long>(ceil_div(slab_total_[d], kT), (long long)sm_count_ * 8);
            kb_bc_edge<<<g2, kT, 0, stream_>>>(d_ctx_, d_bc, d_live_, d_pf, d_slab_off_ + (size_t)d * std::max(nlive_, 1),
                                               nlive_, slab_total_[d], mask, d, e, 1, resistive_only ? 1 : 0);
        }
}

void Batch::bc_fill_dim(unsigned mask, int d, bool resistive_only)
{
    if (nlive_ == 0) return;
    const BcTable *d_bc = d_bc_;
    const unsigned *d_pf = d_pf_;
    const int g2 = (int)std::min<long long>(ceil_div(slab_total_[d], kT), (long long)sm_count_ * 8);
    for (int e = 0; e < 2; ++e)
        kb_bc_edge<<<g2, kT, 0, stream_>>>(d_ctx_, d_bc, d_live_, d_pf, d_slab_off_ + (size_t)d * std::max(nlive_, 1),
                                           nlive_, slab_total_[d], mask, d, e, 0, resistive_only ? 1 : 0);
}

void Batch::enqueue_step()
{
    // ---- Lagrangian predictor ----
    launch<ops::CellPrep>(-1, false);
    launch<ops::NodePrep>(0, false);
    launch<ops::Alpha>(0, false);
    launch_visc();
    if (nlive_) kb_dt_finalize<<<(unsigned)ceil_div(nlive_, 128), 128, 0, stream_>>>(d_ctx_, d_live_, nlive_);
    if (has_resistive_) {
        for (int sub = 0; sub < 2; ++sub) {
            launch<ops::ResistRK>(0, true);
            launch<ops::ResistB>(sub == 1 ? 1 : 0, true);
            bc_fill(FM_BFIELD | FM_ENERGY, true);
        }
    }
    launch<ops::Pred1>(-1, false);
    launch<ops::Pred2>(0, false);
    bc_fill(FM_REMAPV, false);
    // ---- corrector ----
    launch<ops::Corr1>(0, false);
    launch<ops::Corr2>(0, false);
    bc_fill(FM_VELOCITY | FM_ENERGY | FM_DENSITY, false);
    // ---- remap ----
    if (has_rke_) launch<ops::RkeZero>(0, false);
    launch<ops::BScale>(0, false);
    launch<ops::SweepVol<0>>(0, false);
    launch<ops::SweepCvc>(0, false);
    launch<ops::SweepCT<0>>(0, false);
    launch<ops::SweepCTUpd<0>>(0, false);
    launch<ops::SweepMass<0>>(0, false);
    bc_fill_dim(FM_DM, 0, false);
    launch<ops::SweepS6<0>>(0, false);
    launch<ops::SweepS7<0>>(0, false);
    if (has_rke_) {  // solves without rke return at once (Phys::rke)
        launch<ops::SweepRkeDk<0>>(0, false);
        launch<ops::SweepRkeGather<0>>(0, false);
    }
    launch<ops::SweepS8<0>>(0, false);
    bc_fill(FM_ALL9, false);
    launch<ops::SweepVol<1>>(0, false);
    launch<ops::SweepCvc>(0, false);
    launch<ops::SweepCT<1>>(0, false);
    launch<ops::SweepCTUpd<1>>(0, false);
    launch<ops::SweepMass<1>>(0, false);
    bc_fill_dim(FM_DM, 1, false);
    launch<ops::SweepS6<1>>(0, false);
    launch<ops::SweepS7<1>>(0, false);
    if (has_rke_) {  // solves without rke return at once (Phys::rke)
        launch<ops::SweepRkeDk<1>>(0, false);
        launch<ops::SweepRkeGather<1>>(0, false);
    }
    launch<ops::SweepS8<1>>(0, false);
    bc_fill(FM_ALL9, false);
    launch<ops::SweepVol<2>>(0, false);
    launch<ops::SweepCvc>(0, false);
    launch<ops::SweepCT<2>>(0, false);
    launch<ops::SweepCTUpd<2>>(0, false);
    launch<ops::SweepMass<2>>(0, false);
    bc_fill_dim(FM_DM, 2, false);
    if (zfuse_) {
        launch_zsweep();
    } else {
        launch<ops::SweepS6<2>>(0, false);
        launch<ops::SweepS7<2>>(0, false);
        if (has_rke_) {  // solves without rke return at once (Phys::rke)
            launch<ops::SweepRkeDk<2>>(0, false);
            launch<ops::SweepRkeGather<2>>(0, false);
        }
        launch<ops::SweepS8<2>>(0, false);
    }
    bc_fill(FM_ALL9, false);
    launch<ops::BScale>(1, false);
    bc_fill(FM_BFIELD, false);
    if (has_rke_) launch<ops::RkeEnergy>(0, false);
}

int Batch::step(long long nsteps)
{
    if (nsteps < 0) { err = "negative step count"; return SAMS_ERR_INVALID; }
    int rc;
    if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
    if (dirty_ && (rc = rebuild())) return rc;
    for (long long s = 0; s < nsteps; ++s) enqueue_step();
    return check(cudaGetLastError(), "batch step launch");
}

int Batch::step_graph(long long nsteps)
{
    if (nsteps < 0) { err = "negative step count"; return SAMS_ERR_INVALID; }
    if (nsteps == 0) return SAMS_OK;
    int rc;
    if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
    if (dirty_) {
        if ((rc = rebuild())) return rc;
        drop_graphs();
    }
    auto it = graphs_.find(nsteps);
    if (it == graphs_.end()) {
        cudaGraph_t graph;
        if ((rc = check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture"))) return rc;
        for (long long s = 0; s < nsteps; ++s) enqueue_step();
        if ((rc = check(cudaStreamEndCapture(stream_, &graph), "end capture"))) return rc;
        cudaGraphExec_t exec;
        rc = check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
        cudaGraphDestroy(graph);
        if (rc) return rc;
        it = graphs_.emplace(nsteps, exec).first;
    }
    return check(cudaGraphLaunch(it->second, stream_), "graph launch");
}

int Batch::sync() { return check(cudaStreamSynchronize(stream_), "batch synchronize"); }

int Batch::scalars(int id, Scalars &out)
{
    if (id < 0 || id >= (int)slots_.size() || !slots_[id].live) { err = "no such solve"; return SAMS_ERR_INVALID; }
    int rc = check(cudaMemcpyAsync(&out, slots_[id].sc, sizeof(Scalars), cudaMemcpyDeviceToHost, stream_), "scalars");
    if (rc) return rc;
    return check(cudaStreamSynchronize(stream_), "scalars sync");
}

int Batch::set_tuning(int tile_i, int blocks_per_sm)
{
    if (tile_i < 1 || tile_i > 64 || blocks_per_sm < 1 || blocks_per_sm > 32) {
        err = "tile_i must be 1..64 and blocks_per_sm 1..32";
        return SAMS_ERR_INVALID;
    }
    tile_i_ = tile_i;
    blocks_per_sm_ = blocks_per_sm;
    dirty_ = true;
    drop_graphs();
    return SAMS_OK;
}

// Time every candidate tiling on the live batch for trial_steps steps and keep
// the fastest.  The state of every solve (13 fields and its scalars) is
// copied aside first and restored afterwards, so tuning leaves the solves
// exactly where they were.
int Batch::autotune(int trial_steps, int *tile_i, int *blocks_per_sm, double *best_ms)
{
    if (trial_steps < 1) trial_steps = 1;
    int rc;
    if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
    std::vector<double *> backup;
    std::vector<Scalars *> sback;
    for (auto &s : slots_) {
        if (!s.live) { backup.push_back(nullptr); sback.push_back(nullptr); continue; }
        double *b = nullptr;
        Scalars *sb = nullptr;
        size_t n = (size_t)SAMS_NFIELDS * (size_t)s.ctx.g.nelem * sizeof(double);
        if ((rc = check(cudaMalloc(&b, n), "cudaMalloc(autotune backup)"))) break;
        if ((rc = check(cudaMalloc(&sb, sizeof(Scalars)), "cudaMalloc(autotune backup)"))) { cudaFree(b); break; }
        cudaMemcpyAsync(b, s.arena, n, cudaMemcpyDeviceToDevice, stream_);
        cudaMemcpyAsync(sb, s.sc, sizeof(Scalars), cudaMemcpyDeviceToDevice, stream_);
        backup.push_back(b);
        sback.push_back(sb);
    }
    const int tiles[] = {1, 2, 4, 8};
    const int bps[] = {2, 4, 8};
    int bt = tile_i_, bb = blocks_per_sm_;
    double best = 1e300;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int ti : tiles) {
        if (rc) break;
        for (int b : bps) {
            set_tuning(ti, b);
            if ((rc = step(1))) break;  // warm-up (also rebuilds the tables)
            cudaEventRecord(e0, stream_);
            if ((rc = step(trial_steps))) break;
            cudaEventRecord(e1, stream_);
            if ((rc = check(cudaEventSynchronize(e1), "autotune sync"))) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                bt = ti;
                bb = b;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (size_t q = 0; q < slots_.size(); ++q) {
        if (!slots_[q].live || !backup[q]) continue;
        size_t n = (size_t)SAMS_NFIELDS * (size_t)slots_[q].ctx.g.nelem * sizeof(double);
        cudaMemcpyAsync(slots_[q].arena, backup[q], n, cudaMemcpyDeviceToDevice, stream_);
        cudaMemcpyAsync(slots_[q].sc, sback[q], sizeof(Scalars), cudaMemcpyDeviceToDevice, stream_);
    }
    cudaStreamSynchronize(stream_);
    for (auto *b : backup) cudaFree(b);
    for (auto *b : sback) cudaFree(b);
    set_tuning(bt, bb);
    if (tile_i) *tile_i = bt;
    if (blocks_per_sm) *blocks_per_sm = bb;
    if (best_ms) *best_ms = best / trial_steps;
    return rc;
}

long long Batch::device_bytes() const
{
    long long b = (long long)table_cap_bytes_;
    for (auto &s : slots_)
        if (s.live) b += s.bytes;
    return b;
}

int Batch::live_count() const
{
    int n = 0;
    for (auto &s : slots_) n += s.live ? 1 : 0;
    return n;
}

long long Batch::live_cells() const
{
    long long n = 0;
    for (auto &s : slots_)
        if (s.live) n += s.p.nx * s.p.ny * s.p.nz;
    return n;
}

}  // namespace sams
