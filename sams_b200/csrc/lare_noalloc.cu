// lare_noalloc.cu -- a LARE3D step for callers that cannot allocate device
// memory.
//
// Some hosts of this code cannot call cudaMalloc once they are running: a
// Fortran or C simulation whose device memory all comes from its own pool
// allocator, or an application that has handed the rest of the GPU's memory
// to other work and must not grow its footprint.  sams_lare_step_noalloc lets
// them advance a solve held in their own device buffers: they pass the 13
// field arrays (inputs and outputs), and the step's scratch comes from one
// fixed array compiled into this library.
//
// The scratch array is a file-scope __device__ array of
// SAMS_NOALLOC_SCRATCH_BYTES (64 MiB).  Every GPU that loads the library
// holds it until the process exits.  Its device address is looked up once per
// device, on the first call made with that device current (the first call
// should therefore come before any stream capture).  All calls share the
// array and it keeps the previous call's contents: each call clears the part
// it uses before stepping, and calls that overlap on the GPU (two streams,
// two host threads) race on it.
#include "sams_lare.h"
#include "lare_solver.cuh"

#include <cstring>
#include <mutex>
#include <string>

#define SAMS_NOALLOC_SCRATCH_BYTES (64ull << 20)

static __device__ __align__(256) double g_noalloc_scratch[SAMS_NOALLOC_SCRATCH_BYTES / sizeof(double)];

// defined in lare_capi.cu (library-internal)
void sams_capi_set_last_error(const std::string &msg);

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_scratch_addr[kMaxDevices] = {};

// failures are reported through sams_lare_last_error()
int fail(int rc, const std::string &msg)
{
    sams_capi_set_last_error(msg);
    return rc;
}

// The 1-D spacings exactly as the harness builds them (axisRegistry.h:393-430,
// the first delta copied from the next), on the device so that nothing is
// staged through host memory.
__global__ void k_noalloc_axes(double *out, double lo, double hi, long long n, int centred)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x - 2;
    if (i > n + 3) return;
    const double d = (hi - lo) / (double)n;
    auto b = [&](long long q) { return lo + d * (double)q; };
    auto c = [&](long long q) { return 0.5 * (b(q) + b(q - 1)); };
    double v = 0.0;
    if (!centred) {
        long long q = i < -1 ? -1 : i;  // db(-2) = db(-1)
        if (q <= n + 2) v = b(q) - b(q - 1);
    } else {
        long long q = i < 0 ? 0 : i;    // dc(-1) = dc(0); dc(-2) unused
        if (i >= -1 && q <= n + 2) v = c(q) - c(q - 1);
    }
    out[i + 2] = v;
}

__global__ void k_noalloc_scalars(sams::Scalars *sc, double dt, double time)
{
    sams::Scalars s{};
    s.dt = dt;
    s.time = time;
    s.dtmin_bits = 0x7FEFFFFFFFFFFFFFull;  // DBL_MAX
    *sc = s;
}

}  // namespace

extern "C" int sams_lare_step_noalloc(const sams_lare_params *params, const sams_lare_bcs *bcs,
                                      double *const dev_fields[SAMS_NFIELDS], double *dt_inout,
                                      double *time_inout, int64_t nsteps, void *stream)
{
    if (!params || !bcs || !dev_fields || !dt_inout || !time_inout || nsteps < 0)
        return fail(SAMS_ERR_INVALID, "sams_lare_step_noalloc: null argument or negative step count");
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        if (!dev_fields[f]) return fail(SAMS_ERR_INVALID, "sams_lare_step_noalloc: null field pointer");
    const sams_lare_params &p = *params;
    if (p.nx < 1 || p.ny < 1 || p.nz < 1 || !(p.x_max > p.x_min) || !(p.y_max > p.y_min) || !(p.z_max > p.z_min))
        return fail(SAMS_ERR_INVALID, "sams_lare_step_noalloc: empty grid or domain");
    // per-dimension bound first, so that the box products below cannot overflow
    if (p.nx > 60000 || p.ny > 60000 || p.nz > 60000)
        return fail(SAMS_ERR_INVALID, "sams_lare_step_noalloc: grid too large (a dimension above 60000 cells)");

    // Fields are dense box buffers: -2..n+2 per dimension, z fastest.
    sams::Geom g{};
    g.nx = (int)p.nx;
    g.ny = (int)p.ny;
    g.nz = (int)p.nz;
    g.zoff = 2;
    g.sy = (int)(p.nz + 5);
    g.sx = (int)((p.ny + 5) * (p.nz + 5));
    g.nelem = (p.nx + 5) * (p.ny + 5) * (p.nz + 5);
    const unsigned long long axis_len[3] = {(unsigned long long)p.nx + 6, (unsigned long long)p.ny + 6,
                                            (unsigned long long)p.nz + 6};
    const unsigned long long scratch_elems = (unsigned long long)sams::NSCRATCH * (unsigned long long)g.nelem;
    const unsigned long long axes_elems = 2 * (axis_len[0] + axis_len[1] + axis_len[2]);
    const unsigned long long scalar_elems = (sizeof(sams::Scalars) + 255) / 256 * 32;
    const unsigned long long need = (scratch_elems + axes_elems + scalar_elems) * sizeof(double);
    if (need > SAMS_NOALLOC_SCRATCH_BYTES)
        return fail(SAMS_ERR_INVALID,
                    "sams_lare_step_noalloc: grid too large: it needs " + std::to_string(need) +
                        " bytes of scratch and the static array holds " +
                        std::to_string(SAMS_NOALLOC_SCRATCH_BYTES) +
                        " (19 box arrays: about (nx+5)(ny+5)(nz+5) <= 440000)");

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return fail(SAMS_ERR_CUDA, "sams_lare_step_noalloc: no usable current CUDA device");
    double *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_scratch_addr[device]) {
            cudaError_t e = cudaGetSymbolAddress((void **)&g_scratch_addr[device], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_scratch_addr[device] = nullptr;
                return fail(SAMS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            }
        }
        base = g_scratch_addr[device];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Carve the static array: scratch fields, six axes, scalars.
    sams::Ctx ctx{};
    ctx.g = g;
    for (int f = 0; f < SAMS_NFIELDS; ++f) ctx.f[f] = dev_fields[f];
    for (int s = 0; s < sams::NSCRATCH; ++s) ctx.s[s] = base + (size_t)s * (size_t)g.nelem;
    double *ax = base + scratch_elems;
    double *dxb = ax, *dyb = dxb + axis_len[0], *dzb = dyb + axis_len[1];
    double *dxc = dzb + axis_len[2], *dyc = dxc + axis_len[0], *dzc = dyc + axis_len[1];
    ctx.ax = {dxb, dyb, dzb, dxc, dyc, dzc};
    ctx.sc = reinterpret_cast<sams::Scalars *>(ax + axes_elems);
    ctx.p.gamma = p.gas_gamma;
    ctx.p.mu0 = p.mu0;
    ctx.p.visc1 = p.visc1;
    ctx.p.visc2_norm = 0.25 * (p.gas_gamma + 1.0) * p.visc2;
    ctx.p.dt_multiplier = p.dt_multiplier;
    ctx.p.eta_bg = p.eta_background;
    ctx.p.eta0 = p.eta0;
    ctx.p.j_max = p.j_max;

    // Previous calls' contents: clear the scratch this call uses.
    cudaError_t e = cudaMemsetAsync(base, 0, (size_t)need, st);
    if (e != cudaSuccess) return fail(SAMS_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    const double lo[3] = {p.x_min, p.y_min, p.z_min}, hi[3] = {p.x_max, p.y_max, p.z_max};
    const long long n[3] = {p.nx, p.ny, p.nz};
    double *bout[3] = {dxb, dyb, dzb}, *cout[3] = {dxc, dyc, dzc};
    for (int d = 0; d < 3; ++d) {
        unsigned blocks = (unsigned)((n[d] + 6 + 127) / 128);
        k_noalloc_axes<<<blocks, 128, 0, st>>>(bout[d], lo[d], hi[d], n[d], 0);
        k_noalloc_axes<<<blocks, 128, 0, st>>>(cout[d], lo[d], hi[d], n[d], 1);
    }
    k_noalloc_scalars<<<1, 1, 0, st>>>(ctx.sc, *dt_inout, *time_inout);

    sams::Solver solver;
    int rc = solver.init_borrowed(p, *bcs, ctx, device, st);
    if (rc == SAMS_OK) rc = solver.step(nsteps);
    sams::Scalars out{};
    if (rc == SAMS_OK) {
        e = cudaMemcpyAsync(&out, ctx.sc, sizeof(out), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            solver.err = std::string("sams_lare_step_noalloc: ") + cudaGetErrorString(e);
            rc = SAMS_ERR_CUDA;
        }
    }
    std::string msg = solver.err;
    solver.release_borrowed();
    if (rc != SAMS_OK) return fail(rc, msg);
    if (out.status) return fail(SAMS_ERR_NONFINITE, "the CFL timestep became non-finite or non-positive");
    *dt_inout = out.dt;
    *time_inout = out.time;
    return SAMS_OK;
}
