// lare_capi.cu -- the extern "C" boundary (include/sams_lare.h) over
// sams::Solver.
#include "sams_lare.h"
#include "lare_solver.cuh"
#include "lare_dump.cuh"

#include <cstring>
#include <new>
#include <string>
#include <vector>

struct sams_lare_solver {
    sams::Solver s;
};

namespace {
thread_local std::string g_last_error;

int fail(int rc, const std::string &msg)
{
    g_last_error = msg;
    return rc;
}

int pass(sams_lare_solver *h, int rc)
{
    if (rc != SAMS_OK) g_last_error = h->s.err;
    return rc;
}

cudaMemcpyKind host_kind(const void *p)
{
    // pageable and pinned host memory both work with cudaMemcpyDefault
    (void)p;
    return cudaMemcpyDefault;
}
}  // namespace

// Library-internal: lets other translation units report through
// sams_lare_last_error().
__attribute__((visibility("hidden"))) void sams_capi_set_last_error(const std::string &msg)
{
    g_last_error = msg;
}

extern "C" {

int sams_lare_abi_version(void) { return 100; }

const char *sams_lare_last_error(void) { return g_last_error.c_str(); }

int sams_lare_create(const sams_lare_params *params, const sams_lare_bcs *bcs, int device, sams_lare_solver **out)
{
    if (!params || !bcs || !out) return fail(SAMS_ERR_INVALID, "sams_lare_create: null argument");
    *out = nullptr;
    sams_lare_solver *h = new (std::nothrow) sams_lare_solver();
    if (!h) return fail(SAMS_ERR_NOMEM, "sams_lare_create: host allocation failed");
    int rc = h->s.init(*params, *bcs, device);
    if (rc != SAMS_OK) {
        g_last_error = h->s.err;
        delete h;
        return rc;
    }
    *out = h;
    return SAMS_OK;
}

int sams_lare_destroy(sams_lare_solver *h)
{
    if (!h) return fail(SAMS_ERR_INVALID, "sams_lare_destroy: null handle");
    delete h;
    return SAMS_OK;
}

int sams_lare_set_stream(sams_lare_solver *h, void *stream)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.set_stream(static_cast<cudaStream_t>(stream)));
}

int sams_lare_set_bc(sams_lare_solver *h, int field, int dim, int edge, int kind, double value)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.set_bc(field, dim, edge, kind, value));
}

int sams_lare_upload_field(sams_lare_solver *h, int field, const double *host_box)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.upload(field, host_box, host_kind(host_box)));
}

int sams_lare_download_field(sams_lare_solver *h, int field, double *host_box)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.download(field, host_box, host_kind(host_box)));
}

int sams_lare_upload_field_device(sams_lare_solver *h, int field, const double *dev_box)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.upload(field, dev_box, cudaMemcpyDeviceToDevice));
}

int sams_lare_download_field_device(sams_lare_solver *h, int field, double *dev_box)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.download(field, dev_box, cudaMemcpyDeviceToDevice));
}

int sams_lare_step(sams_lare_solver *h, int64_t nsteps)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.step(nsteps));
}

int sams_lare_step_graph(sams_lare_solver *h, int64_t nsteps)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.step_graph(nsteps));
}

int sams_lare_synchronize(sams_lare_solver *h)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null handle");
    return pass(h, h->s.sync());
}

int sams_lare_get_dt(sams_lare_solver *h, double *dt)
{
    if (!h || !dt) return fail(SAMS_ERR_INVALID, "null argument");
    sams::Scalars s;
    int rc = h->s.scalars(s);
    if (rc) return pass(h, rc);
    *dt = s.dt;
    return SAMS_OK;
}

int sams_lare_get_time(sams_lare_solver *h, double *time)
{
    if (!h || !time) return fail(SAMS_ERR_INVALID, "null argument");
    sams::Scalars s;
    int rc = h->s.scalars(s);
    if (rc) return pass(h, rc);
    *time = s.time;
    return SAMS_OK;
}

int sams_lare_get_step(sams_lare_solver *h, int64_t *step)
{
    if (!h || !step) return fail(SAMS_ERR_INVALID, "null argument");
    sams::Scalars s;
    int rc = h->s.scalars(s);
    if (rc) return pass(h, rc);
    *step = s.step;
    return SAMS_OK;
}

int sams_lare_field_device_ptr(sams_lare_solver *h, int field, double **ptr, int64_t strides[3], int64_t *zoff)
{
    if (!h || !ptr || !strides || !zoff || field < 0 || field >= SAMS_NFIELDS)
        return fail(SAMS_ERR_INVALID, "invalid argument");
    const sams::Geom &g = h->s.geom();
    *ptr = h->s.field_ptr(field);
    strides[0] = g.sx;
    strides[1] = g.sy;
    strides[2] = 1;
    *zoff = g.zoff;
    return SAMS_OK;
}

int sams_lare_device_bytes(sams_lare_solver *h, int64_t *bytes)
{
    if (!h || !bytes) return fail(SAMS_ERR_INVALID, "invalid argument");
    *bytes = h->s.device_bytes();
    return SAMS_OK;
}

int sams_lare_save(sams_lare_solver *h, const char *path)
{
    if (!h || !path) return fail(SAMS_ERR_INVALID, "sams_lare_save: null argument");
    const sams::Geom &g = h->s.geom();
    const size_t n = (size_t)(g.nx + 5) * (g.ny + 5) * (g.nz + 5);
    std::vector<std::vector<double>> bufs(SAMS_NFIELDS, std::vector<double>(n));
    const double *box[SAMS_NFIELDS];
    int rc;
    for (int f = 0; f < SAMS_NFIELDS; ++f) {
        if ((rc = h->s.download(f, bufs[f].data(), cudaMemcpyDefault))) return pass(h, rc);
        box[f] = bufs[f].data();
    }
    sams::Scalars sc;
    if ((rc = h->s.scalars(sc))) return pass(h, rc);
    sams::DumpState st{g.nx, g.ny, g.nz, sc.step, sc.time, sc.dt};
    std::string err;
    if ((rc = sams::dump_write(path, st, box, err))) return fail(rc, "sams_lare_save: " + err);
    return SAMS_OK;
}

int sams_lare_load(sams_lare_solver *h, const char *path)
{
    if (!h || !path) return fail(SAMS_ERR_INVALID, "sams_lare_load: null argument");
    const sams::Geom &g = h->s.geom();
    const size_t n = (size_t)(g.nx + 5) * (g.ny + 5) * (g.nz + 5);
    std::vector<std::vector<double>> bufs(SAMS_NFIELDS, std::vector<double>(n, 0.0));
    double *box[SAMS_NFIELDS];
    for (int f = 0; f < SAMS_NFIELDS; ++f) box[f] = bufs[f].data();
    bool present[SAMS_NFIELDS];
    sams::DumpState st{g.nx, g.ny, g.nz, 0, 0.0, 0.0};
    std::string err;
    int rc = sams::dump_read(path, st, box, present, err);
    if (rc) return fail(rc, "sams_lare_load: " + err);
    const int state[9] = {SAMS_F_RHO, SAMS_F_ENERGY_ELECTRON, SAMS_F_ENERGY_ION, SAMS_F_VX, SAMS_F_VY,
                          SAMS_F_VZ, SAMS_F_BX, SAMS_F_BY, SAMS_F_BZ};
    for (int f : state)
        if (!present[f])
            return fail(SAMS_ERR_INVALID, std::string("sams_lare_load: ") + path + " lacks state field " +
                                              sams_lare_field_names[f]);
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        if (present[f] && (rc = h->s.upload(f, box[f], cudaMemcpyDefault))) return pass(h, rc);
    return pass(h, h->s.set_scalars(st.dt, st.time, st.step));
}

int sams_lare_phase_times(sams_lare_solver *h, double ms[5])
{
    if (!h || !ms) return fail(SAMS_ERR_INVALID, "invalid argument");
    return pass(h, h->s.phase_times(ms));
}

int sams_lare_launches_per_step(sams_lare_solver *h, int64_t *launches)
{
    if (!h || !launches) return fail(SAMS_ERR_INVALID, "invalid argument");
    *launches = h->s.launches_per_step();
    return SAMS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched solves (include/sams_lare.h, "batch" section)
// ---------------------------------------------------------------------------
#include "lare_batch.cuh"

struct sams_lare_batch {
    sams::Batch b;
};

namespace {
int bpass(sams_lare_batch *h, int rc)
{
    if (rc != SAMS_OK) g_last_error = h->b.err;
    return rc;
}
}  // namespace

extern "C" {

int sams_lare_batch_create(int device, sams_lare_batch **out)
{
    if (!out) return fail(SAMS_ERR_INVALID, "sams_lare_batch_create: null argument");
    *out = nullptr;
    sams_lare_batch *h = new (std::nothrow) sams_lare_batch();
    if (!h) return fail(SAMS_ERR_NOMEM, "host allocation failed");
    int rc = h->b.init(device);
    if (rc != SAMS_OK) {
        g_last_error = h->b.err;
        delete h;
        return rc;
    }
    *out = h;
    return SAMS_OK;
}

int sams_lare_batch_destroy(sams_lare_batch *h)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    delete h;
    return SAMS_OK;
}

int sams_lare_batch_set_stream(sams_lare_batch *h, void *stream)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.set_stream(static_cast<cudaStream_t>(stream)));
}

int sams_lare_batch_add(sams_lare_batch *h, const sams_lare_params *p, const sams_lare_bcs *bcs, int *id)
{
    if (!h || !p || !bcs || !id) return fail(SAMS_ERR_INVALID, "null argument");
    return bpass(h, h->b.add(*p, *bcs, id));
}

int sams_lare_batch_remove(sams_lare_batch *h, int id)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.remove(id));
}

int sams_lare_batch_upload_field(sams_lare_batch *h, int id, int field, const double *host_box)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.upload(id, field, host_box, cudaMemcpyDefault));
}

int sams_lare_batch_download_field(sams_lare_batch *h, int id, int field, double *host_box)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.download(id, field, host_box, cudaMemcpyDefault));
}

int sams_lare_batch_step(sams_lare_batch *h, int64_t nsteps)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.step(nsteps));
}

int sams_lare_batch_step_graph(sams_lare_batch *h, int64_t nsteps)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.step_graph(nsteps));
}

int sams_lare_batch_synchronize(sams_lare_batch *h)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.sync());
}

int sams_lare_batch_get_state(sams_lare_batch *h, int id, double *dt, double *time, int64_t *step)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    sams::Scalars s;
    int rc = h->b.scalars(id, s);
    if (rc) return bpass(h, rc);
    if (s.status) return fail(SAMS_ERR_NONFINITE, "the CFL timestep of this solve became non-finite");
    if (dt) *dt = s.dt;
    if (time) *time = s.time;
    if (step) *step = s.step;
    return SAMS_OK;
}

int sams_lare_batch_set_tuning(sams_lare_batch *h, int tile_planes, int blocks_per_sm)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.set_tuning(tile_planes, blocks_per_sm));
}

int sams_lare_batch_autotune(sams_lare_batch *h, int trial_steps, int *tile_planes, int *blocks_per_sm,
                             double *ms_per_step)
{
    if (!h) return fail(SAMS_ERR_INVALID, "null batch");
    return bpass(h, h->b.autotune(trial_steps, tile_planes, blocks_per_sm, ms_per_step));
}

int sams_lare_batch_device_bytes(sams_lare_batch *h, int64_t *bytes)
{
    if (!h || !bytes) return fail(SAMS_ERR_INVALID, "null argument");
    *bytes = h->b.device_bytes();
    return SAMS_OK;
}

}  // extern "C"
