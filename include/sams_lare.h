/*
 * sams_lare.h -- C ABI of the B200 LARE3D timestep.
 *
 * This is the drop-in boundary for the reference's LARE3D physics package
 * (src/PhysicsPackages/LARE/shared_data.h:229-508).  In the reference the
 * package is a C++ class driven by SAMS::runner events; here the same state
 * and the same step are owned by an opaque solver handle whose memory lives
 * on one GPU.  Plain pointers, sizes and status codes only: no C++ or torch
 * types cross this boundary.  Host buffers use the box layout of
 * sams_lare_layout.h.
 *
 * Every function returns SAMS_OK (0) or a negative status; the message of
 * the last failure on the calling thread is available from
 * sams_lare_last_error().  Calls on one handle are not thread-safe.
 */
#ifndef SAMS_LARE_H
#define SAMS_LARE_H

#include <stddef.h>
#include <stdint.h>
#include "sams_lare_layout.h"
#include "sams_lare_ic.h"

#ifdef __cplusplus
extern "C" {
#endif

enum sams_status {
    SAMS_OK = 0,
    SAMS_ERR_INVALID = -1,      /* bad argument or unsupported option      */
    SAMS_ERR_NOMEM = -2,        /* device or host allocation failed         */
    SAMS_ERR_CUDA = -3,         /* a CUDA runtime call failed               */
    SAMS_ERR_UNSUPPORTED = -4,  /* geometry or option not built            */
    SAMS_ERR_NONFINITE = -5,    /* the timestep became NaN or infinite      */
    SAMS_ERR_TIMEOUT = -6,      /* a bounded wait ran out                   */
    SAMS_ERR_BUDGET = -7        /* request exceeds the memory budget        */
};

typedef struct sams_lare_solver sams_lare_solver;

/* Version of this ABI (major * 100 + minor). */
int sams_lare_abi_version(void);

/* Message of the last failure on this thread ("" if none). */
const char *sams_lare_last_error(void);

/* Create a solver on a CUDA device: allocates the 13 harness variables and
 * the step's scratch on that device and builds the grid metrics.
 * Replaces LARE3D::registerAxes/registerVariables/allocate/grid
 * (setup.cpp:27-437) and the runner's decomposeAndAllocate
 * (include/runner/runner.h:456-464).  Boundary conditions are copied; they
 * replace the IC package's setBoundaryConditions
 * (variableDef::addBoundaryCondition, include/harness/variableDef.h:402-481).
 * Supported: Cartesian, cylindrical and spherical geometry (params.geometry
 * 0, 1, 2), rke on or off. */
int sams_lare_create(const sams_lare_params *params, const sams_lare_bcs *bcs,
                     int device, sams_lare_solver **out);

/* Free all device memory of the solver. */
int sams_lare_destroy(sams_lare_solver *h);

/* Run the solver's work on this CUDA stream (cudaStream_t passed as void*);
 * NULL selects the solver's own stream. */
int sams_lare_set_stream(sams_lare_solver *h, void *stream);

/* Replace one (field, dim, edge) boundary condition; see sams_lare_bc_kind.
 * Replaces variableDef::addBoundaryCondition(dim, edge, bc). */
int sams_lare_set_bc(sams_lare_solver *h, int field, int dim, int edge,
                     int kind, double value);

/* Copy one field from a host box buffer to the device (asynchronous on the
 * solver's stream when the buffer is pinned).  Together they replace the IC
 * package's initialConditions writes into variableRegistry arrays
 * (src/InitialConditions/OrszagTang/OrszagTang.cpp:104-156). */
int sams_lare_upload_field(sams_lare_solver *h, int field, const double *host_box);
int sams_lare_download_field(sams_lare_solver *h, int field, double *host_box);

/* Checkpoint / restart.  save writes the 13 harness variables over their
 * local ranges, the step count, the time and the last step's dt (which the
 * next step's edge viscosity reads) as a SAMSDUMP1 file: a text magic line,
 * a one-line JSON header with an array directory, then little-endian float64
 * arrays -- the dump format the oracle's reference harness writes for the
 * reference's own state (the reference itself writes no field data,
 * src/PhysicsPackages/LARE/io/writerSimple.h:151).  load reads such a file of the same grid
 * (the nine state fields must be present; extra arrays are skipped), so a
 * run resumes bit for bit, also from a state the reference produced.
 * Replaces the runner's output/restart hooks (include/runner/runner.h:505-525)
 * for this path.  Both synchronise the solver's stream. */
int sams_lare_save(sams_lare_solver *h, const char *path);
int sams_lare_load(sams_lare_solver *h, const char *path);

/* Same, from / to a device box buffer (e.g. a CUDA tensor's storage). */
int sams_lare_upload_field_device(sams_lare_solver *h, int field, const double *dev_box);
int sams_lare_download_field_device(sams_lare_solver *h, int field, double *dev_box);

/* Advance nsteps full timesteps, asynchronously on the solver's stream.
 * One step is the runner's startOfTimestep -> halfTimestep -> step/time
 * update -> endOfTimestep sequence (include/runner/runner.h:564-586) over
 * LARE3D::lagrangian_step, corrector_step and eulerian_remap
 * (shared_data.h:397-419).  The CFL timestep is reduced on the device
 * (lagran.cpp:380-443) and never read back. */
int sams_lare_step(sams_lare_solver *h, int64_t nsteps);

/* Same, but the nsteps are recorded once into a CUDA graph and replayed. */
int sams_lare_step_graph(sams_lare_solver *h, int64_t nsteps);

/* Wait for the solver's stream. */
int sams_lare_synchronize(sams_lare_solver *h);

/* Current dt / time / step count (these synchronise).  Replace
 * SAMS::timeState (runner.h:20-25) and LARE3D::getTimestep. */
int sams_lare_get_dt(sams_lare_solver *h, double *dt);
int sams_lare_get_time(sams_lare_solver *h, double *time);
int sams_lare_get_step(sams_lare_solver *h, int64_t *step);

/* Device address of a field's box storage and its element strides
 * (x, y, z; z stride is 1) and z offset: element (i,j,k) lives at
 * ptr[(i+2)*sx + (j+2)*sy + (k+zoff)]. */
int sams_lare_field_device_ptr(sams_lare_solver *h, int field, double **ptr,
                               int64_t strides[3], int64_t *zoff);

/* Device bytes held by the solver. */
int sams_lare_device_bytes(sams_lare_solver *h, int64_t *bytes);

/* Advance one step and report the device time (ms) of its five phases:
 * Lagrangian predictor (startOfTimestep), corrector (halfTimestep), and the
 * x, y and z remap sweeps (endOfTimestep).  Replaces the reference's
 * per-event timers (include/runner/runnerMacros.h:113-150). */
int sams_lare_phase_times(sams_lare_solver *h, double ms[5]);

/* Number of kernel launches one sams_lare_step(h, 1) issues. */
int sams_lare_launches_per_step(sams_lare_solver *h, int64_t *launches);

/* No counterpart in the reference (it has no performance model).  Measured
 * FP64 throughput of `device`, in thread-level operations per second, for
 * the compute roof of the step: rates[0] add, [1] multiply, [2] fused
 * multiply-add, [3] IEEE division by data, [4] IEEE square root (with one
 * multiply), [5] correctly rounded reciprocal (with one multiply).  Runs
 * for about a second on an idle B200. */
int sams_lare_fp64_rates(int device, double rates[6]);

/* ---- Batched solves ----------------------------------------------------
 * Many independent LARE3D solves (any mix of sizes, parameters and boundary
 * conditions) stepped together: each phase of the step is one persistent
 * launch over a worklist of tiles drawn from every solve in the batch, and
 * each solve keeps its own CFL timestep.  The reference runs one
 * simulationData per runner (shared_data.h:60-226, runner.h:564-586); a
 * batch replaces N runners stepping one after another. */
typedef struct sams_lare_batch sams_lare_batch;

int sams_lare_batch_create(int device, sams_lare_batch **out);
int sams_lare_batch_destroy(sams_lare_batch *b);
int sams_lare_batch_set_stream(sams_lare_batch *b, void *stream);
/* Add a solve (allocates its device state); *id identifies it. */
int sams_lare_batch_add(sams_lare_batch *b, const sams_lare_params *params,
                        const sams_lare_bcs *bcs, int *id);
/* Remove a solve and free its device memory. */
int sams_lare_batch_remove(sams_lare_batch *b, int id);
int sams_lare_batch_upload_field(sams_lare_batch *b, int id, int field, const double *host_box);
int sams_lare_batch_download_field(sams_lare_batch *b, int id, int field, double *host_box);
/* Advance every solve in the batch nsteps steps (asynchronous). */
int sams_lare_batch_step(sams_lare_batch *b, int64_t nsteps);
/* Same, replaying a CUDA graph of nsteps batched steps. */
int sams_lare_batch_step_graph(sams_lare_batch *b, int64_t nsteps);
int sams_lare_batch_synchronize(sams_lare_batch *b);
/* dt, time and step count of one solve (any pointer may be NULL). */
int sams_lare_batch_get_state(sams_lare_batch *b, int id, double *dt, double *time, int64_t *step);
/* Tile shape: x planes per tile and resident blocks per SM of the
 * persistent launches. */
int sams_lare_batch_set_tuning(sams_lare_batch *b, int tile_planes, int blocks_per_sm);
/* Time each candidate tile shape on the live batch for trial_steps steps
 * and keep the fastest; the solves' states are restored afterwards. */
int sams_lare_batch_autotune(sams_lare_batch *b, int trial_steps, int *tile_planes,
                             int *blocks_per_sm, double *ms_per_step);
int sams_lare_batch_device_bytes(sams_lare_batch *b, int64_t *bytes);

/* ---- Serving: continuous batching under a device-memory budget ----------
 * A scheduler thread keeps the running solves resident on the GPU and
 * advances them together one step at a time: solves whose z lines fill the
 * single-solve path's fused kernels each launch their own step graph on their
 * own stream, the rest share one batched step, and all of these overlap on
 * the device.  Queued requests are admitted in arrival order as soon as
 * their device footprint fits the budget, and each finished solve's state is
 * copied to the host and its memory freed.  A solve's result is the same
 * bits on either path.  The reference has no serving layer (one runner = one
 * solve, runner.h:564-586). */
typedef struct sams_lare_server sams_lare_server;

enum sams_serve_status {
    SAMS_SERVE_QUEUED = 0,
    SAMS_SERVE_RUNNING = 1,
    SAMS_SERVE_DONE = 2,
    SAMS_SERVE_FAILED = 3,
    SAMS_SERVE_CANCELLED = 4
};

typedef struct sams_lare_serve_stats {
    int64_t submitted, completed, failed, queued, running;
    double p50_latency_s, p99_latency_s, mean_latency_s;  /* submit -> result on host */
    double cell_updates, wall_s, cell_updates_per_s;      /* since creation */
    int64_t device_bytes_in_use;
    /* outstanding work: interior cells x steps still to run, summed over the
     * queued and running requests, and the device bytes the queued ones will
     * take when admitted */
    double pending_cell_updates;
    int64_t queued_bytes;
} sams_lare_serve_stats;

int sams_lare_serve_create(int device, int64_t budget_bytes, sams_lare_server **out);
/* Queue a solve of nsteps steps.  ic[f] are 13 host box buffers read when the
 * solve is admitted (keep them valid until the status is RUNNING or later).
 * out[q] receive the final rho, e_e, e_i, vx, vy, vz, bx, by, bz (box
 * buffers, valid until DONE); with out == NULL the server keeps the result
 * for sams_lare_serve_fetch.  Rejects a solve larger than the whole budget
 * with SAMS_ERR_BUDGET. */
int sams_lare_serve_submit(sams_lare_server *s, const sams_lare_params *params,
                           const sams_lare_bcs *bcs, const double *const ic[SAMS_NFIELDS],
                           int64_t nsteps, double *const out[9], int64_t *ticket);
/* Device bytes a solve takes while a server runs it (what admission charges
 * against the budget). */
int sams_lare_serve_solve_bytes(const sams_lare_params *params, int64_t *bytes);
/* Cap the interior cells (nx*ny*nz summed) of the solves running at once;
 * 0 (the default) leaves only the memory budget.  Under a backlog a smaller
 * running set finishes each solve sooner, so a cap just large enough to keep
 * the GPU busy lowers latency at the same throughput.  Admission stays in
 * arrival order: a request that does not fit waits at the head of the queue
 * (one solve larger than the cap still runs, alone). */
int sams_lare_serve_set_max_cells(sams_lare_server *s, int64_t max_cells);
/* Status (sams_serve_status) and latency so far / at completion. */
int sams_lare_serve_poll(sams_lare_server *s, int64_t ticket, int *status, double *latency_s);
/* Copy one of the nine kept result fields (index as for out[]). */
int sams_lare_serve_fetch(sams_lare_server *s, int64_t ticket, int state_index, double *host_box);
/* Withdraw a request: a queued one leaves the queue at once; a running one
 * is retired (its device memory freed, no result) before the scheduler's
 * next step, after which its status is SAMS_SERVE_CANCELLED.  A request that
 * already finished is refused with SAMS_ERR_INVALID. */
int sams_lare_serve_cancel(sams_lare_server *s, int64_t ticket);
/* Forget a finished or cancelled request (frees a kept result). */
int sams_lare_serve_release(sams_lare_server *s, int64_t ticket);
/* Wait until nothing is queued or running (SAMS_ERR_TIMEOUT otherwise). */
int sams_lare_serve_drain(sams_lare_server *s, double timeout_s);
int sams_lare_serve_get_stats(sams_lare_server *s, sams_lare_serve_stats *stats);
/* Stop the scheduler and free everything. */
int sams_lare_serve_destroy(sams_lare_server *s);

/* ---- Serving on several GPUs --------------------------------------------
 * No counterpart in the reference (its runner is one solve per MPI job).
 * Independent solves need no exchange, so a host router owns one server per
 * listed device (each with its own scheduler thread, stream and budget) and
 * sends each submitted solve to the least-loaded one: among the devices
 * whose budget can hold the solve, those where it fits next to what is
 * already admitted or queued come first, then the least outstanding work
 * (pending_cell_updates), then the fewest committed bytes, then the lowest
 * index.  A device may be listed more than once (two servers share it).
 * Tickets are the router's own; every call mirrors its sams_lare_serve_*
 * counterpart. */
typedef struct sams_lare_router sams_lare_router;

int sams_lare_router_create(const int *devices, int ndevices, int64_t budget_bytes_per_device,
                            sams_lare_router **out);
int sams_lare_router_submit(sams_lare_router *r, const sams_lare_params *params,
                            const sams_lare_bcs *bcs, const double *const ic[SAMS_NFIELDS],
                            int64_t nsteps, double *const out[9], int64_t *ticket);
/* Index (into the create call's device list) of the server a ticket went to. */
int sams_lare_router_placement(sams_lare_router *r, int64_t ticket, int *index);
int sams_lare_router_set_max_cells(sams_lare_router *r, int64_t max_cells_per_device);
int sams_lare_router_poll(sams_lare_router *r, int64_t ticket, int *status, double *latency_s);
int sams_lare_router_fetch(sams_lare_router *r, int64_t ticket, int state_index, double *host_box);
int sams_lare_router_cancel(sams_lare_router *r, int64_t ticket);
int sams_lare_router_release(sams_lare_router *r, int64_t ticket);
int sams_lare_router_drain(sams_lare_router *r, double timeout_s);
/* Totals over every server; latency percentiles over all completed requests. */
int sams_lare_router_get_stats(sams_lare_router *r, sams_lare_serve_stats *stats);
/* One server's own statistics (index into the device list). */
int sams_lare_router_server_stats(sams_lare_router *r, int index, sams_lare_serve_stats *stats);
int sams_lare_router_destroy(sams_lare_router *r);

/* The router's placement rule on its own (host only, no device): loads of n
 * servers, a solve of request_bytes; *index receives the choice.  Returns
 * SAMS_ERR_BUDGET when no server's budget can hold the solve. */
int sams_lare_route_pick(int n, const double *pending_cell_updates, const int64_t *committed_bytes,
                         const int64_t *budget_bytes, int64_t request_bytes, int *index);

/* ---- One solve on several GPUs -------------------------------------------
 * The reference's MPI decomposition with MPIManager::haloExchange
 * (include/harness/mpiManager.h:1246-1277), for grids larger than one GPU:
 * the grid is cut along x into nparts slabs of nx/nparts (+1) cells, slab q
 * on devices[q] (a device may hold several slabs).  At every boundary fill of
 * the step each slab pulls its x ghost planes from the neighbouring slabs by
 * peer copies; the CFL minimum is taken over all slabs.  The result equals
 * the undivided solve's bit for bit.  Needs at least three cells per slab;
 * rke is not available (its correction gathers over the whole grid in order). */
typedef struct sams_lare_dist sams_lare_dist;

/* Host only: offsets[0..nparts] with slab q covering cells offsets[q]+1 ..
 * offsets[q+1] (the partition sams_lare_dist_create uses). */
int sams_lare_dist_partition(int64_t nx, int nparts, int64_t *offsets);
int sams_lare_dist_create(const sams_lare_params *params, const sams_lare_bcs *bcs, const int *devices, int nparts,
                          sams_lare_dist **out);
/* First global cell index (1-based) and cell count of slab `part`. */
int sams_lare_dist_slab(sams_lare_dist *d, int part, int64_t *first_cell, int64_t *ncells);
/* Whole-grid box buffers (-2..n+2 per dimension, z fastest), as for a single solve. */
int sams_lare_dist_upload_field(sams_lare_dist *d, int field, const double *host_box);
int sams_lare_dist_download_field(sams_lare_dist *d, int field, double *host_box);
/* Advance nsteps timesteps on every slab; returns when they are done. */
int sams_lare_dist_step(sams_lare_dist *d, int64_t nsteps);
int sams_lare_dist_get_state(sams_lare_dist *d, double *dt, double *time, int64_t *step);
int sams_lare_dist_destroy(sams_lare_dist *d);

/* No counterpart in the reference.  Advance nsteps timesteps of a solve whose
 * 13 fields live in the caller's own device memory, allocating nothing: for
 * callers that cannot call cudaMalloc while running (a host code whose device
 * memory all comes from its own pool, or one that must not grow its device
 * footprint).  dev_fields[f] are dense box buffers on the current device
 * (-2..n+2 per dimension, z fastest, no padding), read and written in place.
 * *dt_inout is the previous step's dt (0 before the first step) and
 * *time_inout the time; both are updated.  Runs on `stream` (NULL = legacy
 * default stream) and returns when the steps are done.
 * The step's scratch is a static 64 MiB device array inside the library
 * (held by every GPU that loads it until exit), enough for
 * (nx+5)(ny+5)(nz+5) up to about 440000; larger grids are rejected with
 * SAMS_ERR_INVALID.  The first call on a device looks up that array's address
 * and should come before any stream capture.  Calls share the array: calls
 * that overlap on the GPU race. */
int sams_lare_step_noalloc(const sams_lare_params *params, const sams_lare_bcs *bcs,
                           double *const dev_fields[SAMS_NFIELDS], double *dt_inout,
                           double *time_inout, int64_t nsteps, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SAMS_LARE_H */
