// lare_solver.cuh -- one LARE3D solve resident on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "lare_device.cuh"
#include "lare_bc.cuh"
#include "sams_lare.h"

namespace sams {

// Sets of fields filled together (the LARE3D *_bcs groups,
// src/PhysicsPackages/LARE/boundary.cpp:27-97).
enum : unsigned {
    FM_BFIELD = (1u << SAMS_F_BX) | (1u << SAMS_F_BY) | (1u << SAMS_F_BZ),
    FM_ENERGY = (1u << SAMS_F_ENERGY_ELECTRON) | (1u << SAMS_F_ENERGY_ION),
    FM_DENSITY = (1u << SAMS_F_RHO),
    FM_VELOCITY = (1u << SAMS_F_VX) | (1u << SAMS_F_VY) | (1u << SAMS_F_VZ),
    FM_REMAPV = (1u << SAMS_F_VX1) | (1u << SAMS_F_VY1) | (1u << SAMS_F_VZ1),
    FM_DM = (1u << SAMS_F_DM),
    FM_ALL9 = FM_BFIELD | FM_ENERGY | FM_DENSITY | FM_VELOCITY
};

class Solver;

// A solve split along x into slabs (lare_dist.cu): the slab's place in the
// whole grid, and the hooks that replace the x boundary fills (halo
// exchange with the neighbouring slabs) and complete the CFL minimum over
// all slabs.
struct XSlab {
    long long off = 0;        // global index of the slab's cell 0 (cells off+1 .. off+nx)
    long long nx_global = 0;  // cells of the whole grid along x
};

class Halo {
public:
    virtual ~Halo() = default;
    // Fill the x ghost planes of the fields in mask (exchange at slab
    // edges, the boundary condition at the grid's own edges).
    virtual void fill_x(Solver &s, unsigned mask) = 0;
    // Replace this slab's CFL candidate minimum by the minimum over all slabs.
    virtual void reduce_dt(Solver &s) = 0;
};

class Solver {
public:
    Solver() = default;
    ~Solver();
    Solver(const Solver &) = delete;
    Solver &operator=(const Solver &) = delete;

    // Returns a sams_status; on failure err holds the reason.
    int init(const sams_lare_params &p, const sams_lare_bcs &bcs, int device);
    // Device bytes a solve of these parameters takes: state and scratch
    // arrays, the host-transfer staging buffer, axes and metric tables (an
    // upper bound, for admission under a memory budget).
    static long long bytes_for(const sams_lare_params &p);
    // Whether the step of a solve of these parameters runs the fused
    // marching and windowed kernels (its z lines fill their tiles).
    static bool fused_path(const sams_lare_params &p);
    // One x slab of a larger grid: p.nx is the slab's own cell count, the
    // x axis and metric tables are those of the whole grid (slab.nx_global
    // cells over x_min..x_max) from the slab's offset on.
    int init_slab(const sams_lare_params &p, const sams_lare_bcs &bcs, int device, const XSlab &slab);
    void set_halo(Halo *h) { halo_ = h; }
    cudaStream_t stream() const { return stream_; }
    Scalars *scalars_ptr() const { return sc_; }
    int device() const { return device_; }
    const BcTable &bc_table() const { return bc_; }
    // Boundary-condition fill of one (dimension, edge) for the fields in mask.
    void bc_fill_edge(unsigned mask, int dim, int edge);
    // Set up over memory the solver does not own (fields, scratch, axes and
    // scalars already placed in ctx); allocates nothing and frees nothing.
    int init_borrowed(const sams_lare_params &p, const sams_lare_bcs &bcs, const Ctx &ctx, int device,
                      cudaStream_t stream);
    // Forget borrowed memory (call before destroying a borrowed solver).
    void release_borrowed();
    int set_bc(int field, int dim, int edge, int kind, double value);
    int set_stream(cudaStream_t s);
    int upload(int field, const double *src, cudaMemcpyKind kind);
    int download(int field, double *dst, cudaMemcpyKind kind);
    int step(long long nsteps);
    int step_graph(long long nsteps);
    int sync();
    int scalars(Scalars &out);
    // Restart: the dt of the last step taken, the time and the step count.
    int set_scalars(double dt, double time, long long step);
    long long device_bytes() const { return bytes_; }
    long long launches_per_step() const { return launches_per_step_; }
    const Geom &geom() const { return ctx_.g; }
    double *field_ptr(int f) const { return ctx_.f[f]; }

    std::string err;

    // Enqueue one step on the current stream (no synchronisation).  With
    // marks != nullptr, records marks[0..5] around the step's phases:
    // Lagrangian predictor, corrector, x, y and z remap sweeps.
    void enqueue_step(cudaEvent_t *marks = nullptr);
    // Run one step and return the device time of each phase in ms.
    int phase_times(double ms[5]);

private:
    int check(cudaError_t e, const char *what);
    void bc_fill(unsigned mask);
    void bc_fill_dim(unsigned mask, int dim);
    bool all_periodic(unsigned mask) const;
    bool ghosts_refilled(unsigned mask) const;
    template <class Op> void launch(int arg);
    template <int DIR> void launch_psweep(int ct_arg);
    template <class P> void launch_cellnode(int arg);
    template <class P> void launch_edges();
    void launch_pred(int resistive);
    void launch_resist(bool last);
    // true when the kernel also wrote dm's periodic ghost images along DIR
    template <int DIR> bool launch_ctmass(int scale);
    int setup_psweep();
    int staging(double **out);
    void free_all();

    int init_impl(const sams_lare_params &p, const sams_lare_bcs &bcs, int device, const XSlab *slab);

    sams_lare_params p_{};
    BcTable bc_{};
    Halo *halo_ = nullptr;
    bool psweep_ok_ = false;  // the fused x / y sweep's shared memory fits this device
    int device_ = 0;
    int sm_count_ = 148;  // multiprocessors of device_ (grid sizing)
    cudaStream_t own_stream_ = nullptr;
    cudaStream_t stream_ = nullptr;
    Ctx ctx_{};
    double *arena_ = nullptr;
    double *axes_ = nullptr;
    Scalars *sc_ = nullptr;
    double *staging_ = nullptr;  // dense box buffer for host transfers (on first use)
    long long bytes_ = 0;
    long long launches_ = 0;
    long long launches_per_step_ = 0;
    std::map<long long, cudaGraphExec_t> graphs_;
};

}  // namespace sams
