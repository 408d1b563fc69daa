// lare_batch.cuh -- many independent LARE3D solves stepped together.
//
// Every phase of the step is ONE persistent launch over a worklist of tiles
// drawn from all live solves (a tile = one solve, a slab of tile_i planes
// along x, one chunk of 256 points of the (y, z) plane).  Each solve keeps its
// own state, scratch, metrics and device scalars, so each advances with its
// own CFL timestep; the batch shares only the launches.  The whole batched
// step is recorded once into a CUDA graph and replayed until the set of
// solves or the tiling changes.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "lare_device.cuh"
#include "lare_solver.cuh"
#include "sams_lare.h"

namespace sams {

struct Tile {
    int inst;  // slot of the solve in the batch's Ctx table
    int i0;    // first x plane of the slab
    int p0;    // first flattened (y, z) point of the chunk
    int pad;
};

struct BatchSlot {
    bool live = false;
    sams_lare_params p{};
    BcTable bc{};
    Ctx ctx{};
    double *arena = nullptr;
    double *axes = nullptr;
    Scalars *sc = nullptr;
    long long bytes = 0;
    unsigned periodic_groups = 0;  // bit g set: field group g all-periodic
};

class Batch {
public:
    Batch() = default;
    ~Batch();
    Batch(const Batch &) = delete;
    Batch &operator=(const Batch &) = delete;

    int init(int device);
    int set_stream(cudaStream_t s);
    int add(const sams_lare_params &p, const sams_lare_bcs &bcs, int *id);
    int remove(int id);
    int upload(int id, int field, const double *src, cudaMemcpyKind kind);
    int download(int id, int field, double *dst, cudaMemcpyKind kind);
    int download_async(int id, int field, double *dst);
    int step(long long nsteps);
    int step_graph(long long nsteps);
    int sync();
    int scalars(int id, Scalars &out);
    int set_tuning(int tile_i, int blocks_per_sm);
    int autotune(int trial_steps, int *tile_i, int *blocks_per_sm, double *best_ms);
    long long device_bytes() const;
    int live_count() const;
    long long live_cells() const;
    static long long bytes_for(const sams_lare_params &p);
    cudaStream_t stream() const { return stream_; }

    std::string err;

private:
    int check(cudaError_t e, const char *what);
    int rebuild();
    void enqueue_step();
    template <class Op> void launch(int arg, bool resistive_only);
    void launch_visc();
    void launch_zsweep();
    void bc_fill(unsigned mask, bool resistive_only);
    void bc_fill_dim(unsigned mask, int dim, bool resistive_only);
    void drop_graphs();
    void free_slot(BatchSlot &s);

    int device_ = 0;
    cudaStream_t own_stream_ = nullptr;
    cudaStream_t stream_ = nullptr;
    std::vector<BatchSlot> slots_;
    bool dirty_ = true;
    int tile_i_ = 2;
    int blocks_per_sm_ = 4;
    int sm_count_ = 148;
    // device tables (rebuilt when the set of solves changes)
    Ctx *d_ctx_ = nullptr;
    Tile *d_tiles_ = nullptr;  // plane tiles, then (when zfuse_) the z-line tiles
    int ntiles_ = 0;
    int nztiles_ = 0;
    bool zfuse_ = false;  // the z sweep's S6-S8 run as one kernel (kb_zsweep)
    int *d_live_ = nullptr;
    unsigned *d_pf_ = nullptr;          // per live solve: fields that are all-periodic
    BcTable *d_bc_ = nullptr;           // per slot boundary conditions
    long long *d_shell_off_ = nullptr;  // prefix of ghost-shell points per live solve
    long long *d_slab_off_ = nullptr;   // 3 x prefix of one-edge slab points per live solve
    long long shell_total_ = 0, slab_total_[3] = {0, 0, 0};
    int nlive_ = 0;
    int has_resistive_ = 0;
    int has_rke_ = 0;
    int has_geo_ = 0;
    int all_pow2_ = 0;  // every live solve has a power-of-two grid
    size_t table_cap_bytes_ = 0;
    std::map<long long, cudaGraphExec_t> graphs_;
};

}  // namespace sams
