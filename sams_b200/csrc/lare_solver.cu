// lare_solver.cu -- kernels and step orchestration of one LARE3D solve.
//
// One step on the device, in launch order (reference events in brackets;
// the standard path: Cartesian or curvilinear, no rke, every dimension at
// least three cells, every B edge with a condition):
//   [startOfTimestep -> lagrangian_step, lagran.cpp:95-173]
//     k_cellnode_march (CellPrep + NodePrep), Alpha, k_visc_split (Visc +
//     CFL block minima), DtFinalize, resistive only: 2 x {k_resist_march (ResistRK +
//     ResistB), fill B + energies}, k_pred_march (Pred1 + Pred2), fill v1
//   [halfTimestep -> corrector_step, lagran.cpp:739-804]
//     k_edge_march (Corr1 from per-node edge terms), Corr2, fill v +
//     energies + rho
//   [endOfTimestep -> eulerian_remap, remap.cpp:23-111]
//     x: k_cellnode_march (SweepVol + SweepCvc), k_ctmass (SweepCT +
//        SweepMass), SweepCTUpd (with B to flux form, BScale), fill dm along
//        x, k_psweep (S6-S8 out of place), fill the nine state fields
//     y: k_cellnode_march, k_ctmass, fill dm along y, k_psweep (S6-S8 out
//        of place, with SweepCTUpd), fill the nine state fields
//     z: k_cellnode_march (SweepVol + SweepCvc), k_ctmass_z, fill dm along
//        z, k_zsweep (S6-S8 in place, with SweepCTUpd bringing B back from
//        flux form), fill the nine state fields
// Other solves take the separate kernels (CellPrep, NodePrep, Corr1,
// SweepVol, SweepCvc, BScale, SweepS6/S7/S8, the rke kernels, k_copy_shell) where a
// condition above fails (thin grids, rke, a field edge without a condition).
// The runner's step++/time += dt (runner.h:573-574) happens in DtFinalize.
// Nothing is read back to the host inside a step.
#include "lare_solver.cuh"
#include "lare_ops.cuh"
#include "lare_bc.cuh"
#include "lare_geom_host.h"

#include <algorithm>
#include <cstdio>
#include <cstring>

namespace sams {

namespace {

constexpr int kThreads = 256;

// One thread per (j, k) of a plane, blockIdx.y walks i.  GEO: the solve's
// geometry is curvilinear (its metric factors are applied); the Cartesian
// instantiation has no trace of them.
template <class Op, bool GEO, bool P2>
__global__ void __launch_bounds__(kThreads, (MinBlocks<Op, P2>::value)) k_op(Ctx c, int arg)
{
    int lo[3], hi[3];
    Op::bounds(c.g, arg, lo, hi);
    const int nk = hi[2] - lo[2] + 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long plane = (long long)(hi[1] - lo[1] + 1) * nk;
    if (t >= plane) return;
    const int j = lo[1] + (int)(t / nk);
    const int k = lo[2] + (int)(t % nk);
    for (int i = lo[0] + (int)blockIdx.y; i <= hi[0]; i += gridDim.y) Op::template run<GEO, P2>(c, arg, i, j, k);
}

// The z sweep's stages S6, S7 and S8 (ops::SweepFused<2>) over whole z
// lines: a block holds kZThreads / (nz + 4) lines of (i, j) in 0..nx x
// 0..ny, one thread per k = -2..nz+1 of each.
constexpr int kZThreads = ops::kZLineThreads;

// ct_arg >= 0: each point of 0..n also takes the z sweep's CT update of B
// (SweepCTUpd<2> with that argument), which nothing else in the kernel reads
// or writes.
template <bool GEO>
__global__ void __launch_bounds__(kZThreads, 5) k_zsweep(Ctx c, int ct_arg)  // 5 blocks per SM, tuned on B200
{
    using F = ops::SweepFused<2>;
    extern __shared__ double zsm[];
    static_assert(!F::kSharedFluxSlots, "the z passes of stage B run without a barrier between them");
    const Geom &g = c.g;
    const int W = g.nz + 4, lines = kZThreads / W, S = lines * W;
    const int line = (int)threadIdx.x / W, k = (int)threadIdx.x % W - 2;
    const long long q = (long long)blockIdx.x * lines + line;
    const bool on = line < lines && q < (long long)(g.nx + 1) * (g.ny + 1);
    const int i = on ? (int)(q / (g.ny + 1)) : 0, j = on ? (int)(q % (g.ny + 1)) : 0;
    const ops::LineStore st{zsm, S, line * W + k + 2};
    const ops::SweepOut w = ops::sweep_in_place(c);
    if (on) F::stage_a<GEO>(c, i, j, k, st, w, true);
    __syncthreads();
    if (on && k >= 1 && k <= g.nz) F::stage_b_energy(c, i, j, k, st, w);
    if (on && k >= -1 && k <= g.nz) F::stage_b_mom<GEO>(c, i, j, k, st);  // its own slots: no barrier between
    __syncthreads();
    if (on && k >= 0 && k <= g.nz) F::stage_c(c, i, j, k, st, w);
    if (ct_arg >= 0 && on && k >= 0 && k <= g.nz) ops::SweepCTUpd<2>::run<GEO, false>(c, ct_arg, i, j, k);
}

// The x or y sweep's stages (ops::SweepFused<DIR>) out of place, over
// windows of kWinK adjacent k in 0..nz times kWinS own points along DIR, for
// one value of the third index (j for x, i for y) in 0..n.  The solve's
// state arrays are only read; the new rho, energies and velocities go to w.
// Halo points recompute stage A (two before, one after) and stage B (one
// before) without writing the state.  ct_arg >= 0: each own point (0..n in
// every dimension) also takes the sweep's CT update of B (SweepCTUpd<DIR>
// with that argument); no stage reads B.
template <int DIR, bool GEO>
__global__ void __launch_bounds__(ops::kWinThreads, 4) k_psweep(Ctx c, ops::SweepOut w, int ct_arg)  // window shape and cap tuned on B200
{
    using F = ops::SweepFused<DIR>;
    constexpr int TK = ops::kWinK, TS = ops::kWinThreads / ops::kWinK;
    extern __shared__ double psm[];
    const Geom &g = c.g;
    const int nd = DIR == 0 ? g.nx : g.ny;
    const int nkt = (g.nz + TK) / TK, nwin = (nd + ops::kWinS) / ops::kWinS;
    const int b = (int)blockIdx.x;
    const int win = b % nwin, kt = (b / nwin) % nkt, a = b / (nwin * nkt);
    const int s0 = win * ops::kWinS, s1 = min(s0 + ops::kWinS - 1, nd);  // own points
    const int kc = (int)threadIdx.x % TK, sl = (int)threadIdx.x / TK;
    const int k = kt * TK + kc;
    const bool on = k <= g.nz;
    auto at = [&](int s) { return ops::WinStore{psm, s - s0 + 2, kc}; };
    const int a_lo = max(s0 - 2, -2), a_hi = min(s1 + 1, nd + 1);
    for (int s = a_lo + sl; s <= a_hi; s += TS)
        if (on) F::template stage_a<GEO>(c, DIR == 0 ? s : a, DIR == 0 ? a : s, k, at(s), w, s >= s0 && s <= s1);
    __syncthreads();
    for (int s = s0 + sl; s <= s1; s += TS)
        if (on) F::stage_b_energy(c, DIR == 0 ? s : a, DIR == 0 ? a : s, k, at(s), w);
    __syncthreads();
    const int b_lo = max(s0 - 1, -1);
    for (int s = b_lo + sl; s <= s1; s += TS)
        if (on) F::template stage_b_mom<GEO>(c, DIR == 0 ? s : a, DIR == 0 ? a : s, k, at(s));
    __syncthreads();
    for (int s = s0 + sl; s <= s1; s += TS)
        if (on) F::stage_c(c, DIR == 0 ? s : a, DIR == 0 ? a : s, k, at(s), w);
    if (ct_arg >= 0)
        for (int s = s0 + sl; s <= s1; s += TS)
            if (on) ops::SweepCTUpd<DIR>::template run<GEO, false>(c, ct_arg, DIR == 0 ? s : a, DIR == 0 ? a : s, k);
}

// The predictor (ops::Pred1 then ops::Pred2) in one kernel.  A block owns
// kMK x kMJ nodes of a y-z plane (k fastest) and a chunk of kMI planes along
// x, and marches along x: for each plane i it computes Pred1 for the cells of
// plane i+1 that its nodes read (its kMJ+1 x kMK+1 cells: the +1 halo in y
// and z is recomputed by the neighbouring block too) into a ring of three
// planes in shared memory, then Pred2 for its nodes of plane i from the
// ring.  cv1 and the half-step B never go to global memory.  The half-step
// p_e and p_i of the block's own cells go to pe_out / pi_out: in resistive
// runs Pred1 reads the step-start p_e / p_i at cells that other blocks own,
// so those arrays cannot be overwritten in place.
// The ring plane is (kMK+1) x (kMJ+1) cells, one per thread of a block of
// kMThreads: 32 x 9, nine full warps, so the producer is one pass; the
// consumer maps thread t to (t / (kMK+1), t % (kMK+1)) and leaves the last
// lane of each row and the last row idle.
constexpr int kMK = 31, kMJ = 8, kMI = 16;
constexpr int kRP = (kMK + 1) * (kMJ + 1);  // cells of one ring plane
constexpr int kMThreads = (kRP + 31) / 32 * 32;

struct RingSrc {
    const double *ring;
    __device__ double operator()(int arr, int q) const { return ring[arr * 3 * kRP + q]; }
};
// The predictor's ring: Pred1's outputs with p_e + p_i in the PE slot (Pred2
// reads only that sum), five arrays.
struct PredRingSrc {
    static constexpr bool kPressureSum = true;
    static constexpr int NR = ops::Pred1::PI;  // CV1, B1X, B1Y, B1Z, PE (= p_e + p_i)
    const double *ring;
    __device__ double operator()(int arr, int q) const { return ring[arr * 3 * kRP + q]; }
};

template <bool GEO, bool P2>
__global__ void __launch_bounds__(kMThreads, 3) k_pred_march(Ctx c, int resistive, double *pe_out, double *pi_out)
{
    using P1 = ops::Pred1;
    extern __shared__ double ring[];  // [PredRingSrc::NR][3 planes][kRP]
    const Geom &g = c.g;
    const int nkt = (g.nz + kMK) / kMK, njt = (g.ny + kMJ) / kMJ;  // tiles over nodes 0..n
    int b = (int)blockIdx.x;
    const int tk = b % nkt;
    b /= nkt;
    const int tj = b % njt;
    const int i0 = (b / njt) * kMI, i1 = min(i0 + kMI - 1, g.nx);
    const int k0 = tk * kMK, j0 = tj * kMJ;
    const int t = (int)threadIdx.x;
    // Pred1 at the block's cells of plane i (cells 0..n+1: what Pred2 reads)
    auto produce = [&](int i) {
        const int slot = i % 3;
        for (int p = t; p < kRP; p += kMThreads) {
            const int pj = p / (kMK + 1), pk = p - pj * (kMK + 1);
            const int j = j0 + pj, k = k0 + pk;
            if (j > g.ny + 1 || k > g.nz + 1) continue;
            double out[P1::NOUT];
            bool half_p;
            P1::compute<GEO, P2>(c, resistive, i, j, k, out, half_p);
#pragma unroll
            for (int a = 0; a < P1::PE; ++a) ring[(a * 3 + slot) * kRP + p] = out[a];
            ring[(P1::PE * 3 + slot) * kRP + p] = out[P1::PE] + out[P1::PI];
            if (pj < kMJ && pk < kMK && i <= i1 && j <= g.ny && k <= g.nz) {
                const int o = box_off(g, i, j, k);
                pe_out[o] = out[P1::PE];
                pi_out[o] = out[P1::PI];
            }
        }
    };
    const int kc = t % (kMK + 1), jc = t / (kMK + 1);
    const int j = j0 + jc, k = k0 + kc;
    const bool on = kc < kMK && jc < kMJ && j <= g.ny && k <= g.nz;
    const PredRingSrc src{ring};
    produce(i0);
    for (int i = i0; i <= i1; ++i) {
        produce(i + 1);
        __syncthreads();  // the ring's planes i and i+1 are complete
        if (on) {
            const int s0 = i % 3, s1 = (i + 1) % 3;
            ops::Pred2::run_src<GEO, P2>(c, i, j, k, src, s0 * kRP + jc * (kMK + 1) + kc, (s1 - s0) * kRP, kMK + 1, 1);
        }
        // three ring planes: the next iteration's producer writes the plane
        // this one read as i-1, which no thread reads after this barrier
    }
}

// A cell op feeding a node op that reads it at the node's eight cells, in
// one kernel: the same march as k_pred_march over nodes -1..n+1 of every
// dimension, with the cell op over cells -1..n+2.  P::produce computes a
// cell's ring values (P::NR of them) and, where `own`, stores its outputs
// (each cell is owned by one block: a chunk, row or column holds its own
// cells and, at the grid's upper end, the +1 halo cell too);
// P::consume runs the node op from the ring.
template <class P, bool GEO, bool P2>
__global__ void __launch_bounds__(kMThreads, P::kMinBlocks) k_cellnode_march(Ctx c, int arg)
{
    extern __shared__ double ring[];  // [P::NR][3 planes][kRP]
    const Geom &g = c.g;
    const int nkt = (g.nz + 2 + kMK) / kMK, njt = (g.ny + 2 + kMJ) / kMJ;  // tiles over nodes -1..n+1
    int b = (int)blockIdx.x;
    const int tk = b % nkt;
    b /= nkt;
    const int tj = b % njt;
    const int i0 = -1 + (b / njt) * kMI, i1 = min(i0 + kMI - 1, g.nx + 1);
    const int k0 = -1 + tk * kMK, j0 = -1 + tj * kMJ;
    const int t = (int)threadIdx.x;
    auto produce = [&](int i) {
        const int slot = (i + 3) % 3;
        for (int p = t; p < kRP; p += kMThreads) {
            const int pj = p / (kMK + 1), pk = p - pj * (kMK + 1);
            const int j = j0 + pj, k = k0 + pk;
            if (j > g.ny + 2 || k > g.nz + 2) continue;
            const bool own = (pj < kMJ || j == g.ny + 2) && (pk < kMK || k == g.nz + 2) && (i <= i1 || i == g.nx + 2);
            double out[P::NR];
            P::template produce<GEO, P2>(c, arg, i, j, k, own, out);
#pragma unroll
            for (int a = 0; a < P::NR; ++a) ring[(a * 3 + slot) * kRP + p] = out[a];
        }
    };
    const int kc = t % (kMK + 1), jc = t / (kMK + 1);
    const int j = j0 + jc, k = k0 + kc;
    const bool on = kc < kMK && jc < kMJ && j <= g.ny + 1 && k <= g.nz + 1;
    const RingSrc src{ring};
    produce(i0);
    for (int i = i0; i <= i1; ++i) {
        produce(i + 1);
        __syncthreads();  // the ring's planes i and i+1 are complete
        if (on) {
            const int s0 = (i + 3) % 3, s1 = (i + 4) % 3;
            P::template consume<GEO, P2>(c, arg, i, j, k, src, s0 * kRP + jc * (kMK + 1) + kc, (s1 - s0) * kRP,
                                         kMK + 1, 1);
        }
    }
}

// CellPrep + NodePrep: each cell's rho and sound speed go into the ring for
// the node averages, so cs never goes to global memory; in resistive runs
// (arg 1) the cell's step-start p_e, p_i are stored.
struct PrepMarch {
    static constexpr int NR = 2, kMinBlocks = 5;  // register cap tuned on B200
    template <bool GEO, bool P2>
    __device__ static void produce(const Ctx &c, int resistive, int i, int j, int k, bool own, double *out)
    {
        const int o = box_off(c.g, i, j, k);
        double pe, pi;
        out[1] = ops::CellPrep::sound_speed(c, o, out[0], pe, pi);
        if (resistive && own) {
            c.s[S_PE][o] = pe;
            c.s[S_PI][o] = pi;
        }
    }
    template <bool GEO, bool P2, class S>
    __device__ static void consume(const Ctx &c, int, int i, int j, int k, const S &src, int q0, int QX, int QY, int QZ)
    {
        ops::NodePrep::run_src<GEO, P2>(c, i, j, k, src, q0, QX, QY, QZ);
    }
};

// SweepVol + SweepCvc of one sweep: cv1 goes into the ring for the node
// volumes cvc1.
template <int DIR>
struct VolMarch {
    static constexpr int NR = 1, kMinBlocks = DIR == 2 ? 5 : 4;  // register cap tuned on B200
    template <bool GEO, bool P2>
    __device__ static void produce(const Ctx &c, int arg, int i, int j, int k, bool own, double *out)
    {
        out[0] = ops::SweepVol<DIR>::template compute<GEO, P2>(c, arg, i, j, k, own);
    }
    template <bool GEO, bool P2, class S>
    __device__ static void consume(const Ctx &c, int, int i, int j, int k, const S &src, int q0, int QX, int QY, int QZ)
    {
        ops::SweepCvc::node(c, box_off(c.g, i, j, k), src, q0, QX, QY, QZ);
    }
};

// An edge term feeding a cell op that reads it on twelve edges around the
// cell, in one kernel (used for the shock heating, whose twelve products of
// velocity jumps per cell, lagran.cpp:888-979, are terms of the edges
// between the cell's corner nodes).  Each term is formed once, at the node
// where its edge ends, instead of once for each of the four cells that share
// the edge.  The march of k_pred_march over cells 0..n+1: for each plane i
// the block forms the x, y and z edge terms of the nodes of plane i that its
// cells read (rows j0-1 .. j0+kMJ-1, kMK+1 columns from k0 + P::KOFF) into a
// ring of three planes in shared memory, then runs the cell op for its cells
// of plane i from the ring's planes i-1 and i.
template <class P, bool GEO, bool P2>
__global__ void __launch_bounds__(kMThreads, (P2 ? P::kMinBlocksP2 : P::kMinBlocks)) k_edge_march(Ctx c)
{
    extern __shared__ double ring[];  // [3 edge directions][3 planes][kRP]
    const Geom &g = c.g;
    const int nkt = (g.nz + 1 + kMK) / kMK, njt = (g.ny + 1 + kMJ) / kMJ;  // tiles over cells 0..n+1
    int b = (int)blockIdx.x;
    const int tk = b % nkt;
    b /= nkt;
    const int tj = b % njt;
    const int i0 = (b / njt) * kMI, i1 = min(i0 + kMI - 1, g.nx + 1);
    const int k0 = tk * kMK, j0 = tj * kMJ;
    const int t = (int)threadIdx.x;
    const int kmax = g.nz + 2 + P::KOFF;  // last node column the cells read
    auto produce = [&](int i) {
        const int slot = (i + 3) % 3;
        for (int p = t; p < kRP; p += kMThreads) {
            const int pj = p / (kMK + 1), pk = p - pj * (kMK + 1);
            const int j = j0 - 1 + pj, k = k0 + P::KOFF + pk;
            if (j > g.ny + 1 || k > kmax) continue;
            double e[3];
            P::Op::node_edges(c, box_off(g, i, j, k), e);
#pragma unroll
            for (int a = 0; a < 3; ++a) ring[(a * 3 + slot) * kRP + p] = e[a];
        }
    };
    const int kc = t % (kMK + 1), jc = t / (kMK + 1);
    const int j = j0 + jc, k = k0 + kc;
    const bool on = kc < kMK && jc < kMJ && j <= g.ny + 1 && k <= g.nz + 1;
    const RingSrc src{ring};
    produce(i0 - 1);
    for (int i = i0; i <= i1; ++i) {
        produce(i);
        __syncthreads();  // the ring's planes i-1 and i are complete
        if (on) {
            const int s0 = (i + 3) % 3, sm = (i + 2) % 3;
            double a[12];
            P::Op::ring_edges(src, s0 * kRP + (jc + 1) * (kMK + 1) + (kc - P::KOFF), (s0 - sm) * kRP, kMK + 1, a);
            P::template finish<GEO, P2>(c, i, j, k, a);
        }
        // three ring planes: the next iteration's producer writes the plane
        // this one read as i-2, which no thread reads any more
    }
}

// Corr1 from the ring of products of velocity jumps: the shock heating.
// (Corr2's energy and density update folded in here, with only its velocity
// update left as a kernel, measured slower on B200: 0.83 + 0.25 ms against
// 0.43 + 0.60.)
struct HeatEdges {
    using Op = ops::Corr1;
    static constexpr int KOFF = 0, kMinBlocks = 4, kMinBlocksP2 = 4;  // register cap tuned on B200
    template <bool GEO, bool P2>
    __device__ static void finish(const Ctx &c, int i, int j, int k, const double *a)
    {
        c.s[S_VH][box_off(c.g, i, j, k)] = Op::heating_finish<GEO, P2>(c, i, j, k, a);
    }
};

// One resistive sub-step (ops::ResistRK then ops::ResistB) in one kernel,
// out of place for B.  A block owns kMK x kMJ points of a y-z plane of the
// whole box (-2..n+2) and a chunk of kMI planes along x, and marches along x:
// ResistRK for the cells of plane i that its points read (the -1 halo in y
// and z is recomputed by the neighbouring block) goes into a ring of three
// planes in shared memory, then ResistB for its points of plane i reads the
// ring's planes i-1 and i.  ResistRK reads B at +1 neighbours that other
// blocks update, so the new B goes to nbx/nby/nbz (every box point: updated
// or copied); the electron energy is updated in place (nothing else reads
// it here).
template <bool GEO, bool P2>
__global__ void __launch_bounds__(kMThreads, 5) k_resist_march(Ctx c, double *nbx, double *nby, double *nbz)
{
    using RK = ops::ResistRK;
    extern __shared__ double ring[];  // [RK::NOUT][3 planes][kRP]
    const Geom &g = c.g;
    const int nkt = (g.nz + 4 + kMK) / kMK, njt = (g.ny + 4 + kMJ) / kMJ;  // tiles over -2..n+2
    int b = (int)blockIdx.x;
    const int tk = b % nkt;
    b /= nkt;
    const int tj = b % njt;
    const int i0 = -2 + (b / njt) * kMI, i1 = min(i0 + kMI - 1, g.nx + 2);
    const int k0 = -2 + tk * kMK, j0 = -2 + tj * kMJ;
    const int t = (int)threadIdx.x;
    // ResistRK at the block's cells of plane i (ring index (j - j0 + 1, k - k0 + 1)),
    // where it is defined (0..n)
    auto produce = [&](int i) {
        if (i < 0 || i > g.nx) return;
        const int slot = (i + 6) % 3;
        for (int p = t; p < kRP; p += kMThreads) {
            const int pj = p / (kMK + 1), pk = p - pj * (kMK + 1);
            const int j = j0 - 1 + pj, k = k0 - 1 + pk;
            if (j < 0 || j > g.ny || k < 0 || k > g.nz) continue;
            double out[RK::NOUT];
            RK::compute<GEO, P2>(c, i, j, k, out);
#pragma unroll
            for (int a = 0; a < RK::NOUT; ++a) ring[(a * 3 + slot) * kRP + p] = out[a];
        }
    };
    const int kc = t % (kMK + 1), jc = t / (kMK + 1);
    const int j = j0 + jc, k = k0 + kc;
    const bool on = kc < kMK && jc < kMJ && j <= g.ny + 2 && k <= g.nz + 2;
    const RingSrc src{ring};
    produce(i0 - 1);
    for (int i = i0; i <= i1; ++i) {
        produce(i);
        __syncthreads();  // the ring's planes i-1 and i are complete
        if (on) {
            const int s0 = (i + 6) % 3, sm = (i + 5) % 3;
            ops::ResistB::run_src<P2>(c, i, j, k, src, s0 * kRP + (jc + 1) * (kMK + 1) + (kc + 1), (s0 - sm) * kRP,
                                      kMK + 1, 1, nbx, nby, nbz);
        }
    }
}

// SweepCT + SweepMass of the x or y sweep (ops::SweepCTMass<DIR>) over
// windows of kWinK adjacent k times kWinS own points along DIR, for one value
// a of the third index (j for x, i for y).  The CT quotients of the window's
// points and of a halo of one before and two after go to shared memory first.
// CT fluxes where a and k are in 0..n, mass fluxes where they are in 0..n+1.
constexpr int kCtS = 21;              // own points of a window along the sweep (tuned on B200)
constexpr int kCtP = kCtS + 3;         // with the quotient halo (one before, two after)
struct CtStore {
    double *sm;
    int at, kc;
    __device__ double get(int a, int ds) const { return sm[(a * kCtP + at + ds) * ops::kWinK + kc]; }
    __device__ void put(int a, double v) const { sm[(a * kCtP + at) * ops::kWinK + kc] = v; }
};

template <int DIR, bool GEO>
__global__ void __launch_bounds__(ops::kWinThreads, 5) k_ctmass(Ctx c, int scale, int images)  // cap tuned on B200
{
    using F = ops::SweepCTMass<DIR>;
    constexpr int TK = ops::kWinK, TS = ops::kWinThreads / ops::kWinK;
    extern __shared__ double csm[];
    const Geom &g = c.g;
    const int nd = DIR == 0 ? g.nx : g.ny, na = DIR == 0 ? g.ny : g.nx;
    const int nkt = (g.nz + 1 + TK) / TK, nwin = (nd + kCtS) / kCtS;
    const int b = (int)blockIdx.x;
    const int win = b % nwin, kt = (b / nwin) % nkt, a = b / (nwin * nkt);
    const int s0 = win * kCtS, s1 = min(s0 + kCtS - 1, nd);
    const int kc = (int)threadIdx.x % TK, sl = (int)threadIdx.x / TK;
    const int k = kt * TK + kc;
    const bool ct = a <= na && k <= g.nz, mass = k <= g.nz + 1;
    auto at = [&](int s) { return CtStore{csm, s - s0 + 1, kc}; };
    if (ct)
        for (int s = s0 - 1 + sl; s <= s1 + 2; s += TS)
            F::template quot<GEO>(c, DIR == 0 ? s : a, DIR == 0 ? a : s, k, at(s), scale != 0);
    __syncthreads();
    if (mass)
        for (int s = s0 + sl; s <= s1; s += TS)
            F::template fluxes<GEO>(c, DIR == 0 ? s : a, DIR == 0 ? a : s, k, at(s), ct, images != 0);
}

// SweepCT + SweepMass of the z sweep: kZRows lines (i, j) in 0..nx+1 x
// 0..ny+1 per block (CT fluxes on the lines in 0..n), 32 own k in 0..nz each;
// the quotients of k0-1 .. k0+34 (up to nz+2) of each line go to shared
// memory first.
constexpr int kZRows = 8, kZOwn = 64, kZSpan = kZOwn + 3;
struct ZRowStore {
    double *sm;
    int at;
    __device__ double get(int a, int ds) const { return sm[a * (kZRows * kZSpan) + at + ds]; }
    __device__ void put(int a, double v) const { sm[a * (kZRows * kZSpan) + at] = v; }
};

template <bool GEO>
__global__ void __launch_bounds__(256, 5) k_ctmass_z(Ctx c, int images)  // cap tuned on B200
{
    using F = ops::SweepCTMass<2>;
    __shared__ double zsm[F::NARR * kZRows * kZSpan];
    const Geom &g = c.g;
    const int r = (int)threadIdx.x / 32, kc = (int)threadIdx.x % 32;
    const long long line = (long long)blockIdx.x * kZRows + r;
    const bool on = line < (long long)(g.nx + 2) * (g.ny + 2);
    const int i = on ? (int)(line / (g.ny + 2)) : 0, j = on ? (int)(line % (g.ny + 2)) : 0;
    const int k0 = (int)blockIdx.y * kZOwn;
    const bool ct = on && i <= g.nx && j <= g.ny;
    if (ct)
        for (int kk = kc; kk < kZSpan; kk += 32) {
            const int k = k0 - 1 + kk;
            if (k <= g.nz + 2) F::quot<GEO>(c, i, j, k, ZRowStore{zsm, r * kZSpan + kk}, false);
        }
    __syncthreads();
    for (int kk = kc; kk < kZOwn; kk += 32) {
        const int k = k0 + kk;  // along the sweep: 0..nz for both fluxes
        if (on && k <= g.nz) F::fluxes<GEO>(c, i, j, k, ZRowStore{zsm, r * kZSpan + kk + 1}, ct, images != 0);
    }
}

// The points of the out-of-place sweep's arrays it does not compute (rho and
// energies outside 1..n, velocities outside 0..n in some dimension): copied
// from the solve's arrays, so the new arrays are complete boxes.  One
// thread per shell point: the rho / energy shell, then the velocity shell.
__global__ void __launch_bounds__(kThreads) k_copy_shell(Ctx c, ops::SweepOut w)
{
    const Geom &g = c.g;
    const BoxShell cell{{g.nx, g.ny, g.nz}, 1, 0}, node{{g.nx, g.ny, g.nz}, 0, 0};
    const long long nc = cell.count(), n = nc + node.count();
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (t < nc) {
            cell.point(t, i, j, k);
            const int o = box_off(g, i, j, k);
            w.rho[o] = c.f[SAMS_F_RHO][o];
            w.ee[o] = c.f[SAMS_F_ENERGY_ELECTRON][o];
            w.ei[o] = c.f[SAMS_F_ENERGY_ION][o];
        } else {
            node.point(t - nc, i, j, k);
            const int o = box_off(g, i, j, k);
            w.ux[o] = c.f[SAMS_F_VX][o];
            w.uy[o] = c.f[SAMS_F_VY][o];
            w.uz[o] = c.f[SAMS_F_VZ][o];
        }
    }
}

// Visc with two threads per cell: a block holds 128 consecutive (j, k)
// points of a y-z plane (walking i); its first four warps run the viscous heating and forces
// (ops::Visc::heat_forces), the other four the viscous pressure and CFL
// candidate (ops::Visc::cfl), so each thread carries half the work's live
// values.  Both halves read the same corners, which the block's L1 serves.
// The block's minimum candidate goes to Scalars::dtmin_bits: positive
// doubles order like their bit patterns, so an integer atomicMin is an
// exact, order-free minimum.
template <bool GEO, bool P2>
__global__ void __launch_bounds__(kThreads, 4) k_visc_split(Ctx c)  // 4 blocks per SM, tuned on B200
{
    int lo[3], hi[3];
    ops::Visc::bounds(c.g, 0, lo, hi);
    const int nk = hi[2] - lo[2] + 1;
    const int half = (int)threadIdx.x >> 7;
    const long long t = (long long)blockIdx.x * (kThreads / 2) + (threadIdx.x & (kThreads / 2 - 1));
    const long long plane = (long long)(hi[1] - lo[1] + 1) * nk;
    double best = DBL_MAX;
    bool bad = false;
    if (t < plane) {
        const int j = lo[1] + (int)(t / nk);
        const int k = lo[2] + (int)(t % nk);
        for (int i = lo[0] + (int)blockIdx.y; i <= hi[0]; i += gridDim.y) {
            if (half == 0)
                ops::Visc::heat_forces<GEO, P2>(c, i, j, k, bad);
            else if (i <= c.g.nx && j <= c.g.ny && k <= c.g.nz)
                best = dev::pmin(best, ops::Visc::cfl<GEO, P2>(c, i, j, k, bad));
        }
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&c.sc->status, 1);
    for (int off = 16; off > 0; off >>= 1) best = dev::pmin(best, __shfl_xor_sync(0xffffffffu, best, off));
    __shared__ double wmin[kThreads / 32];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = wmin[0];
        for (int w = 1; w < kThreads / 32; ++w) m = dev::pmin(m, wmin[w]);
        if (m < DBL_MAX) atomicMin(&c.sc->dtmin_bits, (unsigned long long)__double_as_longlong(m));
    }
}

// Dense box buffer <-> padded device rows (to_padded = 1: dense -> padded).
__global__ void k_repack(const double *__restrict__ src, double *__restrict__ dst, Geom g, int to_padded)
{
    const long long n = (long long)(g.nx + 5) * (g.ny + 5) * (g.nz + 5);
    const int ez = g.nz + 5;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const long long row = t / ez;
        const long long p = row * g.sy + (g.zoff - 2) + (t - row * ez);
        if (to_padded)
            dst[p] = src[t];
        else
            dst[t] = src[p];
    }
}

// dt = dt_multiplier * min (lagran.cpp:387-442), then the runner's
// min-with-DBL_MAX (runner.h:161-167, shared_data.h:428-440); the resistive
// sub-step is dt / (int(dt/dtr) + 1) (lagran.cpp:159-163); dtr == dt, so
// that count is 2.  Also the runner's time += dt, step++.
__global__ void k_dt_finalize(Scalars *sc, double dt_multiplier, int resistive)
{
    double m = __longlong_as_double((long long)sc->dtmin_bits);
    double dt = dt_multiplier * m;
    sc->dtr = dt;
    dt = dt < DBL_MAX ? dt : DBL_MAX;
    sc->dt = dt;
    if (resistive) {
        int nsub = (int)(dt / sc->dtr) + 1;
        sc->nsub = nsub;
        sc->dt_sub = dt / (double)nsub;
    }
    sc->dtmin_bits = (unsigned long long)__double_as_longlong(DBL_MAX);
    if (!(m < DBL_MAX) || !(dt > 0.0) || !(dt < DBL_MAX)) sc->status = 1;
    sc->time += dt;
    sc->step += 1;
}

// ---------------------------------------------------------------------------
// Boundary fills (variableDef::applyBoundaryConditions order,
// include/harness/variableDef.h:539-605; built-in conditions of
// include/boundaryConditions/builtInBoundaryConditions.h).
// ---------------------------------------------------------------------------

struct FieldList {
    int n;
    int id[SAMS_NFIELDS];
};

__device__ __forceinline__ int field_lb(int f, int d) { return field_half(f, d) ? -2 : -1; }

// All-periodic fields: applying the lower then upper periodic copy in x, y
// and z in turn leaves every ghost point equal to the interior point it
// wraps to, w(q) = q + n for q <= 0 and q - n for q >= n + 1 (a half-cell
// index n keeps its value), so all ghosts are filled by one gather.
__global__ void __launch_bounds__(kThreads) k_bc_periodic(Ctx c, FieldList fl)
{
    const int f = fl.id[blockIdx.y];
    const Geom &g = c.g;
    const int n[3] = {g.nx, g.ny, g.nz};
    int lb[3], ext[3], gh[3];
    for (int d = 0; d < 3; ++d) {
        lb[d] = field_lb(f, d);
        ext[d] = n[d] + 3 - lb[d];
        gh[d] = ext[d] - n[d];
    }
    // 32-bit index arithmetic: a field's shell has fewer points than the
    // field, and a field has fewer than 2^31 (checked at set-up)
    const int A = gh[0] * ext[1] * ext[2];
    const int B = n[0] * gh[1] * ext[2];
    const int C = n[0] * n[1] * gh[2];
    int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    int q[3];
    if (t < A) {
        const int pl = ext[1] * ext[2];
        const int gi = t / pl, r = t - gi * pl;
        q[0] = gi < 1 - lb[0] ? lb[0] + gi : n[0] + 1 + (gi - (1 - lb[0]));
        q[1] = lb[1] + r / ext[2];
        q[2] = lb[2] + r % ext[2];
    } else if ((t -= A) < B) {
        const int pl = gh[1] * ext[2];
        const int i = t / pl, r = t - i * pl;
        const int gj = r / ext[2];
        q[0] = 1 + i;
        q[1] = gj < 1 - lb[1] ? lb[1] + gj : n[1] + 1 + (gj - (1 - lb[1]));
        q[2] = lb[2] + (r - gj * ext[2]);
    } else if ((t -= B) < C) {
        const int pl = n[1] * gh[2];
        const int i = t / pl, r = t - i * pl;
        const int gk = r % gh[2];
        q[0] = 1 + i;
        q[1] = 1 + r / gh[2];
        q[2] = gk < 1 - lb[2] ? lb[2] + gk : n[2] + 1 + (gk - (1 - lb[2]));
    } else {
        return;
    }
    int s[3];
    for (int d = 0; d < 3; ++d) s[d] = q[d] <= 0 ? q[d] + n[d] : (q[d] >= n[d] + 1 ? q[d] - n[d] : q[d]);
    double *a = c.f[f];
    a[box_off(g, q[0], q[1], q[2])] = a[box_off(g, s[0], s[1], s[2])];
}

// One (dimension, edge) of the given fields, exactly as the reference's
// boundary-condition objects apply it (lare_bc.cuh).
__global__ void __launch_bounds__(kThreads) k_bc_edge(Ctx c, FieldList fl, BcTable bt, int d, int e)
{
    const int f = fl.id[blockIdx.y];
    const int kind = bt.kind[f][d][e];
    if (kind == SAMS_BC_NONE) return;
    const Geom &g = c.g;
    const BcEdge sl = bc_edge_slab(g, f, d, e);
    const int e1 = sl.hi[1] - sl.lo[1] + 1, e2 = sl.hi[2] - sl.lo[2] + 1;
    const long long total = (long long)(sl.hi[0] - sl.lo[0] + 1) * e1 * e2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int q[3];
    q[0] = sl.lo[0] + (int)(t / ((long long)e1 * e2));
    q[1] = sl.lo[1] + (int)((t / e2) % e1);
    q[2] = sl.lo[2] + (int)(t % e2);
    bc_edge_apply(c.f[f], g, sl, bt, f, d, e, q);
}

FieldList make_list(unsigned mask)
{
    FieldList fl{};
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        if (mask & (1u << f)) fl.id[fl.n++] = f;
    return fl;
}

long long ceil_div(long long a, long long b) { return (a + b - 1) / b; }

// Whether n values split into tiles of w lanes keep at least three quarters
// of the lanes busy (thin grids, e.g. n x n x 4 solves, leave most idle).
bool lanes_full(long long n, long long w) { return 4 * n >= 3 * w * ceil_div(n, w); }

}  // namespace

// ---------------------------------------------------------------------------

long long Solver::bytes_for(const sams_lare_params &p)
{
    const long long zrow = ((p.nz + 6) + 7) / 8 * 8;
    const long long nelem = (p.nx + 5) * (p.ny + 5) * zrow;
    const long long narr = SAMS_NFIELDS + NSCRATCH + (p.rke ? 1 : 0);
    const long long staging = (p.nx + 5) * (p.ny + 5) * (p.nz + 5);
    long long axes = 6 * (p.nx + p.ny + p.nz + 18);
    if (p.geometry) axes += 5 * (p.nx + 6) * (p.ny + 6) + 8 * (p.nx + p.ny + 12);
    return (narr * nelem + staging + axes) * (long long)sizeof(double) + (long long)sizeof(Scalars) + 4096;
}

bool Solver::fused_path(const sams_lare_params &p) { return lanes_full(p.nz + 1, kMK); }

Solver::~Solver() { free_all(); }

void Solver::free_all()
{
    if (device_ >= 0) cudaSetDevice(device_);
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    if (arena_) cudaFree(arena_);
    if (axes_) cudaFree(axes_);
    if (sc_) cudaFree(sc_);
    if (staging_) cudaFree(staging_);
    if (own_stream_) cudaStreamDestroy(own_stream_);
    arena_ = nullptr;
    axes_ = nullptr;
    sc_ = nullptr;
    staging_ = nullptr;
    own_stream_ = nullptr;
}

int Solver::check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return SAMS_OK;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? SAMS_ERR_NOMEM : SAMS_ERR_CUDA;
}

static void axis_host(double lo, double hi, long long n, std::vector<double> &db, std::vector<double> &dc)
{
    // axisRegistry: b(i) = lo + d*i, c(i) = 0.5*(b(i) + b(i-1)), deltas with
    // the first one copied from the next (non-periodic axes).
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

int Solver::init(const sams_lare_params &p, const sams_lare_bcs &bcs, int device)
{
    return init_impl(p, bcs, device, nullptr);
}

int Solver::init_slab(const sams_lare_params &p, const sams_lare_bcs &bcs, int device, const XSlab &slab)
{
    if (slab.off < 0 || slab.off + p.nx > slab.nx_global) {
        err = "slab outside the grid";
        return SAMS_ERR_INVALID;
    }
    if (p.rke) {
        err = "the remap kinetic-energy correction (rke) gathers over the whole grid in order; not on slabs";
        return SAMS_ERR_UNSUPPORTED;
    }
    return init_impl(p, bcs, device, &slab);
}

int Solver::init_impl(const sams_lare_params &p, const sams_lare_bcs &bcs, int device, const XSlab *slab)
{
    if (p.nx < 1 || p.ny < 1 || p.nz < 1) { err = "grid sizes must be >= 1"; return SAMS_ERR_INVALID; }
    if (p.nx > 60000 || p.ny > 60000 || p.nz > 60000) { err = "grid size too large"; return SAMS_ERR_INVALID; }
    if (p.geometry < 0 || p.geometry > 2) { err = "geometry must be 0 (Cartesian), 1 (cylindrical) or 2 (spherical)"; return SAMS_ERR_UNSUPPORTED; }
    if (!(p.x_max > p.x_min) || !(p.y_max > p.y_min) || !(p.z_max > p.z_min)) {
        err = "empty domain";
        return SAMS_ERR_INVALID;
    }
    p_ = p;
    device_ = device;
    {
        const long long n[3] = {p.nx, p.ny, p.nz};
        if (!bc_table_from(bc_, bcs, n, &err)) return SAMS_ERR_INVALID;
    }
    int rc;
    if ((rc = check(cudaSetDevice(device), "cudaSetDevice"))) return rc;
    if ((rc = check(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device), "sm count")))
        return rc;
    if ((rc = check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "cudaStreamCreate"))) return rc;
    stream_ = own_stream_;

    Geom &g = ctx_.g;
    g.nx = (int)p.nx;
    g.ny = (int)p.ny;
    g.nz = (int)p.nz;
    g.zoff = 3;
    const long long zrow = ((p.nz + 6) + 7) / 8 * 8;
    const long long sx = (long long)(p.ny + 5) * zrow;
    if ((long long)(p.nx + 5) * sx > INT32_MAX) {
        err = "one array of this grid exceeds 2^31 elements";
        return SAMS_ERR_UNSUPPORTED;
    }
    g.sy = (int)zrow;
    g.sx = (int)sx;
    g.nelem = (long long)(p.nx + 5) * sx;
    // the rke correction keeps one more array (delta_ke) across the sweeps
    const long long narr = SAMS_NFIELDS + NSCRATCH + (p.rke ? 1 : 0);
    const size_t abytes = (size_t)narr * (size_t)g.nelem * sizeof(double);
    if ((rc = check(cudaMalloc(&arena_, abytes), "cudaMalloc(state)"))) return rc;
    if ((rc = check(cudaMemsetAsync(arena_, 0, abytes, stream_), "cudaMemset(state)"))) return rc;
    for (int f = 0; f < SAMS_NFIELDS; ++f) ctx_.f[f] = arena_ + (size_t)f * g.nelem;
    for (int s = 0; s < NSCRATCH; ++s) ctx_.s[s] = arena_ + (size_t)(SAMS_NFIELDS + s) * g.nelem;
    ctx_.dke = p.rke ? arena_ + (size_t)(SAMS_NFIELDS + NSCRATCH) * g.nelem : nullptr;

    // 1-D spacings: dxb, dyb, dzb, dxc, dyc, dzc, each (n + 6) long.
    std::vector<double> dxb, dyb, dzb, dxc, dyc, dzc;
    if (slab) {  // the whole grid's x axis from the slab's offset on
        std::vector<double> gb, gc;
        axis_host(p.x_min, p.x_max, slab->nx_global, gb, gc);
        dxb.assign(gb.begin() + slab->off, gb.begin() + slab->off + p.nx + 6);
        dxc.assign(gc.begin() + slab->off, gc.begin() + slab->off + p.nx + 6);
    } else {
        axis_host(p.x_min, p.x_max, p.nx, dxb, dxc);
    }
    axis_host(p.y_min, p.y_max, p.ny, dyb, dyc);
    axis_host(p.z_min, p.z_max, p.nz, dzb, dzc);
    std::vector<double> packed;
    for (auto *v : {&dxb, &dyb, &dzb, &dxc, &dyc, &dzc}) packed.insert(packed.end(), v->begin(), v->end());
    const size_t geo_off = packed.size();
    if (p.geometry) {  // metric factors after the spacings
        std::vector<double> t = slab ? geom_tables_slab(p, slab->off, slab->nx_global) : geom_tables(p);
        packed.insert(packed.end(), t.begin(), t.end());
    }
    if ((rc = check(cudaMalloc(&axes_, packed.size() * sizeof(double)), "cudaMalloc(axes)"))) return rc;
    if ((rc = check(cudaMemcpy(axes_, packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice), "axes upload"))) return rc;
    size_t off = 0;
    const double **slots[6] = {&ctx_.ax.dxb, &ctx_.ax.dyb, &ctx_.ax.dzb, &ctx_.ax.dxc, &ctx_.ax.dyc, &ctx_.ax.dzc};
    const size_t lens[6] = {dxb.size(), dyb.size(), dzb.size(), dxc.size(), dyc.size(), dzc.size()};
    for (int a = 0; a < 6; ++a) {
        *slots[a] = axes_ + off;
        off += lens[a];
    }
    ctx_.gf = GeomF{};
    if (p.geometry) geom_bind(ctx_.gf, axes_ + geo_off, p);
    ctx_.p.geometry = (int)p.geometry;
    ctx_.p.pow2 = p.geometry == 0 && pow2_grid(dxb, dyb, dzb, dxc, dyc, dzc, p.mu0, &ctx_.rc) ? 1 : 0;

    ctx_.p.gamma = p.gas_gamma;
    ctx_.p.mu0 = p.mu0;
    ctx_.p.visc1 = p.visc1;
    ctx_.p.visc2_norm = 0.25 * (p.gas_gamma + 1.0) * p.visc2;  // lagran.cpp:178
    ctx_.p.dt_multiplier = p.dt_multiplier;
    ctx_.p.eta_bg = p.eta_background;
    ctx_.p.eta0 = p.eta0;
    ctx_.p.j_max = p.j_max;
    ctx_.p.resistive = p.resistive_mhd ? 1 : 0;
    ctx_.p.rke = p.rke ? 1 : 0;

    if ((rc = check(cudaMalloc(&sc_, sizeof(Scalars)), "cudaMalloc(scalars)"))) return rc;
    Scalars s0{};
    s0.dt = 0.0;  // value-initialised runner data: the first step's viscosity sees dt = 0
    s0.dtmin_bits = 0x7FEFFFFFFFFFFFFFull;  // DBL_MAX
    if ((rc = check(cudaMemcpy(sc_, &s0, sizeof(s0), cudaMemcpyHostToDevice), "scalars upload"))) return rc;
    ctx_.sc = sc_;
    bytes_ = (long long)abytes + (long long)(packed.size() * sizeof(double)) + (long long)sizeof(Scalars);
    if ((rc = setup_psweep())) return rc;
    return check(cudaStreamSynchronize(stream_), "init sync");
}

int Solver::init_borrowed(const sams_lare_params &p, const sams_lare_bcs &bcs, const Ctx &ctx, int device,
                          cudaStream_t stream)
{
    if (p.geometry != 0) {
        err = "only Cartesian geometry is available on this entry point (no room for the metric tables)";
        return SAMS_ERR_UNSUPPORTED;
    }
    if (p.rke != 0) {
        err = "the remap kinetic-energy correction (rke) needs an array this entry point does not have";
        return SAMS_ERR_UNSUPPORTED;
    }
    p_ = p;
    device_ = device;
    {
        const long long n[3] = {p.nx, p.ny, p.nz};
        if (!bc_table_from(bc_, bcs, n, &err)) return SAMS_ERR_INVALID;
    }
    ctx_ = ctx;
    sc_ = ctx.sc;  // borrowed: release_borrowed() must clear it before destruction
    stream_ = stream;
    int rc;
    if ((rc = check(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device), "sm count")))
        return rc;
    return setup_psweep();
}

void Solver::release_borrowed()
{
    sc_ = nullptr;
    for (int f = 0; f < SAMS_NFIELDS; ++f) ctx_.f[f] = nullptr;
    for (int s = 0; s < NSCRATCH; ++s) ctx_.s[s] = nullptr;
}

int Solver::set_bc(int field, int dim, int edge, int kind, double value)
{
    if (field < 0 || field >= SAMS_NFIELDS || dim < 0 || dim > 2 || edge < 0 || edge > 1) {
        err = "invalid boundary-condition slot or kind";
        return SAMS_ERR_INVALID;
    }
    const long long n[3] = {p_.nx, p_.ny, p_.nz};
    BcTable t = bc_;
    if (!bc_slot_set(t, field, dim, edge, kind, value, n, &err)) return SAMS_ERR_INVALID;
    bc_ = t;
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    return SAMS_OK;
}

int Solver::set_stream(cudaStream_t s)
{
    stream_ = s ? s : own_stream_;
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    return SAMS_OK;
}

// Box rows are (nz+5) doubles; device rows are padded to g.sy with the row
// starting at offset zoff-2.  Copies from or to host memory go through a
// dense device staging buffer (one contiguous transfer at full link speed)
// and a repacking kernel; device-to-device copies are strided copies.
int Solver::staging(double **out)
{
    if (!staging_) {
        const size_t bytes = (size_t)(ctx_.g.nx + 5) * (ctx_.g.ny + 5) * (ctx_.g.nz + 5) * sizeof(double);
        int rc;
        if ((rc = check(cudaMalloc(&staging_, bytes), "cudaMalloc(staging)"))) return rc;
        bytes_ += (long long)bytes;
    }
    *out = staging_;
    return SAMS_OK;
}

int Solver::upload(int field, const double *src, cudaMemcpyKind kind)
{
    if (field < 0 || field >= SAMS_NFIELDS || !src) { err = "invalid field or buffer"; return SAMS_ERR_INVALID; }
    const Geom &g = ctx_.g;
    const size_t w = (size_t)(g.nz + 5) * sizeof(double);
    const size_t rows = (size_t)(g.nx + 5) * (size_t)(g.ny + 5);
    double *dst = ctx_.f[field] + (g.zoff - 2);
    if (kind == cudaMemcpyDeviceToDevice)
        return check(cudaMemcpy2DAsync(dst, (size_t)g.sy * sizeof(double), src, w, w, rows, kind, stream_), "upload");
    double *st;
    int rc;
    if ((rc = staging(&st))) return rc;
    if ((rc = check(cudaMemcpyAsync(st, src, w * rows, kind, stream_), "upload"))) return rc;
    k_repack<<<(unsigned)std::min<long long>(ceil_div((long long)(w / sizeof(double) * rows), kThreads), 8L * sm_count_),
               kThreads, 0, stream_>>>(st, ctx_.f[field], g, 1);
    return check(cudaGetLastError(), "repack");
}

int Solver::download(int field, double *dst, cudaMemcpyKind kind)
{
    if (field < 0 || field >= SAMS_NFIELDS || !dst) { err = "invalid field or buffer"; return SAMS_ERR_INVALID; }
    const Geom &g = ctx_.g;
    const size_t w = (size_t)(g.nz + 5) * sizeof(double);
    const size_t rows = (size_t)(g.nx + 5) * (size_t)(g.ny + 5);
    const double *src = ctx_.f[field] + (g.zoff - 2);
    int rc;
    if (kind == cudaMemcpyDeviceToDevice) {
        rc = check(cudaMemcpy2DAsync(dst, w, src, (size_t)g.sy * sizeof(double), w, rows, kind, stream_), "download");
    } else {
        double *st;
        if ((rc = staging(&st))) return rc;
        k_repack<<<(unsigned)std::min<long long>(ceil_div((long long)(w / sizeof(double) * rows), kThreads),
                                                 8L * sm_count_),
                   kThreads, 0, stream_>>>(ctx_.f[field], st, g, 0);
        if ((rc = check(cudaGetLastError(), "repack"))) return rc;
        rc = check(cudaMemcpyAsync(dst, st, w * rows, kind, stream_), "download");
    }
    if (rc) return rc;
    return check(cudaStreamSynchronize(stream_), "download sync");
}

// The x or y sweep's S6-S8 out of place into six scratch arrays free during
// the remap (the intermediates of the separate kernels live on chip here),
// then the solve's state pointers move to them; the y sweep writes back into
// the arrays the x sweep left, so after the two sweeps every pointer is
// where it started.
template <int DIR>
void Solver::launch_psweep(int ct_arg)
{
    static const int kOut[6] = {S_FX, S_FY, S_FZ, S_VH, S_FXV, S_FYV};
    static const int kState[6] = {SAMS_F_RHO, SAMS_F_ENERGY_ELECTRON, SAMS_F_ENERGY_ION,
                                  SAMS_F_VX, SAMS_F_VY, SAMS_F_VZ};
    const Geom &g = ctx_.g;
    const ops::SweepOut w{ctx_.s[kOut[0]], ctx_.s[kOut[1]], ctx_.s[kOut[2]],
                          ctx_.s[kOut[3]], ctx_.s[kOut[4]], ctx_.s[kOut[5]]};
    const int nd = DIR == 0 ? g.nx : g.ny, na = (DIR == 0 ? g.ny : g.nx) + 1;
    const long long blocks = (long long)na * ((g.nz + ops::kWinK) / ops::kWinK) * ((nd + ops::kWinS) / ops::kWinS);
    const size_t smem = (size_t)ops::SweepFused<DIR>::NARR * ops::WinStore::P * ops::kWinK * sizeof(double);
    // rho1 (rho before the sweep) is rho itself here: the sweep writes the new
    // rho elsewhere (SweepVol skipped the copy)
    Ctx cc = ctx_;
    cc.s[S_R_RHO1] = ctx_.f[SAMS_F_RHO];
    if (ctx_.p.geometry)
        k_psweep<DIR, true><<<(unsigned)blocks, ops::kWinThreads, smem, stream_>>>(cc, w, ct_arg);
    else
        k_psweep<DIR, false><<<(unsigned)blocks, ops::kWinThreads, smem, stream_>>>(cc, w, ct_arg);
    ++launches_;
    // The points the sweep does not compute are ghost points of each array;
    // the fill that follows the sweep rewrites all of them from domain values
    // when every edge of these fields has a condition and every dimension at
    // least three cells (see enqueue_step).  Otherwise copy them over.
    if (!ghosts_refilled(FM_DENSITY | FM_ENERGY | FM_VELOCITY)) {
        const long long shell = BoxShell{{g.nx, g.ny, g.nz}, 1, 0}.count() + BoxShell{{g.nx, g.ny, g.nz}, 0, 0}.count();
        k_copy_shell<<<(unsigned)std::min<long long>(ceil_div(shell, kThreads), 8L * sm_count_), kThreads, 0,
                       stream_>>>(ctx_, w);
        ++launches_;
    }
    for (int q = 0; q < 6; ++q) std::swap(ctx_.f[kState[q]], ctx_.s[kOut[q]]);
}

// Whether the fused x / y sweep runs for this solve (its windows must be at
// least three quarters full of k values), and its shared memory: allow the
// device's opt-in maximum (the attribute belongs to the kernel, so it is
// the same for every solve).
int Solver::setup_psweep()
{
    int maxsm = 0, rc;
    if ((rc = check(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_), "smem limit")))
        return rc;
    const size_t need = (size_t)ops::SweepFused<0>::NARR * ops::WinStore::P * ops::kWinK * sizeof(double);
    // a window holds kWinK adjacent k; thin grids would leave most lanes idle
    const int kw = ops::kWinK, nk = ctx_.g.nz + 1;
    const bool lanes_full = 4 * nk >= 3 * kw * ((nk + kw - 1) / kw);
    psweep_ok_ = need <= (size_t)maxsm && lanes_full;
    if (!psweep_ok_) return SAMS_OK;
    const void *fn[4] = {(const void *)k_psweep<0, false>, (const void *)k_psweep<0, true>,
                         (const void *)k_psweep<1, false>, (const void *)k_psweep<1, true>};
    for (const void *f : fn)
        if ((rc = check(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm), "psweep smem")))
            return rc;
    return SAMS_OK;
}

// A cell op + node op pair (k_cellnode_march) over the whole box.
template <class P>
void Solver::launch_cellnode(int arg)
{
    const Geom &g = ctx_.g;
    const long long blocks =
        (long long)((g.nz + 2 + kMK) / kMK) * ((g.ny + 2 + kMJ) / kMJ) * ((g.nx + 2 + kMI) / kMI);
    const size_t smem = (size_t)P::NR * 3 * kRP * sizeof(double);
    if (ctx_.p.geometry)
        k_cellnode_march<P, true, false><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, arg);
    else if (ctx_.p.pow2)
        k_cellnode_march<P, false, true><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, arg);
    else
        k_cellnode_march<P, false, false><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, arg);
    ++launches_;
}

// A marching edge-term kernel (k_edge_march) over cells 0..n+1.
template <class P>
void Solver::launch_edges()
{
    const Geom &g = ctx_.g;
    const long long blocks =
        (long long)((g.nz + 1 + kMK) / kMK) * ((g.ny + 1 + kMJ) / kMJ) * ((g.nx + 1 + kMI) / kMI);
    const size_t smem = (size_t)3 * 3 * kRP * sizeof(double);
    if (ctx_.p.geometry)
        k_edge_march<P, true, false><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_);
    else if (ctx_.p.pow2)
        k_edge_march<P, false, true><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_);
    else
        k_edge_march<P, false, false><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_);
    ++launches_;
}

// Pred1 + Pred2 fused (k_pred_march); the half-step pressures land in the
// S_CS / S_CSV arrays (free from here to the remap), whose slots then swap
// with S_PE / S_PI.
void Solver::launch_pred(int resistive)
{
    const Geom &g = ctx_.g;
    const long long blocks = (long long)((g.nz + kMK) / kMK) * ((g.ny + kMJ) / kMJ) * ((g.nx + kMI) / kMI);
    const size_t smem = (size_t)PredRingSrc::NR * 3 * kRP * sizeof(double);
    double *pe = ctx_.s[S_CS], *pi = ctx_.s[S_CSV];
    if (ctx_.p.geometry)
        k_pred_march<true, false><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, resistive, pe, pi);
    else if (ctx_.p.pow2)
        k_pred_march<false, true><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, resistive, pe, pi);
    else
        k_pred_march<false, false><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, resistive, pe, pi);
    ++launches_;
    std::swap(ctx_.s[S_PE], ctx_.s[S_CS]);
    std::swap(ctx_.s[S_PI], ctx_.s[S_CSV]);
}

// One resistive sub-step fused (k_resist_march): the new B goes to the
// S_CS / S_CSV / S_CV1 arrays (free during the sub-steps), whose slots then
// swap with the field's, so after the two sub-steps B is back in its own
// arrays and those three slots hold B as it was at the start of the last
// sub-step: the predictor's b1 (resistive_effects' copy, lagran.cpp:482-484).
void Solver::launch_resist(bool last)
{
    const Geom &g = ctx_.g;
    const long long blocks =
        (long long)((g.nz + 4 + kMK) / kMK) * ((g.ny + 4 + kMJ) / kMJ) * ((g.nx + 4 + kMI) / kMI);
    const size_t smem = (size_t)ops::ResistRK::NOUT * 3 * kRP * sizeof(double);
    double *nb[3] = {ctx_.s[S_CS], ctx_.s[S_CSV], ctx_.s[S_CV1]};
    if (ctx_.p.geometry)
        k_resist_march<true, false><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, nb[0], nb[1], nb[2]);
    else if (ctx_.p.pow2)
        k_resist_march<false, true><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, nb[0], nb[1], nb[2]);
    else
        k_resist_march<false, false><<<(unsigned)blocks, kMThreads, smem, stream_>>>(ctx_, nb[0], nb[1], nb[2]);
    ++launches_;
    std::swap(ctx_.f[SAMS_F_BX], ctx_.s[S_CS]);
    std::swap(ctx_.f[SAMS_F_BY], ctx_.s[S_CSV]);
    std::swap(ctx_.f[SAMS_F_BZ], ctx_.s[S_CV1]);
    if (last) {
        std::swap(ctx_.s[S_B1X], ctx_.s[S_CS]);
        std::swap(ctx_.s[S_B1Y], ctx_.s[S_CSV]);
        std::swap(ctx_.s[S_B1Z], ctx_.s[S_CV1]);
    }
}

// SweepCT + SweepMass of one sweep (k_ctmass / k_ctmass_z).
template <int DIR>
bool Solver::launch_ctmass(int scale)
{
    const Geom &g = ctx_.g;
    // windows over k (x, y: kWinK lanes over 0..nz+1; z: kZOwn own k per
    // line): on thin grids the separate kernels keep more lanes busy
    const bool window = DIR == 2 ? lanes_full(g.nz + 1, kZOwn) : lanes_full(g.nz + 2, ops::kWinK);
    if (!window) {  // (the solver folds the B scaling in only where the x window runs: scale == 0 here)
        launch<ops::SweepCT<DIR>>(0);
        launch<ops::SweepMass<DIR>>(0);
        return false;
    }
    // dm's periodic fill along the sweep folded into the kernel (the slabs'
    // x fill is an exchange between slabs and stays)
    const int nd = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
    const int images = !(halo_ && DIR == 0) && nd >= kBcSequentialBelow &&
                       bc_.kind[SAMS_F_DM][DIR][0] == SAMS_BC_PERIODIC && bc_.kind[SAMS_F_DM][DIR][1] == SAMS_BC_PERIODIC;
    if (DIR == 2) {
        const long long lines = (long long)(g.nx + 2) * (g.ny + 2);
        dim3 grid((unsigned)ceil_div(lines, kZRows), (unsigned)ceil_div(g.nz + 1, kZOwn));
        if (ctx_.p.geometry)
            k_ctmass_z<true><<<grid, 256, 0, stream_>>>(ctx_, images);
        else
            k_ctmass_z<false><<<grid, 256, 0, stream_>>>(ctx_, images);
    } else {
        const int na = DIR == 0 ? g.ny : g.nx;
        const long long blocks = (long long)(na + 2) * ((g.nz + 1 + ops::kWinK) / ops::kWinK) *
                                 ((nd + kCtS) / kCtS);
        const size_t smem = (size_t)ops::SweepCTMass<DIR>::NARR * kCtP * ops::kWinK * sizeof(double);
        if (ctx_.p.geometry)
            k_ctmass<DIR, true><<<(unsigned)blocks, ops::kWinThreads, smem, stream_>>>(ctx_, scale, images);
        else
            k_ctmass<DIR, false><<<(unsigned)blocks, ops::kWinThreads, smem, stream_>>>(ctx_, scale, images);
    }
    ++launches_;
    return images != 0;
}

template <class Op>
void Solver::launch(int arg)
{
    int lo[3], hi[3];
    Op::bounds(ctx_.g, arg, lo, hi);
    const long long plane = (long long)(hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
    dim3 grid((unsigned)ceil_div(plane, kThreads), (unsigned)(hi[0] - lo[0] + 1));
    if (ctx_.p.geometry)
        k_op<Op, true, false><<<grid, kThreads, 0, stream_>>>(ctx_, arg);
    else if (ctx_.p.pow2)
        k_op<Op, false, true><<<grid, kThreads, 0, stream_>>>(ctx_, arg);
    else
        k_op<Op, false, false><<<grid, kThreads, 0, stream_>>>(ctx_, arg);
    ++launches_;
}

// Whether a boundary fill of the fields in mask rewrites every ghost point
// from domain values, whatever the ghosts held before: every (dim, edge) of
// those fields has a condition (none is SAMS_BC_NONE), and every dimension
// has at least three cells (with fewer, an edge copy reads ghost planes it
// wrote).  Each condition reads domain planes of its own dimension; the fills
// run x, then y, then z, so a point that is a ghost in several dimensions
// ends with the value the last of them computes from the earlier ones.
bool Solver::ghosts_refilled(unsigned mask) const
{
    if (std::min(ctx_.g.nx, std::min(ctx_.g.ny, ctx_.g.nz)) < kBcSequentialBelow) return false;
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        if (mask & (1u << f))
            for (int d = 0; d < 3; ++d)
                for (int e = 0; e < 2; ++e)
                    if (bc_.kind[f][d][e] == SAMS_BC_NONE) return false;
    return true;
}

bool Solver::all_periodic(unsigned mask) const
{
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        if (mask & (1u << f))
            for (int d = 0; d < 3; ++d)
                for (int e = 0; e < 2; ++e)
                    if (bc_.kind[f][d][e] != SAMS_BC_PERIODIC) return false;
    return true;
}

void Solver::bc_fill(unsigned mask)
{
    FieldList fl = make_list(mask);
    if (fl.n == 0) return;
    if (halo_) {  // a slab: x by exchange, then y and z in the same order as below
        halo_->fill_x(*this, mask);
        bc_fill_dim(mask, 1);
        bc_fill_dim(mask, 2);
        return;
    }
    const Geom &g = ctx_.g;
    // the one-pass gather needs every source inside the domain (n >= 3)
    if (all_periodic(mask) && std::min(g.nx, std::min(g.ny, g.nz)) >= kBcSequentialBelow) {
        // the largest ghost shell is the all-half-cell one
        const long long e0 = g.nx + 5, e1 = g.ny + 5, e2 = g.nz + 5;
        const long long cnt = 5 * e1 * e2 + (long long)g.nx * 5 * e2 + (long long)g.nx * g.ny * 5;
        dim3 grid((unsigned)ceil_div(cnt, kThreads), (unsigned)fl.n);
        k_bc_periodic<<<grid, kThreads, 0, stream_>>>(ctx_, fl);
        ++launches_;
        (void)e0;
        return;
    }
    for (int d = 0; d < 3; ++d) bc_fill_dim(mask, d);
}

void Solver::bc_fill_dim(unsigned mask, int d)
{
    if (halo_ && d == 0) {
        halo_->fill_x(*this, mask);
        return;
    }
    for (int e = 0; e < 2; ++e) bc_fill_edge(mask, d, e);
}

void Solver::bc_fill_edge(unsigned mask, int d, int e)
{
    FieldList fl = make_list(mask);
    if (fl.n == 0) return;
    const Geom &g = ctx_.g;
    const long long ext[3] = {g.nx + 5, g.ny + 5, g.nz + 5};
    long long slab = 3;
    for (int q = 0; q < 3; ++q)
        if (q != d) slab *= ext[q];
    dim3 grid((unsigned)ceil_div(slab, kThreads), (unsigned)fl.n);
    k_bc_edge<<<grid, kThreads, 0, stream_>>>(ctx_, fl, bc_, d, e);
    ++launches_;
}

void Solver::enqueue_step(cudaEvent_t *marks)
{
    const int resistive = p_.resistive_mhd ? 1 : 0;
    auto mark = [&](int m) {
        if (marks) cudaEventRecord(marks[m], stream_);
    };
    mark(0);
    // ---- Lagrangian predictor ----
    // the marching kernels tile k by kMK: on thin grids the separate kernels
    // (one thread per (j, k) of a plane) keep more lanes busy
    const bool march = lanes_full(ctx_.g.nz + 1, kMK);
    if (march) {
        launch_cellnode<PrepMarch>(resistive);
    } else {
        launch<ops::CellPrep>(resistive);
        launch<ops::NodePrep>(0);
    }
    launch<ops::Alpha>(0);
    {
        // Visc with two threads per cell (k_visc_split): 1.21 -> 1.12 ms at
        // 256^3 against one thread per cell at 128 registers
        int lo[3], hi[3];
        ops::Visc::bounds(ctx_.g, 0, lo, hi);
        const long long plane = (long long)(hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
        const int ni = hi[0] - lo[0] + 1;
        dim3 grid((unsigned)ceil_div(plane, kThreads / 2), (unsigned)(ni < 16 ? ni : 16));
        if (ctx_.p.geometry)
            k_visc_split<true, false><<<grid, kThreads, 0, stream_>>>(ctx_);
        else if (ctx_.p.pow2)
            k_visc_split<false, true><<<grid, kThreads, 0, stream_>>>(ctx_);
        else
            k_visc_split<false, false><<<grid, kThreads, 0, stream_>>>(ctx_);
        ++launches_;
    }
    if (halo_) halo_->reduce_dt(*this);
    k_dt_finalize<<<1, 1, 0, stream_>>>(sc_, p_.dt_multiplier, resistive);
    ++launches_;
    if (resistive) {
        for (int sub = 0; sub < 2; ++sub) {
            if (march) {
                launch_resist(sub == 1);
            } else {
                launch<ops::ResistRK>(0);
                launch<ops::ResistB>(sub == 1 ? 1 : 0);
            }
            bc_fill(FM_BFIELD | FM_ENERGY);
        }
    }
    if (march) {
        launch_pred(resistive);
    } else {
        launch<ops::Pred1>(resistive);
        launch<ops::Pred2>(0);
    }
    bc_fill(FM_REMAPV);
    mark(1);
    // ---- corrector ----
    // (Corr1 and Corr2 as one pass, with the velocities written out of place,
    // was measured slower on B200: Corr2 runs at 6 blocks per SM alone, at
    // Corr1's 2 when fused.)
    if (march)
        launch_edges<HeatEdges>();
    else
        launch<ops::Corr1>(0);
    launch<ops::Corr2>(0);
    bc_fill(FM_VELOCITY | FM_ENERGY | FM_DENSITY);
    mark(2);
    // ---- remap ----
    // B to and from flux form (BScale) folded into the x and z sweeps' CT
    // updates when the B fills rewrite every ghost point (ghosts_refilled):
    // the z sweep then unscales 0..n only, and the final B fill sets the
    // ghosts from those values, as it does after BScale's pass over the
    // whole box.
    // The x-sweep half of the fold forms b * area inside k_ctmass, so it also
    // needs that window kernel (not used on thin grids).
    const bool b_fill_all = ghosts_refilled(FM_BFIELD) && lanes_full(ctx_.g.nz + 2, ops::kWinK);
    if (p_.rke) launch<ops::RkeZero>(0);
    if (!b_fill_all) launch<ops::BScale>(0);
    if (march) {
        launch_cellnode<VolMarch<0>>(!p_.rke && psweep_ok_ ? 1 : 0);
    } else {
        launch<ops::SweepVol<0>>(!p_.rke && psweep_ok_ ? 1 : 0);
        launch<ops::SweepCvc>(0);
    }
    const bool dm_x = launch_ctmass<0>(b_fill_all ? 1 : 0);
    // The CT update changes only B, which the dm fill and the stages S6-S8
    // do not read, so the y and z sweeps' fused stages take it at their
    // points 0..n (its whole range).  In the x sweep, with the B scaling
    // folded in, it stays a kernel of its own: inside k_psweep it measured
    // slower on B200 (14 us per step), in the y and z sweeps faster (13 and
    // 40 us).
    const bool fused_xy = !p_.rke && psweep_ok_;  // k_psweep runs the x and y stages
    launch<ops::SweepCTUpd<0>>(b_fill_all ? 1 : 0);
    if (!dm_x) bc_fill_dim(FM_DM, 0);
    if (fused_xy) {
        launch_psweep<0>(-1);
    } else {
        launch<ops::SweepS6<0>>(0);
        launch<ops::SweepS7<0>>(0);
        if (p_.rke) {
            launch<ops::SweepRkeDk<0>>(0);
            launch<ops::SweepRkeGather<0>>(0);
        }
        launch<ops::SweepS8<0>>(0);
    }
    bc_fill(FM_ALL9);
    mark(3);
    if (march) {
        launch_cellnode<VolMarch<1>>(!p_.rke && psweep_ok_ ? 1 : 0);
    } else {
        launch<ops::SweepVol<1>>(!p_.rke && psweep_ok_ ? 1 : 0);
        launch<ops::SweepCvc>(0);
    }
    const bool dm_y = launch_ctmass<1>(0);
    if (!fused_xy) launch<ops::SweepCTUpd<1>>(0);
    if (!dm_y) bc_fill_dim(FM_DM, 1);
    if (fused_xy) {
        launch_psweep<1>(0);
    } else {
        launch<ops::SweepS6<1>>(0);
        launch<ops::SweepS7<1>>(0);
        if (p_.rke) {
            launch<ops::SweepRkeDk<1>>(0);
            launch<ops::SweepRkeGather<1>>(0);
        }
        launch<ops::SweepS8<1>>(0);
    }
    bc_fill(FM_ALL9);
    mark(4);
    if (march) {
        launch_cellnode<VolMarch<2>>(0);
    } else {
        launch<ops::SweepVol<2>>(0);
        launch<ops::SweepCvc>(0);
    }
    const bool dm_z = launch_ctmass<2>(0);
    const bool zfused = !p_.rke && ctx_.g.nz + 4 <= kZThreads;
    if (!zfused) launch<ops::SweepCTUpd<2>>(b_fill_all ? 2 : 0);
    if (!dm_z) bc_fill_dim(FM_DM, 2);
    if (zfused) {
        const Geom &g = ctx_.g;
        const int W = g.nz + 4, lines = kZThreads / W;
        const long long nl = (long long)(g.nx + 1) * (g.ny + 1);
        const size_t smem = (size_t)ops::SweepFused<2>::NARR * lines * W * sizeof(double);
        const unsigned blocks = (unsigned)ceil_div(nl, lines);
        const int ct_arg = b_fill_all ? 2 : 0;
        if (ctx_.p.geometry)
            k_zsweep<true><<<blocks, kZThreads, smem, stream_>>>(ctx_, ct_arg);
        else
            k_zsweep<false><<<blocks, kZThreads, smem, stream_>>>(ctx_, ct_arg);
        ++launches_;
    } else {
        launch<ops::SweepS6<2>>(0);
        launch<ops::SweepS7<2>>(0);
        if (p_.rke) {
            launch<ops::SweepRkeDk<2>>(0);
            launch<ops::SweepRkeGather<2>>(0);
        }
        launch<ops::SweepS8<2>>(0);
    }
    // with the B scaling folded into the z sweep's CT update, B needs no pass
    // of its own before the fill, so all nine fields take one fill (the fill
    // of each field is independent of the others')
    bc_fill(FM_ALL9);
    if (!b_fill_all) {
        launch<ops::BScale>(1);
        bc_fill(FM_BFIELD);
    }
    if (p_.rke) launch<ops::RkeEnergy>(0);  // after the remap (shared_data.h:414-417)
    mark(5);
}

int Solver::phase_times(double ms[5])
{
    int rc;
    if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
    cudaEvent_t ev[6];
    for (int i = 0; i < 6; ++i)
        if ((rc = check(cudaEventCreate(&ev[i]), "cudaEventCreate"))) return rc;
    enqueue_step(ev);
    rc = check(cudaEventSynchronize(ev[5]), "phase sync");
    for (int i = 0; i < 5 && !rc; ++i) {
        float t = 0.f;
        rc = check(cudaEventElapsedTime(&t, ev[i], ev[i + 1]), "cudaEventElapsedTime");
        ms[i] = t;
    }
    for (int i = 0; i < 6; ++i) cudaEventDestroy(ev[i]);
    return rc;
}

int Solver::step(long long nsteps)
{
    if (nsteps < 0) { err = "negative step count"; return SAMS_ERR_INVALID; }
    int rc;
    if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
    for (long long s = 0; s < nsteps; ++s) {
        long long before = launches_;
        enqueue_step();
        launches_per_step_ = launches_ - before;
        if ((rc = check(cudaGetLastError(), "step launch"))) return rc;
    }
    return SAMS_OK;
}

int Solver::step_graph(long long nsteps)
{
    if (nsteps < 0) { err = "negative step count"; return SAMS_ERR_INVALID; }
    if (nsteps == 0) return SAMS_OK;
    int rc;
    if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
    auto it = graphs_.find(nsteps);
    if (it == graphs_.end()) {
        cudaGraph_t graph;
        if ((rc = check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture"))) return rc;
        for (long long s = 0; s < nsteps; ++s) {
            long long before = launches_;
            enqueue_step();
            launches_per_step_ = launches_ - before;
        }
        if ((rc = check(cudaStreamEndCapture(stream_, &graph), "end capture"))) return rc;
        cudaGraphExec_t exec;
        rc = check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
        cudaGraphDestroy(graph);
        if (rc) return rc;
        it = graphs_.emplace(nsteps, exec).first;
    }
    return check(cudaGraphLaunch(it->second, stream_), "graph launch");
}

int Solver::sync()
{
    int rc = check(cudaStreamSynchronize(stream_), "synchronize");
    if (rc) return rc;
    Scalars s;
    if ((rc = scalars(s))) return rc;
    if (s.status) {
        err = "the CFL timestep became non-finite or non-positive";
        return SAMS_ERR_NONFINITE;
    }
    return SAMS_OK;
}

int Solver::set_scalars(double dt, double time, long long step)
{
    Scalars h{};
    h.dt = dt;
    h.dtr = dt;
    h.time = time;
    h.step = step;
    const double big = DBL_MAX;
    std::memcpy(&h.dtmin_bits, &big, sizeof big);
    int rc = check(cudaMemcpyAsync(sc_, &h, sizeof(Scalars), cudaMemcpyHostToDevice, stream_), "scalars write");
    if (rc) return rc;
    return check(cudaStreamSynchronize(stream_), "scalars sync");
}

int Solver::scalars(Scalars &out)
{
    int rc = check(cudaMemcpyAsync(&out, sc_, sizeof(Scalars), cudaMemcpyDeviceToHost, stream_), "scalars read");
    if (rc) return rc;
    return check(cudaStreamSynchronize(stream_), "scalars sync");
}

}  // namespace sams
