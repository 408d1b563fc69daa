// lare_ops.cuh -- the fused phases of one LARE3D timestep as per-point
// device operations.  Each Op has
//   bounds(g, arg, lo, hi)   the index box the phase covers, and
//   run(c, arg, i, j, k)     the work of one (i, j, k) of that box,
// so the same code runs under the single-solve launcher (one grid per
// phase) and the batched launcher (one grid over a worklist of tiles from
// many solves).
//
// Fusion plan (reference kernels each op replaces in brackets):
//   CellPrep   cs                                  [lagran.cpp:113-125, 192-198]
//   NodePrep   rho_v, cs_v                         [lagran.cpp:128-153, 201-215]
//   Alpha      alpha1..3                           [lagran.cpp:218-279]
//   Visc       visc_heat, f*_visc, CFL candidate   [lagran.cpp:284-376, 388-439]
//   ResistRK   eta (on the fly), edge E, curlb     [lagran.cpp:449-474, 511-533]
//   ResistB    B update, Ohmic heating, b1 copy    [lagran.cpp:482-499, 541-587]
//   Pred1      cv1, half-step B*cv1, p_e/p_i       [lagran.cpp:598-614, 810-880]
//   Pred2      forces, v1                          [lagran.cpp:619-733]
//   Corr1      shock heating                       [lagran.cpp:888-992]
//   Corr2      velocity, energies, density         [lagran.cpp:754-798]
//   BScale / BUnscale  B <-> flux form             [remap.cpp:46-50, 91-95]
//   SweepVol   cv1, cv2, db1, rho1, dm = 0         [xremap.cpp:24-70 + y/z]
//   SweepCvc   cvc1                                [xremap.cpp:74-81]
//   SweepCT    both CT fluxes                      [xremap.cpp:269-371]
//   SweepCTUpd both CT updates                     [xremap.cpp:87-115]
//   SweepMass  dm                                  [xremap.cpp:373-422]
//   SweepS6    rho, energy fluxes, vertex rho_v,   [xremap.cpp:121-221]
//              cv2 (node), dm (node), v1 shift
//   SweepS7    energy updates, momentum fluxes*dm  [xremap.cpp:130-152, 485-566]
//   SweepS8    momentum updates (rho_v1 inline)    [xremap.cpp:226-261]
// Metric arrays (cv, dxab, ...) are products of the 1-D spacings in
// Cartesian geometry (setup.cpp:337-390) and are formed on the fly in the
// same multiplication order.
#pragma once

#include "lare_device.cuh"
#include "sams_lare_layout.h"

namespace sams {
namespace ops {

using namespace dev;

#define LOFF(i, j, k) box_off(g, (i), (j), (k))

// Metric terms of LARE3D::grid (setup.cpp:337-390), formed on the fly: the
// product of the 1-D spacings in the reference's order, then, outside
// Cartesian geometry, its metric factors in the reference's order (in
// Cartesian geometry they are 1.0 and are skipped).
__device__ __forceinline__ int h2_index(const Ctx &c, int i, int j) { return (i + 2) * (c.g.ny + 5) + (j + 2); }
template <bool GEO>
__device__ __forceinline__ double cv_at(const Ctx &c, int i, int j, int k)
{
    double v = c.ax.dxb[i + 2] * (c.ax.dyb[j + 2] * c.ax.dzb[k + 2]);
    if (GEO && c.p.geometry) v = v * c.gf.hyc[i + 2] * c.gf.hzc[h2_index(c, i, j)];
    return v;
}
template <bool GEO>
__device__ __forceinline__ double dxab_at(const Ctx &c, int i, int j, int k)
{
    double v = c.ax.dyb[j + 2] * c.ax.dzb[k + 2];
    if (GEO && c.p.geometry) v = v * c.gf.hy[i + 2] * c.gf.hz1[h2_index(c, i, j)];
    return v;
}
template <bool GEO>
__device__ __forceinline__ double dyab_at(const Ctx &c, int i, int j, int k)
{
    double v = c.ax.dxb[i + 2] * c.ax.dzb[k + 2];
    if (GEO && c.p.geometry) v = v * c.gf.hz2[h2_index(c, i, j)];
    return v;
}
// dzab at k = -2 is set last with hyc (setup.cpp:368-371)
template <bool GEO>
__device__ __forceinline__ double dzab_at(const Ctx &c, int i, int j, int k)
{
    double v = c.ax.dxb[i + 2] * c.ax.dyb[j + 2];
    if (GEO && c.p.geometry) v = v * (k == -2 ? c.gf.hyc[i + 2] : c.gf.hy[i + 2]);
    return v;
}
template <bool GEO>
__device__ __forceinline__ double dxac_at(const Ctx &c, int i, int j, int k)
{
    double v = c.ax.dyb[j + 2] * c.ax.dzc[k + 2];
    if (GEO && c.p.geometry) v = v * c.gf.hyc[i + 2] * c.gf.hz2[h2_index(c, i, j)];
    return v;
}
template <bool GEO>
__device__ __forceinline__ double dyac_at(const Ctx &c, int i, int j, int k)
{
    double v = c.ax.dxb[i + 2] * c.ax.dzc[k + 2];
    if (GEO && c.p.geometry) v = v * c.gf.hz1[h2_index(c, i, j)];
    return v;
}

__host__ __device__ inline void set_bounds(int *lo, int *hi, int a0, int b0, int a1, int b1, int a2, int b2)
{
    lo[0] = a0; hi[0] = b0;
    lo[1] = a1; hi[1] = b1;
    lo[2] = a2; hi[2] = b2;
}

// ---------------------------------------------------------------------------
// Lagrangian phase
// ---------------------------------------------------------------------------

// Per-point outputs of one op as another op reads them from global memory:
// src(arr, q) is array arr at offset q.  (The fused kernels read the same
// values from a shared-memory ring instead.)
struct ArraySrc {
    static constexpr bool kPressureSum = false;  // p_e and p_i are separate arrays (see Pred2)
    const double *a[6];
    __device__ double operator()(int arr, int q) const { return __ldg(a[arr] + q); }
};

// Sound speed on cells; with resistive MHD also keeps p_e and p_i, which the
// predictor reads as they were at the start of the step (lagran.cpp:121-123,
// 606-607): between the two, the resistive sub-steps heat the electrons and
// refill the energies' ghost cells (energy_bcs), so recomputing them there
// would differ wherever a ghost was not already its boundary value.
struct CellPrep {
    static constexpr int kMinBlocks = 6;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -1, g.nx + 2, -1, g.ny + 2, -1, g.nz + 2);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int resistive, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        double rho, pe, pi;
        c.s[S_CS][o] = sound_speed(c, o, rho, pe, pi);
        if (resistive) {
            c.s[S_PE][o] = pe;
            c.s[S_PI][o] = pi;
        }
    }
    // cs of the cell at offset o, with its rho, p_e and p_i
    __device__ static double sound_speed(const Ctx &c, int o, double &rho, double &pe, double &pi)
    {
        const Geom &g = c.g;
        const RO bx{c.f[SAMS_F_BX]}, by{c.f[SAMS_F_BY]}, bz{c.f[SAMS_F_BZ]};
        double bx1 = 0.5 * (bx[o] + bx[o - g.sx]);
        double by1 = 0.5 * (by[o] + by[o - g.sy]);
        double bz1 = 0.5 * (bz[o] + bz[o - 1]);
        const double gm = c.p.gamma;
        rho = __ldg(c.f[SAMS_F_RHO] + o);
        pe = (gm - 1.0) * rho * __ldg(c.f[SAMS_F_ENERGY_ELECTRON] + o);
        pi = (gm - 1.0) * rho * __ldg(c.f[SAMS_F_ENERGY_ION] + o);
        double p = pe + pi;
        double rmin = pmax(rho, NONE_ZERO);
        double b2 = bx1 * bx1 + by1 * by1 + bz1 * bz1;
        return sqrt((gm * p + b2) / rmin);
    }
};

// Node density and sound speed (8-cell volume-weighted averages).
struct NodePrep {
    static constexpr int kMinBlocks = 4;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -1, g.nx + 1, -1, g.ny + 1, -1, g.nz + 1);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const ArraySrc src{{c.f[SAMS_F_RHO], c.s[S_CS]}};
        run_src<GEO, P2>(c, i, j, k, src, LOFF(i, j, k), g.sx, g.sy, 1);
    }
    // rho (array 0) and cs (array 1) of the node's eight cells read through
    // src(array, q), q = q0 + dx*QX + dy*QY + dz*QZ (dx, dy, dz in {0, 1})
    template <bool GEO, bool P2, class S>
    __device__ static void run_src(const Ctx &c, int i, int j, int k, const S &src, int q0, int QX, int QY, int QZ)
    {
        const Geom &g = c.g;
        struct Arr {
            const S &s;
            int a;
            __device__ double operator[](int q) const { return s(a, q); }
        };
        const Arr rho{src, 0}, cs{src, 1};
        const int ip = i + 1, jp = j + 1, kp = k + 1;
        double cv0 = cv_at<GEO>(c, i, j, k), cv1 = cv_at<GEO>(c, ip, j, k), cv2 = cv_at<GEO>(c, i, jp, k), cv3 = cv_at<GEO>(c, ip, jp, k);
        double cv4 = cv_at<GEO>(c, i, j, kp), cv5 = cv_at<GEO>(c, ip, j, kp), cv6 = cv_at<GEO>(c, i, jp, kp), cv7 = cv_at<GEO>(c, ip, jp, kp);
        const int o0 = q0, o1 = q0 + QX, o2 = q0 + QY, o3 = q0 + QX + QY;
        const int o4 = q0 + QZ, o5 = q0 + QX + QZ, o6 = q0 + QY + QZ, o7 = q0 + QX + QY + QZ;
        const int on = LOFF(i, j, k);
        double sum_rho_cv = rho[o0] * cv0 + rho[o1] * cv1 + rho[o2] * cv2 + rho[o3] * cv3 +
                            rho[o4] * cv4 + rho[o5] * cv5 + rho[o6] * cv6 + rho[o7] * cv7;
        double sum_cv = cv0 + cv1 + cv2 + cv3 + cv4 + cv5 + cv6 + cv7;
        c.s[S_RHOV][on] = div_by<P2>(sum_rho_cv, sum_cv, 0.125 * c.rc.cv);
        double cv_v = 0.125 * sum_cv;
        double sum = cs[o0] * cv0 + cs[o1] * cv1 + cs[o2] * cv2 + cs[o3] * cv3 +
                     cs[o4] * cv4 + cs[o5] * cv5 + cs[o6] * cv6 + cs[o7] * cv7;
        c.s[S_CSV][on] = div_by<P2>(0.125 * sum, cv_v, c.rc.cv);
    }
};

// Edge viscosities.  dt is the previous step's (the CFL reduction of this
// step runs later, lagran.cpp:155-156).
struct Alpha {
    static constexpr int kMinBlocks = 4;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -1, g.nx + 1, -1, g.ny + 2, 0, g.nz + 2);
    }
    // the edge viscosity of direction E (0 x, 1 y, 2 z) at (i, j, k), where
    // that direction's range holds the point
    template <int E, bool GEO, bool P2>
    __device__ static void edge(const Ctx &c, int i, int j, int k)
    {
        const Geom &g = c.g;
        const RO vx{c.f[SAMS_F_VX]}, vy{c.f[SAMS_F_VY]}, vz{c.f[SAMS_F_VZ]};
        const RO rho_v{c.s[S_RHOV]}, cs_v{c.s[S_CSV]};
        const double dt = c.sc->dt, visc1 = c.p.visc1, v2n = c.p.visc2_norm;
        const int o = LOFF(i, j, k);
        if (E == 0 && i >= 0 && j >= 0) {  // alpha1: (0..nx+1, 0..ny+2, 0..nz+2)
            int o1 = LOFF(i - 1, j - 1, k - 1), o2 = LOFF(i, j - 1, k - 1);
            int o0 = o1 - g.sx, o3 = o2 + g.sx;
            double dx = c.ax.dxb[i + 2], dxp = c.ax.dxb[i + 3], dxm = c.ax.dxb[i + 1];
            double dvdots = -(vx[o1] - vx[o2]);
            double cs_edge = pmin(cs_v[o1], cs_v[o2]);
            c.s[S_A1][o] = edge_viscosity<P2>(dt, visc1, v2n, vx, vy, vz, rho_v, dvdots, dx, dxm, dxp, cs_edge, o0, o1, o2, o3, c.rc.xb);
        }
        if (E == 1 && j >= 0 && j <= g.ny + 1) {  // alpha2: (-1..nx+1, 0..ny+1, 0..nz+2)
            int o1 = LOFF(i, j - 1, k - 1), o2 = LOFF(i, j, k - 1);
            int o0 = o1 - g.sy, o3 = o2 + g.sy;
            double dx = c.ax.dyb[j + 2], dxp = c.ax.dyb[j + 3], dxm = c.ax.dyb[j + 1];
            if (GEO && c.p.geometry) {  // lagran.cpp:251-253
                const double h = c.gf.hy[i + 2];
                dx = dx * h; dxp = dxp * h; dxm = dxm * h;
            }
            double dvdots = -(vy[o1] - vy[o2]);
            double cs_edge = pmin(cs_v[o1], cs_v[o2]);
            c.s[S_A2][o] = edge_viscosity<P2>(dt, visc1, v2n, vx, vy, vz, rho_v, dvdots, dx, dxm, dxp, cs_edge, o0, o1, o2, o3, c.rc.yb);
        }
        if (E == 2 && j <= g.ny + 1 && k <= g.nz + 1) {  // alpha3: (-1..nx+1, -1..ny+1, 0..nz+1)
            int o1 = o - 1, o2 = o;
            int o0 = o1 - 1, o3 = o2 + 1;
            double dx = c.ax.dzb[k + 2], dxp = c.ax.dzb[k + 3], dxm = c.ax.dzb[k + 1];
            if (GEO && c.p.geometry) {  // lagran.cpp:270-272
                const double h = c.gf.hz[h2_index(c, i, j)];
                dx = dx * h; dxp = dxp * h; dxm = dxm * h;
            }
            double dvdots = -(vz[o1] - vz[o2]);
            double cs_edge = pmin(cs_v[o1], cs_v[o2]);
            c.s[S_A3][o] = edge_viscosity<P2>(dt, visc1, v2n, vx, vy, vz, rho_v, dvdots, dx, dxm, dxp, cs_edge, o0, o1, o2, o3, c.rc.zb);
        }
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        edge<0, GEO, P2>(c, i, j, k);
        edge<1, GEO, P2>(c, i, j, k);
        edge<2, GEO, P2>(c, i, j, k);
    }
};

// Viscous pressure and heating on cells, viscous forces on nodes and the
// cell's CFL candidate (p_visc is consumed here and never stored).
// Returns the candidate (DBL_MAX outside the CFL range).
struct Visc {
    // (launched by k_visc_split and kb_visc, each with its own register cap)
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, g.nx + 1, 0, g.ny + 1, 0, g.nz + 1);
    }
    // The cell's work in two halves, which the single-solve kernel
    // (k_visc_split) gives to different threads: heat_forces is the viscous
    // heating of cell (i, j, k) (lagran.cpp:283-326) and the viscous forces
    // on node (i, j, k) (:329-376); cfl is the cell's viscous pressure
    // (:303-305, with the three edge jumps it needs formed again, the same
    // expressions) and its CFL candidate (set_dt, :380-443).
    template <bool GEO, bool P2>
    __device__ static void heat_forces(const Ctx &c, int i, int j, int k, bool &nonfinite)
    {
        const Geom &g = c.g;
        const RO vx{c.f[SAMS_F_VX]}, vy{c.f[SAMS_F_VY]}, vz{c.f[SAMS_F_VZ]};
        const RO a1a{c.s[S_A1]}, a2a{c.s[S_A2]}, a3a{c.s[S_A3]};
        const int SX = g.sx, SY = g.sy;
        const int o = LOFF(i, j, k);
        const double dx = c.ax.dxb[i + 2], dyp = c.ax.dyb[j + 2], dzp = c.ax.dzb[k + 2];
        // edge lengths of the heating and forces (lagran.cpp:307-309, 338-340)
        const double dy = (GEO && c.p.geometry) ? dyp * c.gf.hyc[i + 2] : dyp;
        const double dz = (GEO && c.p.geometry) ? dzp * c.gf.hz2[h2_index(c, i, j)] : dzp;
#define DV2(a, b) ((vx[a] - vx[b]) * (vx[a] - vx[b]) + (vy[a] - vy[b]) * (vy[a] - vy[b]) + (vz[a] - vz[b]) * (vz[a] - vz[b]))
        // cell (ix, iy, iz) corners: m = minus one along that axis
        const int c_mmm = o - SX - SY - 1, c_0mm = o - SY - 1, c_00m = o - 1, c_m0m = o - SX - 1;
        const int c_mm0 = o - SX - SY, c_0m0 = o - SY, c_000 = o, c_m00 = o - SX;
        double a1 = DV2(c_mmm, c_0mm);
        double a2 = DV2(c_0mm, c_00m);
        double a3 = DV2(c_00m, c_m0m);
        double a4 = DV2(c_m0m, c_mmm);
        double a5 = DV2(c_mm0, c_0m0);
        double a6 = DV2(c_0m0, c_000);
        double a7 = DV2(c_000, c_m00);
        double a8 = DV2(c_m00, c_mm0);
        double a9 = DV2(c_00m, c_000);
        double a10 = DV2(c_m0m, c_m00);
        double a11 = DV2(c_mmm, c_mm0);
        double a12 = DV2(c_0mm, c_0m0);
#undef DV2
        double vh = -0.25 * dy * dz * a1a[o] * a1
                    - 0.25 * dx * dz * a2a[o] * a2
                    - 0.25 * dy * dz * a1a[o + SY] * a3
                    - 0.25 * dx * dz * a2a[o - SX] * a4
                    - 0.25 * dy * dz * a1a[o + 1] * a5
                    - 0.25 * dx * dz * a2a[o + 1] * a6
                    - 0.25 * dy * dz * a1a[o + SY + 1] * a7
                    - 0.25 * dx * dz * a2a[o - SX + 1] * a8
                    - 0.25 * dx * dy * a3a[o] * a9
                    - 0.25 * dx * dy * a3a[o - SX] * a10
                    - 0.25 * dx * dy * a3a[o - SX - SY] * a11
                    - 0.25 * dx * dy * a3a[o - SY] * a12;
        const double cv = (GEO && c.p.geometry) ? cv_at<GEO>(c, i, j, k) : dx * (dyp * dzp);
        c.s[S_VH][o] = div_by<P2>(vh, cv, c.rc.cv);
        if (i > g.nx || j > g.ny || k > g.nz) return;
        // checked where run checks it: the cells of the CFL range
        if (!(GEO && c.p.geometry && i < 1) && !(fabs(vh) <= DBL_MAX)) nonfinite = true;
        double e1 = a1a[o + SY + 1] * dy * dz;
        double e2 = a1a[o + SX + SY + 1] * dy * dz;
        double e3 = a2a[o + 1] * dx * dz;
        double e4 = a2a[o + SY + 1] * dx * dz;
        double e5 = a3a[o] * dx * dy;
        double e6 = a3a[o + 1] * dx * dy;
        // cv_v = 0.125 * (8-cell sum of cv) (lagran.cpp:142-151)
        const int ip = i + 1, jp = j + 1, kp = k + 1;
        double sum_cv = cv_at<GEO>(c, i, j, k) + cv_at<GEO>(c, ip, j, k) + cv_at<GEO>(c, i, jp, k) + cv_at<GEO>(c, ip, jp, k) +
                        cv_at<GEO>(c, i, j, kp) + cv_at<GEO>(c, ip, j, kp) + cv_at<GEO>(c, i, jp, kp) + cv_at<GEO>(c, ip, jp, kp);
        double cv_v = 0.125 * sum_cv;
#define FV(v) div_by<P2>(e1 * (v[o] - v[o - SX]) + e2 * (v[o] - v[o + SX]) + e3 * (v[o] - v[o - SY]) + \
                e4 * (v[o] - v[o + SY]) + e5 * (v[o] - v[o - 1]) + e6 * (v[o] - v[o + 1]), cv_v, c.rc.cv)
        c.s[S_FXV][o] = FV(vx);
        c.s[S_FYV][o] = FV(vy);
        c.s[S_FZV][o] = FV(vz);
#undef FV
    }
    // (cells 0..n; DBL_MAX outside the CFL range)
    template <bool GEO, bool P2>
    __device__ static double cfl(const Ctx &c, int i, int j, int k, bool &nonfinite)
    {
        const Geom &g = c.g;
        const RO vx{c.f[SAMS_F_VX]}, vy{c.f[SAMS_F_VY]}, vz{c.f[SAMS_F_VZ]};
        const RO a1a{c.s[S_A1]}, a2a{c.s[S_A2]}, a3a{c.s[S_A3]};
        const int SX = g.sx, SY = g.sy;
        const int o = LOFF(i, j, k);
        const double dx = c.ax.dxb[i + 2], dyp = c.ax.dyb[j + 2], dzp = c.ax.dzb[k + 2];
#define DV2(a, b) ((vx[a] - vx[b]) * (vx[a] - vx[b]) + (vy[a] - vy[b]) * (vy[a] - vy[b]) + (vz[a] - vz[b]) * (vz[a] - vz[b]))
        const int c_mmm = o - SX - SY - 1, c_0mm = o - SY - 1, c_00m = o - 1, c_m0m = o - SX - 1;
        const int c_mm0 = o - SX - SY, c_0m0 = o - SY, c_000 = o, c_m00 = o - SX;
        const double a1 = DV2(c_mmm, c_0mm), a2 = DV2(c_0mm, c_00m), a9 = DV2(c_00m, c_000);
#undef DV2
        double p_visc = 0.0;
        p_visc = pmax(p_visc, -a1a[o] * sqrt(a1));
        p_visc = pmax(p_visc, -a2a[o] * sqrt(a2));
        p_visc = pmax(p_visc, -a3a[o] * sqrt(a9));
        const double cv = (GEO && c.p.geometry) ? cv_at<GEO>(c, i, j, k) : dx * (dyp * dzp);
        const double gm = c.p.gamma;
        const RO bx{c.f[SAMS_F_BX]}, by{c.f[SAMS_F_BY]}, bz{c.f[SAMS_F_BZ]};
        double rho = __ldg(c.f[SAMS_F_RHO] + o);
        double pressure = (gm - 1.0) * rho * __ldg(c.f[SAMS_F_ENERGY_ELECTRON] + o) +
                          (gm - 1.0) * rho * __ldg(c.f[SAMS_F_ENERGY_ION] + o);
        double rho0 = pmax(rho, NONE_ZERO);
        double cs2 = gm * pressure / rho0;
        double w1 = div_by<P2>(bx[o] * bx[o] + by[o] * by[o] + bz[o] * bz[o], c.p.mu0, c.rc.mu0) / rho0;
        double c_visc2 = p_visc / rho0;
        // outside Cartesian geometry the CFL range starts at x index 1 (lagran.cpp:384)
        if (GEO && c.p.geometry && i < 1) return DBL_MAX;
        // lagran.cpp:396-398
        const double dhy = (GEO && c.p.geometry) ? dyp * c.gf.hyc[i + 2] : dyp;
        const double dhz = (GEO && c.p.geometry) ? dzp * c.gf.hzc[h2_index(c, i, j)] : dzp;
        double length = pmin(pmin(dx, dhy), dhz);
        double dt1 = length / (sqrt(c_visc2) + sqrt(cs2 + w1 + c_visc2));
        double ax = 0.25 * (dyp * dzp), ay = 0.25 * (dx * dzp), az = 0.25 * (dx * dyp);
        if (GEO && c.p.geometry) {  // lagran.cpp:404-406 reads the metric arrays
            ax = 0.25 * dxab_at<GEO>(c, i, j, k);
            ay = 0.25 * dyab_at<GEO>(c, i, j, k);
            az = 0.25 * dzab_at<GEO>(c, i, j, k);
        }
        double vxbm = (vx[c_m00] + vx[c_mm0] + vx[c_m0m] + vx[c_mmm]) * ax;
        double vxbp = (vx[c_000] + vx[c_0m0] + vx[c_00m] + vx[c_0mm]) * ax;
        double vybm = (vy[c_0m0] + vy[c_mm0] + vy[c_0mm] + vy[c_mmm]) * ay;
        double vybp = (vy[c_000] + vy[c_m00] + vy[c_00m] + vy[c_m0m]) * ay;
        double vzbm = (vz[c_00m] + vz[c_m0m] + vz[c_0mm] + vz[c_mmm]) * az;
        double vzbp = (vz[c_000] + vz[c_m00] + vz[c_0m0] + vz[c_mm0]) * az;
        double dvx = fabs(vxbp - vxbm), dvy = fabs(vybp - vybm), dvz = fabs(vzbp - vzbm);
        double avxm = fabs(vxbm), avxp = fabs(vxbp), avym = fabs(vybm);
        double avyp = fabs(vybp), avzm = fabs(vzbm), avzp = fabs(vzbp);
        double volume = cv;
        double dt2 = volume / pmax(pmax(pmax(avxm, avxp), dvx), 1.0e-10 * volume);
        double dt3 = volume / pmax(pmax(pmax(avym, avyp), dvy), 1.0e-10 * volume);
        double dt4 = volume / pmax(pmax(pmax(avzm, avzp), dvz), 1.0e-10 * volume);
        const double chk = dt1 + dt2 + dt3 + dt4 + p_visc;
        if (!(fabs(chk) <= DBL_MAX)) nonfinite = true;
        return pmin(pmin(pmin(dt1, dt2), dt3), dt4);
    }
    // nonfinite is set when a NaN or infinity shows up in this cell's viscous
    // pressure, heating or CFL terms (the solve's state is no longer finite;
    // the min itself would hide it, as LARE's min does).
    template <bool GEO, bool P2>
    __device__ static double run(const Ctx &c, int, int i, int j, int k, bool &nonfinite)
    {
        heat_forces<GEO, P2>(c, i, j, k, nonfinite);
        if (i > c.g.nx || j > c.g.ny || k > c.g.nz) return DBL_MAX;
        return cfl<GEO, P2>(c, i, j, k, nonfinite);
    }
};

// Resistive sub-step, part 1: current density, eta (lagran.cpp:449-474,
// evaluated at the same point from the same B, so computed once), edge
// electric fields and Ohmic heating rate.
struct ResistRK {
    static constexpr int kMinBlocks = 6;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, g.nx, 0, g.ny, 0, g.nz);
    }
    // outputs: the three edge fluxes and the Ohmic heating rate
    enum { FX, FY, FZ, CURLB, NOUT };
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        double out[NOUT];
        compute<GEO, P2>(c, i, j, k, out);
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        c.s[S_FLUXX][o] = out[FX];
        c.s[S_FLUXY][o] = out[FY];
        c.s[S_FLUXZ][o] = out[FZ];
        c.s[S_CURLB][o] = out[CURLB];
    }
    template <bool GEO, bool P2>
    __device__ static void compute(const Ctx &c, int i, int j, int k, double *out)
    {
        const Geom &g = c.g;
        const RO bx{c.f[SAMS_F_BX]}, by{c.f[SAMS_F_BY]}, bz{c.f[SAMS_F_BZ]};
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const double dxc = c.ax.dxc[i + 2], dyc = c.ax.dyc[j + 2], dzc = c.ax.dzc[k + 2];
        const double rx = c.rc.xc, ry = c.rc.yc, rz = c.rc.zc;
        double jx1 = div_by<P2>(bz[o + SY] - bz[o], dyc, ry) - div_by<P2>(by[o + 1] - by[o], dzc, rz);
        double jx2 = div_by<P2>(bz[o + SX + SY] - bz[o + SX], dyc, ry) - div_by<P2>(by[o + SX + 1] - by[o + SX], dzc, rz);
        double jy1 = div_by<P2>(bx[o + 1] - bx[o], dzc, rz) - div_by<P2>(bz[o + SX] - bz[o], dxc, rx);
        double jy2 = div_by<P2>(bx[o + SY + 1] - bx[o + SY], dzc, rz) - div_by<P2>(bz[o + SX + SY] - bz[o + SY], dxc, rx);
        double jz1 = div_by<P2>(by[o + SX] - by[o], dxc, rx) - div_by<P2>(bx[o + SY] - bx[o], dyc, ry);
        double jz2 = div_by<P2>(by[o + SX + 1] - by[o + 1], dxc, rx) - div_by<P2>(bx[o + SY + 1] - bx[o + 1], dyc, ry);
        double jx = 0.5 * (jx1 + jx2), jy = 0.5 * (jy1 + jy2), jz = 0.5 * (jz1 + jz2);
        // eta_bg + eta0 where |J| > j_max, else eta_bg.  When the two have the
        // same bits (eta0 = 0: the configurations' uniform eta) the choice
        // cannot show and the square root of |J|^2 is skipped.
        const double eta_hi = c.p.eta_bg + c.p.eta0;
        const bool same = __double_as_longlong(eta_hi) == __double_as_longlong(c.p.eta_bg);
        double eta = !same && sqrt(jx * jx + jy * jy + jz * jz) > c.p.j_max ? eta_hi : c.p.eta_bg;
        out[FX] = -jx * eta * dxc * 0.5;
        out[FY] = -jy * eta * dyc * 0.5;
        out[FZ] = -jz * eta * dzc * 0.5;
        out[CURLB] = eta * (jx * jx + jy * jy + jz * jz);
    }
};

// Resistive sub-step, part 2: constrained-transport B update and Ohmic
// heating; on the last sub-step also keeps the pre-update face B as b1,
// which the predictor reads (resistive_effects' copy, lagran.cpp:482-484).
struct ResistB {
    static constexpr int kMinBlocks = 6;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -1, g.nx + 2, -1, g.ny + 2, -1, g.nz + 2);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int last, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        double *bx = c.f[SAMS_F_BX], *by = c.f[SAMS_F_BY], *bz = c.f[SAMS_F_BZ];
        if (last) {
            c.s[S_B1X][o] = bx[o];
            c.s[S_B1Y][o] = by[o];
            c.s[S_B1Z][o] = bz[o];
        }
        const ArraySrc src{{c.s[S_FLUXX], c.s[S_FLUXY], c.s[S_FLUXZ], c.s[S_CURLB]}};
        run_src<P2>(c, i, j, k, src, o, g.sx, g.sy, 1, bx, by, bz);
    }
    // The update at (i, j, k) with the fluxes of ResistRK read through
    // src(array, q) for the cell q = q0 - dx*QX - dy*QY - dz*QZ (dx, dy, dz in
    // {0, 1}); the new B goes to nbx/nby/nbz[o] (unchanged values included),
    // the electron energy is updated in place.
    template <bool P2, class S>
    __device__ static void run_src(const Ctx &c, int i, int j, int k, const S &src, int q0, int QX, int QY, int QZ,
                                   double *nbx, double *nby, double *nbz)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        struct Arr {
            const S &s;
            int a;
            __device__ double operator[](int q) const { return s(a, q); }
        };
        const Arr fx{src, ResistRK::FX}, fy{src, ResistRK::FY}, fz{src, ResistRK::FZ};
        const double dt = c.sc->dt_sub;
        const int q = q0, SX = QX, SY = QY;
        double bxo = __ldg(c.f[SAMS_F_BX] + o), byo = __ldg(c.f[SAMS_F_BY] + o), bzo = __ldg(c.f[SAMS_F_BZ] + o);
        const bool inx = i >= 0 && i <= g.nx, iny = j >= 0 && j <= g.ny, inz = k >= 0 && k <= g.nz;
        const bool inx1 = i >= 1 && i <= g.nx, iny1 = j >= 1 && j <= g.ny, inz1 = k >= 1 && k <= g.nz;
        double bxn = bxo, byn = byo, bzn = bzo;
        if (inx && iny1 && inz1) {
            double area = c.ax.dyb[j + 2] * c.ax.dzb[k + 2];
            bxn = bxo + div_by<P2>((fz[q] - fz[q - SY] + fz[q - QZ] - fz[q - SY - QZ] - fy[q] + fy[q - QZ] - fy[q - SY] + fy[q - SY - QZ]) * dt, area, c.rc.yb * c.rc.zb);
        }
        if (inx1 && iny && inz1) {
            double area = c.ax.dxb[i + 2] * c.ax.dzb[k + 2];
            byn = byo + div_by<P2>((fx[q] - fx[q - QZ] + fx[q - SX] - fx[q - SX - QZ] - fz[q] + fz[q - SX] - fz[q - QZ] + fz[q - SX - QZ]) * dt, area, c.rc.xb * c.rc.zb);
        }
        if (inx1 && iny1 && inz) {
            double area = c.ax.dxb[i + 2] * c.ax.dyb[j + 2];
            bzn = bzo + div_by<P2>((fy[q] - fy[q - SX] + fy[q - SY] - fy[q - SX - SY] - fx[q] + fx[q - SY] - fx[q - SX] + fx[q - SX - SY]) * dt, area, c.rc.xb * c.rc.yb);
        }
        nbx[o] = bxn;
        nby[o] = byn;
        nbz[o] = bzn;
        if (inx1 && iny1 && inz1) {
            const Arr curlb{src, ResistRK::CURLB};
            double sum_curlb = curlb[q] + curlb[q - SX] + curlb[q - SY] + curlb[q - SX - SY] +
                               curlb[q - QZ] + curlb[q - SX - QZ] + curlb[q - SY - QZ] + curlb[q - SX - SY - QZ];
            double *ee = c.f[SAMS_F_ENERGY_ELECTRON];
            ee[o] += sum_curlb * dt / (8.0 * __ldg(c.f[SAMS_F_RHO] + o));
        }
    }
};

// Predictor, part 1: half-step cell volume and B (then scaled by cv1), and
// the half-step pressures (lagran.cpp:598-614, 806-882).
struct Pred1 {
    static constexpr int kMinBlocks = 4;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -1, g.nx + 2, -1, g.ny + 2, -1, g.nz + 2);
    }
    // Outputs of one cell, in this order: cv1, b1x*cv1, b1y*cv1, b1z*cv1 and
    // (where the cell is in 0..n+1 in every dimension, `half_p` set) the
    // half-step p_e, p_i.  Reads the step-start p_e/p_i of resistive runs
    // from S_PE/S_PI.
    enum { CV1, B1X, B1Y, B1Z, PE, PI, NOUT };
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int resistive, int i, int j, int k)
    {
        double out[NOUT];
        bool half_p;
        compute<GEO, P2>(c, resistive, i, j, k, out, half_p);
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        c.s[S_B1X][o] = out[B1X];
        c.s[S_B1Y][o] = out[B1Y];
        c.s[S_B1Z][o] = out[B1Z];
        c.s[S_CV1][o] = out[CV1];
        if (!half_p) return;
        c.s[S_PE][o] = out[PE];
        c.s[S_PI][o] = out[PI];
    }
    template <bool GEO, bool P2>
    __device__ static void compute(const Ctx &c, int resistive, int i, int j, int k, double *out, bool &half_p)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const RO vx{c.f[SAMS_F_VX]}, vy{c.f[SAMS_F_VY]}, vz{c.f[SAMS_F_VZ]};
        const double dt = c.sc->dt;
        const double dxab0 = dxab_at<GEO>(c, i, j, k), dxabm = dxab_at<GEO>(c, i - 1, j, k);
        const double dyab0 = dyab_at<GEO>(c, i, j, k), dyabm = dyab_at<GEO>(c, i, j - 1, k);
        const double dzab0 = dzab_at<GEO>(c, i, j, k), dzabm = dzab_at<GEO>(c, i, j, k - 1);
        const int a = o, am = o - SX, bm = o - SY, cm = o - 1;
        double vxb = 0.25 * (vx[a] + vx[bm] + vx[cm] + vx[bm - 1]);
        double vxbm = 0.25 * (vx[am] + vx[am - SY] + vx[am - 1] + vx[am - SY - 1]);
        double vyb = 0.25 * (vy[a] + vy[am] + vy[cm] + vy[am - 1]);
        double vybm = 0.25 * (vy[bm] + vy[bm - SX] + vy[bm - 1] + vy[bm - SX - 1]);
        double vzb = 0.25 * (vz[a] + vz[am] + vz[bm] + vz[am - SY]);
        double vzbm = 0.25 * (vz[cm] + vz[am - 1] + vz[bm - 1] + vz[am - SY - 1]);
        double vol = cv_at<GEO>(c, i, j, k);
        double dvxdx = div_by<P2>(vxb * dxab0 - vxbm * dxabm, vol, c.rc.cv);
        double dvydy = div_by<P2>(vyb * dyab0 - vybm * dyabm, vol, c.rc.cv);
        double dvzdz = div_by<P2>(vzb * dzab0 - vzbm * dzabm, vol, c.rc.cv);
        double dv = (dvxdx + dvydy + dvzdz) * dt / 2.0;
        double cv1 = vol * (1.0 + dv);

        vxb = 0.25 * (vx[a] + vx[am] + vx[cm] + vx[am - 1]);
        vxbm = 0.25 * (vx[bm] + vx[bm - SX] + vx[bm - 1] + vx[bm - SX - 1]);
        vyb = 0.25 * (vy[a] + vy[bm] + vy[cm] + vy[bm - 1]);
        vybm = 0.25 * (vy[am] + vy[am - SY] + vy[am - 1] + vy[am - SY - 1]);
        double dvxdy = div_by<P2>(vxb * dyab0 - vxbm * dyabm, vol, c.rc.cv);
        double dvydx = div_by<P2>(vyb * dxab0 - vybm * dxabm, vol, c.rc.cv);

        vxb = 0.25 * (vx[a] + vx[am] + vx[bm] + vx[am - SY]);
        vxbm = 0.25 * (vx[cm] + vx[am - 1] + vx[bm - 1] + vx[am - SY - 1]);
        double vzb2 = 0.25 * (vz[a] + vz[bm] + vz[cm] + vz[bm - 1]);
        double vzbm2 = 0.25 * (vz[am] + vz[am - SY] + vz[am - 1] + vz[am - SY - 1]);
        double dvxdz = div_by<P2>(vxb * dzab0 - vxbm * dzabm, vol, c.rc.cv);
        double dvzdx = div_by<P2>(vzb2 * dxab0 - vzbm2 * dxabm, vol, c.rc.cv);

        vyb = 0.25 * (vy[a] + vy[am] + vy[bm] + vy[am - SY]);
        vybm = 0.25 * (vy[cm] + vy[am - 1] + vy[bm - 1] + vy[am - SY - 1]);
        vzb2 = 0.25 * (vz[a] + vz[am] + vz[cm] + vz[am - 1]);
        vzbm2 = 0.25 * (vz[bm] + vz[bm - SX] + vz[bm - 1] + vz[bm - SX - 1]);
        double dvydz = div_by<P2>(vyb * dzab0 - vybm * dzabm, vol, c.rc.cv);
        double dvzdy = div_by<P2>(vzb2 * dyab0 - vzbm2 * dyabm, vol, c.rc.cv);

        double b1x, b1y, b1z;
        if (resistive) {
            b1x = __ldg(c.s[S_B1X] + o);
            b1y = __ldg(c.s[S_B1Y] + o);
            b1z = __ldg(c.s[S_B1Z] + o);
        } else {
            const RO bx{c.f[SAMS_F_BX]}, by{c.f[SAMS_F_BY]}, bz{c.f[SAMS_F_BZ]};
            b1x = 0.5 * (bx[o] + bx[o - SX]);
            b1y = 0.5 * (by[o] + by[o - SY]);
            b1z = 0.5 * (bz[o] + bz[o - 1]);
        }
        double w3 = b1x * dvxdx + b1y * dvxdy + b1z * dvxdz;
        double w4 = b1x * dvydx + b1y * dvydy + b1z * dvydz;
        double w5 = b1x * dvzdx + b1y * dvzdy + b1z * dvzdz;
        b1x = (b1x + w3 * dt / 2.0) / (1.0 + dv);
        b1y = (b1y + w4 * dt / 2.0) / (1.0 + dv);
        b1z = (b1z + w5 * dt / 2.0) / (1.0 + dv);
        out[B1X] = b1x * cv1;
        out[B1Y] = b1y * cv1;
        out[B1Z] = b1z * cv1;
        out[CV1] = cv1;

        half_p = !(i < 0 || i > g.nx + 1 || j < 0 || j > g.ny + 1 || k < 0 || k > g.nz + 1);
        if (!half_p) return;
        const double gm = c.p.gamma;
        double rho = __ldg(c.f[SAMS_F_RHO] + o), ee = __ldg(c.f[SAMS_F_ENERGY_ELECTRON] + o);
        double ei = __ldg(c.f[SAMS_F_ENERGY_ION] + o);
        double pe = resistive ? __ldg(c.s[S_PE] + o) : (gm - 1.0) * rho * ee;
        double pi = resistive ? __ldg(c.s[S_PI] + o) : (gm - 1.0) * rho * ei;
        double dvv = div_by<P2>(cv1, vol, c.rc.cv) - 1.0;
        double e1_e = ee - pe * dvv / rho;
        double e1_i = ei - pi * dvv / rho;
        e1_i += __ldg(c.s[S_VH] + o) * dt / 2.0 / rho;
        out[PE] = e1_e * (gm - 1.0) * rho * vol / cv1;
        out[PI] = e1_i * (gm - 1.0) * rho * vol / cv1;
    }
};

// Predictor, part 2: pressure and J x B forces on nodes and the half-step
// velocity (lagran.cpp:619-733, Cartesian).
struct Pred2 {
    static constexpr int kMinBlocks = 4;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, g.nx, 0, g.ny, 0, g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const ArraySrc src{{c.s[S_CV1], c.s[S_B1X], c.s[S_B1Y], c.s[S_B1Z], c.s[S_PE], c.s[S_PI]}};
        run_src<GEO, P2>(c, i, j, k, src, LOFF(i, j, k), g.sx, g.sy, 1);
    }
    // The node's update with Pred1's outputs read through src(array, q) for
    // the cell q = q0 + dx*QX + dy*QY + dz*QZ (dx, dy, dz in {0, 1}).
    template <bool GEO, bool P2, class S>
    __device__ static void run_src(const Ctx &c, int i, int j, int k, const S &src, int q0, int QX, int QY, int QZ)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        struct Arr {
            const S &s;
            int a;
            __device__ double operator[](int q) const { return s(a, q); }
        };
        const Arr pe{src, Pred1::PE}, pi{src, Pred1::PI}, cv1{src, Pred1::CV1};
        // p_e + p_i of cell q: a source with kPressureSum holds that sum (the
        // same addition, made where the values were produced) under PE
        auto ptot = [&](int q) { return S::kPressureSum ? pe[q] : pe[q] + pi[q]; };
        const Arr bx1{src, Pred1::B1X}, by1{src, Pred1::B1Y}, bz1{src, Pred1::B1Z};
        const double dx = c.ax.dxc[i + 2], dy = c.ax.dyc[j + 2], dz = c.ax.dzc[k + 2];
        // metric factors (lagran.cpp:627-630; all 1.0 in Cartesian geometry)
        const bool geo = GEO && c.p.geometry != 0;
        double h2 = 1.0, h2x = 1.0, h3 = 1.0, h3x = 1.0, h3y = 1.0, h2c = 1.0, h3c = 1.0;
        if (geo) {
            h2 = c.gf.hy[i + 2];
            h2x = c.gf.hy[i + 3];
            h3 = c.gf.hz[h2_index(c, i, j)];
            h3x = c.gf.hz[h2_index(c, i + 1, j)];
            h3y = c.gf.hz[h2_index(c, i, j + 1)];
            h2c = c.gf.hyc[i + 2];
            h3c = c.gf.hzc[h2_index(c, i, j)];
        }
        const double dhy = geo ? h2c * dy : dy, dhz = geo ? h3c * dz : dz;
        const int qx = q0 + QX, qy = q0 + QY, qz = q0 + QZ, qxy = q0 + QX + QY, qxz = q0 + QX + QZ,
                  qyz = q0 + QY + QZ, qxyz = q0 + QX + QY + QZ;
        double pp = ptot(q0), ppx = ptot(qx), ppy = ptot(qy), ppz = ptot(qz);
        double ppxy = ptot(qxy), ppxz = ptot(qxz), ppyz = ptot(qyz), ppxyz = ptot(qxyz);
        double w1 = pp + ppy + ppz + ppyz;
        double w2 = ppx + ppxy + ppxz + ppxyz;
        double fx = div_by<P2>((w1 - w2) * 0.25, dx, c.rc.xc);
        w1 = pp + ppx + ppz + ppxz;
        w2 = ppy + ppxy + ppyz + ppxyz;
        double fy = div_by<P2>((w1 - w2) * 0.25, dhy, c.rc.yc);
        w1 = pp + ppx + ppy + ppxy;
        w2 = ppz + ppxz + ppyz + ppxyz;
        double fz = div_by<P2>((w1 - w2) * 0.25, dhz, c.rc.zc);

        double cvx = cv1[q0] + cv1[qy] + cv1[qz] + cv1[qyz];
        double cvxp = cv1[qx] + cv1[qxy] + cv1[qxz] + cv1[qxyz];
        double cvy = cv1[q0] + cv1[qx] + cv1[qz] + cv1[qxz];
        double cvyp = cv1[qy] + cv1[qxy] + cv1[qyz] + cv1[qxyz];
        double cvz = cv1[q0] + cv1[qx] + cv1[qy] + cv1[qxy];
        double cvzp = cv1[qz] + cv1[qxz] + cv1[qyz] + cv1[qxyz];

        double jx;
        if (geo) {
            w1 = (bz1[q0] + bz1[qx] + bz1[qz] + bz1[qxz]) * h3 / cvy;
            w2 = (bz1[qy] + bz1[qxy] + bz1[qyz] + bz1[qxyz]) * h3y / cvyp;
            jx = (w2 - w1) / dhy / h3c;
        } else {
            w1 = (bz1[q0] + bz1[qx] + bz1[qz] + bz1[qxz]) / cvy;
            w2 = (bz1[qy] + bz1[qxy] + bz1[qyz] + bz1[qxyz]) / cvyp;
            jx = div_by<P2>(w2 - w1, dhy, c.rc.yc);
        }
        w1 = (by1[q0] + by1[qx] + by1[qy] + by1[qxy]) / cvz;
        w2 = (by1[qz] + by1[qxz] + by1[qyz] + by1[qxyz]) / cvzp;
        jx -= div_by<P2>(w2 - w1, dhz, c.rc.zc);

        double jy;
        if (geo) {
            w1 = (bz1[q0] + bz1[qy] + bz1[qz] + bz1[qyz]) * h3 / cvx;
            w2 = (bz1[qx] + bz1[qxy] + bz1[qxz] + bz1[qxyz]) * h3x / cvxp;
            jy = -(w2 - w1) / dx / h3c;
        } else {
            w1 = (bz1[q0] + bz1[qy] + bz1[qz] + bz1[qyz]) / cvx;
            w2 = (bz1[qx] + bz1[qxy] + bz1[qxz] + bz1[qxyz]) / cvxp;
            jy = div_by<P2>(-(w2 - w1), dx, c.rc.xc);
        }
        w1 = (bx1[q0] + bx1[qx] + bx1[qy] + bx1[qxy]) / cvz;
        w2 = (bx1[qz] + bx1[qxz] + bx1[qyz] + bx1[qxyz]) / cvzp;
        jy += div_by<P2>(w2 - w1, dhz, c.rc.zc);

        double jz;
        if (geo) {
            w1 = (by1[q0] + by1[qy] + by1[qz] + by1[qyz]) * h2 / cvx;
            w2 = (by1[qx] + by1[qxy] + by1[qxz] + by1[qxyz]) * h2x / cvxp;
            jz = (w2 - w1) / dx / h2c;
        } else {
            w1 = (by1[q0] + by1[qy] + by1[qz] + by1[qyz]) / cvx;
            w2 = (by1[qx] + by1[qxy] + by1[qxz] + by1[qxyz]) / cvxp;
            jz = div_by<P2>(w2 - w1, dx, c.rc.xc);
        }
        w1 = (bx1[q0] + bx1[qx] + bx1[qz] + bx1[qxz]) / cvy;
        w2 = (bx1[qy] + bx1[qxy] + bx1[qyz] + bx1[qxyz]) / cvyp;
        jz -= div_by<P2>(w2 - w1, dhy, c.rc.yc);

#define SUM8(a) (a[q0] + a[qx] + a[qy] + a[qxy] + a[qz] + a[qxz] + a[qyz] + a[qxyz])
        double bxv = SUM8(bx1) / (cvx + cvxp);
        double byv = SUM8(by1) / (cvx + cvxp);
        double bzv = SUM8(bz1) / (cvx + cvxp);
#undef SUM8
        const double mu0 = c.p.mu0;
        fx += div_by<P2>(jy * bzv - jz * byv, mu0, c.rc.mu0);
        fy += div_by<P2>(jz * bxv - jx * bzv, mu0, c.rc.mu0);
        fz += div_by<P2>(jx * byv - jy * bxv, mu0, c.rc.mu0);
        if (geo) {  // geometric source terms (lagran.cpp:711-721)
            const double rv = __ldg(c.s[S_RHOV] + o), r = c.gf.xb[i + 2];
            const double ux = __ldg(c.f[SAMS_F_VX] + o), uy = __ldg(c.f[SAMS_F_VY] + o), uz = __ldg(c.f[SAMS_F_VZ] + o);
            if (c.p.geometry == 2) {
                const double cotantheta = c.gf.cot[j + 2];
                fx += rv * (uy * uy + uz * uz) / r;
                fy -= rv * (uy * ux - cotantheta * uz * uz) / r;
                fz -= rv * (uz * ux + cotantheta * uz * uy) / r;
            } else {
                fx += rv * uy * uy / r;
                fy -= rv * uy * ux / r;
            }
        }
        // the total force f_visc + f is what both half-steps add (here and in
        // Corr2, lagran.cpp:757-759): kept as that sum, one array per component
        const double sx = __ldg(c.s[S_FXV] + o) + fx, sy = __ldg(c.s[S_FYV] + o) + fy,
                     sz = __ldg(c.s[S_FZV] + o) + fz;
        c.s[S_FX][o] = sx;
        c.s[S_FY][o] = sy;
        c.s[S_FZ][o] = sz;
        const double dt = c.sc->dt;
        const double rho_v = __ldg(c.s[S_RHOV] + o);
        c.f[SAMS_F_VX1][o] = __ldg(c.f[SAMS_F_VX] + o) + dt / 2.0 * sx / rho_v;
        c.f[SAMS_F_VY1][o] = __ldg(c.f[SAMS_F_VY] + o) + dt / 2.0 * sy / rho_v;
        c.f[SAMS_F_VZ1][o] = __ldg(c.f[SAMS_F_VZ] + o) + dt / 2.0 * sz / rho_v;
    }
};

// Corrector, part 1: shock heating with the half-step velocities
// (lagran.cpp:884-993, including its dy*dy factors at :987).
struct Corr1 {
    static constexpr int kMinBlocks = 2;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, g.nx + 1, 0, g.ny + 1, 0, g.nz + 1);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        c.s[S_VH][LOFF(i, j, k)] = heating<GEO, P2>(c, i, j, k);
    }
    // Product of the velocity jumps at the start of the step and of the
    // half step along an edge.  Swapping a and b negates both factors, which
    // gives the same product up to the sign of a zero; a cell's heating is
    // clamped at +0.0, so the sign of a zero never shows.
    __device__ __forceinline__ static double dd(const Ctx &c, int a, int b)
    {
        const RO vx{c.f[SAMS_F_VX]}, vy{c.f[SAMS_F_VY]}, vz{c.f[SAMS_F_VZ]};
        const RO vx1{c.f[SAMS_F_VX1]}, vy1{c.f[SAMS_F_VY1]}, vz1{c.f[SAMS_F_VZ1]};
        return 1 * ((vx[a] - vx[b]) * (vx1[a] - vx1[b]) + (vy[a] - vy[b]) * (vy1[a] - vy1[b]) +
                    (vz[a] - vz[b]) * (vz1[a] - vz1[b]));
    }
    // The products of the x, y and z edges that end at node o, formed once
    // per node by the marching kernel (k_edge_march).
    __device__ __forceinline__ static void node_edges(const Ctx &c, int o, double *e)
    {
        e[0] = dd(c, o - c.g.sx, o);
        e[1] = dd(c, o - c.g.sy, o);
        e[2] = dd(c, o - 1, o);
    }
    // a1..a12 of cell (i, j, k) from the marching kernel's ring (q0: node
    // (i, j, k)).  The shock heating's x and y edges are at k and k+1 and
    // its z edges end at k (lagran.cpp:888-979).
    template <class S>
    __device__ __forceinline__ static void ring_edges(const S &src, int q0, int QX, int QY, double *a)
    {
        a[0] = src(0, q0 - QY);
        a[1] = src(1, q0);
        a[2] = src(0, q0);
        a[3] = src(1, q0 - QX);
        a[4] = src(0, q0 - QY + 1);
        a[5] = src(1, q0 + 1);
        a[6] = src(0, q0 + 1);
        a[7] = src(1, q0 - QX + 1);
        a[8] = src(2, q0);
        a[9] = src(2, q0 - QX);
        a[10] = src(2, q0 - QX - QY);
        a[11] = src(2, q0 - QY);
    }
    // visc_heat of cell (i, j, k) (the corrector's shock_heating)
    template <bool GEO, bool P2>
    __device__ static double heating(const Ctx &c, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const int mm0 = o - SX - SY, m00 = o - SX, om0 = o - SY;
        double a[12];
        a[0] = dd(c, mm0, om0);
        a[1] = dd(c, om0, o);
        a[2] = dd(c, o, m00);
        a[3] = dd(c, m00, mm0);
        a[4] = dd(c, mm0 + 1, om0 + 1);
        a[5] = dd(c, om0 + 1, o + 1);
        a[6] = dd(c, o + 1, m00 + 1);
        a[7] = dd(c, m00 + 1, mm0 + 1);
        a[8] = dd(c, o - 1, o);
        a[9] = dd(c, m00 - 1, m00);
        a[10] = dd(c, mm0 - 1, mm0);
        a[11] = dd(c, om0 - 1, om0);
        return heating_finish<GEO, P2>(c, i, j, k, a);
    }
    template <bool GEO, bool P2>
    __device__ __forceinline__ static double heating_finish(const Ctx &c, int i, int j, int k, const double *a)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const RO a1a{c.s[S_A1]}, a2a{c.s[S_A2]}, a3a{c.s[S_A3]};
        const double a1 = a[0], a2 = a[1], a3 = a[2], a4 = a[3], a5 = a[4], a6 = a[5];
        const double a7 = a[6], a8 = a[7], a9 = a[8], a10 = a[9], a11 = a[10], a12 = a[11];
        const double dx = c.ax.dxb[i + 2];
        double dy = c.ax.dyb[j + 2], dz = c.ax.dzb[k + 2];
        if (GEO && c.p.geometry) {  // lagran.cpp:980-982
            dy = dy * c.gf.hyc[i + 2];
            dz = dz * c.gf.hz2[h2_index(c, i, j)];
        }
        double vh = (-0.25 * dy * dz * a1a[o] * a1 - 0.25 * dx * dz * a2a[o] * a2 - 0.25 * dy * dz * a1a[o + SY] * a3 -
                     0.25 * dx * dz * a2a[o - SX] * a4 - 0.25 * dy * dz * a1a[o + 1] * a5 - 0.25 * dx * dz * a2a[o + 1] * a6 -
                     0.25 * dy * dz * a1a[o + SY + 1] * a7 - 0.25 * dx * dz * a2a[o - SX + 1] * a8 - 0.25 * dy * dy * a3a[o] * a9 -
                     0.25 * dx * dy * a3a[o - SX] * a10 - 0.25 * dy * dy * a3a[o - SX - SY] * a11 - 0.25 * dx * dy * a3a[o - SY] * a12);
        return pmax(div_by<P2>(vh, cv_at<GEO>(c, i, j, k), c.rc.cv), 0.0);
    }
};

// Corrector, part 2: final velocities on nodes; energies, density on cells
// (lagran.cpp:754-798).  The corrector's cv1 is not kept: the x sweep
// recomputes it over the whole range before any read.
struct Corr2 {
    static constexpr int kMinBlocks = 6;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, g.nx, 0, g.ny, 0, g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        velocity(c, o, c.f[SAMS_F_VX], c.f[SAMS_F_VY], c.f[SAMS_F_VZ]);
        if (i < 1 || j < 1 || k < 1) return;
        energy<GEO, P2>(c, i, j, k, __ldg(c.s[S_VH] + o));
    }
    // the node's final velocity into nvx/nvy/nvz[o] (the solve's own
    // arrays in place, or the fused corrector's out-of-place arrays)
    __device__ static void velocity(const Ctx &c, int o, double *nvx, double *nvy, double *nvz)
    {
        const double dt = c.sc->dt;
        const double rho_v = __ldg(c.s[S_RHOV] + o);
        const double vxo = c.f[SAMS_F_VX][o], vyo = c.f[SAMS_F_VY][o], vzo = c.f[SAMS_F_VZ][o];
        // S_FX..S_FZ hold the total force f_visc + f (Pred2)
        nvx[o] = vxo + dt * __ldg(c.s[S_FX] + o) / rho_v;
        nvy[o] = vyo + dt * __ldg(c.s[S_FY] + o) / rho_v;
        nvz[o] = vzo + dt * __ldg(c.s[S_FZ] + o) / rho_v;
    }
    // the cell's energies and density with its visc_heat vh (cells 1..n)
    template <bool GEO, bool P2>
    __device__ static void energy(const Ctx &c, int i, int j, int k, double vh)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const double dt = c.sc->dt;
        const RO vx1{c.f[SAMS_F_VX1]}, vy1{c.f[SAMS_F_VY1]}, vz1{c.f[SAMS_F_VZ1]};
        const int a = o, am = o - SX, bm = o - SY, cm = o - 1;
        double vxb = 0.25 * (vx1[a] + vx1[bm] + vx1[cm] + vx1[bm - 1]);
        double vxbm = 0.25 * (vx1[am] + vx1[am - SY] + vx1[am - 1] + vx1[am - SY - 1]);
        double vyb = 0.25 * (vy1[a] + vy1[am] + vy1[cm] + vy1[am - 1]);
        double vybm = 0.25 * (vy1[bm] + vy1[bm - SX] + vy1[bm - 1] + vy1[bm - SX - 1]);
        double vzb = 0.25 * (vz1[a] + vz1[am] + vz1[bm] + vz1[am - SY]);
        double vzbm = 0.25 * (vz1[cm] + vz1[am - 1] + vz1[bm - 1] + vz1[am - SY - 1]);
        double vol = cv_at<GEO>(c, i, j, k);
        double dvxdx = div_by<P2>(vxb * dxab_at<GEO>(c, i, j, k) - vxbm * dxab_at<GEO>(c, i - 1, j, k), vol, c.rc.cv);
        double dvydy = div_by<P2>(vyb * dyab_at<GEO>(c, i, j, k) - vybm * dyab_at<GEO>(c, i, j - 1, k), vol, c.rc.cv);
        double dvzdz = div_by<P2>(vzb * dzab_at<GEO>(c, i, j, k) - vzbm * dzab_at<GEO>(c, i, j, k - 1), vol, c.rc.cv);
        double dv = (dvxdx + dvydy + dvzdz) * dt;
        double *rho = c.f[SAMS_F_RHO], *ee = c.f[SAMS_F_ENERGY_ELECTRON], *ei = c.f[SAMS_F_ENERGY_ION];
        double r = rho[o];
        ee[o] -= dv * __ldg(c.s[S_PE] + o) / r;
        ei[o] += (dt * vh - dv * __ldg(c.s[S_PI] + o)) / r;
        rho[o] = r / (1.0 + dv);
    }
};

// ---------------------------------------------------------------------------
// Remap
// ---------------------------------------------------------------------------

// B to flux form (remap.cpp:46-50) when arg = 0, back to B with the
// none_zero guard (remap.cpp:91-95) when arg = 1.
struct BScale {
    static constexpr int kMinBlocks = 6;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -2, g.nx + 2, -2, g.ny + 2, -2, g.nz + 2);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int back, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        if (j >= -1 && k >= -1) {
            double a = dxab_at<GEO>(c, i, j, k);
            double *b = c.f[SAMS_F_BX];
            b[o] = back ? b[o] / (a + NONE_ZERO) : b[o] * a;
        }
        if (i >= -1 && k >= -1) {
            double a = dyab_at<GEO>(c, i, j, k);
            double *b = c.f[SAMS_F_BY];
            b[o] = back ? b[o] / (a + NONE_ZERO) : b[o] * a;
        }
        if (i >= -1 && j >= -1) {
            double a = dzab_at<GEO>(c, i, j, k);
            double *b = c.f[SAMS_F_BZ];
            b[o] = back ? b[o] / (a + NONE_ZERO) : b[o] * a;
        }
    }
};

__device__ __forceinline__ int dir_stride(const Geom &g, int dir)
{
    return dir == 0 ? g.sx : (dir == 1 ? g.sy : 1);
}

// First pass of a sweep: volumes before/after the sweep and the sweep-axis
// cell length before it (xremap.cpp:28-70, yremap.cpp:27-80,
// zremap.cpp:28-81); also rho1 = rho and dm = 0 (xremap.cpp:24-25).
// Terms multiplied by a zero pass flag are left out: 0 * finite = 0 and
// adding zero does not change the sum.
template <int DIR>
struct SweepVol {
    static constexpr int kMinBlocks = 6;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -1, g.nx + 2, -1, g.ny + 2, -1, g.nz + 2);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int arg, int i, int j, int k)
    {
        compute<GEO, P2>(c, arg, i, j, k, true);
    }
    // cv1 of the cell (i, j, k); its outputs are stored where `store`
    template <bool GEO, bool P2>
    __device__ static double compute(const Ctx &c, int arg, int i, int j, int k, bool store)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const double dt = c.sc->dt;
        const double dxb0 = c.ax.dxb[i + 2], dyb0 = c.ax.dyb[j + 2], dzb0 = c.ax.dzb[k + 2];
        const double vol = cv_at<GEO>(c, i, j, k);
        const int am = o - SX, bm = o - SY, cm = o - 1;
        double tx = 0.0, ty = 0.0, tz = 0.0, vxb = 0.0, vxbm = 0.0, vyb = 0.0, vybm = 0.0, vzb = 0.0, vzbm = 0.0;
        if (DIR == 0) {
            const RO vx1{c.f[SAMS_F_VX1]};
            vxb = (vx1[o] + vx1[bm] + vx1[cm] + vx1[bm - 1]) * 0.25;
            vxbm = (vx1[am] + vx1[am - SY] + vx1[am - 1] + vx1[am - SY - 1]) * 0.25;
            tx = vxb * dxab_at<GEO>(c, i, j, k) - vxbm * dxab_at<GEO>(c, i - 1, j, k);
        }
        if (DIR <= 1) {
            const RO vy1{c.f[SAMS_F_VY1]};
            vyb = (vy1[o] + vy1[am] + vy1[cm] + vy1[am - 1]) * 0.25;
            vybm = (vy1[bm] + vy1[bm - SX] + vy1[bm - 1] + vy1[bm - SX - 1]) * 0.25;
            ty = vyb * dyab_at<GEO>(c, i, j, k) - vybm * dyab_at<GEO>(c, i, j - 1, k);
        }
        {
            const RO vz1{c.f[SAMS_F_VZ1]};
            vzb = (vz1[o] + vz1[am] + vz1[bm] + vz1[am - SY]) * 0.25;
            vzbm = (vz1[cm] + vz1[am - 1] + vz1[bm - 1] + vz1[am - SY - 1]) * 0.25;
            tz = vzb * dzab_at<GEO>(c, i, j, k) - vzbm * dzab_at<GEO>(c, i, j, k - 1);
        }
        double dv, cv2, db1;
        if (DIR == 0) {
            double dvxdx = div_by<P2>(tx, vol, c.rc.cv), dvydy = div_by<P2>(1.0 * ty, vol, c.rc.cv), dvzdz = div_by<P2>(1.0 * tz, vol, c.rc.cv);
            dv = (dvydy + dvzdz) * dt;
            cv2 = vol * (1.0 + dv);
            dv = dv + dvxdx * dt;
            db1 = dxb0 + (vxb - vxbm) * dt;
        } else if (DIR == 1) {
            double dvydy = div_by<P2>(ty, vol, c.rc.cv), dvzdz = div_by<P2>(1.0 * tz, vol, c.rc.cv);
            dv = dvzdz * dt;
            cv2 = vol * (1.0 + dv);
            dv = dv + dvydy * dt;
            // hyc * dyb (yremap.cpp:78); hyc = 1 in Cartesian geometry
            db1 = ((GEO && c.p.geometry) ? c.gf.hyc[i + 2] * dyb0 : dyb0) + (vyb - vybm) * dt;
        } else {
            double dvzdz = div_by<P2>(tz, vol, c.rc.cv);
            dv = 0.0 * dt;
            cv2 = vol * (1.0 + dv);
            dv = dv + dvzdz * dt;
            // hzc * dzb (zremap.cpp:79)
            db1 = ((GEO && c.p.geometry) ? c.gf.hzc[h2_index(c, i, j)] * dzb0 : dzb0) + (vzb - vzbm) * dt;
        }
        const double cv1 = vol * (1.0 + dv);
        if (store) {
            c.s[S_R_CV2][o] = cv2;
            c.s[S_R_CV1][o] = cv1;
            c.s[S_R_DB1][o] = db1;
            // rho1 = rho before the sweep; arg 1: the sweep runs out of place
            // (k_psweep) and reads rho itself, which it does not change
            if (!arg) c.s[S_R_RHO1][o] = __ldg(c.f[SAMS_F_RHO] + o);
            c.f[SAMS_F_DM][o] = 0.0;
        }
        return cv1;
    }
};

struct SweepCvc {
    static constexpr int kMinBlocks = 4;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -1, g.nx + 1, -1, g.ny + 1, -1, g.nz + 1);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const ArraySrc src{{c.s[S_R_CV1]}};
        const int o = LOFF(i, j, k);
        node(c, o, src, o, g.sx, g.sy, 1);
    }
    // cvc1 at the node at offset o from cv1 of its eight cells read through
    // src(0, q), q = q0 + dx*QX + dy*QY + dz*QZ (dx, dy, dz in {0, 1})
    template <class S>
    __device__ static void node(const Ctx &c, int o, const S &src, int q0, int QX, int QY, int QZ)
    {
        c.s[S_R_CVC1][o] = 0.125 * (src(0, q0) + src(0, q0 + QX) + src(0, q0 + QY) + src(0, q0 + QX + QY) +
                                    src(0, q0 + QZ) + src(0, q0 + QX + QZ) + src(0, q0 + QY + QZ) +
                                    src(0, q0 + QX + QY + QZ));
    }
};

// Both constrained-transport fluxes of a sweep.
template <int DIR>
struct SweepCT {
    static constexpr int kMinBlocks = 4;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, g.nx, 0, g.ny, 0, g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const double dt = c.sc->dt;
        const RO db1{c.s[S_R_DB1]}, cvc1{c.s[S_R_CVC1]}, cv1{c.s[S_R_CV1]};
        const RO v1{c.f[SAMS_F_VX1 + DIR]};
        // transverse offsets of the two db1 samples averaged for each flux
        int t1, t2, va1, va2;
        RO b1, b2;
        if (DIR == 0) {        // vx_by (avg +y, v avg -z), vx_bz (avg +z, v avg -y)
            t1 = SY; va1 = -1; b1.p = c.f[SAMS_F_BY];
            t2 = 1;  va2 = -SY; b2.p = c.f[SAMS_F_BZ];
        } else if (DIR == 1) { // vy_bx (avg +x, v avg -z), vy_bz (avg +z, v avg -x)
            t1 = SX; va1 = -1; b1.p = c.f[SAMS_F_BX];
            t2 = 1;  va2 = -SX; b2.p = c.f[SAMS_F_BZ];
        } else {               // vz_bx (avg +x, v avg -y), vz_by (avg +y, v avg -x)
            t1 = SX; va1 = -SY; b1.p = c.f[SAMS_F_BX];
            t2 = SY; va2 = -SX; b2.p = c.f[SAMS_F_BY];
        }
        const double dci = cvc1[o], dcm = cvc1[o - d], dcp = cvc1[o + d], cvi = cv1[o], cvp = cv1[o + d];
        {
            double v = (v1[o] + v1[o + va1]) * 0.5;
            double dbm = (db1[o - d] + db1[o - d + t1]) * 0.5, dbi = (db1[o] + db1[o + t1]) * 0.5;
            double dbp = (db1[o + d] + db1[o + d + t1]) * 0.5, dbp2 = (db1[o + 2 * d] + db1[o + 2 * d + t1]) * 0.5;
            c.s[S_R_CT1][o] = ct_flux(v, dt, b1[o - d], b1[o], b1[o + d], b1[o + 2 * d], dbm, dbi, dbp, dbp2,
                                      dci, dcm, dcp, cvi, cvp);
        }
        {
            double v = (v1[o] + v1[o + va2]) * 0.5;
            double dbm = (db1[o - d] + db1[o - d + t2]) * 0.5, dbi = (db1[o] + db1[o + t2]) * 0.5;
            double dbp = (db1[o + d] + db1[o + d + t2]) * 0.5, dbp2 = (db1[o + 2 * d] + db1[o + 2 * d + t2]) * 0.5;
            c.s[S_R_CT2][o] = ct_flux(v, dt, b2[o - d], b2[o], b2[o + d], b2[o + 2 * d], dbm, dbi, dbp, dbp2,
                                      dci, dcm, dcp, cvi, cvp);
        }
        (void)SX;
    }
};

// Both constrained-transport updates of a sweep (xremap.cpp:87-115,
// yremap.cpp:97-127, zremap.cpp:103-121), in the reference's order.
// arg 0: the updates over 0..n.  arg 1 (x sweep, when the solver folds the
// remap's B scaling in): first B to flux form (BScale's b * area,
// remap.cpp:46-50) at every box point, then the updates.  arg 2 (z sweep):
// the updates, then B back from flux form (BScale's b / (area + none_zero),
// remap.cpp:91-95) over 0..n.  Each value gets the same single multiply or
// divide as in BScale, so the results are the same bits.
template <int DIR>
struct SweepCTUpd {
    static constexpr int kMinBlocks = 4;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int arg, int *lo, int *hi)
    {
        if (arg == 1)
            set_bounds(lo, hi, -2, g.nx + 2, -2, g.ny + 2, -2, g.nz + 2);
        else
            set_bounds(lo, hi, 0, g.nx, 0, g.ny, 0, g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int arg, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const RO f1{c.s[S_R_CT1]}, f2{c.s[S_R_CT2]};
        double *bx = c.f[SAMS_F_BX], *by = c.f[SAMS_F_BY], *bz = c.f[SAMS_F_BZ];
        double vx = bx[o], vy = by[o], vz = bz[o];
        bool wx = false, wy = false, wz = false;  // components to store
        if (arg == 1) {
            if (j >= -1 && k >= -1) { vx = vx * dxab_at<GEO>(c, i, j, k); wx = true; }
            if (i >= -1 && k >= -1) { vy = vy * dyab_at<GEO>(c, i, j, k); wy = true; }
            if (i >= -1 && j >= -1) { vz = vz * dzab_at<GEO>(c, i, j, k); wz = true; }
        }
        const bool in = i >= 0 && i <= g.nx && j >= 0 && j <= g.ny && k >= 0 && k <= g.nz;
        const bool xb = in, xc = in && i >= 1, yb = in, yc = in && j >= 1, zb = in, zc = in && k >= 1;
        if (DIR == 0) {
            if (xc && yb && zc) { vy = vy - f1[o] + f1[o - SX]; wy = true; }
            if (xc && yc && zb) { vz = vz - f2[o] + f2[o - SX]; wz = true; }
            if (xb && yc && zc) {
                double t = vx + f1[o] - f1[o - SY];
                vx = t + f2[o] - f2[o - 1];
                wx = true;
            }
        } else if (DIR == 1) {
            if (xb && yc && zc) { vx = vx - f1[o] + f1[o - SY]; wx = true; }
            if (xc && yc && zb) { vz = vz - f2[o] + f2[o - SY]; wz = true; }
            if (xc && yb && zc) {
                double t = vy + f1[o] - f1[o - SX];
                vy = t + f2[o] - f2[o - 1];
                wy = true;
            }
        } else {
            if (xb && yc && zc) { vx = vx - f1[o] + f1[o - 1]; wx = true; }
            if (xc && yb && zc) { vy = vy - f2[o] + f2[o - 1]; wy = true; }
            if (xc && yc && zb) {
                double t = vz + f1[o] - f1[o - SX];
                vz = t + f2[o] - f2[o - SY];
                wz = true;
            }
        }
        if (arg == 2) {  // every point of 0..n meets BScale's conditions
            vx = vx / (dxab_at<GEO>(c, i, j, k) + NONE_ZERO);
            vy = vy / (dyab_at<GEO>(c, i, j, k) + NONE_ZERO);
            vz = vz / (dzab_at<GEO>(c, i, j, k) + NONE_ZERO);
            wx = wy = wz = true;
        }
        if (wx) bx[o] = vx;
        if (wy) by[o] = vy;
        if (wz) bz[o] = vz;
    }
};

// Node-average advection velocity of a cell face along the sweep
// (x/y/z_mass_flux and x/y/z_energy_flux use the same 4-point sums).
template <int DIR>
__device__ __forceinline__ double face_velocity(const Ctx &c, int o)
{
    const Geom &g = c.g;
    const int SX = g.sx, SY = g.sy;
    if (DIR == 0) {
        const RO v{c.f[SAMS_F_VX1]};
        return (v[o] + v[o - SY] + v[o - 1] + v[o - SY - 1]) * 0.25;
    } else if (DIR == 1) {
        const RO v{c.f[SAMS_F_VY1]};
        return (v[o - SX] + v[o] + v[o - SX - 1] + v[o - 1]) * 0.25;
    } else {
        const RO v{c.f[SAMS_F_VZ1]};
        return (v[o - SX] + v[o] + v[o - SX - SY] + v[o - SY]) * 0.25;
    }
}

template <int DIR, bool GEO>
__device__ __forceinline__ double face_area(const Ctx &c, int i, int j, int k)
{
    return DIR == 0 ? dxab_at<GEO>(c, i, j, k) : (DIR == 1 ? dyab_at<GEO>(c, i, j, k) : dzab_at<GEO>(c, i, j, k));
}

template <int DIR>
struct SweepMass {
    static constexpr int kMinBlocks = 5;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, DIR == 0 ? g.nx : g.nx + 1, 0, DIR == 1 ? g.ny : g.ny + 1, 0,
                   DIR == 2 ? g.nz : g.nz + 1);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const RO rho{c.f[SAMS_F_RHO]}, cvc1{c.s[S_R_CVC1]}, cv1{c.s[S_R_CV1]};
        double v = face_velocity<DIR>(c, o);
        c.f[SAMS_F_DM][o] = mass_flux(v, c.sc->dt, face_area<DIR, GEO>(c, i, j, k), rho[o - d], rho[o], rho[o + d],
                                      rho[o + 2 * d], cvc1[o], cvc1[o - d], cvc1[o + d], cv1[o], cv1[o + d]);
    }
};

// SweepCT and SweepMass of one sweep in one kernel (k_ctmass): every
// quotient b/db of the CT fluxes is formed once per point into a window store
// and read by the four fluxes along the sweep that use it (the separate
// kernel forms each four times).  quot() at one point along the sweep, then
// fluxes() at the window's own points.
template <int DIR>
struct SweepCTMass {
    enum { F1, F2, DB1, DB2, NARR };  // the two quotients and their db averages
    // t1 / t2: transverse offset of the db1 sample averaged for flux 1 / 2;
    // va1 / va2: offset of the second v1 sample of its advection velocity
    __device__ static void offsets(const Geom &g, int &t1, int &t2, int &va1, int &va2)
    {
        if (DIR == 0) { t1 = g.sy; va1 = -1; t2 = 1; va2 = -g.sy; }
        else if (DIR == 1) { t1 = g.sx; va1 = -1; t2 = 1; va2 = -g.sx; }
        else { t1 = g.sx; va1 = -g.sy; t2 = g.sy; va2 = -g.sx; }
    }
    // scale: B is not yet in flux form (the x sweep with the scaling folded
    // into SweepCTUpd<0>): form BScale's b * area here, the same product
    template <bool GEO, class A>
    __device__ static void quot(const Ctx &c, int i, int j, int k, A st, bool scale)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        int t1, t2, va1, va2;
        offsets(g, t1, t2, va1, va2);
        const RO db1{c.s[S_R_DB1]};
        const RO b1{c.f[DIR == 0 ? SAMS_F_BY : SAMS_F_BX]}, b2{c.f[DIR == 2 ? SAMS_F_BY : SAMS_F_BZ]};
        const double dba1 = (db1[o] + db1[o + t1]) * 0.5, dba2 = (db1[o] + db1[o + t2]) * 0.5;
        double v1 = b1[o], v2 = b2[o];
        if (DIR == 0 && scale) {  // by and bz at i >= -1, k >= 0: BScale scales both
            v1 = v1 * dyab_at<GEO>(c, i, j, k);
            v2 = v2 * dzab_at<GEO>(c, i, j, k);
        }
        st.put(F1, v1 / dba1);
        st.put(F2, v2 / dba2);
        st.put(DB1, dba1);
        st.put(DB2, dba2);
    }
    // CT fluxes where `ct` ((i, j, k) in 0..n), the mass flux everywhere it
    // is called (0..n along the sweep, 0..n+1 across).  With `images` (dm
    // periodic along the sweep, at least three cells) the mass flux also goes
    // to the ghost points that the periodic fill along the sweep would copy it
    // to (sweep index n-1, n -> -1, 0 and 1, 2 -> n+1, n+2), and index 0,
    // which that fill overwrites, is left alone, so the fill is not needed.
    template <bool GEO, class A>
    __device__ static void fluxes(const Ctx &c, int i, int j, int k, A st, bool ct, bool images = false)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const double dt = c.sc->dt;
        const RO cvc1{c.s[S_R_CVC1]}, cv1{c.s[S_R_CV1]};
        const double dci = cvc1[o], dcm = cvc1[o - d], dcp = cvc1[o + d], cvi = cv1[o], cvp = cv1[o + d];
        if (ct) {
            int t1, t2, va1, va2;
            offsets(g, t1, t2, va1, va2);
            const RO v1{c.f[SAMS_F_VX1 + DIR]};
            const double v1o = v1[o];
            c.s[S_R_CT1][o] = ct_flux_q((v1o + v1[o + va1]) * 0.5, dt, st.get(F1, -1), st.get(F1, 0), st.get(F1, 1),
                                        st.get(F1, 2), st.get(DB1, 0), st.get(DB1, 1), dci, dcm, dcp, cvi, cvp);
            c.s[S_R_CT2][o] = ct_flux_q((v1o + v1[o + va2]) * 0.5, dt, st.get(F2, -1), st.get(F2, 0), st.get(F2, 1),
                                        st.get(F2, 2), st.get(DB2, 0), st.get(DB2, 1), dci, dcm, dcp, cvi, cvp);
        }
        const RO rho{c.f[SAMS_F_RHO]};
        const double m = mass_flux(face_velocity<DIR>(c, o), dt, face_area<DIR, GEO>(c, i, j, k), rho[o - d],
                                   rho[o], rho[o + d], rho[o + 2 * d], dci, dcm, dcp, cvi, cvp);
        double *dm = c.f[SAMS_F_DM];
        if (!images) {
            dm[o] = m;
            return;
        }
        const int s = DIR == 0 ? i : (DIR == 1 ? j : k);
        const int nd = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
        if (s >= 1) dm[o] = m;
        if (s >= nd - 1) dm[o - nd * d] = m;
        if (s >= 1 && s <= 2) dm[o + nd * d] = m;
    }
};

// Range lo/hi of index q in dimension DIM for a sweep-direction-dependent
// interval: [alo, ahi] along the sweep, [blo, bhi] across it.
template <int DIR, int DIM>
__device__ __forceinline__ bool in_sweep_range(int q, int n, int alo, int ahi_off, int blo, int bhi_off)
{
    return DIM == DIR ? (q >= alo && q <= n + ahi_off) : (q >= blo && q <= n + bhi_off);
}

// rho update, energy fluxes, vertex density, node cv2, node dm and the v1
// shift (xremap.cpp:121-221 and the y/z analogues).
template <int DIR>
struct SweepS6 {
    static constexpr int kMinBlocks = 4;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, DIR == 0 ? -2 : 0, DIR == 0 ? g.nx + 1 : g.nx, DIR == 1 ? -2 : 0,
                   DIR == 1 ? g.ny + 1 : g.ny, DIR == 2 ? -2 : 0, DIR == 2 ? g.nz + 1 : g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const double dt = c.sc->dt;
        const RO rho1{c.s[S_R_RHO1]}, cv1{c.s[S_R_CV1]}, cv2{c.s[S_R_CV2]}, cvc1{c.s[S_R_CVC1]};
        const RO dm{c.f[SAMS_F_DM]};
        const int nd = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
        const int qd = DIR == 0 ? i : (DIR == 1 ? j : k);
        const bool all0n = i >= 0 && i <= g.nx && j >= 0 && j <= g.ny && k >= 0 && k <= g.nz;
        // density (1..n)^3
        if (i >= 1 && j >= 1 && k >= 1 && i <= g.nx && j <= g.ny && k <= g.nz)
            c.f[SAMS_F_RHO][o] = (rho1[o] * cv1[o] + dm[o - d] - dm[o]) / cv2[o];
        // energy fluxes (0..n)^3
        if (all0n) {
            double v = face_velocity<DIR>(c, o);
            double area = face_area<DIR, GEO>(c, i, j, k);
            const RO ee{c.f[SAMS_F_ENERGY_ELECTRON]}, ei{c.f[SAMS_F_ENERGY_ION]};
            c.s[S_R_FE1][o] = energy_flux(v, dt, area, ee[o - d], ee[o], ee[o + d], ee[o + 2 * d], cvc1[o], cvc1[o - d],
                                          cvc1[o + d], cv1[o], cv1[o + d], rho1[o], rho1[o + d], dm[o]);
            c.s[S_R_FE2][o] = energy_flux(v, dt, area, ei[o - d], ei[o], ei[o + d], ei[o + 2 * d], cvc1[o], cvc1[o - d],
                                          cvc1[o + d], cv1[o], cv1[o + d], rho1[o], rho1[o + d], dm[o]);
            // node cv2 (0..n)^3
            c.s[S_R_CV2N][o] = (cv2[o] + cv2[o + SX] + cv2[o + SY] + cv2[o + SX + SY] +
                                cv2[o + 1] + cv2[o + SX + 1] + cv2[o + SY + 1] + cv2[o + SX + SY + 1]) * 0.125;
        }
        // vertex density: -1..n+1 along the sweep, 0..n across
        if (qd >= -1) {
            double sum = rho1[o] * cv1[o] + rho1[o + SX] * cv1[o + SX] + rho1[o + SY] * cv1[o + SY] +
                         rho1[o + SX + SY] * cv1[o + SX + SY] + rho1[o + 1] * cv1[o + 1] +
                         rho1[o + SX + 1] * cv1[o + SX + 1] + rho1[o + SY + 1] * cv1[o + SY + 1] +
                         rho1[o + SX + SY + 1] * cv1[o + SX + SY + 1];
            c.s[S_R_RVN][o] = DIR == 0 ? sum * 0.125 / cvc1[o] : sum * (0.125 / cvc1[o]);
        }
        // node dm: -1..n along the sweep, 0..n across
        if (qd >= -1 && qd <= nd) {
            c.s[S_R_DMN][o] = (dm[o] + dm[o + SX] + dm[o + SY] + dm[o + SX + SY] +
                               dm[o + 1] + dm[o + SX + 1] + dm[o + SY + 1] + dm[o + SX + SY + 1]) * 0.125;
        }
        // sweep-direction v1 moved to the face centre: -2..n+1 along, 0..n across
        {
            const RO v1{c.f[SAMS_F_VX1 + DIR]};
            c.s[S_R_V1S][o] = (v1[o] + v1[o + d]) * 0.5;
        }
    }
};

// Energy updates (1..n)^3 and the three momentum fluxes (times dm).
template <int DIR>
struct SweepS7 {
    static constexpr int kMinBlocks = 6;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, DIR == 0 ? -1 : 0, g.nx, DIR == 1 ? -1 : 0, g.ny, DIR == 2 ? -1 : 0, g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const double dt = c.sc->dt;
        const RO rho1{c.s[S_R_RHO1]}, cv1{c.s[S_R_CV1]}, cv2{c.s[S_R_CV2]}, cvc1{c.s[S_R_CVC1]};
        if (i >= 1 && j >= 1 && k >= 1) {
            const RO f1{c.s[S_R_FE1]}, f2{c.s[S_R_FE2]};
            double *ee = c.f[SAMS_F_ENERGY_ELECTRON], *ei = c.f[SAMS_F_ENERGY_ION];
            double den = cv2[o] * __ldg(c.f[SAMS_F_RHO] + o);
            ee[o] = (ee[o] * cv1[o] * rho1[o] + f1[o - d] - f1[o]) / den;
            ei[o] = (ei[o] * cv1[o] * rho1[o] + f2[o - d] - f2[o]) / den;
        }
        const RO v1s{c.s[S_R_V1S]}, rv{c.s[S_R_RVN]}, dmn{c.s[S_R_DMN]};
        // x sweep uses dxac; the y and z sweeps both use dyac (zremap.cpp:475)
        double area = DIR == 0 ? dxac_at<GEO>(c, i, j, k) : dyac_at<GEO>(c, i, j, k);
        const double v = v1s[o], dmv = dmn[o];
        const double dci = cv1[o + d], dcm = cv1[o], dcp = cv1[o + 2 * d], cvi = cvc1[o], cvp = cvc1[o + d];
        const double rvi = rv[o], rvp = rv[o + d];
        const RO ux{c.f[SAMS_F_VX]}, uy{c.f[SAMS_F_VY]}, uz{c.f[SAMS_F_VZ]};
        const double f1 = mom_flux<DIR == 2>(v, dt, area, ux[o - d], ux[o], ux[o + d], ux[o + 2 * d], dci, dcm, dcp,
                                             cvi, cvp, rvi, rvp, dmv);
        const double f2 = mom_flux<DIR == 2>(v, dt, area, uy[o - d], uy[o], uy[o + d], uy[o + 2 * d], dci, dcm, dcp,
                                             cvi, cvp, rvi, rvp, dmv);
        const double f3 = mom_flux<DIR == 2>(v, dt, area, uz[o - d], uz[o], uz[o + d], uz[o + 2 * d], dci, dcm, dcp,
                                             cvi, cvp, rvi, rvp, dmv);
        // with the rke correction the flux is kept as is (its kinetic-energy
        // error needs it) and SweepS8 takes the product with dm
        const bool raw = c.p.rke != 0;
        c.s[S_R_FM1][o] = raw ? f1 : f1 * dmv;
        c.s[S_R_FM2][o] = raw ? f2 : f2 * dmv;
        c.s[S_R_FM3][o] = raw ? f3 : f3 * dmv;
    }
};

// Momentum updates with the vertex density after the sweep formed inline
// (xremap.cpp:226-261).
template <int DIR>
struct SweepS8 {
    static constexpr int kMinBlocks = 6;  // blocks of 256 per SM (register cap), tuned on B200
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, g.nx, 0, g.ny, 0, g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const RO rv{c.s[S_R_RVN]}, cvc1{c.s[S_R_CVC1]}, cv2n{c.s[S_R_CV2N]}, dmn{c.s[S_R_DMN]};
        const double rvo = rv[o], cvco = cvc1[o], cv2o = cv2n[o];
        const double rho_v1 = (rvo * cvco + dmn[o - d] - dmn[o]) / cv2o;
        const double den = cv2o * rho_v1;
        double *ux = c.f[SAMS_F_VX], *uy = c.f[SAMS_F_VY], *uz = c.f[SAMS_F_VZ];
        const RO f1{c.s[S_R_FM1]}, f2{c.s[S_R_FM2]}, f3{c.s[S_R_FM3]};
        if (c.p.rke) {  // raw fluxes: the reference's flux *= dm, then the update
            const double dm0 = dmn[o - d], dm1 = dmn[o];
            ux[o] = (rvo * ux[o] * cvco + f1[o - d] * dm0 - f1[o] * dm1) / den;
            uy[o] = (rvo * uy[o] * cvco + f2[o - d] * dm0 - f2[o] * dm1) / den;
            uz[o] = (rvo * uz[o] * cvco + f3[o - d] * dm0 - f3[o] * dm1) / den;
            return;
        }
        ux[o] = (rvo * ux[o] * cvco + f1[o - d] - f1[o]) / den;
        uy[o] = (rvo * uy[o] * cvco + f2[o - d] - f2[o]) / den;
        uz[o] = (rvo * uz[o] * cvco + f3[o - d] - f3[o]) / den;
    }
};

// The state arrays a fused sweep writes: in place (the solve's own rho,
// energies and velocities) or into six free scratch arrays (x and y sweeps,
// see k_psweep), in which case the solve's arrays are only read.
struct SweepOut {
    double *rho, *ee, *ei, *ux, *uy, *uz;
};

__device__ __forceinline__ SweepOut sweep_in_place(const Ctx &c)
{
    return SweepOut{c.f[SAMS_F_RHO], c.f[SAMS_F_ENERGY_ELECTRON], c.f[SAMS_F_ENERGY_ION],
                    c.f[SAMS_F_VX], c.f[SAMS_F_VY], c.f[SAMS_F_VZ]};
}

// SweepS6, SweepS7 and SweepS8 of one sweep as three stages of one kernel.
// Every value a stage passes to the next (energy fluxes, vertex density,
// node dm, momentum fluxes) is read only along the sweep direction on the
// same line, so a block that holds a stretch of lines runs the stages over
// it with __syncthreads in between and keeps those intermediates in shared
// memory:
//   k_zsweep (z): whole z lines, one thread per k, in place (every array
//     the stages write is read only along its own line);
//   k_psweep (x, y): 32 adjacent z values x a window of the line plus a
//     recomputed halo, writing rho, energies and velocities out of place
//     (SweepOut), so no block reads a value another block has updated.
// Stage A and B at halo points (own == false) compute the intermediates
// only; the state is written at the window's own points.  The arithmetic of
// each stage is the separate kernel's; node cv2 and the shifted v1 are formed
// where they are used (same expressions).  Not used with rke (its correction
// needs the raw momentum fluxes in memory).
// A is the intermediate store at one point: get(array, ds) reads it ds
// points along the sweep, put(array, v) writes it here.
template <int DIR>
struct SweepFused {
    // In the x and y windows the momentum fluxes FM1, FM2 take the energy
    // fluxes' slots: stage B runs as two passes with a barrier between them
    // (stage_b_energy reads the energy fluxes at s-1 and s, then stage_b_mom
    // writes the momentum fluxes), so a window holds five arrays instead of
    // seven and leaves more of the SM's memory to L1 (measured 15 and 28 us
    // faster per x and y sweep at 256^3).  The z sweep's line store is small
    // and keeps seven arrays, with no barrier between the passes (13 us
    // faster than five).
    enum { FE1, FE2, RVN, DMN, FM3, FM1 = DIR == 2 ? 5 : FE1, FM2 = DIR == 2 ? 6 : FE2, NARR = DIR == 2 ? 7 : 5 };
    static constexpr bool kSharedFluxSlots = DIR != 2;

    // SweepS6 at (i, j, k), sweep index -2..n+1.
    template <bool GEO, class A>
    __device__ static void stage_a(const Ctx &c, int i, int j, int k, A b, const SweepOut &w, bool own)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const double dt = c.sc->dt;
        const RO rho1{c.s[S_R_RHO1]}, cv1{c.s[S_R_CV1]}, cv2{c.s[S_R_CV2]}, cvc1{c.s[S_R_CVC1]};
        const RO dm{c.f[SAMS_F_DM]};
        const int nd = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
        const int qd = DIR == 0 ? i : (DIR == 1 ? j : k);
        if (own && i >= 1 && j >= 1 && k >= 1 && i <= g.nx && j <= g.ny && k <= g.nz)
            w.rho[o] = (rho1[o] * cv1[o] + dm[o - d] - dm[o]) / cv2[o];
        if (qd >= 0 && qd <= nd) {  // the lines are 0..n across the sweep
            double v = face_velocity<DIR>(c, o);
            double area = face_area<DIR, GEO>(c, i, j, k);
            const RO ee{c.f[SAMS_F_ENERGY_ELECTRON]}, ei{c.f[SAMS_F_ENERGY_ION]};
            b.put(FE1, energy_flux(v, dt, area, ee[o - d], ee[o], ee[o + d], ee[o + 2 * d], cvc1[o], cvc1[o - d],
                                   cvc1[o + d], cv1[o], cv1[o + d], rho1[o], rho1[o + d], dm[o]));
            b.put(FE2, energy_flux(v, dt, area, ei[o - d], ei[o], ei[o + d], ei[o + 2 * d], cvc1[o], cvc1[o - d],
                                   cvc1[o + d], cv1[o], cv1[o + d], rho1[o], rho1[o + d], dm[o]));
        }
        if (qd >= -1) {
            double sum = rho1[o] * cv1[o] + rho1[o + SX] * cv1[o + SX] + rho1[o + SY] * cv1[o + SY] +
                         rho1[o + SX + SY] * cv1[o + SX + SY] + rho1[o + 1] * cv1[o + 1] +
                         rho1[o + SX + 1] * cv1[o + SX + 1] + rho1[o + SY + 1] * cv1[o + SY + 1] +
                         rho1[o + SX + SY + 1] * cv1[o + SX + SY + 1];
            b.put(RVN, DIR == 0 ? sum * 0.125 / cvc1[o] : sum * (0.125 / cvc1[o]));
        }
        if (qd >= -1 && qd <= nd)
            b.put(DMN, (dm[o] + dm[o + SX] + dm[o + SY] + dm[o + SX + SY] + dm[o + 1] + dm[o + SX + 1] +
                        dm[o + SY + 1] + dm[o + SX + SY + 1]) * 0.125);
    }

    // SweepS7 at (i, j, k), first pass: the energy updates at the own points
    // (sweep index 1..n), after stage A everywhere.
    template <class A>
    __device__ static void stage_b_energy(const Ctx &c, int i, int j, int k, A b, const SweepOut &w)
    {
        if (i < 1 || j < 1 || k < 1) return;
        const int o = box_off(c.g, i, j, k);
        const RO rho1{c.s[S_R_RHO1]}, cv1{c.s[S_R_CV1]}, cv2{c.s[S_R_CV2]};
        const double *ee = c.f[SAMS_F_ENERGY_ELECTRON], *ei = c.f[SAMS_F_ENERGY_ION];
        double den = cv2[o] * w.rho[o];  // stage A's rho (a coherent load)
        const double e_new = (ee[o] * cv1[o] * rho1[o] + b.get(FE1, -1) - b.get(FE1, 0)) / den;
        const double i_new = (ei[o] * cv1[o] * rho1[o] + b.get(FE2, -1) - b.get(FE2, 0)) / den;
        w.ee[o] = e_new;
        w.ei[o] = i_new;
    }

    // SweepS7 at (i, j, k), second pass: the momentum fluxes, sweep index
    // -1..n (after stage_b_energy everywhere: they overwrite the energy
    // fluxes).
    template <bool GEO, class A>
    __device__ static void stage_b_mom(const Ctx &c, int i, int j, int k, A b)
    {
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const double dt = c.sc->dt;
        const RO cv1{c.s[S_R_CV1]}, cvc1{c.s[S_R_CVC1]};
        // x sweep uses dxac; the y and z sweeps both use dyac (zremap.cpp:475)
        double area = DIR == 0 ? dxac_at<GEO>(c, i, j, k) : dyac_at<GEO>(c, i, j, k);
        const RO v1{c.f[SAMS_F_VX1 + DIR]};
        const double v = (v1[o] + v1[o + d]) * 0.5, dmv = b.get(DMN, 0);
        const double dci = cv1[o + d], dcm = cv1[o], dcp = cv1[o + 2 * d], cvi = cvc1[o], cvp = cvc1[o + d];
        const double rvi = b.get(RVN, 0), rvp = b.get(RVN, 1);
        const double *ux = c.f[SAMS_F_VX], *uy = c.f[SAMS_F_VY], *uz = c.f[SAMS_F_VZ];
        const double f1 = mom_flux<DIR == 2>(v, dt, area, ux[o - d], ux[o], ux[o + d], ux[o + 2 * d], dci, dcm, dcp,
                                             cvi, cvp, rvi, rvp, dmv);
        const double f2 = mom_flux<DIR == 2>(v, dt, area, uy[o - d], uy[o], uy[o + d], uy[o + 2 * d], dci, dcm, dcp,
                                             cvi, cvp, rvi, rvp, dmv);
        const double f3 = mom_flux<DIR == 2>(v, dt, area, uz[o - d], uz[o], uz[o + d], uz[o + 2 * d], dci, dcm, dcp,
                                             cvi, cvp, rvi, rvp, dmv);
        b.put(FM1, f1 * dmv);
        b.put(FM2, f2 * dmv);
        b.put(FM3, f3 * dmv);
    }

    // SweepS8 at (i, j, k), sweep index 0..n (after stage B everywhere).
    template <class A>
    __device__ static void stage_c(const Ctx &c, int i, int j, int k, A b, const SweepOut &w)
    {
        const Geom &g = c.g;
        const int SX = g.sx, SY = g.sy, o = LOFF(i, j, k);
        const RO cv2{c.s[S_R_CV2]};
        const double cv2o = (cv2[o] + cv2[o + SX] + cv2[o + SY] + cv2[o + SX + SY] + cv2[o + 1] + cv2[o + SX + 1] +
                             cv2[o + SY + 1] + cv2[o + SX + SY + 1]) * 0.125;
        const double rvo = b.get(RVN, 0), cvco = __ldg(c.s[S_R_CVC1] + o);
        const double rho_v1 = (rvo * cvco + b.get(DMN, -1) - b.get(DMN, 0)) / cv2o;
        const double den = cv2o * rho_v1;
        const double *ux = c.f[SAMS_F_VX], *uy = c.f[SAMS_F_VY], *uz = c.f[SAMS_F_VZ];
        const double nx = (rvo * ux[o] * cvco + b.get(FM1, -1) - b.get(FM1, 0)) / den;
        const double ny = (rvo * uy[o] * cvco + b.get(FM2, -1) - b.get(FM2, 0)) / den;
        const double nz = (rvo * uz[o] * cvco + b.get(FM3, -1) - b.get(FM3, 0)) / den;
        w.ux[o] = nx;
        w.uy[o] = ny;
        w.uz[o] = nz;
    }
};

// Threads per block of the fused z sweep: whole z lines of nz+4 threads.
constexpr int kZLineThreads = 288;

// Intermediates of the block's z lines: array a at sm[a * S + at], at =
// line base + k + 2.
struct LineStore {
    double *sm;
    int S, at;
    __device__ double get(int a, int ds) const { return sm[a * S + at + ds]; }
    __device__ void put(int a, double v) const { sm[a * S + at] = v; }
};

// Fused x / y sweep windows: kWinK adjacent z values (a warp) x kWinS own
// points along the line, plus stage A's halo of two points before and one
// after and stage B's of one before.  Array a of the window at
// sm[((a * P) + p) * kWinK + kc], p = s - s0 + 2, P = kWinS + 3.
constexpr int kWinK = 32, kWinS = 21, kWinThreads = 256;  // 31 KB of shared memory; 4 blocks per SM (window tuned on B200)
struct WinStore {
    double *sm;
    int at, kc;
    static constexpr int P = kWinS + 3;
    __device__ double get(int a, int ds) const { return sm[(a * P + at + ds) * kWinK + kc]; }
    __device__ void put(int a, double v) const { sm[(a * P + at) * kWinK + kc] = v; }
};

// ---------------------------------------------------------------------------
// Remap kinetic-energy correction (rke; Phys::rke, Ctx::dke)
// ---------------------------------------------------------------------------

// delta_ke = 0 before the sweeps (remap.cpp:38-41).
struct RkeZero {
    static constexpr int kMinBlocks = 6;
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, -2, g.nx + 2, -2, g.ny + 2, -2, g.nz + 2);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        if (c.p.rke) c.dke[box_off(c.g, i, j, k)] = 0.0;
    }
};

// Kinetic-energy error of the sweep's three momentum fluxes at each face,
// the dk of x_mom_flux (xremap.cpp:534-558) and its y/z analogues
// (yremap.cpp:557-583, zremap.cpp:513-536), one per velocity component into
// S_FX/S_FY/S_FZ.  Reads the raw fluxes of SweepS7 and the velocities before
// SweepS8 updates them; the post-sweep vertex density is formed as in S8.
template <int DIR>
struct SweepRkeDk {
    static constexpr int kMinBlocks = 4;
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 0, DIR == 0 ? g.nx - 1 : g.nx, 0, DIR == 1 ? g.ny - 1 : g.ny, 0,
                   DIR == 2 ? g.nz - 1 : g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        if (!c.p.rke) return;
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        const int d = dir_stride(g, DIR);
        const int op = o + d, om = o - d;
        const RO rv{c.s[S_R_RVN]}, cvc1{c.s[S_R_CVC1]}, cv2n{c.s[S_R_CV2N]}, dmn{c.s[S_R_DMN]};
        const double rv1o = (rv[o] * cvc1[o] + dmn[om] - dmn[o]) / cv2n[o];
        const double rv1p = (rv[op] * cvc1[op] + dmn[o] - dmn[op]) / cv2n[op];
        const double m = rv1o * cv2n[o];
        const double mp = rv1p * cv2n[op];
        const double dmm = dmn[om], dm0 = dmn[o], dmp = dmn[op];
        const int fluxes[3] = {S_R_FM1, S_R_FM2, S_R_FM3};
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const RO u{c.f[SAMS_F_VX + q]}, fl{c.s[fluxes[q]]};
            const double uo = u[o], up = u[op], flm = fl[om], fl0 = fl[o], flp = fl[op];
            const double ai = (uo - flm) * dmm / m - (uo - fl0) * dm0 / m;
            const double aip = (up - fl0) * dm0 / mp - (up - flp) * dmp / mp;
            double dk = (up - uo) * (fl0 - 0.5 * (up + uo)) - 0.5 * ai * (uo - fl0) + 0.5 * aip * (up - fl0);
            dk = dk * dm0 * 0.5;
            c.s[S_FX + q][o] = dk;
        }
    }
};

// delta_ke gathers the dk of the four faces around each node, for vx, vy and
// vz in turn, adding in the order the reference's loops add them serially
// (source faces in index order).  The reference adds with atomics from
// parallel loops, so its own result is this one only when run on one thread.
template <int DIR>
struct SweepRkeGather {
    static constexpr int kMinBlocks = 6;
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, DIR == 0 ? 1 : 0, DIR == 0 ? g.nx : g.nx + 1, DIR == 1 ? 1 : 0,
                   DIR == 1 ? g.ny : g.ny + 1, DIR == 2 ? 1 : 0, DIR == 2 ? g.nz : g.nz + 1);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        if (!c.p.rke) return;
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        // the two transverse dimensions, lower index first, and their extents
        const int t1 = DIR == 0 ? 1 : 0, t2 = DIR == 2 ? 1 : 2;
        const int q[3] = {i, j, k};
        const int n[3] = {g.nx, g.ny, g.nz};
        const int st[3] = {g.sx, g.sy, 1};
        const int src0 = o - st[DIR];
        double acc = c.dke[o];
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
            const RO dk{c.s[S_FX + comp]};
#pragma unroll
            for (int a = -1; a <= 0; ++a) {
                const int qa = q[t1] + a;
                if (qa < 0 || qa > n[t1]) continue;
#pragma unroll
                for (int b = -1; b <= 0; ++b) {
                    const int qb = q[t2] + b;
                    if (qb < 0 || qb > n[t2]) continue;
                    acc += dk[src0 + a * st[t1] + b * st[t2]];
                }
            }
        }
        c.dke[o] = acc;
    }
};

// energy_correction (diagnostics.cpp:125-135) after the remap's last
// boundary fill; the energies' ghosts are left as that fill set them.
struct RkeEnergy {
    static constexpr int kMinBlocks = 6;
    __host__ __device__ static void bounds(const Geom &g, int, int *lo, int *hi)
    {
        set_bounds(lo, hi, 1, g.nx, 1, g.ny, 1, g.nz);
    }
    template <bool GEO, bool P2>
    __device__ static void run(const Ctx &c, int, int i, int j, int k)
    {
        if (!c.p.rke) return;
        const Geom &g = c.g;
        const int o = LOFF(i, j, k);
        const double d = pmax(-c.dke[o], 0.0) / (__ldg(c.f[SAMS_F_RHO] + o) * cv_at<GEO>(c, i, j, k));
        double *ee = c.f[SAMS_F_ENERGY_ELECTRON], *ei = c.f[SAMS_F_ENERGY_ION];
        ee[o] += 0.5 * d;
        ei[o] += 0.5 * d;
    }
};

#undef LOFF

// Register cap (blocks of 256 per SM) of an op's power-of-two instantiation:
// multiplying by reciprocals instead of calling the division routine lets
// the compiler keep more values live, so these caps were tuned separately
// on B200 (the same sweep as kMinBlocks, on the 256^3 step).
template <class Op>
struct CapP2 {
    static constexpr int value = Op::kMinBlocks;
};
template <>
struct CapP2<NodePrep> {
    static constexpr int value = 5;
};
template <>
struct CapP2<ResistRK> {
    static constexpr int value = 5;
};
template <>
struct CapP2<Pred1> {
    static constexpr int value = 6;
};

// Register cap of an op in the batched engine (lare_batch.cu), whose solves
// are typically thin (n x n x 4): rows of nine doubles, tiles of eight
// planes.  Swept on B200 like kMinBlocks, on the batched step of 64
// Orszag-Tang solves; ops not listed keep kMinBlocks.
template <class Op>
struct CapBatch {
    static constexpr int value = Op::kMinBlocks;
};
template <> struct CapBatch<BScale> { static constexpr int value = 8; };
template <> struct CapBatch<SweepCvc> { static constexpr int value = 8; };
template <> struct CapBatch<Corr2> { static constexpr int value = 5; };
template <int D> struct CapBatch<SweepVol<D>> { static constexpr int value = 4; };
template <int D> struct CapBatch<SweepCTUpd<D>> { static constexpr int value = 8; };
template <int D> struct CapBatch<SweepMass<D>> { static constexpr int value = 4; };
template <int D> struct CapBatch<SweepS7<D>> { static constexpr int value = 4; };
template <int D> struct CapBatch<SweepS8<D>> { static constexpr int value = 8; };

}  // namespace ops

// Blocks-per-SM bound of a kernel running Op.
template <class Op, bool P2>
struct MinBlocks {
    static constexpr int value = P2 ? ops::CapP2<Op>::value : Op::kMinBlocks;
};
template <class Op, bool P2>
struct MinBlocksBatch {
    static constexpr int value = P2 ? ops::CapP2<Op>::value : ops::CapBatch<Op>::value;
};

}  // namespace sams
