// lare_device.cuh -- device-side data layout and point formulas of the
// LARE3D timestep on B200.
//
// Layout: every field is one "box" over indices -2..n+2 per dimension, z
// fastest, with the z row padded so that interior index k = 1 starts on a
// 32-byte boundary (zoff = 3) and rows are a multiple of 8 doubles.  All
// fields share one geometry, so one offset serves every array.
//
// Arithmetic: this translation unit is compiled with --fmad=false and the
// formulas below keep the reference's evaluation order term by term
// (left-to-right sums, the same parenthesisation), so results are identical
// to the reference CPU build with -ffp-contract=off.  Double division and
// sqrt are IEEE round-to-nearest on the GPU as on the CPU.
#pragma once

#include <cfloat>
#include <cstdint>

#include "sams_lare_layout.h"

namespace sams {

struct Geom {
    int nx, ny, nz;
    int sx, sy;        // element strides of i and j (k stride is 1)
    int zoff;          // k + zoff is the position of index k in its row
    long long nelem;   // doubles per field allocation
};

// Host/device helpers for the box geometry.
// Offsets are 32-bit: the 32 arrays of a solve must fit one GPU, so a single
// array holds far fewer than 2^31 elements (checked when a solve is set up).
__host__ __device__ inline int box_off(const Geom &g, int i, int j, int k)
{
    return (i + 2) * g.sx + (j + 2) * g.sy + (k + g.zoff);
}

// The points of a box (-2..n+2 in each dimension) outside the cube
// lo..n+hi in every dimension, one per index t in 0 .. count()-1:
// first the x slabs (whole y-z planes), then the y slabs inside the cube's
// x range, then the z slabs inside its x and y ranges.
struct BoxShell {
    int n[3];
    int lo, hi;
    __host__ __device__ long long ext(int d) const { return (long long)n[d] + 5; }
    __host__ __device__ long long in(int d) const { return (long long)n[d] + hi - lo + 1; }
    // box index of the q-th ghost layer of dimension d (lo+2 below, the rest above)
    __host__ __device__ int ghost(int d, long long q) const
    {
        return q < lo + 2 ? (int)q - 2 : n[d] + hi + 1 + (int)(q - (lo + 2));
    }
    __host__ __device__ long long count() const
    {
        return (ext(0) - in(0)) * ext(1) * ext(2) + in(0) * (ext(1) - in(1)) * ext(2) +
               in(0) * in(1) * (ext(2) - in(2));
    }
    __host__ __device__ void point(long long t, int &i, int &j, int &k) const
    {
        const long long cx = (ext(0) - in(0)) * ext(1) * ext(2);
        if (t < cx) {
            i = ghost(0, t / (ext(1) * ext(2)));
            j = (int)((t / ext(2)) % ext(1)) - 2;
            k = (int)(t % ext(2)) - 2;
            return;
        }
        t -= cx;
        const long long gy = ext(1) - in(1), cy = in(0) * gy * ext(2);
        if (t < cy) {
            i = lo + (int)(t / (gy * ext(2)));
            j = ghost(1, (t / ext(2)) % gy);
            k = (int)(t % ext(2)) - 2;
            return;
        }
        t -= cy;
        const long long gz = ext(2) - in(2);
        i = lo + (int)(t / (in(1) * gz));
        j = lo + (int)((t / gz) % in(1));
        k = ghost(2, t % gz);
    }
};

// Staggering of a field in one dimension (1 = half cell), the device-side
// copy of sams_lare_field_stagger.
__host__ __device__ constexpr int field_half(int f, int d)
{
    return (f >= SAMS_F_VX && f <= SAMS_F_VZ1) ? 1
           : (f == SAMS_F_BX) ? (d == 0)
           : (f == SAMS_F_BY) ? (d == 1)
           : (f == SAMS_F_BZ) ? (d == 2)
           : 0;
}

// 1-D axes (index i at [i + 2]); Cartesian metrics are products of these.
struct Axes {
    const double *dxb, *dyb, *dzb, *dxc, *dyc, *dzc;
};

struct Phys {
    double gamma, mu0, visc1, visc2_norm, dt_multiplier, eta_bg, eta0, j_max;
    int resistive;  // per-solve resistive flag (read by the batched launcher)
    int rke;        // remap kinetic-energy correction on (Ctx::dke allocated)
    int geometry;   // 0 Cartesian, 1 cylindrical, 2 spherical (Ctx::gf set)
    int pow2;       // Cartesian grid whose spacings are all one power of two each (Ctx::rc set)
};

// Reciprocals of the spacings and of the cell volume of a uniform Cartesian
// grid whose spacings are powers of two.  Dividing by a power of two and
// multiplying by its reciprocal give the same correctly rounded result for
// every operand, so kernels built for such grids multiply instead.
struct Recip {
    double xb, yb, zb, xc, yc, zc, cv;
    double mu0;  // 1 / mu0 (mu0 is a power of two too)
};

// Metric factors of a cylindrical or spherical solve, as LARE3D::grid builds
// them (setup.cpp:277-335), computed on the host.  All null in Cartesian
// geometry, where every factor is 1.0 and the kernels skip them.
struct GeomF {
    const double *hy, *hyc, *hyv, *xb;   // per x, index i + 2
    const double *hz, *hz1, *hz2, *hzc;  // per (x, y), index (i + 2) * (ny + 5) + (j + 2)
    const double *cot;                   // 1 / tan(yb) per y, index j + 2
};

// Per-solve device scalars.
struct Scalars {
    double dt;        // timestep of the step in progress (previous step's
                      // value until the CFL reduction has run)
    double dtr;       // LARE's dtr (equals the reduced dt)
    double dt_sub;    // resistive sub-step
    double time;      // simulation time
    unsigned long long dtmin_bits;  // running min of the CFL candidates
    long long step;
    int nsub;         // resistive sub-steps this step
    int status;       // 0 ok, nonzero: non-finite dt seen
};

// LARE uses the same 32 arrays for every solve: the 13 harness variables and
// 19 scratch arrays whose roles change with the phase of the step.
enum ScratchId {
    // Lagrangian phase
    S_CS = 0, S_RHOV, S_CSV, S_A1, S_A2, S_A3, S_VH, S_FXV, S_FYV, S_FZV,
    S_CV1, S_B1X, S_B1Y, S_B1Z, S_PE, S_PI, S_FX, S_FY, S_FZ,
    NSCRATCH
};
// Resistive sub-step aliases (live between the CFL reduction and the
// predictor, when cs, cs_v, cv1 and fx are free; pe holds the cell
// electron pressure from before the Ohmic heating).
#define S_FLUXX S_CS
#define S_FLUXY S_CSV
#define S_FLUXZ S_CV1
#define S_CURLB S_FX
// Remap aliases (the whole Lagrangian scratch is dead by then).
#define S_R_CV1 S_CV1
#define S_R_CV2 S_CS
#define S_R_DB1 S_RHOV
#define S_R_RHO1 S_CSV
#define S_R_CVC1 S_A1
#define S_R_CT1 S_A2
#define S_R_CT2 S_A3
#define S_R_FE1 S_VH
#define S_R_FE2 S_FXV
#define S_R_RVN S_FYV
#define S_R_CV2N S_FZV
#define S_R_DMN S_B1X
#define S_R_V1S S_B1Y
#define S_R_FM1 S_B1Z
#define S_R_FM2 S_PE
#define S_R_FM3 S_PI

struct Ctx {
    Geom g;
    Axes ax;
    Phys p;
    double *f[13];
    double *s[NSCRATCH];
    double *dke;  // delta_ke of the rke correction (null unless Phys::rke)
    GeomF gf;     // metric factors (null in Cartesian geometry)
    Recip rc;     // reciprocals (valid when Phys::pow2)
    Scalars *sc;
};

namespace dev {

constexpr double NONE_ZERO = DBL_EPSILON;  // LARE simulationData::none_zero
constexpr double SIXTH = 1.0 / 6.0;

// An array that no thread of the running kernel writes.  Its loads take the
// read-only (non-coherent) path, so the compiler may move them across the
// kernel's stores to other arrays and keep more of them in flight.
struct RO {
    const double *p;
    __device__ __forceinline__ double operator[](int i) const { return __ldg(p + i); }
};

// x / d, or x * r where the kernel is built for a power-of-two grid (r = 1/d
// exactly; see Recip).
template <bool P2>
__device__ __forceinline__ double div_by(double x, double d, double r)
{
    if constexpr (P2) {
        (void)d;
        return x * r;
    } else {
        (void)r;
        return x / d;
    }
}

// portableWrapper min/max semantics (include/pp/utils.h:277-335).
__device__ __forceinline__ double pmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double pmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double pmin_list3(double a, double b, double c)
{
    double m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    return m;
}
__device__ __forceinline__ double pmin_list4(double a, double b, double c, double d)
{
    double m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    if (d < m) m = d;
    return m;
}

// Da, ss and Di of the van Leer limiter written in every remap flux function
// (e.g. xremap.cpp:309-314).
__device__ __forceinline__ double limiter_Di(double sign_v, double phi, double dfi, double dfu,
                                             double dxci, double dxcu, double dxbu)
{
    double Da = (2.0 - phi) * fabs(dfi) / dxci + (1.0 + phi) * fabs(dfu) / dxcu;
    Da = Da * SIXTH;
    double ss = 0.5 * ((dfi >= 0.0 ? 1.0 : -1.0) + (dfu >= 0.0 ? 1.0 : -1.0));
    return sign_v * ss * pmin_list3(fabs(Da) * dxbu, fabs(dfi), fabs(dfu));
}

// Evans-Hawley constrained-transport flux of a transverse face field
// (vx_by_flux xremap.cpp:269-319 and the five analogues in x/y/zremap.cpp).
// With the four quotients b/db along the sweep given (fm = bm / dbm, ...):
// each is the same value at its point for every flux that reads it, so a
// kernel can form it once per point.
__device__ __forceinline__ double ct_flux_q(double v_advect, double dt, double fm, double fi, double fp, double fp2,
                                            double dbi, double dbp, double dci, double dcm, double dcp,
                                            double cv1i, double cv1p)
{
    double o_v = v_advect * dt;
    double dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
    double sign_v = (v_advect >= 0.0) ? 1.0 : -1.0;
    double vad_p = (sign_v + 1.0) * 0.5;
    double vad_m = 1.0 - vad_p;
    double fu = fi * vad_p + fp * vad_m;
    double dfu = dfm * vad_p + dfp * vad_m;
    double dxcu = dcm * vad_p + dcp * vad_m;
    double dxbu = cv1i * vad_p + cv1p * vad_m;
    double dxu = dbi * vad_p + dbp * vad_m;
    double phi = fabs(o_v) / dxu;
    double Di = limiter_Di(sign_v, phi, dfi, dfu, dci, dxcu, dxbu);
    return (fu + Di * (1.0 - phi)) * o_v;
}

__device__ __forceinline__ double ct_flux(double v_advect, double dt, double bm, double bi, double bp,
                                          double bp2, double dbm, double dbi, double dbp, double dbp2,
                                          double dci, double dcm, double dcp, double cv1i, double cv1p)
{
    double o_v = v_advect * dt;
    double fm = bm / dbm, fi = bi / dbi, fp = bp / dbp, fp2 = bp2 / dbp2;
    double dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
    double sign_v = (v_advect >= 0.0) ? 1.0 : -1.0;
    double vad_p = (sign_v + 1.0) * 0.5;
    double vad_m = 1.0 - vad_p;
    double fu = fi * vad_p + fp * vad_m;
    double dfu = dfm * vad_p + dfp * vad_m;
    double dxcu = dcm * vad_p + dcp * vad_m;
    double dxbu = cv1i * vad_p + cv1p * vad_m;
    double dxu = dbi * vad_p + dbp * vad_m;
    double phi = fabs(o_v) / dxu;
    double Di = limiter_Di(sign_v, phi, dfi, dfu, dci, dxcu, dxbu);
    return (fu + Di * (1.0 - phi)) * o_v;
}

// Mass flux through a face (x_mass_flux xremap.cpp:373-422 and analogues).
__device__ __forceinline__ double mass_flux(double v_advect, double dt, double area, double fm, double fi,
                                            double fp, double fp2, double dci, double dcm, double dcp,
                                            double cv1i, double cv1p)
{
    double o_v = v_advect * dt * area;
    double dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
    double sign_v = (v_advect >= 0.0) ? 1.0 : -1.0;
    double vad_p = (sign_v + 1.0) * 0.5;
    double vad_m = 1.0 - vad_p;
    double fu = fi * vad_p + fp * vad_m;
    double dfu = dfm * vad_p + dfp * vad_m;
    double dxcu = dcm * vad_p + dcp * vad_m;
    double dxbu = cv1i * vad_p + cv1p * vad_m;
    double phi = fabs(o_v) / dxbu;
    double Di = limiter_Di(sign_v, phi, dfi, dfu, dci, dxcu, dxbu);
    return (fu + Di * (1.0 - phi)) * o_v;
}

// Specific-energy flux (x_energy_flux xremap.cpp:429-483 and analogues).
__device__ __forceinline__ double energy_flux(double v_advect, double dt, double area, double fm, double fi,
                                              double fp, double fp2, double dci, double dcm, double dcp,
                                              double cv1i, double cv1p, double rho1i, double rho1p, double dm)
{
    double o_v = v_advect * dt * area;
    double dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
    double sign_v = (v_advect >= 0.0) ? 1.0 : -1.0;
    double vad_p = (sign_v + 1.0) * 0.5;
    double vad_m = 1.0 - vad_p;
    double fu = fi * vad_p + fp * vad_m;
    double dfu = dfm * vad_p + dfp * vad_m;
    double dxcu = dcm * vad_p + dcp * vad_m;
    double dxbu = cv1i * vad_p + cv1p * vad_m;
    double phi = fabs(o_v) / dxbu;
    double Di = limiter_Di(sign_v, phi, dfi, dfu, dci, dxcu, dxbu);
    double rhou = rho1i * vad_p + rho1p * vad_m;
    double dmu = fabs(dm) / dxbu / rhou;
    return (fu + Di * (1.0 - dmu)) * dm;
}

// Momentum flux before its product with dm (x_mom_flux xremap.cpp:485-566
// and analogues; the z sweep divides |dm| by (dzbu * rhou) in one step,
// zremap.cpp:509).
template <bool ZFORM>
__device__ __forceinline__ double mom_flux(double v_advect, double dt, double area, double fm, double fi,
                                           double fp, double fp2, double dci, double dcm, double dcp,
                                           double cvci, double cvcp, double rvi, double rvp, double dm)
{
    double o_v = v_advect * dt * area;
    double dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
    double sign_v = (o_v >= 0.0) ? 1.0 : -1.0;
    double vad_p = (sign_v + 1.0) * 0.5;
    double vad_m = 1.0 - vad_p;
    double fu = fi * vad_p + fp * vad_m;
    double dfu = dfm * vad_p + dfp * vad_m;
    double dxcu = dcm * vad_p + dcp * vad_m;
    double dxbu = cvci * vad_p + cvcp * vad_m;
    double phi = fabs(o_v) / dxbu;
    double Di = limiter_Di(sign_v, phi, dfi, dfu, dci, dxcu, dxbu);
    double rhou = rvi * vad_p + rvp * vad_m;
    double dmu = ZFORM ? fabs(dm) / (dxbu * rhou) : fabs(dm) / dxbu / rhou;
    return fu + Di * (1.0 - dmu);
}

// Caramana edge viscosity (lagran.cpp:56-93).  v[a] are the four points
// along the edge direction, o1/o2 the edge ends.
template <bool P2, class A>
__device__ __forceinline__ double edge_viscosity(double dt, double visc1, double v2n, const A &vx,
                                                 const A &vy, const A &vz, const A &rho_v,
                                                 double dvdots, double dx, double dxm, double dxp,
                                                 double cs_edge, int o0, int o1, int o2, int o3, double rdx = 0.0)
{
    dvdots = pmin(0.0, dvdots);
    double rv1 = rho_v[o1], rv2 = rho_v[o2];
    double rho_edge = 2.0 * rv1 * rv2 / (rv1 + rv2);
    double vx1 = vx[o1], vx2 = vx[o2], vy1 = vy[o1], vy2 = vy[o2], vz1 = vz[o1], vz2 = vz[o2];
    double dvx = vx1 - vx2, dvy = vy1 - vy2, dvz = vz1 - vz2;
    double dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
    double dv = sqrt(dv2);
    bool small = div_by<P2>(dv * dt, dx, rdx) < 1.e-14;
    dvdots = small ? 0.0 : dvdots / dv;
    double dvxm = vx[o0] - vx1, dvxp = vx2 - vx[o3];
    double dvym = vy[o0] - vy1, dvyp = vy2 - vy[o3];
    double dvzm = vz[o0] - vz1, dvzp = vz2 - vz[o3];
    double rl = small ? 1.0 : (dvxp * dvx + dvyp * dvy + dvzp * dvz) * dx / (dxp * dv2);
    double rr = small ? 1.0 : (dvxm * dvx + dvym * dvy + dvzm * dvz) * dx / (dxm * dv2);
    double psi = pmin_list4(0.5 * (rr + rl), 2.0 * rl, 2.0 * rr, 1.0);
    psi = pmax(0.0, psi);
    double q_k_bar = rho_edge * (v2n * dv + sqrt(v2n * v2n * dv2 + (visc1 * cs_edge) * (visc1 * cs_edge)));
    return q_k_bar * (1.0 - psi) * dvdots;
}

}  // namespace dev
}  // namespace sams
