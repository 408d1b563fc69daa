/*
 * lare_oracle.c -- CPU restatement of the reference LARE3D timestep.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): the product never links, loads or
 * calls this file.  Every loop below restates one reference kernel with the
 * same index range and the same floating-point expression order, so that
 * built with -ffp-contract=off it reproduces the reference bit for bit.
 * Reference locations are cited per function (paths relative to the
 * reference project root).
 *
 * Geometry: Cartesian, cylindrical and spherical.  The metric factors hy,
 * hyc, hyv (per x) and hz, hz1, hz2, hzc (per x and y) are built as
 * LARE3D::grid builds them (setup.cpp:260-335); in Cartesian geometry they
 * are 1.0 and multiplying or dividing by them changes nothing.  The
 * Lagrangian position arrays x, y, z are diagnostics (never read by the
 * physics) and are not kept.  The second rkstep of resistive_effects (lagran.cpp:504) writes only
 * flux_x/y/z and curlb, which nothing reads before they are recomputed, so it
 * is not repeated.
 */
#include "lare_oracle.h"
#include "sams_lare_bc_other.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

struct lo_state {
    sams_lare_params p;
    sams_lare_bcs bcs;
    int64_t nx, ny, nz, nbox;
    double *f[SAMS_NFIELDS];
    /* metrics (setup.cpp:260-390) */
    double *cv, *cvc, *dxab, *dyab, *dzab, *dxac, *dyac, *dzac;
    /* axes, index i at [i + 2] */
    double *xb, *yb, *zb, *xc, *yc, *zc, *dxb, *dyb, *dzb, *dxc, *dyc, *dzc;
    /* Lagrangian intermediates (shared_data.h:194-216) */
    double *p_visc, *visc_heat, *alpha1, *alpha2, *alpha3, *pressure, *p_e, *p_i;
    double *rho_v, *cv_v, *fx, *fy, *fz, *fx_visc, *fy_visc, *fz_visc;
    double *bx1, *by1, *bz1, *cv1, *eta, *flux_x, *flux_y, *flux_z, *curlb;
    double *cs, *cs_v;
    /* remap temporaries (remapData.h:23-32) */
    double *rho1, *cv2, *cvc1, *db1, *r_rho_v, *rho_v1, *flux;
    double *delta_ke; /* remap kinetic-energy correction (rke only, setup.cpp:251) */
    /* geometry factors (setup.cpp:277-335): per x at [x + 2], per (x, y) at H2 */
    double *hy, *hyc, *hyv, *hz, *hz1, *hz2, *hzc, *cot_yb;
    double dt, dtr, time, visc2_norm;
    int64_t step;
    double xpass, ypass, zpass;
};

#define DIMS(s)                                                   \
    const int64_t nx = (s)->nx, ny = (s)->ny, nz = (s)->nz;       \
    const int64_t sy = ny + 5, sz = nz + 5;                       \
    (void)nx; (void)ny; (void)nz; (void)sy; (void)sz
#define I3(i, j, k) ((((int64_t)(i) + 2) * sy + ((int64_t)(j) + 2)) * sz + ((int64_t)(k) + 2))
#define A1(i) ((int64_t)(i) + 2)
#define H2(i, j) (((int64_t)(i) + 2) * sy + ((int64_t)(j) + 2))

#define LOOP3(ilo, ihi, jlo, jhi, klo, khi)                        \
    _Pragma("omp parallel for schedule(static)")                   \
    for (int64_t ix = (ilo); ix <= (ihi); ++ix)                    \
        for (int64_t iy = (jlo); iy <= (jhi); ++iy)                \
            for (int64_t iz = (klo); iz <= (khi); ++iz)

/* include/pp/utils.h:277-335 */
static inline double pmin(double a, double b) { return a < b ? a : b; }
static inline double pmax(double a, double b) { return a > b ? a : b; }
static inline double pmin_list3(double a, double b, double c)
{
    double m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    return m;
}
static inline double pmin_list4(double a, double b, double c, double d)
{
    double m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    if (d < m) m = d;
    return m;
}

static const double NONE_ZERO = DBL_EPSILON;   /* shared_data.h:92 */
static const double SIXTH = 1.0 / 6.0;         /* constants.h:46 */

/* ------------------------------------------------------------------ */
/* Boundary conditions: variableDef::applyBoundaryConditions order      */
/* (include/harness/variableDef.h:539-605) with the built-in conditions */
/* of include/boundaryConditions/builtInBoundaryConditions.h.           */
/* ------------------------------------------------------------------ */

static void bc_apply_edge(lo_state *s, int f, int d, int e)
{
    DIMS(s);
    const int kind = s->bcs.kind[f][d][e];
    if (kind == SAMS_BC_NONE) return;
    double *A = s->f[f];
    const int64_t n[3] = {nx, ny, nz};
    const int st = sams_lare_field_stagger[f][d];
    /* local ranges of the field in all dims */
    int64_t lo[3], hi[3];
    for (int q = 0; q < 3; ++q) {
        lo[q] = sams_lare_field_lb(f, q);
        hi[q] = n[q] + 2;
    }
    if (kind == SAMS_BC_LARE_OTHER) {
        /* LARE BC_OTHER (src/InitialConditions/LARE/boundary.cpp): whole-plane
         * copies or zeroed planes, one pw::assign after another */
        int32_t dst[3], src[3];
        const int np = sams_lare_other_planes(f, d, e, n[d], dst, src);
        for (int q = 0; q < np; ++q) {
            int64_t a[3] = {lo[0], lo[1], lo[2]}, b[3] = {hi[0], hi[1], hi[2]};
            a[d] = b[d] = dst[q];
            for (int64_t i = a[0]; i <= b[0]; ++i)
                for (int64_t j = a[1]; j <= b[1]; ++j)
                    for (int64_t k = a[2]; k <= b[2]; ++k) {
                        int64_t p3[3] = {i, j, k};
                        p3[d] = src[q];
                        A[I3(i, j, k)] = src[q] == SAMS_PLANE_ZERO ? 0.0 : A[I3(p3[0], p3[1], p3[2])];
                    }
        }
        return;
    }
    const int64_t dlb = st ? 0 : 1, dub = n[d];                 /* domain   */
    const int64_t glo = e == 0 ? lo[d] : (st ? n[d] : n[d] + 1); /* ghosts   */
    const int64_t ghi = e == 0 ? 0 : n[d] + 2;
    const int64_t cnt = ghi - glo + 1;
    lo[d] = glo;
    hi[d] = ghi;
    for (int64_t i = lo[0]; i <= hi[0]; ++i)
        for (int64_t j = lo[1]; j <= hi[1]; ++j)
            for (int64_t k = lo[2]; k <= hi[2]; ++k) {
                int64_t idx[3] = {i, j, k};
                int64_t g = idx[d];
                int64_t src[3] = {i, j, k};
                double v;
                switch (kind) {
                case SAMS_BC_PERIODIC: /* :252-300 */
                    src[d] = e == 0 ? dub - cnt + 1 + (g - glo) : dlb + (g - glo);
                    v = A[I3(src[0], src[1], src[2])];
                    break;
                case SAMS_BC_ZERO_GRADIENT: /* :200-249 */
                    src[d] = e == 0 ? dlb : dub;
                    v = A[I3(src[0], src[1], src[2])];
                    break;
                case SAMS_BC_MIRROR: { /* :96-171 */
                    int64_t last = e == 0 ? dlb : dub;
                    int64_t first = e == 0 ? ghi : glo;
                    int64_t lt[3] = {i, j, k};
                    lt[d] = last;
                    double a = A[I3(lt[0], lt[1], lt[2])];
                    double bv = (a + a) / 2.0;
                    src[d] = last - (g - first);
                    double delta = A[I3(src[0], src[1], src[2])] - bv;
                    v = bv - delta;
                    break;
                }
                case SAMS_BC_CLAMP: /* :55-83 */
                    v = s->bcs.value[f][d][e];
                    break;
                default:
                    continue;
                }
                A[I3(i, j, k)] = v;
            }
}

static void bc_dim(lo_state *s, int f, int d)
{
    bc_apply_edge(s, f, d, 0);
    bc_apply_edge(s, f, d, 1);
}

static void bc_field(lo_state *s, int f)
{
    for (int d = 0; d < 3; ++d) bc_dim(s, f, d);
}

/* boundary.cpp:27-97 */
static void bfield_bcs(lo_state *s) { bc_field(s, SAMS_F_BX); bc_field(s, SAMS_F_BY); bc_field(s, SAMS_F_BZ); }
static void energy_bcs(lo_state *s) { bc_field(s, SAMS_F_ENERGY_ELECTRON); bc_field(s, SAMS_F_ENERGY_ION); }
static void density_bcs(lo_state *s) { bc_field(s, SAMS_F_RHO); }
static void velocity_bcs(lo_state *s) { bc_field(s, SAMS_F_VX); bc_field(s, SAMS_F_VY); bc_field(s, SAMS_F_VZ); }
static void remap_v_bcs(lo_state *s) { bc_field(s, SAMS_F_VX1); bc_field(s, SAMS_F_VY1); bc_field(s, SAMS_F_VZ1); }
static void boundary_conditions(lo_state *s)
{
    bfield_bcs(s);
    energy_bcs(s);
    density_bcs(s);
    velocity_bcs(s);
}

/* ------------------------------------------------------------------ */
/* Grid: axisRegistry (axisRegistry.h:134-200, 393-430, 973-985) and    */
/* LARE3D::grid (setup.cpp:260-390), Cartesian.                         */
/* ------------------------------------------------------------------ */

static void build_axis(double lo, double hi, int64_t n, double *b, double *c, double *db, double *dc)
{
    double d = (hi - lo) / (double)n;
    for (int64_t i = -2; i <= n + 2; ++i) b[A1(i)] = lo + d * (double)i;
    for (int64_t i = -1; i <= n + 2; ++i) c[A1(i)] = 0.5 * (b[A1(i)] + b[A1(i - 1)]);
    for (int64_t i = -1; i <= n + 2; ++i) db[A1(i)] = b[A1(i)] - b[A1(i - 1)];
    db[A1(-2)] = db[A1(-1)]; /* non-periodic axis: first delta = next */
    for (int64_t i = 0; i <= n + 2; ++i) dc[A1(i)] = c[A1(i)] - c[A1(i - 1)];
    dc[A1(-1)] = dc[A1(0)];
    c[A1(-2)] = 0.0;
    dc[A1(-2)] = 0.0;
}

static void build_grid(lo_state *s)
{
    DIMS(s);
    build_axis(s->p.x_min, s->p.x_max, nx, s->xb, s->xc, s->dxb, s->dxc);
    build_axis(s->p.y_min, s->p.y_max, ny, s->yb, s->yc, s->dyb, s->dyc);
    build_axis(s->p.z_min, s->p.z_max, nz, s->zb, s->zc, s->dzb, s->dzc);
    const double *dxb = s->dxb, *dyb = s->dyb, *dzb = s->dzb, *dzc = s->dzc, *dyc = s->dyc;
    double *hy = s->hy, *hyc = s->hyc, *hyv = s->hyv, *hz = s->hz, *hz1 = s->hz1, *hz2 = s->hz2, *hzc = s->hzc;
    const int geo = s->p.geometry;
    /* setup.cpp:277-292; LARE::none_zero = DBL_MIN (constants.h:43) */
    for (int64_t ix = -2; ix <= nx + 2; ++ix) {
        if (geo == 0) {
            hy[A1(ix)] = hyc[A1(ix)] = hyv[A1(ix)] = 1.0;
        } else {
            hy[A1(ix)] = fabs(s->xb[A1(ix)]);
            hyc[A1(ix)] = fabs(s->xc[A1(ix)]);
            hyv[A1(ix)] = (fabs(s->xc[A1(0)]) < DBL_MIN && ix == 1) ? fabs(s->xc[A1(ix)]) : 0.25 * fabs(s->xc[A1(ix)]);
        }
    }
    /* setup.cpp:294-334 */
    for (int64_t ix = -2; ix <= nx + 2; ++ix)
        for (int64_t iy = -2; iy <= ny + 2; ++iy)
            hz[H2(ix, iy)] = hz1[H2(ix, iy)] = hz2[H2(ix, iy)] = hzc[H2(ix, iy)] = 1.0;
    if (geo == 2) {
        for (int64_t iy = -2; iy <= ny + 2; ++iy) {
            double sn = fabs(sin(s->yb[A1(iy)]));
            hz[H2(-2, iy)] = hy[A1(-2)] * sn;
            for (int64_t ix = -1; ix <= nx + 2; ++ix) {
                hz[H2(ix, iy)] = hy[A1(ix)] * sn;
                hz2[H2(ix, iy)] = hyc[A1(ix)] * sn;
            }
        }
        for (int64_t iy = -1; iy <= ny + 2; ++iy) {
            double sc = fabs(sin(s->yc[A1(iy)]));
            hz1[H2(-2, iy)] = hy[A1(-2)] * sc;
            for (int64_t ix = -1; ix <= nx + 2; ++ix) {
                hz1[H2(ix, iy)] = hy[A1(ix)] * sc;
                hzc[H2(ix, iy)] = hyc[A1(ix)] * sc;
            }
        }
    }
    /* 1/tan(yb) of the spherical force terms (lagran.cpp:713) */
    for (int64_t iy = -2; iy <= ny + 2; ++iy) s->cot_yb[A1(iy)] = geo == 2 ? 1.0 / tan(s->yb[A1(iy)]) : 0.0;
    /* cell-centred areas and volumes (setup.cpp:337-354) */
    for (int64_t iy = -1; iy <= ny + 2; ++iy)
        for (int64_t iz = -1; iz <= nz + 2; ++iz) {
            double dy = dyb[A1(iy)], dz = dzb[A1(iz)], dydz = dy * dz;
            s->dxab[I3(-2, iy, iz)] = dydz * hy[A1(-2)] * hz1[H2(-2, iy)];
            for (int64_t ix = -1; ix <= nx + 2; ++ix) {
                double dx = dxb[A1(ix)];
                s->dxab[I3(ix, iy, iz)] = dydz * hy[A1(ix)] * hz1[H2(ix, iy)];
                s->dyab[I3(ix, iy, iz)] = dx * dz * hz2[H2(ix, iy)];
                s->dzab[I3(ix, iy, iz)] = dx * dy * hy[A1(ix)];
                s->cv[I3(ix, iy, iz)] = dx * dydz * hyc[A1(ix)] * hzc[H2(ix, iy)];
            }
        }
    /* negative y and z boundaries (setup.cpp:356-374; the dzab(-2) pass with
     * dyc is overwritten by the one with dyb) */
    for (int64_t ix = -1; ix <= nx + 2; ++ix)
        for (int64_t iz = -1; iz <= nz + 2; ++iz)
            s->dyab[I3(ix, -2, iz)] = dxb[A1(ix)] * dzb[A1(iz)] * hz2[H2(ix, -2)];
    (void)dyc;
    for (int64_t ix = -1; ix <= nx + 2; ++ix)
        for (int64_t iy = -1; iy <= ny + 2; ++iy)
            s->dzab[I3(ix, iy, -2)] = dxb[A1(ix)] * dyb[A1(iy)] * hyc[A1(ix)];
    /* node-centred areas and volumes (setup.cpp:375-390) */
    for (int64_t ix = -1; ix <= nx + 2; ++ix)
        for (int64_t iy = -1; iy <= ny + 2; ++iy)
            for (int64_t iz = -1; iz <= nz + 2; ++iz) {
                double dx = dxb[A1(ix)], dy = dyb[A1(iy)], dz = dzc[A1(iz)];
                double dydz = dy * dz;
                s->dxac[I3(ix, iy, iz)] = dydz * hyc[A1(ix)] * hz2[H2(ix, iy)];
                s->dyac[I3(ix, iy, iz)] = dx * dz * hz1[H2(ix, iy)];
                s->dzac[I3(ix, iy, iz)] = dx * dy * hy[A1(ix)];
                s->cvc[I3(ix, iy, iz)] = dx * dydz * hyv[A1(ix)] * hz[H2(ix, iy)];
            }
}

/* ------------------------------------------------------------------ */
/* Lagrangian step (lagran.cpp)                                        */
/* ------------------------------------------------------------------ */

/* lagran.cpp:56-93 */
static inline double edge_viscosity(const lo_state *s, const double *vx, const double *vy,
                                    const double *vz, const double *rho_v, double dvdots,
                                    double dx, double dxm, double dxp, double cs_edge,
                                    int64_t o0, int64_t o1, int64_t o2, int64_t o3)
{
    dvdots = pmin(0.0, dvdots);
    double rho_edge = 2.0 * rho_v[o1] * rho_v[o2] / (rho_v[o1] + rho_v[o2]);
    double dvx = vx[o1] - vx[o2];
    double dvy = vy[o1] - vy[o2];
    double dvz = vz[o1] - vz[o2];
    double dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
    double dv = sqrt(dv2);
    double psi;
    int small = dv * s->dt / dx < 1.e-14;
    dvdots = small ? 0.0 : dvdots / dv;
    double dvxm = vx[o0] - vx[o1];
    double dvxp = vx[o2] - vx[o3];
    double dvym = vy[o0] - vy[o1];
    double dvyp = vy[o2] - vy[o3];
    double dvzm = vz[o0] - vz[o1];
    double dvzp = vz[o2] - vz[o3];
    double rl = small ? 1.0 : (dvxp * dvx + dvyp * dvy + dvzp * dvz) * dx / (dxp * dv2);
    double rr = small ? 1.0 : (dvxm * dvx + dvym * dvy + dvzm * dvz) * dx / (dxm * dv2);
    psi = pmin_list4(0.5 * (rr + rl), 2.0 * rl, 2.0 * rr, 1.0);
    psi = pmax(0.0, psi);
    double v2n = s->visc2_norm, v1 = s->p.visc1;
    double q_k_bar = rho_edge * (v2n * dv + sqrt(v2n * v2n * dv2 + (v1 * cs_edge) * (v1 * cs_edge)));
    return q_k_bar * (1.0 - psi) * dvdots;
}

#define SQ(a) ((a) * (a))

/* lagran.cpp:175-378 */
static void shock_viscosity(lo_state *s)
{
    DIMS(s);
    const double g = s->p.gas_gamma;
    s->visc2_norm = 0.25 * (g + 1.0) * s->p.visc2;
    double *vx = s->f[SAMS_F_VX], *vy = s->f[SAMS_F_VY], *vz = s->f[SAMS_F_VZ];
    double *rho = s->f[SAMS_F_RHO];
    double *cs = s->cs, *cs_v = s->cs_v, *cv = s->cv, *cv_v = s->cv_v, *rho_v = s->rho_v;
    double *a1a = s->alpha1, *a2a = s->alpha2, *a3a = s->alpha3;
    double *bx1 = s->bx1, *by1 = s->by1, *bz1 = s->bz1, *pressure = s->pressure;
    const double *dxb = s->dxb, *dyb = s->dyb, *dzb = s->dzb;

    for (int64_t o = 0; o < s->nbox; ++o) { s->p_visc[o] = 0.0; s->visc_heat[o] = 0.0; }

    LOOP3(-1, nx + 2, -1, ny + 2, -1, nz + 2)
    {
        double rmin = pmax(rho[I3(ix, iy, iz)], NONE_ZERO);
        double b2 = bx1[I3(ix, iy, iz)] * bx1[I3(ix, iy, iz)] +
                    by1[I3(ix, iy, iz)] * by1[I3(ix, iy, iz)] +
                    bz1[I3(ix, iy, iz)] * bz1[I3(ix, iy, iz)];
        double p = pressure[I3(ix, iy, iz)];
        cs[I3(ix, iy, iz)] = sqrt((g * p + b2) / rmin);
    }
    LOOP3(-1, nx + 1, -1, ny + 1, -1, nz + 1)
    {
        int64_t ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
        double sum = cs[I3(ix, iy, iz)] * cv[I3(ix, iy, iz)] +
                     cs[I3(ixp, iy, iz)] * cv[I3(ixp, iy, iz)] +
                     cs[I3(ix, iyp, iz)] * cv[I3(ix, iyp, iz)] +
                     cs[I3(ixp, iyp, iz)] * cv[I3(ixp, iyp, iz)] +
                     cs[I3(ix, iy, izp)] * cv[I3(ix, iy, izp)] +
                     cs[I3(ixp, iy, izp)] * cv[I3(ixp, iy, izp)] +
                     cs[I3(ix, iyp, izp)] * cv[I3(ix, iyp, izp)] +
                     cs[I3(ixp, iyp, izp)] * cv[I3(ixp, iyp, izp)];
        cs_v[I3(ix, iy, iz)] = 0.125 * sum / cv_v[I3(ix, iy, iz)];
    }
    /* alpha1 */
    LOOP3(0, nx + 1, 0, ny + 2, 0, nz + 2)
    {
        int64_t i1 = ix - 1, j1 = iy - 1, k1 = iz - 1;
        int64_t i2 = ix, j2 = iy - 1, k2 = iz - 1;
        int64_t o1 = I3(i1, j1, k1), o2 = I3(i2, j2, k2);
        int64_t o0 = I3(i1 - 1, j1, k1), o3 = I3(i2 + 1, j2, k2);
        double dx = dxb[A1(ix)], dxp = dxb[A1(ix + 1)], dxm = dxb[A1(ix - 1)];
        double dvdots = -(vx[o1] - vx[o2]);
        double cs_edge = pmin(cs_v[o1], cs_v[o2]);
        a1a[I3(ix, iy, iz)] = edge_viscosity(s, vx, vy, vz, rho_v, dvdots, dx, dxm, dxp, cs_edge, o0, o1, o2, o3);
    }
    /* alpha2 */
    LOOP3(-1, nx + 1, 0, ny + 1, 0, nz + 2)
    {
        int64_t o1 = I3(ix, iy - 1, iz - 1), o2 = I3(ix, iy, iz - 1);
        int64_t o0 = I3(ix, iy - 2, iz - 1), o3 = I3(ix, iy + 1, iz - 1);
        const double h = s->hy[A1(ix)];
        double dx = dyb[A1(iy)] * h, dxp = dyb[A1(iy + 1)] * h, dxm = dyb[A1(iy - 1)] * h;
        double dvdots = -(vy[o1] - vy[o2]);
        double cs_edge = pmin(cs_v[o1], cs_v[o2]);
        a2a[I3(ix, iy, iz)] = edge_viscosity(s, vx, vy, vz, rho_v, dvdots, dx, dxm, dxp, cs_edge, o0, o1, o2, o3);
    }
    /* alpha3 */
    LOOP3(-1, nx + 1, -1, ny + 1, 0, nz + 1)
    {
        int64_t o1 = I3(ix, iy, iz - 1), o2 = I3(ix, iy, iz);
        int64_t o0 = I3(ix, iy, iz - 2), o3 = I3(ix, iy, iz + 1);
        const double h = s->hz[H2(ix, iy)];
        double dx = dzb[A1(iz)] * h, dxp = dzb[A1(iz + 1)] * h, dxm = dzb[A1(iz - 1)] * h;
        double dvdots = -(vz[o1] - vz[o2]);
        double cs_edge = pmin(cs_v[o1], cs_v[o2]);
        a3a[I3(ix, iy, iz)] = edge_viscosity(s, vx, vy, vz, rho_v, dvdots, dx, dxm, dxp, cs_edge, o0, o1, o2, o3);
    }
    /* p_visc and visc_heat */
    double *p_visc = s->p_visc, *visc_heat = s->visc_heat;
    LOOP3(0, nx + 1, 0, ny + 1, 0, nz + 1)
    {
        int64_t izm = iz - 1, izp = iz + 1, iym = iy - 1, iyp = iy + 1, ixm = ix - 1;
#define DV2(a, b) (SQ(vx[a] - vx[b]) + SQ(vy[a] - vy[b]) + SQ(vz[a] - vz[b]))
        double a1 = DV2(I3(ixm, iym, izm), I3(ix, iym, izm));
        double a2 = DV2(I3(ix, iym, izm), I3(ix, iy, izm));
        double a3 = DV2(I3(ix, iy, izm), I3(ixm, iy, izm));
        double a4 = DV2(I3(ixm, iy, izm), I3(ixm, iym, izm));
        double a5 = DV2(I3(ixm, iym, iz), I3(ix, iym, iz));
        double a6 = DV2(I3(ix, iym, iz), I3(ix, iy, iz));
        double a7 = DV2(I3(ix, iy, iz), I3(ixm, iy, iz));
        double a8 = DV2(I3(ixm, iy, iz), I3(ixm, iym, iz));
        double a9 = DV2(I3(ix, iy, izm), I3(ix, iy, iz));
        double a10 = DV2(I3(ixm, iy, izm), I3(ixm, iy, iz));
        double a11 = DV2(I3(ixm, iym, izm), I3(ixm, iym, iz));
        double a12 = DV2(I3(ix, iym, izm), I3(ix, iym, iz));
#undef DV2
        int64_t o = I3(ix, iy, iz);
        p_visc[o] = pmax(p_visc[o], -a1a[o] * sqrt(a1));
        p_visc[o] = pmax(p_visc[o], -a2a[o] * sqrt(a2));
        p_visc[o] = pmax(p_visc[o], -a3a[o] * sqrt(a9));
        double dx = dxb[A1(ix)], dy = dyb[A1(iy)] * s->hyc[A1(ix)], dz = dzb[A1(iz)] * s->hz2[H2(ix, iy)];
        visc_heat[o] =
            -0.25 * dy * dz * a1a[I3(ix, iy, iz)] * a1
            - 0.25 * dx * dz * a2a[I3(ix, iy, iz)] * a2
            - 0.25 * dy * dz * a1a[I3(ix, iyp, iz)] * a3
            - 0.25 * dx * dz * a2a[I3(ixm, iy, iz)] * a4
            - 0.25 * dy * dz * a1a[I3(ix, iy, izp)] * a5
            - 0.25 * dx * dz * a2a[I3(ix, iy, izp)] * a6
            - 0.25 * dy * dz * a1a[I3(ix, iyp, izp)] * a7
            - 0.25 * dx * dz * a2a[I3(ixm, iy, izp)] * a8
            - 0.25 * dx * dy * a3a[I3(ix, iy, iz)] * a9
            - 0.25 * dx * dy * a3a[I3(ixm, iy, iz)] * a10
            - 0.25 * dx * dy * a3a[I3(ixm, iym, iz)] * a11
            - 0.25 * dx * dy * a3a[I3(ix, iym, iz)] * a12;
        visc_heat[o] = visc_heat[o] / cv[o];
    }
    /* viscous forces */
    double *fxv = s->fx_visc, *fyv = s->fy_visc, *fzv = s->fz_visc;
    LOOP3(0, nx, 0, ny, 0, nz)
    {
        int64_t izm = iz - 1, izp = iz + 1, iym = iy - 1, iyp = iy + 1, ixm = ix - 1, ixp = ix + 1;
        double dx = dxb[A1(ix)], dy = dyb[A1(iy)] * s->hyc[A1(ix)], dz = dzb[A1(iz)] * s->hz2[H2(ix, iy)];
        double a1 = a1a[I3(ix, iyp, izp)] * dy * dz;
        double a2 = a1a[I3(ixp, iyp, izp)] * dy * dz;
        double a3 = a2a[I3(ix, iy, izp)] * dx * dz;
        double a4 = a2a[I3(ix, iyp, izp)] * dx * dz;
        double a5 = a3a[I3(ix, iy, iz)] * dx * dy;
        double a6 = a3a[I3(ix, iy, izp)] * dx * dy;
        int64_t o = I3(ix, iy, iz);
#define FV(v) ((a1 * (v[o] - v[I3(ixm, iy, iz)]) + a2 * (v[o] - v[I3(ixp, iy, iz)]) + \
                a3 * (v[o] - v[I3(ix, iym, iz)]) + a4 * (v[o] - v[I3(ix, iyp, iz)]) + \
                a5 * (v[o] - v[I3(ix, iy, izm)]) + a6 * (v[o] - v[I3(ix, iy, izp)])) / cv_v[o])
        fxv[o] = FV(vx);
        fyv[o] = FV(vy);
        fzv[o] = FV(vz);
#undef FV
    }
}

/* lagran.cpp:380-443 with runner::calculateTimestep (runner.h:158-169) and
 * LARE3D::calculateTimestep/getTimestep (shared_data.h:428-440). */
static void set_dt(lo_state *s)
{
    DIMS(s);
    const double g = s->p.gas_gamma, mu0 = s->p.mu0;
    const double *rho = s->f[SAMS_F_RHO], *bx = s->f[SAMS_F_BX], *by = s->f[SAMS_F_BY], *bz = s->f[SAMS_F_BZ];
    const double *vx = s->f[SAMS_F_VX], *vy = s->f[SAMS_F_VY], *vz = s->f[SAMS_F_VZ];
    const double *dxb = s->dxb, *dyb = s->dyb, *dzb = s->dzb;
    double best = DBL_MAX;
    const int64_t i0 = s->p.geometry == 0 ? 0 : 1; /* lagran.cpp:384 */
#pragma omp parallel for reduction(min : best) schedule(static)
    for (int64_t ix = i0; ix <= nx; ++ix)
        for (int64_t iy = 0; iy <= ny; ++iy)
            for (int64_t iz = 0; iz <= nz; ++iz) {
                int64_t izm = iz - 1, iym = iy - 1, ixm = ix - 1;
                int64_t o = I3(ix, iy, iz);
                double dx = dxb[A1(ix)], dy = dyb[A1(iy)], dz = dzb[A1(iz)];
                double dhx = dx, dhy = dy * s->hyc[A1(ix)], dhz = dz * s->hzc[H2(ix, iy)];
                double rho0 = pmax(rho[o], NONE_ZERO);
                double cs2 = g * s->pressure[o] / rho0;
                double w1 = (bx[o] * bx[o] + by[o] * by[o] + bz[o] * bz[o]) / mu0 / rho0;
                double c_visc2 = s->p_visc[o] / rho0;
                double length = pmin(pmin(dhx, dhy), dhz);
                double dt1 = length / (sqrt(c_visc2) + sqrt(cs2 + w1 + c_visc2));
                double ax = 0.25 * s->dxab[o], ay = 0.25 * s->dyab[o], az = 0.25 * s->dzab[o];
                double vxbm = (vx[I3(ixm, iy, iz)] + vx[I3(ixm, iym, iz)] + vx[I3(ixm, iy, izm)] + vx[I3(ixm, iym, izm)]) * ax;
                double vxbp = (vx[I3(ix, iy, iz)] + vx[I3(ix, iym, iz)] + vx[I3(ix, iy, izm)] + vx[I3(ix, iym, izm)]) * ax;
                double vybm = (vy[I3(ix, iym, iz)] + vy[I3(ixm, iym, iz)] + vy[I3(ix, iym, izm)] + vy[I3(ixm, iym, izm)]) * ay;
                double vybp = (vy[I3(ix, iy, iz)] + vy[I3(ixm, iy, iz)] + vy[I3(ix, iy, izm)] + vy[I3(ixm, iy, izm)]) * ay;
                double vzbm = (vz[I3(ix, iy, izm)] + vz[I3(ixm, iy, izm)] + vz[I3(ix, iym, izm)] + vz[I3(ixm, iym, izm)]) * az;
                double vzbp = (vz[I3(ix, iy, iz)] + vz[I3(ixm, iy, iz)] + vz[I3(ix, iym, iz)] + vz[I3(ixm, iym, iz)]) * az;
                double dvx = fabs(vxbp - vxbm), dvy = fabs(vybp - vybm), dvz = fabs(vzbp - vzbm);
                double avxm = fabs(vxbm), avxp = fabs(vxbp), avym = fabs(vybm);
                double avyp = fabs(vybp), avzm = fabs(vzbm), avzp = fabs(vzbp);
                double volume = s->cv[o];
                double dt2 = volume / pmax(pmax(pmax(avxm, avxp), dvx), 1.0e-10 * volume);
                double dt3 = volume / pmax(pmax(pmax(avym, avyp), dvy), 1.0e-10 * volume);
                double dt4 = volume / pmax(pmax(pmax(avzm, avzp), dvz), 1.0e-10 * volume);
                double r = pmin(pmin(pmin(dt1, dt2), dt3), dt4);
                best = pmin(best, r);
            }
    double dt = s->p.dt_multiplier * best;
    s->dtr = dt;
    /* runner: tData.dt = max; tData.dt = data.dt < tData.dt ? data.dt : tData.dt */
    s->dt = dt < DBL_MAX ? dt : DBL_MAX;
}

/* lagran.cpp:445-476 */
static void eta_calc(lo_state *s)
{
    DIMS(s);
    const double *bx = s->f[SAMS_F_BX], *by = s->f[SAMS_F_BY], *bz = s->f[SAMS_F_BZ];
    const double *dxc = s->dxc, *dyc = s->dyc, *dzc = s->dzc;
    double *eta = s->eta;
    const double jmax = s->p.j_max, e_bg = s->p.eta_background, e0 = s->p.eta0;
    LOOP3(-1, nx + 1, -1, ny + 1, -1, nz + 1)
    {
        int64_t izp = iz + 1, iyp = iy + 1, ixp = ix + 1;
        double jx = (bz[I3(ix, iyp, iz)] - bz[I3(ix, iy, iz)]) / dyc[A1(iy)] - (by[I3(ix, iy, izp)] - by[I3(ix, iy, iz)]) / dzc[A1(iz)];
        double jxp = (bz[I3(ixp, iyp, iz)] - bz[I3(ixp, iy, iz)]) / dyc[A1(iy)] - (by[I3(ixp, iy, izp)] - by[I3(ixp, iy, iz)]) / dzc[A1(iz)];
        double jy = (bx[I3(ix, iy, izp)] - bx[I3(ix, iy, iz)]) / dzc[A1(iz)] - (bz[I3(ixp, iy, iz)] - bz[I3(ix, iy, iz)]) / dxc[A1(ix)];
        double jyp = (bx[I3(ix, iyp, izp)] - bx[I3(ix, iyp, iz)]) / dzc[A1(iz)] - (bz[I3(ixp, iyp, iz)] - bz[I3(ix, iyp, iz)]) / dxc[A1(ix)];
        double jz = (by[I3(ixp, iy, iz)] - by[I3(ix, iy, iz)]) / dxc[A1(ix)] - (bx[I3(ix, iyp, iz)] - bx[I3(ix, iy, iz)]) / dyc[A1(iy)];
        double jzp = (by[I3(ixp, iy, izp)] - by[I3(ix, iy, izp)]) / dxc[A1(ix)] - (bx[I3(ix, iyp, izp)] - bx[I3(ix, iy, izp)]) / dyc[A1(iy)];
        jx = (jx + jxp) * 0.5;
        jy = (jy + jyp) * 0.5;
        jz = (jz + jzp) * 0.5;
        double j_local = sqrt(jx * jx + jy * jy + jz * jz);
        eta[I3(ix, iy, iz)] = j_local > jmax ? e_bg + e0 : e_bg;
    }
}

/* lagran.cpp:507-535 */
static void rkstep(lo_state *s)
{
    DIMS(s);
    const double *bx = s->f[SAMS_F_BX], *by = s->f[SAMS_F_BY], *bz = s->f[SAMS_F_BZ];
    const double *dxc = s->dxc, *dyc = s->dyc, *dzc = s->dzc, *eta = s->eta;
    LOOP3(0, nx, 0, ny, 0, nz)
    {
        int64_t izp = iz + 1, iyp = iy + 1, ixp = ix + 1;
        double jx1 = (bz[I3(ix, iyp, iz)] - bz[I3(ix, iy, iz)]) / dyc[A1(iy)] - (by[I3(ix, iy, izp)] - by[I3(ix, iy, iz)]) / dzc[A1(iz)];
        double jx2 = (bz[I3(ixp, iyp, iz)] - bz[I3(ixp, iy, iz)]) / dyc[A1(iy)] - (by[I3(ixp, iy, izp)] - by[I3(ixp, iy, iz)]) / dzc[A1(iz)];
        double jy1 = (bx[I3(ix, iy, izp)] - bx[I3(ix, iy, iz)]) / dzc[A1(iz)] - (bz[I3(ixp, iy, iz)] - bz[I3(ix, iy, iz)]) / dxc[A1(ix)];
        double jy2 = (bx[I3(ix, iyp, izp)] - bx[I3(ix, iyp, iz)]) / dzc[A1(iz)] - (bz[I3(ixp, iyp, iz)] - bz[I3(ix, iyp, iz)]) / dxc[A1(ix)];
        double jz1 = (by[I3(ixp, iy, iz)] - by[I3(ix, iy, iz)]) / dxc[A1(ix)] - (bx[I3(ix, iyp, iz)] - bx[I3(ix, iy, iz)]) / dyc[A1(iy)];
        double jz2 = (by[I3(ixp, iy, izp)] - by[I3(ix, iy, izp)]) / dxc[A1(ix)] - (bx[I3(ix, iyp, izp)] - bx[I3(ix, iy, izp)]) / dyc[A1(iy)];
        double jx = 0.5 * (jx1 + jx2), jy = 0.5 * (jy1 + jy2), jz = 0.5 * (jz1 + jz2);
        int64_t o = I3(ix, iy, iz);
        s->flux_x[o] = -jx * eta[o] * dxc[A1(ix)] * 0.5;
        s->flux_y[o] = -jy * eta[o] * dyc[A1(iy)] * 0.5;
        s->flux_z[o] = -jz * eta[o] * dzc[A1(iz)] * 0.5;
        s->curlb[o] = eta[o] * (jx * jx + jy * jy + jz * jz);
    }
}

/* lagran.cpp:537-590 */
static void bstep(lo_state *s)
{
    DIMS(s);
    double *bx = s->f[SAMS_F_BX], *by = s->f[SAMS_F_BY], *bz = s->f[SAMS_F_BZ];
    const double *fx = s->flux_x, *fy = s->flux_y, *fz = s->flux_z, *dxb = s->dxb, *dyb = s->dyb, *dzb = s->dzb;
    const double dt = s->dt;
    LOOP3(0, nx, 1, ny, 1, nz)
    {
        int64_t izm = iz - 1, iym = iy - 1;
        double area = dyb[A1(iy)] * dzb[A1(iz)];
        bx[I3(ix, iy, iz)] = s->bx1[I3(ix, iy, iz)] +
            (fz[I3(ix, iy, iz)] - fz[I3(ix, iym, iz)] + fz[I3(ix, iy, izm)] - fz[I3(ix, iym, izm)] -
             fy[I3(ix, iy, iz)] + fy[I3(ix, iy, izm)] - fy[I3(ix, iym, iz)] + fy[I3(ix, iym, izm)]) * dt / area;
    }
    LOOP3(1, nx, 0, ny, 1, nz)
    {
        int64_t izm = iz - 1, ixm = ix - 1;
        double area = dxb[A1(ix)] * dzb[A1(iz)];
        by[I3(ix, iy, iz)] = s->by1[I3(ix, iy, iz)] +
            (fx[I3(ix, iy, iz)] - fx[I3(ix, iy, izm)] + fx[I3(ixm, iy, iz)] - fx[I3(ixm, iy, izm)] -
             fz[I3(ix, iy, iz)] + fz[I3(ixm, iy, iz)] - fz[I3(ix, iy, izm)] + fz[I3(ixm, iy, izm)]) * dt / area;
    }
    LOOP3(1, nx, 1, ny, 0, nz)
    {
        int64_t iym = iy - 1, ixm = ix - 1;
        double area = dxb[A1(ix)] * dyb[A1(iy)];
        bz[I3(ix, iy, iz)] = s->bz1[I3(ix, iy, iz)] +
            (fy[I3(ix, iy, iz)] - fy[I3(ixm, iy, iz)] + fy[I3(ix, iym, iz)] - fy[I3(ixm, iym, iz)] -
             fx[I3(ix, iy, iz)] + fx[I3(ix, iym, iz)] - fx[I3(ixm, iy, iz)] + fx[I3(ixm, iym, iz)]) * dt / area;
    }
    bfield_bcs(s);
}

/* lagran.cpp:478-505; the bx1/by1/bz1 copies at :482-484 cover the index
 * range the face and cell arrays share (the shipped pw::assign throws). */
static void resistive_effects(lo_state *s)
{
    DIMS(s);
    for (int64_t ix = -1; ix <= nx + 2; ++ix)
        for (int64_t iy = -1; iy <= ny + 2; ++iy)
            for (int64_t iz = -1; iz <= nz + 2; ++iz) {
                int64_t o = I3(ix, iy, iz);
                s->bx1[o] = s->f[SAMS_F_BX][o];
                s->by1[o] = s->f[SAMS_F_BY][o];
                s->bz1[o] = s->f[SAMS_F_BZ][o];
            }
    rkstep(s);
    bstep(s);
    double *ee = s->f[SAMS_F_ENERGY_ELECTRON];
    const double *rho = s->f[SAMS_F_RHO], *curlb = s->curlb;
    const double dt = s->dt;
    LOOP3(1, nx, 1, ny, 1, nz)
    {
        int64_t izm = iz - 1, iym = iy - 1, ixm = ix - 1;
        double sum_curlb = curlb[I3(ix, iy, iz)] + curlb[I3(ixm, iy, iz)] +
                           curlb[I3(ix, iym, iz)] + curlb[I3(ixm, iym, iz)] +
                           curlb[I3(ix, iy, izm)] + curlb[I3(ixm, iy, izm)] +
                           curlb[I3(ix, iym, izm)] + curlb[I3(ixm, iym, izm)];
        ee[I3(ix, iy, iz)] += sum_curlb * dt / (8.0 * rho[I3(ix, iy, iz)]);
    }
    energy_bcs(s);
}

/* lagran.cpp:806-882 */
static void b_field_and_cv1_update(lo_state *s)
{
    DIMS(s);
    const double *vx = s->f[SAMS_F_VX], *vy = s->f[SAMS_F_VY], *vz = s->f[SAMS_F_VZ];
    const double *dxab = s->dxab, *dyab = s->dyab, *dzab = s->dzab, *cv = s->cv;
    double *bx1 = s->bx1, *by1 = s->by1, *bz1 = s->bz1, *cv1 = s->cv1;
    const double dt = s->dt;
    LOOP3(-1, nx + 2, -1, ny + 2, -1, nz + 2)
    {
        int64_t izm = iz - 1, iym = iy - 1, ixm = ix - 1;
        int64_t o = I3(ix, iy, iz);
        double vxb = 0.25 * (vx[I3(ix, iy, iz)] + vx[I3(ix, iym, iz)] + vx[I3(ix, iy, izm)] + vx[I3(ix, iym, izm)]);
        double vxbm = 0.25 * (vx[I3(ixm, iy, iz)] + vx[I3(ixm, iym, iz)] + vx[I3(ixm, iy, izm)] + vx[I3(ixm, iym, izm)]);
        double vyb = 0.25 * (vy[I3(ix, iy, iz)] + vy[I3(ixm, iy, iz)] + vy[I3(ix, iy, izm)] + vy[I3(ixm, iy, izm)]);
        double vybm = 0.25 * (vy[I3(ix, iym, iz)] + vy[I3(ixm, iym, iz)] + vy[I3(ix, iym, izm)] + vy[I3(ixm, iym, izm)]);
        double vzb = 0.25 * (vz[I3(ix, iy, iz)] + vz[I3(ixm, iy, iz)] + vz[I3(ix, iym, iz)] + vz[I3(ixm, iym, iz)]);
        double vzbm = 0.25 * (vz[I3(ix, iy, izm)] + vz[I3(ixm, iy, izm)] + vz[I3(ix, iym, izm)] + vz[I3(ixm, iym, izm)]);
        double vol = cv[o];
        double dvxdx = (vxb * dxab[I3(ix, iy, iz)] - vxbm * dxab[I3(ixm, iy, iz)]) / vol;
        double dvydy = (vyb * dyab[I3(ix, iy, iz)] - vybm * dyab[I3(ix, iym, iz)]) / vol;
        double dvzdz = (vzb * dzab[I3(ix, iy, iz)] - vzbm * dzab[I3(ix, iy, izm)]) / vol;
        double dv = (dvxdx + dvydy + dvzdz) * dt / 2.0;
        cv1[o] = vol * (1.0 + dv);

        vxb = 0.25 * (vx[I3(ix, iy, iz)] + vx[I3(ixm, iy, iz)] + vx[I3(ix, iy, izm)] + vx[I3(ixm, iy, izm)]);
        vxbm = 0.25 * (vx[I3(ix, iym, iz)] + vx[I3(ixm, iym, iz)] + vx[I3(ix, iym, izm)] + vx[I3(ixm, iym, izm)]);
        vyb = 0.25 * (vy[I3(ix, iy, iz)] + vy[I3(ix, iym, iz)] + vy[I3(ix, iy, izm)] + vy[I3(ix, iym, izm)]);
        vybm = 0.25 * (vy[I3(ixm, iy, iz)] + vy[I3(ixm, iym, iz)] + vy[I3(ixm, iy, izm)] + vy[I3(ixm, iym, izm)]);
        double dvxdy = (vxb * dyab[I3(ix, iy, iz)] - vxbm * dyab[I3(ix, iym, iz)]) / vol;
        double dvydx = (vyb * dxab[I3(ix, iy, iz)] - vybm * dxab[I3(ixm, iy, iz)]) / vol;

        vxb = 0.25 * (vx[I3(ix, iy, iz)] + vx[I3(ixm, iy, iz)] + vx[I3(ix, iym, iz)] + vx[I3(ixm, iym, iz)]);
        vxbm = 0.25 * (vx[I3(ix, iy, izm)] + vx[I3(ixm, iy, izm)] + vx[I3(ix, iym, izm)] + vx[I3(ixm, iym, izm)]);
        vzb = 0.25 * (vz[I3(ix, iy, iz)] + vz[I3(ix, iym, iz)] + vz[I3(ix, iy, izm)] + vz[I3(ix, iym, izm)]);
        vzbm = 0.25 * (vz[I3(ixm, iy, iz)] + vz[I3(ixm, iym, iz)] + vz[I3(ixm, iy, izm)] + vz[I3(ixm, iym, izm)]);
        double dvxdz = (vxb * dzab[I3(ix, iy, iz)] - vxbm * dzab[I3(ix, iy, izm)]) / vol;
        double dvzdx = (vzb * dxab[I3(ix, iy, iz)] - vzbm * dxab[I3(ixm, iy, iz)]) / vol;

        vyb = 0.25 * (vy[I3(ix, iy, iz)] + vy[I3(ixm, iy, iz)] + vy[I3(ix, iym, iz)] + vy[I3(ixm, iym, iz)]);
        vybm = 0.25 * (vy[I3(ix, iy, izm)] + vy[I3(ixm, iy, izm)] + vy[I3(ix, iym, izm)] + vy[I3(ixm, iym, izm)]);
        vzb = 0.25 * (vz[I3(ix, iy, iz)] + vz[I3(ixm, iy, iz)] + vz[I3(ix, iy, izm)] + vz[I3(ixm, iy, izm)]);
        vzbm = 0.25 * (vz[I3(ix, iym, iz)] + vz[I3(ixm, iym, iz)] + vz[I3(ix, iym, izm)] + vz[I3(ixm, iym, izm)]);
        double dvydz = (vyb * dzab[I3(ix, iy, iz)] - vybm * dzab[I3(ix, iy, izm)]) / vol;
        double dvzdy = (vzb * dyab[I3(ix, iy, iz)] - vzbm * dyab[I3(ix, iym, iz)]) / vol;

        double w3 = bx1[o] * dvxdx + by1[o] * dvxdy + bz1[o] * dvxdz;
        double w4 = bx1[o] * dvydx + by1[o] * dvydy + bz1[o] * dvydz;
        double w5 = bx1[o] * dvzdx + by1[o] * dvzdy + bz1[o] * dvzdz;
        bx1[o] = (bx1[o] + w3 * dt / 2.0) / (1.0 + dv);
        by1[o] = (by1[o] + w4 * dt / 2.0) / (1.0 + dv);
        bz1[o] = (bz1[o] + w5 * dt / 2.0) / (1.0 + dv);
    }
}

/* lagran.cpp:592-737 (Cartesian) */
static void predictor_step(lo_state *s)
{
    DIMS(s);
    b_field_and_cv1_update(s);
    double *bx1 = s->bx1, *by1 = s->by1, *bz1 = s->bz1, *cv1 = s->cv1;
    LOOP3(-1, nx + 2, -1, ny + 2, -1, nz + 2)
    {
        int64_t o = I3(ix, iy, iz);
        bx1[o] *= cv1[o];
        by1[o] *= cv1[o];
        bz1[o] *= cv1[o];
    }
    const double g = s->p.gas_gamma, dt = s->dt, mu0 = s->p.mu0;
    double *rho = s->f[SAMS_F_RHO], *ee = s->f[SAMS_F_ENERGY_ELECTRON], *ei = s->f[SAMS_F_ENERGY_ION];
    double *p_e = s->p_e, *p_i = s->p_i, *pressure = s->pressure, *cv = s->cv;
    LOOP3(0, nx + 1, 0, ny + 1, 0, nz + 1)
    {
        int64_t o = I3(ix, iy, iz);
        double dv = cv1[o] / cv[o] - 1.0;
        double e1_e = ee[o] - p_e[o] * dv / rho[o];
        double e1_i = ei[o] - p_i[o] * dv / rho[o];
        e1_i += s->visc_heat[o] * dt / 2.0 / rho[o];
        p_e[o] = e1_e * (g - 1.0) * rho[o] * cv[o] / cv1[o];
        p_i[o] = e1_i * (g - 1.0) * rho[o] * cv[o] / cv1[o];
        pressure[o] = p_e[o] + p_i[o];
    }
    const double *vx = s->f[SAMS_F_VX], *vy = s->f[SAMS_F_VY], *vz = s->f[SAMS_F_VZ];
    double *vx1 = s->f[SAMS_F_VX1], *vy1 = s->f[SAMS_F_VY1], *vz1 = s->f[SAMS_F_VZ1];
    const double *dxc = s->dxc, *dyc = s->dyc, *dzc = s->dzc;
    LOOP3(0, nx, 0, ny, 0, nz)
    {
        int64_t izp = iz + 1, iyp = iy + 1, ixp = ix + 1;
        int64_t o = I3(ix, iy, iz);
        double dx = dxc[A1(ix)], dy = dyc[A1(iy)], dz = dzc[A1(iz)];
        double h2 = s->hy[A1(ix)], h2x = s->hy[A1(ixp)];
        double h3 = s->hz[H2(ix, iy)], h3x = s->hz[H2(ixp, iy)], h3y = s->hz[H2(ix, iyp)];
        double h2c = s->hyc[A1(ix)], h3c = s->hzc[H2(ix, iy)];
        double dhy = h2c * dy, dhz = h3c * dz;
        double pp = pressure[I3(ix, iy, iz)];
        double ppx = pressure[I3(ixp, iy, iz)];
        double ppy = pressure[I3(ix, iyp, iz)];
        double ppz = pressure[I3(ix, iy, izp)];
        double ppxy = pressure[I3(ixp, iyp, iz)];
        double ppxz = pressure[I3(ixp, iy, izp)];
        double ppyz = pressure[I3(ix, iyp, izp)];
        double ppxyz = pressure[I3(ixp, iyp, izp)];
        double w1 = pp + ppy + ppz + ppyz;
        double w2 = ppx + ppxy + ppxz + ppxyz;
        double fx = (w1 - w2) * 0.25 / dx;
        w1 = pp + ppx + ppz + ppxz;
        w2 = ppy + ppxy + ppyz + ppxyz;
        double fy = (w1 - w2) * 0.25 / dhy;
        w1 = pp + ppx + ppy + ppxy;
        w2 = ppz + ppxz + ppyz + ppxyz;
        double fz = (w1 - w2) * 0.25 / dhz;

        double cvx = cv1[I3(ix, iy, iz)] + cv1[I3(ix, iyp, iz)] + cv1[I3(ix, iy, izp)] + cv1[I3(ix, iyp, izp)];
        double cvxp = cv1[I3(ixp, iy, iz)] + cv1[I3(ixp, iyp, iz)] + cv1[I3(ixp, iy, izp)] + cv1[I3(ixp, iyp, izp)];
        double cvy = cv1[I3(ix, iy, iz)] + cv1[I3(ixp, iy, iz)] + cv1[I3(ix, iy, izp)] + cv1[I3(ixp, iy, izp)];
        double cvyp = cv1[I3(ix, iyp, iz)] + cv1[I3(ixp, iyp, iz)] + cv1[I3(ix, iyp, izp)] + cv1[I3(ixp, iyp, izp)];
        double cvz = cv1[I3(ix, iy, iz)] + cv1[I3(ixp, iy, iz)] + cv1[I3(ix, iyp, iz)] + cv1[I3(ixp, iyp, iz)];
        double cvzp = cv1[I3(ix, iy, izp)] + cv1[I3(ixp, iy, izp)] + cv1[I3(ix, iyp, izp)] + cv1[I3(ixp, iyp, izp)];

        w1 = (bz1[I3(ix, iy, iz)] + bz1[I3(ixp, iy, iz)] + bz1[I3(ix, iy, izp)] + bz1[I3(ixp, iy, izp)]) * h3 / cvy;
        w2 = (bz1[I3(ix, iyp, iz)] + bz1[I3(ixp, iyp, iz)] + bz1[I3(ix, iyp, izp)] + bz1[I3(ixp, iyp, izp)]) * h3y / cvyp;
        double jx = (w2 - w1) / dhy / h3c;
        w1 = (by1[I3(ix, iy, iz)] + by1[I3(ixp, iy, iz)] + by1[I3(ix, iyp, iz)] + by1[I3(ixp, iyp, iz)]) / cvz;
        w2 = (by1[I3(ix, iy, izp)] + by1[I3(ixp, iy, izp)] + by1[I3(ix, iyp, izp)] + by1[I3(ixp, iyp, izp)]) / cvzp;
        jx -= (w2 - w1) / dhz;

        w1 = (bz1[I3(ix, iy, iz)] + bz1[I3(ix, iyp, iz)] + bz1[I3(ix, iy, izp)] + bz1[I3(ix, iyp, izp)]) * h3 / cvx;
        w2 = (bz1[I3(ixp, iy, iz)] + bz1[I3(ixp, iyp, iz)] + bz1[I3(ixp, iy, izp)] + bz1[I3(ixp, iyp, izp)]) * h3x / cvxp;
        double jy = -(w2 - w1) / dx / h3c;
        w1 = (bx1[I3(ix, iy, iz)] + bx1[I3(ixp, iy, iz)] + bx1[I3(ix, iyp, iz)] + bx1[I3(ixp, iyp, iz)]) / cvz;
        w2 = (bx1[I3(ix, iy, izp)] + bx1[I3(ixp, iy, izp)] + bx1[I3(ix, iyp, izp)] + bx1[I3(ixp, iyp, izp)]) / cvzp;
        jy += (w2 - w1) / dhz;

        w1 = (by1[I3(ix, iy, iz)] + by1[I3(ix, iyp, iz)] + by1[I3(ix, iy, izp)] + by1[I3(ix, iyp, izp)]) * h2 / cvx;
        w2 = (by1[I3(ixp, iy, iz)] + by1[I3(ixp, iyp, iz)] + by1[I3(ixp, iy, izp)] + by1[I3(ixp, iyp, izp)]) * h2x / cvxp;
        double jz = (w2 - w1) / dx / h2c;
        w1 = (bx1[I3(ix, iy, iz)] + bx1[I3(ixp, iy, iz)] + bx1[I3(ix, iy, izp)] + bx1[I3(ixp, iy, izp)]) / cvy;
        w2 = (bx1[I3(ix, iyp, iz)] + bx1[I3(ixp, iyp, iz)] + bx1[I3(ix, iyp, izp)] + bx1[I3(ixp, iyp, izp)]) / cvyp;
        jz -= (w2 - w1) / dhy;

#define SUM8(a) (a[I3(ix, iy, iz)] + a[I3(ixp, iy, iz)] + a[I3(ix, iyp, iz)] + a[I3(ixp, iyp, iz)] + \
                 a[I3(ix, iy, izp)] + a[I3(ixp, iy, izp)] + a[I3(ix, iyp, izp)] + a[I3(ixp, iyp, izp)])
        double bxv = SUM8(bx1) / (cvx + cvxp);
        double byv = SUM8(by1) / (cvx + cvxp);
        double bzv = SUM8(bz1) / (cvx + cvxp);
#undef SUM8
        fx += (jy * bzv - jz * byv) / mu0;
        fy += (jz * bxv - jx * bzv) / mu0;
        fz += (jx * byv - jy * bxv) / mu0;
        /* geometry corrections (lagran.cpp:711-721) */
        if (s->p.geometry == 2) {
            const double cotantheta = s->cot_yb[A1(iy)], rv = s->rho_v[o], r = s->xb[A1(ix)];
            fx += rv * (vy[o] * vy[o] + vz[o] * vz[o]) / r;
            fy -= rv * (vy[o] * vx[o] - cotantheta * vz[o] * vz[o]) / r;
            fz -= rv * (vz[o] * vx[o] + cotantheta * vz[o] * vy[o]) / r;
        } else if (s->p.geometry == 1) {
            const double rv = s->rho_v[o], r = s->xb[A1(ix)];
            fx += rv * vy[o] * vy[o] / r;
            fy -= rv * vy[o] * vx[o] / r;
        }
        s->fx[o] = fx;
        s->fy[o] = fy;
        s->fz[o] = fz;
        vx1[o] = vx[o] + dt / 2.0 * (s->fx_visc[o] + fx) / s->rho_v[o];
        vy1[o] = vy[o] + dt / 2.0 * (s->fy_visc[o] + fy) / s->rho_v[o];
        vz1[o] = vz[o] + dt / 2.0 * (s->fz_visc[o] + fz) / s->rho_v[o];
    }
    remap_v_bcs(s);
}

/* lagran.cpp:95-173 */
static void lagrangian_step(lo_state *s)
{
    DIMS(s);
    const double g = s->p.gas_gamma;
    const double *bx = s->f[SAMS_F_BX], *by = s->f[SAMS_F_BY], *bz = s->f[SAMS_F_BZ];
    const double *rho = s->f[SAMS_F_RHO], *ee = s->f[SAMS_F_ENERGY_ELECTRON], *ei = s->f[SAMS_F_ENERGY_ION];
    const double *cv = s->cv;
    LOOP3(-1, nx + 2, -1, ny + 2, -1, nz + 2)
    {
        int64_t o = I3(ix, iy, iz);
        s->bx1[o] = 0.5 * (bx[o] + bx[I3(ix - 1, iy, iz)]);
        s->by1[o] = 0.5 * (by[o] + by[I3(ix, iy - 1, iz)]);
        s->bz1[o] = 0.5 * (bz[o] + bz[I3(ix, iy, iz - 1)]);
        s->p_e[o] = (g - 1.0) * rho[o] * ee[o];
        s->p_i[o] = (g - 1.0) * rho[o] * ei[o];
        s->pressure[o] = s->p_e[o] + s->p_i[o];
    }
    LOOP3(-1, nx + 1, -1, ny + 1, -1, nz + 1)
    {
        int64_t izp = iz + 1, iyp = iy + 1, ixp = ix + 1;
        double sum_rho_cv = rho[I3(ix, iy, iz)] * cv[I3(ix, iy, iz)] +
                            rho[I3(ixp, iy, iz)] * cv[I3(ixp, iy, iz)] +
                            rho[I3(ix, iyp, iz)] * cv[I3(ix, iyp, iz)] +
                            rho[I3(ixp, iyp, iz)] * cv[I3(ixp, iyp, iz)] +
                            rho[I3(ix, iy, izp)] * cv[I3(ix, iy, izp)] +
                            rho[I3(ixp, iy, izp)] * cv[I3(ixp, iy, izp)] +
                            rho[I3(ix, iyp, izp)] * cv[I3(ix, iyp, izp)] +
                            rho[I3(ixp, iyp, izp)] * cv[I3(ixp, iyp, izp)];
        double sum_cv = cv[I3(ix, iy, iz)] + cv[I3(ixp, iy, iz)] + cv[I3(ix, iyp, iz)] + cv[I3(ixp, iyp, iz)] +
                        cv[I3(ix, iy, izp)] + cv[I3(ixp, iy, izp)] + cv[I3(ix, iyp, izp)] + cv[I3(ixp, iyp, izp)];
        s->rho_v[I3(ix, iy, iz)] = sum_rho_cv / sum_cv;
        s->cv_v[I3(ix, iy, iz)] = 0.125 * sum_cv;
    }
    shock_viscosity(s);
    set_dt(s);
    if (s->p.resistive_mhd) {
        double dt_sub = s->dtr;
        int substeps = (int)(s->dt / dt_sub) + 1;
        double actual_dt = s->dt;
        s->dt /= (double)substeps;
        for (int i = 0; i < substeps; ++i) {
            eta_calc(s);
            resistive_effects(s);
        }
        s->dt = actual_dt;
    }
    predictor_step(s);
}

/* lagran.cpp:884-993 (note the dy*dy factors at :987, kept) */
static void shock_heating(lo_state *s)
{
    DIMS(s);
    const double *vx = s->f[SAMS_F_VX], *vy = s->f[SAMS_F_VY], *vz = s->f[SAMS_F_VZ];
    const double *vx1 = s->f[SAMS_F_VX1], *vy1 = s->f[SAMS_F_VY1], *vz1 = s->f[SAMS_F_VZ1];
    const double *a1a = s->alpha1, *a2a = s->alpha2, *a3a = s->alpha3;
    const double *dxb = s->dxb, *dyb = s->dyb, *dzb = s->dzb;
    LOOP3(0, nx + 1, 0, ny + 1, 0, nz + 1)
    {
        int64_t izm = iz - 1, izp = iz + 1, iym = iy - 1, iyp = iy + 1, ixm = ix - 1;
#define DD(a, b) (1 * ((vx[a] - vx[b]) * (vx1[a] - vx1[b]) + (vy[a] - vy[b]) * (vy1[a] - vy1[b]) + \
                       (vz[a] - vz[b]) * (vz1[a] - vz1[b])))
        double a1 = DD(I3(ixm, iym, iz), I3(ix, iym, iz));
        double a2 = DD(I3(ix, iym, iz), I3(ix, iy, iz));
        double a3 = DD(I3(ix, iy, iz), I3(ixm, iy, iz));
        double a4 = DD(I3(ixm, iy, iz), I3(ixm, iym, iz));
        double a5 = DD(I3(ixm, iym, izp), I3(ix, iym, izp));
        double a6 = DD(I3(ix, iym, izp), I3(ix, iy, izp));
        double a7 = DD(I3(ix, iy, izp), I3(ixm, iy, izp));
        double a8 = DD(I3(ixm, iy, izp), I3(ixm, iym, izp));
        double a9 = DD(I3(ix, iy, izm), I3(ix, iy, iz));
        double a10 = DD(I3(ixm, iy, izm), I3(ixm, iy, iz));
        double a11 = DD(I3(ixm, iym, izm), I3(ixm, iym, iz));
        double a12 = DD(I3(ix, iym, izm), I3(ix, iym, iz));
#undef DD
        double dx = dxb[A1(ix)], dy = dyb[A1(iy)] * s->hyc[A1(ix)], dz = dzb[A1(iz)] * s->hz2[H2(ix, iy)];
        int64_t o = I3(ix, iy, iz);
        double vh =
            (-0.25 * dy * dz * a1a[I3(ix, iy, iz)] * a1 - 0.25 * dx * dz * a2a[I3(ix, iy, iz)] * a2 - 0.25 * dy * dz * a1a[I3(ix, iyp, iz)] * a3 -
             0.25 * dx * dz * a2a[I3(ixm, iy, iz)] * a4 - 0.25 * dy * dz * a1a[I3(ix, iy, izp)] * a5 - 0.25 * dx * dz * a2a[I3(ix, iy, izp)] * a6 -
             0.25 * dy * dz * a1a[I3(ix, iyp, izp)] * a7 - 0.25 * dx * dz * a2a[I3(ixm, iy, izp)] * a8 - 0.25 * dy * dy * a3a[I3(ix, iy, iz)] * a9 -
             0.25 * dx * dy * a3a[I3(ixm, iy, iz)] * a10 - 0.25 * dy * dy * a3a[I3(ixm, iym, iz)] * a11 - 0.25 * dx * dy * a3a[I3(ix, iym, iz)] * a12);
        s->visc_heat[o] = pmax(vh / s->cv[o], 0.0);
    }
}

/* lagran.cpp:739-804 */
static void corrector_step(lo_state *s)
{
    DIMS(s);
    double *bx1 = s->bx1, *by1 = s->by1, *bz1 = s->bz1, *cv1 = s->cv1;
    LOOP3(-1, nx + 2, -1, ny + 2, -1, nz + 2)
    {
        int64_t o = I3(ix, iy, iz);
        bx1[o] /= cv1[o];
        by1[o] /= cv1[o];
        bz1[o] /= cv1[o];
    }
    shock_heating(s);
    double *vx = s->f[SAMS_F_VX], *vy = s->f[SAMS_F_VY], *vz = s->f[SAMS_F_VZ];
    const double dt = s->dt;
    LOOP3(0, nx, 0, ny, 0, nz)
    {
        int64_t o = I3(ix, iy, iz);
        vx[o] += dt * (s->fx_visc[o] + s->fx[o]) / s->rho_v[o];
        vy[o] += dt * (s->fy_visc[o] + s->fy[o]) / s->rho_v[o];
        vz[o] += dt * (s->fz_visc[o] + s->fz[o]) / s->rho_v[o];
    }
    velocity_bcs(s);
    const double *vx1 = s->f[SAMS_F_VX1], *vy1 = s->f[SAMS_F_VY1], *vz1 = s->f[SAMS_F_VZ1];
    double *rho = s->f[SAMS_F_RHO], *ee = s->f[SAMS_F_ENERGY_ELECTRON], *ei = s->f[SAMS_F_ENERGY_ION];
    const double *dxab = s->dxab, *dyab = s->dyab, *dzab = s->dzab, *cv = s->cv;
    LOOP3(1, nx, 1, ny, 1, nz)
    {
        int64_t izm = iz - 1, iym = iy - 1, ixm = ix - 1;
        int64_t o = I3(ix, iy, iz);
        double vxb = 0.25 * (vx1[I3(ix, iy, iz)] + vx1[I3(ix, iym, iz)] + vx1[I3(ix, iy, izm)] + vx1[I3(ix, iym, izm)]);
        double vxbm = 0.25 * (vx1[I3(ixm, iy, iz)] + vx1[I3(ixm, iym, iz)] + vx1[I3(ixm, iy, izm)] + vx1[I3(ixm, iym, izm)]);
        double vyb = 0.25 * (vy1[I3(ix, iy, iz)] + vy1[I3(ixm, iy, iz)] + vy1[I3(ix, iy, izm)] + vy1[I3(ixm, iy, izm)]);
        double vybm = 0.25 * (vy1[I3(ix, iym, iz)] + vy1[I3(ixm, iym, iz)] + vy1[I3(ix, iym, izm)] + vy1[I3(ixm, iym, izm)]);
        double vzb = 0.25 * (vz1[I3(ix, iy, iz)] + vz1[I3(ixm, iy, iz)] + vz1[I3(ix, iym, iz)] + vz1[I3(ixm, iym, iz)]);
        double vzbm = 0.25 * (vz1[I3(ix, iy, izm)] + vz1[I3(ixm, iy, izm)] + vz1[I3(ix, iym, izm)] + vz1[I3(ixm, iym, izm)]);
        double vol = cv[o];
        double dvxdx = (vxb * dxab[I3(ix, iy, iz)] - vxbm * dxab[I3(ixm, iy, iz)]) / vol;
        double dvydy = (vyb * dyab[I3(ix, iy, iz)] - vybm * dyab[I3(ix, iym, iz)]) / vol;
        double dvzdz = (vzb * dzab[I3(ix, iy, iz)] - vzbm * dzab[I3(ix, iy, izm)]) / vol;
        double dv = (dvxdx + dvydy + dvzdz) * dt;
        cv1[o] = vol * (1.0 + dv);
        ee[o] -= dv * s->p_e[o] / rho[o];
        ei[o] += (dt * s->visc_heat[o] - dv * s->p_i[o]) / rho[o];
        rho[o] /= (1.0 + dv);
    }
    energy_bcs(s);
    density_bcs(s);
    velocity_bcs(s);
}

/* ------------------------------------------------------------------ */
/* Remap (remap.cpp, xremap.cpp, yremap.cpp, zremap.cpp)               */
/* ------------------------------------------------------------------ */

/* Limiter core: Da, ss and Di as written in every flux function. */
static inline double limiter_Di(double sign_v, double phi, double dfi, double dfu,
                                double dxci, double dxcu, double dxbu)
{
    double Da = (2.0 - phi) * fabs(dfi) / dxci + (1.0 + phi) * fabs(dfu) / dxcu;
    Da = Da * SIXTH;
    double ss = 0.5 * ((dfi >= 0.0 ? 1.0 : -1.0) + (dfu >= 0.0 ? 1.0 : -1.0));
    return sign_v * ss * pmin_list3(fabs(Da) * dxbu, fabs(dfi), fabs(dfu));
}

/* Constrained-transport flux of a face field (vx_by_flux xremap.cpp:269-319
 * and its five siblings).  b*: the four face values along the sweep,
 * db*: the averaged db1 lengths, v: v_advect. */
static inline double ct_flux(double v_advect, double dt, double bm, double bi, double bp, double bp2,
                             double dbm, double dbi, double dbp, double dbp2,
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

/* Mass flux (x_mass_flux xremap.cpp:373-422 and siblings). */
static inline double mass_flux(double v_advect, double dt, double area, double fm, double fi, double fp,
                               double fp2, double dci, double dcm, double dcp, double cv1i, double cv1p)
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

/* Energy flux (x_energy_flux xremap.cpp:429-483 and siblings). */
static inline double energy_flux(double v_advect, double dt, double area, double fm, double fi, double fp,
                                 double fp2, double dci, double dcm, double dcp, double cv1i, double cv1p,
                                 double rho1i, double rho1p, double dm)
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

/* Momentum flux before the *dm (x_mom_flux xremap.cpp:485-566 and
 * siblings).  zform selects the z-sweep's |dm| / (dzbu * rhou). */
static inline double mom_flux(double v_advect, double dt, double area, double fm, double fi, double fp,
                              double fp2, double dci, double dcm, double dcp, double cvci, double cvcp,
                              double rvi, double rvp, double dm, int zform)
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
    double dmu = zform ? fabs(dm) / (dxbu * rhou) : fabs(dm) / dxbu / rhou;
    return fu + Di * (1.0 - dmu);
}

/* First kernel of every sweep (xremap.cpp:28-70, yremap.cpp:27-80,
 * zremap.cpp:28-81): cv2, cv1, db1. dir = sweep direction. */
static void sweep_volumes(lo_state *s, int dir)
{
    DIMS(s);
    const double *vx1 = s->f[SAMS_F_VX1], *vy1 = s->f[SAMS_F_VY1], *vz1 = s->f[SAMS_F_VZ1];
    const double *dxab = s->dxab, *dyab = s->dyab, *dzab = s->dzab, *cv = s->cv;
    const double dt = s->dt, xpass = s->xpass, ypass = s->ypass, zpass = s->zpass;
    LOOP3(-1, nx + 2, -1, ny + 2, -1, nz + 2)
    {
        int64_t ixm = ix - 1, iym = iy - 1, izm = iz - 1;
        int64_t o = I3(ix, iy, iz);
        double vxb = (vx1[I3(ix, iy, iz)] + vx1[I3(ix, iym, iz)] + vx1[I3(ix, iy, izm)] + vx1[I3(ix, iym, izm)]) * 0.25;
        double vxbm = (vx1[I3(ixm, iy, iz)] + vx1[I3(ixm, iym, iz)] + vx1[I3(ixm, iy, izm)] + vx1[I3(ixm, iym, izm)]) * 0.25;
        double vyb = (vy1[I3(ix, iy, iz)] + vy1[I3(ixm, iy, iz)] + vy1[I3(ix, iy, izm)] + vy1[I3(ixm, iy, izm)]) * 0.25;
        double vybm = (vy1[I3(ix, iym, iz)] + vy1[I3(ixm, iym, iz)] + vy1[I3(ix, iym, izm)] + vy1[I3(ixm, iym, izm)]) * 0.25;
        double vzb = (vz1[I3(ix, iy, iz)] + vz1[I3(ixm, iy, iz)] + vz1[I3(ix, iym, iz)] + vz1[I3(ixm, iym, iz)]) * 0.25;
        double vzbm = (vz1[I3(ix, iy, izm)] + vz1[I3(ixm, iy, izm)] + vz1[I3(ix, iym, izm)] + vz1[I3(ixm, iym, izm)]) * 0.25;
        double vol = cv[o];
        double tx = (vxb * dxab[I3(ix, iy, iz)] - vxbm * dxab[I3(ixm, iy, iz)]);
        double ty = (vyb * dyab[I3(ix, iy, iz)] - vybm * dyab[I3(ix, iym, iz)]);
        double tz = (vzb * dzab[I3(ix, iy, iz)] - vzbm * dzab[I3(ix, iy, izm)]);
        double dv;
        if (dir == 0) {
            double dvxdx = tx / vol, dvydy = ypass * ty / vol, dvzdz = zpass * tz / vol;
            dv = (dvydy + dvzdz) * dt;
            s->cv2[o] = vol * (1.0 + dv);
            dv = dv + dvxdx * dt;
            s->db1[o] = s->dxb[A1(ix)] + (vxb - vxbm) * dt;
        } else if (dir == 1) {
            double dvxdx = xpass * tx / vol, dvydy = ty / vol, dvzdz = zpass * tz / vol;
            dv = (dvxdx + dvzdz) * dt;
            s->cv2[o] = vol * (1.0 + dv);
            dv = dv + dvydy * dt;
            s->db1[o] = s->hyc[A1(ix)] * s->dyb[A1(iy)] + (vyb - vybm) * dt;
        } else {
            double dvxdx = xpass * tx / vol, dvydy = ypass * ty / vol, dvzdz = tz / vol;
            dv = (dvxdx + dvydy) * dt;
            s->cv2[o] = vol * (1.0 + dv);
            dv = dv + dvzdz * dt;
            s->db1[o] = s->hzc[H2(ix, iy)] * s->dzb[A1(iz)] + (vzb - vzbm) * dt;
        }
        s->cv1[o] = vol * (1.0 + dv);
    }
    const double *cv1 = s->cv1;
    LOOP3(-1, nx + 1, -1, ny + 1, -1, nz + 1)
    {
        int64_t ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
        s->cvc1[I3(ix, iy, iz)] = 0.125 * (cv1[I3(ix, iy, iz)] + cv1[I3(ixp, iy, iz)] + cv1[I3(ix, iyp, iz)] + cv1[I3(ixp, iyp, iz)] +
                                           cv1[I3(ix, iy, izp)] + cv1[I3(ixp, iy, izp)] + cv1[I3(ix, iyp, izp)] + cv1[I3(ixp, iyp, izp)]);
    }
}

/* Kinetic-energy error of one momentum flux, added to delta_ke at the four
 * nodes across the face (x_mom_flux xremap.cpp:534-558, y_mom_flux
 * yremap.cpp:557-583, z_mom_flux zremap.cpp:513-536).  The reference adds
 * with atomics inside its parallel loop; this is its serial order (source
 * points in index order, the four adds in statement order), which is the
 * reference's result with one thread.  flux holds the momentum flux before
 * it is multiplied by dm; u the velocity component before its update. */
static void rke_scatter(lo_state *s, int dir, const double *u)
{
    DIMS(s);
    const int64_t d1 = dir == 0 ? (int64_t)sy * sz : (dir == 1 ? sz : 1);
    const double *rv1 = s->rho_v1, *cv2 = s->cv2, *flux = s->flux, *dm = s->f[SAMS_F_DM];
    double *dke = s->delta_ke;
    const int64_t ihi = dir == 0 ? nx - 1 : nx, jhi = dir == 1 ? ny - 1 : ny, khi = dir == 2 ? nz - 1 : nz;
    for (int64_t ix = 0; ix <= ihi; ++ix)
        for (int64_t iy = 0; iy <= jhi; ++iy)
            for (int64_t iz = 0; iz <= khi; ++iz) {
                const int64_t o = I3(ix, iy, iz), op = o + d1, om = o - d1;
                const double m = rv1[o] * cv2[o];
                const double mp = rv1[op] * cv2[op];
                const double ai = (u[o] - flux[om]) * dm[om] / m - (u[o] - flux[o]) * dm[o] / m;
                const double aip = (u[op] - flux[o]) * dm[o] / mp - (u[op] - flux[op]) * dm[op] / mp;
                double dk = (u[op] - u[o]) * (flux[o] - 0.5 * (u[op] + u[o])) - 0.5 * ai * (u[o] - flux[o]) +
                            0.5 * aip * (u[op] - flux[o]);
                dk = dk * dm[o] * 0.5;
                if (dir == 0) {
                    dke[I3(ix + 1, iy, iz)] += dk;
                    dke[I3(ix + 1, iy + 1, iz)] += dk;
                    dke[I3(ix + 1, iy + 1, iz + 1)] += dk;
                    dke[I3(ix + 1, iy, iz + 1)] += dk;
                } else if (dir == 1) {
                    dke[I3(ix + 1, iy + 1, iz)] += dk;
                    dke[I3(ix, iy + 1, iz)] += dk;
                    dke[I3(ix + 1, iy + 1, iz + 1)] += dk;
                    dke[I3(ix, iy + 1, iz + 1)] += dk;
                } else {
                    dke[I3(ix, iy, iz + 1)] += dk;
                    dke[I3(ix + 1, iy, iz + 1)] += dk;
                    dke[I3(ix, iy + 1, iz + 1)] += dk;
                    dke[I3(ix + 1, iy + 1, iz + 1)] += dk;
                }
            }
}

/* energy_correction (diagnostics.cpp:125-135), after the remap (shared_data.h:414-417) */
static void energy_correction(lo_state *s)
{
    DIMS(s);
    double *ee = s->f[SAMS_F_ENERGY_ELECTRON], *ei = s->f[SAMS_F_ENERGY_ION];
    const double *rho = s->f[SAMS_F_RHO], *cv = s->cv, *dke = s->delta_ke;
    LOOP3(1, nx, 1, ny, 1, nz)
    {
        const int64_t o = I3(ix, iy, iz);
        const double d = pmax(-dke[o], 0.0) / (rho[o] * cv[o]);
        ee[o] += 0.5 * d;
        ei[o] += 0.5 * d;
    }
}

/* Offsets of +-1, +2 along a direction. */
#define STEP_OF(dir) ((dir) == 0 ? sy * sz : ((dir) == 1 ? sz : 1))

static void remap_sweep(lo_state *s, int dir)
{
    DIMS(s);
    const double dt = s->dt;
    const int64_t d1 = STEP_OF(dir);
    double *rho = s->f[SAMS_F_RHO], *ee = s->f[SAMS_F_ENERGY_ELECTRON], *ei = s->f[SAMS_F_ENERGY_ION];
    double *bx = s->f[SAMS_F_BX], *by = s->f[SAMS_F_BY], *bz = s->f[SAMS_F_BZ];
    double *vx = s->f[SAMS_F_VX], *vy = s->f[SAMS_F_VY], *vz = s->f[SAMS_F_VZ];
    double *v1d = s->f[SAMS_F_VX1 + dir];
    const double *vx1 = s->f[SAMS_F_VX1], *vy1 = s->f[SAMS_F_VY1], *vz1 = s->f[SAMS_F_VZ1];
    double *dm = s->f[SAMS_F_DM];
    double *cv1 = s->cv1, *cv2 = s->cv2, *cvc1 = s->cvc1, *db1 = s->db1, *rho1 = s->rho1;
    double *rv = s->r_rho_v, *rv1 = s->rho_v1, *flux = s->flux;
    const int64_t SX = sy * sz, SY = sz, SZ = 1;
    (void)SY; (void)SZ;

    for (int64_t o = 0; o < s->nbox; ++o) { dm[o] = 0.0; rho1[o] = rho[o]; }
    sweep_volumes(s, dir);

    /* ---- constrained transport of the two transverse field components ---- */
    /* First CT pair */
    if (dir == 0) {
        /* vx_by_flux xremap.cpp:269-319 */
        LOOP3(0, nx, 0, ny, 0, nz)
        {
            int64_t o = I3(ix, iy, iz), oy = SY;
            double v = (vx1[o] + vx1[I3(ix, iy, iz - 1)]) * 0.5;
            double dbm = (db1[o - d1] + db1[o - d1 + oy]) * 0.5, dbi = (db1[o] + db1[o + oy]) * 0.5;
            double dbp = (db1[o + d1] + db1[o + d1 + oy]) * 0.5, dbp2 = (db1[o + 2 * d1] + db1[o + 2 * d1 + oy]) * 0.5;
            flux[o] = ct_flux(v, dt, by[o - d1], by[o], by[o + d1], by[o + 2 * d1], dbm, dbi, dbp, dbp2,
                              cvc1[o], cvc1[o - d1], cvc1[o + d1], cv1[o], cv1[o + d1]);
        }
        LOOP3(1, nx, 0, ny, 1, nz) { int64_t o = I3(ix, iy, iz); by[o] = by[o] - flux[o] + flux[o - SX]; }
        LOOP3(0, nx, 1, ny, 1, nz) { int64_t o = I3(ix, iy, iz); bx[o] = bx[o] + flux[o] - flux[o - SY]; }
        /* vx_bz_flux xremap.cpp:321-371 */
        LOOP3(0, nx, 0, ny, 0, nz)
        {
            int64_t o = I3(ix, iy, iz);
            double v = (vx1[o] + vx1[I3(ix, iy - 1, iz)]) * 0.5;
            double dbm = (db1[o - d1] + db1[o - d1 + 1]) * 0.5, dbi = (db1[o] + db1[o + 1]) * 0.5;
            double dbp = (db1[o + d1] + db1[o + d1 + 1]) * 0.5, dbp2 = (db1[o + 2 * d1] + db1[o + 2 * d1 + 1]) * 0.5;
            flux[o] = ct_flux(v, dt, bz[o - d1], bz[o], bz[o + d1], bz[o + 2 * d1], dbm, dbi, dbp, dbp2,
                              cvc1[o], cvc1[o - d1], cvc1[o + d1], cv1[o], cv1[o + d1]);
        }
        LOOP3(1, nx, 1, ny, 0, nz) { int64_t o = I3(ix, iy, iz); bz[o] = bz[o] - flux[o] + flux[o - SX]; }
        LOOP3(0, nx, 1, ny, 1, nz) { int64_t o = I3(ix, iy, iz); bx[o] = bx[o] + flux[o] - flux[o - 1]; }
    } else if (dir == 1) {
        /* vy_bx_flux yremap.cpp:291-341 */
        LOOP3(0, nx, 0, ny, 0, nz)
        {
            int64_t o = I3(ix, iy, iz);
            double v = (vy1[o] + vy1[I3(ix, iy, iz - 1)]) * 0.5;
            double dbm = (db1[o - d1] + db1[o - d1 + SX]) * 0.5, dbi = (db1[o] + db1[o + SX]) * 0.5;
            double dbp = (db1[o + d1] + db1[o + d1 + SX]) * 0.5, dbp2 = (db1[o + 2 * d1] + db1[o + 2 * d1 + SX]) * 0.5;
            flux[o] = ct_flux(v, dt, bx[o - d1], bx[o], bx[o + d1], bx[o + 2 * d1], dbm, dbi, dbp, dbp2,
                              cvc1[o], cvc1[o - d1], cvc1[o + d1], cv1[o], cv1[o + d1]);
        }
        LOOP3(0, nx, 1, ny, 1, nz) { int64_t o = I3(ix, iy, iz); bx[o] = bx[o] - flux[o] + flux[o - SY]; }
        LOOP3(1, nx, 0, ny, 1, nz) { int64_t o = I3(ix, iy, iz); by[o] = by[o] + flux[o] - flux[o - SX]; }
        /* vy_bz_flux yremap.cpp:343-393 */
        LOOP3(0, nx, 0, ny, 0, nz)
        {
            int64_t o = I3(ix, iy, iz);
            double v = (vy1[o] + vy1[I3(ix - 1, iy, iz)]) * 0.5;
            double dbm = (db1[o - d1] + db1[o - d1 + 1]) * 0.5, dbi = (db1[o] + db1[o + 1]) * 0.5;
            double dbp = (db1[o + d1] + db1[o + d1 + 1]) * 0.5, dbp2 = (db1[o + 2 * d1] + db1[o + 2 * d1 + 1]) * 0.5;
            flux[o] = ct_flux(v, dt, bz[o - d1], bz[o], bz[o + d1], bz[o + 2 * d1], dbm, dbi, dbp, dbp2,
                              cvc1[o], cvc1[o - d1], cvc1[o + d1], cv1[o], cv1[o + d1]);
        }
        LOOP3(1, nx, 1, ny, 0, nz) { int64_t o = I3(ix, iy, iz); bz[o] = bz[o] - flux[o] + flux[o - SY]; }
        LOOP3(1, nx, 0, ny, 1, nz) { int64_t o = I3(ix, iy, iz); by[o] = by[o] + flux[o] - flux[o - 1]; }
    } else {
        /* vz_bx_flux zremap.cpp:249-299 */
        LOOP3(0, nx, 0, ny, 0, nz)
        {
            int64_t o = I3(ix, iy, iz);
            double v = (vz1[o] + vz1[I3(ix, iy - 1, iz)]) * 0.5;
            double dbm = (db1[o - d1] + db1[o - d1 + SX]) * 0.5, dbi = (db1[o] + db1[o + SX]) * 0.5;
            double dbp = (db1[o + d1] + db1[o + d1 + SX]) * 0.5, dbp2 = (db1[o + 2 * d1] + db1[o + 2 * d1 + SX]) * 0.5;
            flux[o] = ct_flux(v, dt, bx[o - d1], bx[o], bx[o + d1], bx[o + 2 * d1], dbm, dbi, dbp, dbp2,
                              cvc1[o], cvc1[o - d1], cvc1[o + d1], cv1[o], cv1[o + d1]);
        }
        LOOP3(0, nx, 1, ny, 1, nz) { int64_t o = I3(ix, iy, iz); bx[o] = bx[o] - flux[o] + flux[o - 1]; }
        LOOP3(1, nx, 1, ny, 0, nz) { int64_t o = I3(ix, iy, iz); bz[o] = bz[o] + flux[o] - flux[o - SX]; }
        /* vz_by_flux zremap.cpp:301-351 */
        LOOP3(0, nx, 0, ny, 0, nz)
        {
            int64_t o = I3(ix, iy, iz);
            double v = (vz1[o] + vz1[I3(ix - 1, iy, iz)]) * 0.5;
            double dbm = (db1[o - d1] + db1[o - d1 + SY]) * 0.5, dbi = (db1[o] + db1[o + SY]) * 0.5;
            double dbp = (db1[o + d1] + db1[o + d1 + SY]) * 0.5, dbp2 = (db1[o + 2 * d1] + db1[o + 2 * d1 + SY]) * 0.5;
            flux[o] = ct_flux(v, dt, by[o - d1], by[o], by[o + d1], by[o + 2 * d1], dbm, dbi, dbp, dbp2,
                              cvc1[o], cvc1[o - d1], cvc1[o + d1], cv1[o], cv1[o + d1]);
        }
        LOOP3(1, nx, 0, ny, 1, nz) { int64_t o = I3(ix, iy, iz); by[o] = by[o] - flux[o] + flux[o - 1]; }
        LOOP3(1, nx, 1, ny, 0, nz) { int64_t o = I3(ix, iy, iz); bz[o] = bz[o] + flux[o] - flux[o - SY]; }
    }

    /* ---- mass flux (x/y/z_mass_flux) ---- */
    const double *area_c = dir == 0 ? s->dxab : (dir == 1 ? s->dyab : s->dzab);
    {
        int64_t ihi = dir == 0 ? nx : nx + 1, jhi = dir == 1 ? ny : ny + 1, khi = dir == 2 ? nz : nz + 1;
        LOOP3(0, ihi, 0, jhi, 0, khi)
        {
            int64_t o = I3(ix, iy, iz);
            double v;
            if (dir == 0)
                v = (vx1[o] + vx1[I3(ix, iy - 1, iz)] + vx1[I3(ix, iy, iz - 1)] + vx1[I3(ix, iy - 1, iz - 1)]) * 0.25;
            else if (dir == 1)
                v = (vy1[I3(ix - 1, iy, iz)] + vy1[o] + vy1[I3(ix - 1, iy, iz - 1)] + vy1[I3(ix, iy, iz - 1)]) * 0.25;
            else
                v = (vz1[I3(ix - 1, iy, iz)] + vz1[o] + vz1[I3(ix - 1, iy - 1, iz)] + vz1[I3(ix, iy - 1, iz)]) * 0.25;
            dm[o] = mass_flux(v, dt, area_c[o], rho[o - d1], rho[o], rho[o + d1], rho[o + 2 * d1],
                              cvc1[o], cvc1[o - d1], cvc1[o + d1], cv1[o], cv1[o + d1]);
        }
    }
    bc_dim(s, SAMS_F_DM, dir); /* dm_{x,y,z}_bcs */
    LOOP3(1, nx, 1, ny, 1, nz)
    {
        int64_t o = I3(ix, iy, iz);
        rho[o] = (rho1[o] * cv1[o] + dm[o - d1] - dm[o]) / cv2[o];
    }
    /* ---- energy fluxes ---- */
    for (int which = 0; which < 2; ++which) {
        double *e = which == 0 ? ee : ei;
        LOOP3(0, nx, 0, ny, 0, nz)
        {
            int64_t o = I3(ix, iy, iz);
            double v;
            if (dir == 0)
                v = (vx1[o] + vx1[I3(ix, iy - 1, iz)] + vx1[I3(ix, iy, iz - 1)] + vx1[I3(ix, iy - 1, iz - 1)]) * 0.25;
            else if (dir == 1)
                v = (vy1[I3(ix - 1, iy, iz)] + vy1[o] + vy1[I3(ix - 1, iy, iz - 1)] + vy1[I3(ix, iy, iz - 1)]) * 0.25;
            else
                v = (vz1[I3(ix - 1, iy, iz)] + vz1[o] + vz1[I3(ix - 1, iy - 1, iz)] + vz1[I3(ix, iy - 1, iz)]) * 0.25;
            flux[o] = energy_flux(v, dt, area_c[o], e[o - d1], e[o], e[o + d1], e[o + 2 * d1],
                                  cvc1[o], cvc1[o - d1], cvc1[o + d1], cv1[o], cv1[o + d1],
                                  rho1[o], rho1[o + d1], dm[o]);
        }
        LOOP3(1, nx, 1, ny, 1, nz)
        {
            int64_t o = I3(ix, iy, iz);
            e[o] = (e[o] * cv1[o] * rho1[o] + flux[o - d1] - flux[o]) / (cv2[o] * rho[o]);
        }
    }
    /* ---- vertex quantities ---- */
    {
        int64_t ilo = dir == 0 ? -1 : 0, ihi = dir == 0 ? nx + 1 : nx;
        int64_t jlo = dir == 1 ? -1 : 0, jhi = dir == 1 ? ny + 1 : ny;
        int64_t klo = dir == 2 ? -1 : 0, khi = dir == 2 ? nz + 1 : nz;
        LOOP3(ilo, ihi, jlo, jhi, klo, khi)
        {
            int64_t ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
            double sum = rho1[I3(ix, iy, iz)] * cv1[I3(ix, iy, iz)] +
                         rho1[I3(ixp, iy, iz)] * cv1[I3(ixp, iy, iz)] +
                         rho1[I3(ix, iyp, iz)] * cv1[I3(ix, iyp, iz)] +
                         rho1[I3(ixp, iyp, iz)] * cv1[I3(ixp, iyp, iz)] +
                         rho1[I3(ix, iy, izp)] * cv1[I3(ix, iy, izp)] +
                         rho1[I3(ixp, iy, izp)] * cv1[I3(ixp, iy, izp)] +
                         rho1[I3(ix, iyp, izp)] * cv1[I3(ix, iyp, izp)] +
                         rho1[I3(ixp, iyp, izp)] * cv1[I3(ixp, iyp, izp)];
            int64_t o = I3(ix, iy, iz);
            if (dir == 0)
                rv[o] = sum * 0.125 / cvc1[o];   /* xremap.cpp:166-174 */
            else
                rv[o] = sum * (0.125 / cvc1[o]); /* yremap.cpp:190, zremap.cpp:163 */
        }
    }
    LOOP3(0, nx, 0, ny, 0, nz)
    {
        int64_t ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
        flux[I3(ix, iy, iz)] = (cv2[I3(ix, iy, iz)] + cv2[I3(ixp, iy, iz)] + cv2[I3(ix, iyp, iz)] + cv2[I3(ixp, iyp, iz)] +
                                cv2[I3(ix, iy, izp)] + cv2[I3(ixp, iy, izp)] + cv2[I3(ix, iyp, izp)] + cv2[I3(ixp, iyp, izp)]) * 0.125;
    }
    LOOP3(0, nx, 0, ny, 0, nz) { int64_t o = I3(ix, iy, iz); cv2[o] = flux[o]; }
    {
        /* shift the sweep-direction v1 to the face centre */
        int64_t ilo = dir == 0 ? -2 : 0, ihi = dir == 0 ? nx + 1 : nx;
        int64_t jlo = dir == 1 ? -2 : 0, jhi = dir == 1 ? ny + 1 : ny;
        int64_t klo = dir == 2 ? -2 : 0, khi = dir == 2 ? nz + 1 : nz;
        LOOP3(ilo, ihi, jlo, jhi, klo, khi) { int64_t o = I3(ix, iy, iz); flux[o] = (v1d[o] + v1d[o + d1]) * 0.5; }
        LOOP3(ilo, ihi, jlo, jhi, klo, khi) { int64_t o = I3(ix, iy, iz); v1d[o] = flux[o]; }
    }
    {
        /* node mass flux */
        int64_t ilo = dir == 0 ? -1 : 0, jlo = dir == 1 ? -1 : 0, klo = dir == 2 ? -1 : 0;
        LOOP3(ilo, nx, jlo, ny, klo, nz)
        {
            int64_t ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
            flux[I3(ix, iy, iz)] = (dm[I3(ix, iy, iz)] + dm[I3(ixp, iy, iz)] + dm[I3(ix, iyp, iz)] + dm[I3(ixp, iyp, iz)] +
                                    dm[I3(ix, iy, izp)] + dm[I3(ixp, iy, izp)] + dm[I3(ix, iyp, izp)] + dm[I3(ixp, iyp, izp)]) * 0.125;
        }
        LOOP3(ilo, nx, jlo, ny, klo, nz) { int64_t o = I3(ix, iy, iz); dm[o] = flux[o]; }
    }
    {
        int64_t klo = dir == 2 ? -1 : 0, khi = dir == 2 ? nz + 1 : nz;
        LOOP3(0, nx, 0, ny, klo, khi)
        {
            int64_t o = I3(ix, iy, iz);
            rv1[o] = (rv[o] * cvc1[o] + dm[o - d1] - dm[o]) / cv2[o];
        }
    }
    /* ---- momentum fluxes ---- */
    const double *area_n = dir == 0 ? s->dxac : s->dyac; /* zremap.cpp:475 uses dyac */
    double *vel[3] = {vx, vy, vz};
    for (int c = 0; c < 3; ++c) {
        double *u = vel[c];
        int64_t ilo = dir == 0 ? -1 : 0, jlo = dir == 1 ? -1 : 0, klo = dir == 2 ? -1 : 0;
        LOOP3(ilo, nx, jlo, ny, klo, nz)
        {
            int64_t o = I3(ix, iy, iz);
            flux[o] = mom_flux(v1d[o], dt, area_n[o], u[o - d1], u[o], u[o + d1], u[o + 2 * d1],
                               cv1[o + d1], cv1[o], cv1[o + 2 * d1], cvc1[o], cvc1[o + d1],
                               rv[o], rv[o + d1], dm[o], dir == 2);
        }
        if (s->p.rke) rke_scatter(s, dir, u);
        LOOP3(ilo, nx, jlo, ny, klo, nz) { int64_t o = I3(ix, iy, iz); flux[o] *= dm[o]; }
        LOOP3(0, nx, 0, ny, 0, nz)
        {
            int64_t o = I3(ix, iy, iz);
            u[o] = (rv[o] * u[o] * cvc1[o] + flux[o - d1] - flux[o]) / (cv2[o] * rv1[o]);
        }
    }
    if (dir == 0) s->xpass = 0.0;
    if (dir == 1) s->ypass = 0.0;
    if (dir == 2) s->zpass = 0.0;
    boundary_conditions(s);
}

/* remap.cpp:23-111 */
static void eulerian_remap(lo_state *s)
{
    DIMS(s);
    double *bx = s->f[SAMS_F_BX], *by = s->f[SAMS_F_BY], *bz = s->f[SAMS_F_BZ];
    if (s->p.rke) memset(s->delta_ke, 0, (size_t)s->nbox * sizeof(double)); /* remap.cpp:38-41 */
    s->xpass = s->ypass = s->zpass = 1.0;
    LOOP3(-2, nx + 2, -1, ny + 2, -1, nz + 2) { int64_t o = I3(ix, iy, iz); bx[o] *= s->dxab[o]; }
    LOOP3(-1, nx + 2, -2, ny + 2, -1, nz + 2) { int64_t o = I3(ix, iy, iz); by[o] *= s->dyab[o]; }
    LOOP3(-1, nx + 2, -1, ny + 2, -2, nz + 2) { int64_t o = I3(ix, iy, iz); bz[o] *= s->dzab[o]; }
    /* data.step is never advanced (remap.cpp:52), so the order is always x, y, z */
    remap_sweep(s, 0);
    remap_sweep(s, 1);
    remap_sweep(s, 2);
    LOOP3(-2, nx + 2, -1, ny + 2, -1, nz + 2) { int64_t o = I3(ix, iy, iz); bx[o] /= (s->dxab[o] + NONE_ZERO); }
    LOOP3(-1, nx + 2, -2, ny + 2, -1, nz + 2) { int64_t o = I3(ix, iy, iz); by[o] /= (s->dyab[o] + NONE_ZERO); }
    LOOP3(-1, nx + 2, -1, ny + 2, -2, nz + 2) { int64_t o = I3(ix, iy, iz); bz[o] /= (s->dzab[o] + NONE_ZERO); }
    bfield_bcs(s);
}

/* ------------------------------------------------------------------ */

#define ALLOC_BOX(name) do { s->name = (double *)calloc((size_t)s->nbox, sizeof(double)); if (!s->name) goto fail; } while (0)
#define ALLOC_AX(name, n) do { s->name = (double *)calloc((size_t)((n) + 5), sizeof(double)); if (!s->name) goto fail; } while (0)
#define ALLOC_PLANE(name) do { s->name = (double *)calloc((size_t)((p->nx + 5) * (p->ny + 5)), sizeof(double)); if (!s->name) goto fail; } while (0)

lo_state *lo_create(const sams_lare_params *p, const sams_lare_bcs *bcs)
{
    if (!p || !bcs || p->nx < 1 || p->ny < 1 || p->nz < 1 || p->geometry < 0 || p->geometry > 2) return NULL;
    lo_state *s = (lo_state *)calloc(1, sizeof(lo_state));
    if (!s) return NULL;
    s->p = *p;
    s->bcs = *bcs;
    s->nx = p->nx; s->ny = p->ny; s->nz = p->nz;
    s->nbox = sams_box_elems(p->nx, p->ny, p->nz);
    for (int f = 0; f < SAMS_NFIELDS; ++f) {
        s->f[f] = (double *)calloc((size_t)s->nbox, sizeof(double));
        if (!s->f[f]) goto fail;
    }
    ALLOC_BOX(cv); ALLOC_BOX(cvc); ALLOC_BOX(dxab); ALLOC_BOX(dyab); ALLOC_BOX(dzab);
    ALLOC_BOX(dxac); ALLOC_BOX(dyac); ALLOC_BOX(dzac);
    ALLOC_AX(xb, p->nx); ALLOC_AX(xc, p->nx); ALLOC_AX(dxb, p->nx); ALLOC_AX(dxc, p->nx);
    ALLOC_AX(yb, p->ny); ALLOC_AX(yc, p->ny); ALLOC_AX(dyb, p->ny); ALLOC_AX(dyc, p->ny);
    ALLOC_AX(zb, p->nz); ALLOC_AX(zc, p->nz); ALLOC_AX(dzb, p->nz); ALLOC_AX(dzc, p->nz);
    ALLOC_AX(hy, p->nx); ALLOC_AX(hyc, p->nx); ALLOC_AX(hyv, p->nx); ALLOC_AX(cot_yb, p->ny);
    ALLOC_PLANE(hz); ALLOC_PLANE(hz1); ALLOC_PLANE(hz2); ALLOC_PLANE(hzc);
    ALLOC_BOX(p_visc); ALLOC_BOX(visc_heat); ALLOC_BOX(alpha1); ALLOC_BOX(alpha2); ALLOC_BOX(alpha3);
    ALLOC_BOX(pressure); ALLOC_BOX(p_e); ALLOC_BOX(p_i); ALLOC_BOX(rho_v); ALLOC_BOX(cv_v);
    ALLOC_BOX(fx); ALLOC_BOX(fy); ALLOC_BOX(fz); ALLOC_BOX(fx_visc); ALLOC_BOX(fy_visc); ALLOC_BOX(fz_visc);
    ALLOC_BOX(bx1); ALLOC_BOX(by1); ALLOC_BOX(bz1); ALLOC_BOX(cv1); ALLOC_BOX(eta);
    ALLOC_BOX(flux_x); ALLOC_BOX(flux_y); ALLOC_BOX(flux_z); ALLOC_BOX(curlb); ALLOC_BOX(cs); ALLOC_BOX(cs_v);
    ALLOC_BOX(rho1); ALLOC_BOX(cv2); ALLOC_BOX(cvc1); ALLOC_BOX(db1); ALLOC_BOX(r_rho_v); ALLOC_BOX(rho_v1); ALLOC_BOX(flux);
    ALLOC_BOX(delta_ke);
    build_grid(s);
    s->dt = 0.0; /* the runner's value-initialised data pack: dt = 0 before the first step */
    s->time = 0.0;
    s->step = 0;
    return s;
fail:
    lo_destroy(s);
    return NULL;
}

void lo_destroy(lo_state *s)
{
    if (!s) return;
    for (int f = 0; f < SAMS_NFIELDS; ++f) free(s->f[f]);
    double *arrs[] = {s->cv, s->cvc, s->dxab, s->dyab, s->dzab, s->dxac, s->dyac, s->dzac,
                      s->xb, s->yb, s->zb, s->xc, s->yc, s->zc, s->dxb, s->dyb, s->dzb, s->dxc, s->dyc, s->dzc,
                      s->hy, s->hyc, s->hyv, s->cot_yb, s->hz, s->hz1, s->hz2, s->hzc,
                      s->p_visc, s->visc_heat, s->alpha1, s->alpha2, s->alpha3, s->pressure, s->p_e, s->p_i,
                      s->rho_v, s->cv_v, s->fx, s->fy, s->fz, s->fx_visc, s->fy_visc, s->fz_visc,
                      s->bx1, s->by1, s->bz1, s->cv1, s->eta, s->flux_x, s->flux_y, s->flux_z, s->curlb,
                      s->cs, s->cs_v, s->rho1, s->cv2, s->cvc1, s->db1, s->r_rho_v, s->rho_v1, s->flux,
                      s->delta_ke};
    for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); ++i) free(arrs[i]);
    free(s);
}

int lo_set_fields(lo_state *s, const double *const fields[SAMS_NFIELDS])
{
    if (!s) return -1;
    for (int f = 0; f < SAMS_NFIELDS; ++f) {
        if (!fields[f]) return -1;
        memcpy(s->f[f], fields[f], (size_t)s->nbox * sizeof(double));
    }
    return 0;
}

int lo_get_field(lo_state *s, int field, double *out)
{
    if (!s || field < 0 || field >= SAMS_NFIELDS || !out) return -1;
    memcpy(out, s->f[field], (size_t)s->nbox * sizeof(double));
    return 0;
}

int lo_get_named(lo_state *s, const char *name, double *out)
{
    if (!s || !name || !out) return -1;
    struct { const char *n; double *a; } tab[] = {
        {"p_visc", s->p_visc}, {"visc_heat", s->visc_heat}, {"alpha1", s->alpha1}, {"alpha2", s->alpha2},
        {"alpha3", s->alpha3}, {"pressure", s->pressure}, {"p_e", s->p_e}, {"p_i", s->p_i},
        {"rho_v", s->rho_v}, {"cv_v", s->cv_v}, {"fx", s->fx}, {"fy", s->fy}, {"fz", s->fz},
        {"fx_visc", s->fx_visc}, {"fy_visc", s->fy_visc}, {"fz_visc", s->fz_visc},
        {"bx1", s->bx1}, {"by1", s->by1}, {"bz1", s->bz1}, {"cv1", s->cv1}, {"eta", s->eta},
        {"cv", s->cv}, {"cvc", s->cvc}, {"dxab", s->dxab}, {"dyab", s->dyab}, {"dzab", s->dzab},
        {"dxac", s->dxac}, {"dyac", s->dyac}, {"dzac", s->dzac}};
    for (size_t i = 0; i < sizeof(tab) / sizeof(tab[0]); ++i)
        if (strcmp(tab[i].n, name) == 0) {
            memcpy(out, tab[i].a, (size_t)s->nbox * sizeof(double));
            return 0;
        }
    /* 1-D axes: copied into out[0 .. n+4] */
    struct { const char *n; double *a; int64_t len; } ax[] = {
        {"xb", s->xb, s->nx + 5}, {"yb", s->yb, s->ny + 5}, {"zb", s->zb, s->nz + 5},
        {"xc", s->xc, s->nx + 5}, {"yc", s->yc, s->ny + 5}, {"zc", s->zc, s->nz + 5},
        {"dxb", s->dxb, s->nx + 5}, {"dyb", s->dyb, s->ny + 5}, {"dzb", s->dzb, s->nz + 5},
        {"dxc", s->dxc, s->nx + 5}, {"dyc", s->dyc, s->ny + 5}, {"dzc", s->dzc, s->nz + 5}};
    for (size_t i = 0; i < sizeof(ax) / sizeof(ax[0]); ++i)
        if (strcmp(ax[i].n, name) == 0) {
            memcpy(out, ax[i].a, (size_t)ax[i].len * sizeof(double));
            return 0;
        }
    return -2;
}

int lo_step_phase(lo_state *s, int phase)
{
    if (!s) return -1;
    lagrangian_step(s);
    if (phase == 0) return 0;
    corrector_step(s);
    if (phase == 1) return 0;
    s->step++;
    s->time += s->dt;
    eulerian_remap(s);
    if (s->p.rke) energy_correction(s);
    eta_calc(s);
    return 0;
}

int lo_step(lo_state *s, int64_t nsteps)
{
    if (!s) return -1;
    for (int64_t i = 0; i < nsteps; ++i) lo_step_phase(s, 2);
    return 0;
}

double lo_dt(const lo_state *s) { return s ? s->dt : 0.0; }
double lo_time(const lo_state *s) { return s ? s->time : 0.0; }
int64_t lo_steps(const lo_state *s) { return s ? s->step : 0; }
