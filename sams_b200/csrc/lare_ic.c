/*
 * lare_ic.c -- initial-condition generators for the LARE3D workloads
 * (declarations and conventions in include/sams_lare_ic.h).
 *
 * Compiled with -ffp-contract=off and no -ffast-math wherever it is built
 * (product library, CPU checker, reference harness) so every build produces
 * bit-identical fields from the same arguments.
 */
#include "sams_lare_ic.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

double sams_axis_edge(double lo, double hi, int64_t n, int64_t i)
{
    /* axisRegistry::setDomain: delta = (max-min)/(edges-1), edges = n+1;
     * createLinearAxis: lowerBound + delta * i. */
    double d = (hi - lo) / (double)n;
    return lo + d * (double)i;
}

double sams_axis_centre(double lo, double hi, int64_t n, int64_t i)
{
    /* createCentredAxis: 0.5 * (b(i) + b(i-1)). */
    return 0.5 * (sams_axis_edge(lo, hi, n, i) + sams_axis_edge(lo, hi, n, i - 1));
}

static uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

double sams_ic_uniform(uint64_t seed, uint64_t stream, uint64_t counter)
{
    uint64_t h = splitmix64(seed ^ splitmix64(stream * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull));
    h = splitmix64(h ^ (counter * 0x9E3779B97F4A7C15ull));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

static int check_grid(const sams_lare_grid *g, double *const fields[SAMS_NFIELDS])
{
    if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1) return -1;
    if (!(g->x_max > g->x_min) || !(g->y_max > g->y_min) || !(g->z_max > g->z_min)) return -1;
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        if (!fields[f]) return -1;
    return 0;
}

static void zero_all(const sams_lare_grid *g, double *const fields[SAMS_NFIELDS])
{
    int64_t n = sams_box_elems(g->nx, g->ny, g->nz);
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        memset(fields[f], 0, (size_t)n * sizeof(double));
}

/* Loop bounds of field f in dimension d. */
#define FLB(f, d) sams_lare_field_lb((f), (d))

int sams_ic_orszag_tang(const sams_lare_grid *g, double gamma, double B0,
                        double *const fields[SAMS_NFIELDS])
{
    if (check_grid(g, fields)) return -1;
    zero_all(g, fields);
    const int64_t nx = g->nx, ny = g->ny, nz = g->nz;
    const double rho0 = 25.0 / (36.0 * M_PI);
    const double p0 = 5.0 / (12.0 * M_PI);
    const double e0 = p0 / ((gamma - 1.0) * rho0) / 2.0;
    const double twopi = 2.0 * M_PI;

    for (int64_t i = -1; i <= nx + 2; ++i)
        for (int64_t j = -1; j <= ny + 2; ++j)
            for (int64_t k = -1; k <= nz + 2; ++k) {
                int64_t o = sams_box_index(ny, nz, i, j, k);
                fields[SAMS_F_RHO][o] = rho0;
                fields[SAMS_F_ENERGY_ELECTRON][o] = e0;
                fields[SAMS_F_ENERGY_ION][o] = e0;
            }
    for (int64_t i = -2; i <= nx + 2; ++i) {
        double xb = sams_axis_edge(g->x_min, g->x_max, nx, i);
        double vy = sin(twopi * xb);
        for (int64_t j = -2; j <= ny + 2; ++j) {
            double yb = sams_axis_edge(g->y_min, g->y_max, ny, j);
            double vx = -sin(twopi * yb);
            for (int64_t k = -2; k <= nz + 2; ++k) {
                int64_t o = sams_box_index(ny, nz, i, j, k);
                fields[SAMS_F_VX][o] = vx;
                fields[SAMS_F_VY][o] = vy;
            }
        }
    }
    /* bx on x faces (xb, yc, zc) */
    for (int64_t i = FLB(SAMS_F_BX, 0); i <= nx + 2; ++i)
        for (int64_t j = -1; j <= ny + 2; ++j) {
            double yc = sams_axis_centre(g->y_min, g->y_max, ny, j);
            double bx = -B0 * sin(twopi * yc);
            for (int64_t k = -1; k <= nz + 2; ++k)
                fields[SAMS_F_BX][sams_box_index(ny, nz, i, j, k)] = bx;
        }
    /* by on y faces (xc, yb, zc) */
    for (int64_t i = -1; i <= nx + 2; ++i) {
        double xc = sams_axis_centre(g->x_min, g->x_max, nx, i);
        double by = B0 * sin(2.0 * twopi * xc);
        for (int64_t j = FLB(SAMS_F_BY, 1); j <= ny + 2; ++j)
            for (int64_t k = -1; k <= nz + 2; ++k)
                fields[SAMS_F_BY][sams_box_index(ny, nz, i, j, k)] = by;
    }
    return 0;
}

/* One Fourier mode: integer wavevector, unit polarisation, phase, amplitude. */
typedef struct {
    int kx, ky, kz;
    double ex, ey, ez;
    double phase, amp, cp, sp;
} ic_mode;

static int draw_modes(uint64_t seed, uint64_t stream, int kmax, int per_shell,
                      double amp_power, ic_mode *modes)
{
    uint64_t ctr = 0;
    int m = 0;
    for (int s = 1; s <= kmax; ++s) {
        for (int q = 0; q < per_shell; ++q) {
            ic_mode md;
            for (;;) {
                int kx = (int)floor(sams_ic_uniform(seed, stream, ctr++) * (2 * s + 1)) - s;
                int ky = (int)floor(sams_ic_uniform(seed, stream, ctr++) * (2 * s + 1)) - s;
                int kz = (int)floor(sams_ic_uniform(seed, stream, ctr++) * (2 * s + 1)) - s;
                double kk = sqrt((double)(kx * kx + ky * ky + kz * kz));
                if (kk >= s - 0.5 && kk < s + 0.5 && kk >= 1.0) {
                    md.kx = kx; md.ky = ky; md.kz = kz;
                    break;
                }
            }
            for (;;) {
                double a = 2.0 * sams_ic_uniform(seed, stream, ctr++) - 1.0;
                double b = 2.0 * sams_ic_uniform(seed, stream, ctr++) - 1.0;
                double c = 2.0 * sams_ic_uniform(seed, stream, ctr++) - 1.0;
                double r = sqrt(a * a + b * b + c * c);
                if (r > 0.1 && r <= 1.0) {
                    md.ex = a / r; md.ey = b / r; md.ez = c / r;
                    break;
                }
            }
            md.phase = 2.0 * M_PI * sams_ic_uniform(seed, stream, ctr++);
            md.cp = cos(md.phase);
            md.sp = sin(md.phase);
            md.amp = pow((double)s, amp_power);
            modes[m++] = md;
        }
    }
    return m;
}

/* Per-axis phase tables: cos/sin of 2 pi k (x - min)/L for every mode and
 * every index -3..n+2 at edge (b) and centred (c) positions. */
typedef struct {
    int64_t n, off;        /* off = 3: index i lives at [i + off] */
    double *cb, *sb, *cc, *sc;
} axis_tab;

static int axis_tab_build(axis_tab *t, int nm, const ic_mode *modes, int comp,
                          double lo, double hi, int64_t n)
{
    t->n = n; t->off = 3;
    int64_t len = n + 6;
    size_t sz = (size_t)nm * (size_t)len * sizeof(double);
    t->cb = (double *)malloc(sz); t->sb = (double *)malloc(sz);
    t->cc = (double *)malloc(sz); t->sc = (double *)malloc(sz);
    if (!t->cb || !t->sb || !t->cc || !t->sc) return -1;
    double L = hi - lo;
    for (int m = 0; m < nm; ++m) {
        int k = comp == 0 ? modes[m].kx : (comp == 1 ? modes[m].ky : modes[m].kz);
        for (int64_t i = -3; i <= n + 2; ++i) {
            double xb = sams_axis_edge(lo, hi, n, i);
            double xc = sams_axis_centre(lo, hi, n, i);
            double ab = 2.0 * M_PI * (double)k * ((xb - lo) / L);
            double ac = 2.0 * M_PI * (double)k * ((xc - lo) / L);
            size_t o = (size_t)m * (size_t)len + (size_t)(i + 3);
            t->cb[o] = cos(ab); t->sb[o] = sin(ab);
            t->cc[o] = cos(ac); t->sc[o] = sin(ac);
        }
    }
    return 0;
}

static void axis_tab_free(axis_tab *t)
{
    free(t->cb); free(t->sb); free(t->cc); free(t->sc);
}

/* Sum over modes of amp * e_comp * cos(phase + phi_x + phi_y + phi_z), with
 * the per-axis angles taken at edge (1) or centred (0) positions. */
static double mode_sum(int nm, const ic_mode *modes, int comp,
                       const axis_tab *tx, int xb, int64_t i,
                       const axis_tab *ty, int yb, int64_t j,
                       const axis_tab *tz, int zb, int64_t k)
{
    double acc = 0.0;
    int64_t lx = tx->n + 6, ly = ty->n + 6, lz = tz->n + 6;
    for (int m = 0; m < nm; ++m) {
        size_t ox = (size_t)m * lx + (size_t)(i + 3);
        size_t oy = (size_t)m * ly + (size_t)(j + 3);
        size_t oz = (size_t)m * lz + (size_t)(k + 3);
        double cx = xb ? tx->cb[ox] : tx->cc[ox], sx = xb ? tx->sb[ox] : tx->sc[ox];
        double cy = yb ? ty->cb[oy] : ty->cc[oy], sy = yb ? ty->sb[oy] : ty->sc[oy];
        double cz = zb ? tz->cb[oz] : tz->cc[oz], sz = zb ? tz->sb[oz] : tz->sc[oz];
        /* e^{i(ax+ay)} */
        double cxy = cx * cy - sx * sy, sxy = sx * cy + cx * sy;
        double cxyz = cxy * cz - sxy * sz, sxyz = sxy * cz + cxy * sz;
        double re = cxyz * modes[m].cp - sxyz * modes[m].sp;
        double e = comp == 0 ? modes[m].ex : (comp == 1 ? modes[m].ey : modes[m].ez);
        acc += modes[m].amp * e * re;
    }
    return acc;
}

int sams_ic_random_field(const sams_lare_grid *g, double gamma, uint64_t seed,
                         int kmax, int modes_per_shell, double b_rms,
                         double v_rms, double rho0, double p0,
                         double *const fields[SAMS_NFIELDS])
{
    if (check_grid(g, fields) || kmax < 1 || modes_per_shell < 1) return -1;
    zero_all(g, fields);
    const int64_t nx = g->nx, ny = g->ny, nz = g->nz;
    const int nmax = kmax * modes_per_shell;
    ic_mode *am = (ic_mode *)malloc(sizeof(ic_mode) * (size_t)nmax);
    ic_mode *vm = (ic_mode *)malloc(sizeof(ic_mode) * (size_t)nmax);
    if (!am || !vm) { free(am); free(vm); return -2; }
    int na = draw_modes(seed, 1, kmax, modes_per_shell, -2.0, am);
    int nv = draw_modes(seed, 2, kmax, modes_per_shell, -1.0, vm);

    axis_tab ax, ay, az, vx_t, vy_t, vz_t;
    if (axis_tab_build(&ax, na, am, 0, g->x_min, g->x_max, nx) ||
        axis_tab_build(&ay, na, am, 1, g->y_min, g->y_max, ny) ||
        axis_tab_build(&az, na, am, 2, g->z_min, g->z_max, nz) ||
        axis_tab_build(&vx_t, nv, vm, 0, g->x_min, g->x_max, nx) ||
        axis_tab_build(&vy_t, nv, vm, 1, g->y_min, g->y_max, ny) ||
        axis_tab_build(&vz_t, nv, vm, 2, g->z_min, g->z_max, nz)) {
        free(am); free(vm);
        return -2;
    }

    /* Vector potential on cell edges, index range -3..n+2 per dimension:
     * Ax at (xc, yb, zb), Ay at (xb, yc, zb), Az at (xb, yb, zc). */
    const int64_t ex = nx + 6, ey = ny + 6, ez = nz + 6;
    size_t asz = (size_t)ex * ey * ez;
    double *A[3];
    for (int c = 0; c < 3; ++c) {
        A[c] = (double *)malloc(asz * sizeof(double));
        if (!A[c]) return -2;
    }
#define AIX(i, j, k) ((((size_t)((i) + 3)) * ey + (size_t)((j) + 3)) * ez + (size_t)((k) + 3))
#pragma omp parallel for schedule(static)
    for (int64_t i = -3; i <= nx + 2; ++i)
        for (int64_t j = -3; j <= ny + 2; ++j)
            for (int64_t k = -3; k <= nz + 2; ++k) {
                size_t o = AIX(i, j, k);
                A[0][o] = mode_sum(na, am, 0, &ax, 0, i, &ay, 1, j, &az, 1, k);
                A[1][o] = mode_sum(na, am, 1, &ax, 1, i, &ay, 0, j, &az, 1, k);
                A[2][o] = mode_sum(na, am, 2, &ax, 1, i, &ay, 1, j, &az, 0, k);
            }

    /* B = curl A on faces, differences divided by the edge spacing. */
    const double dx = (g->x_max - g->x_min) / (double)nx;
    const double dy = (g->y_max - g->y_min) / (double)ny;
    const double dz = (g->z_max - g->z_min) / (double)nz;
    double *bx = fields[SAMS_F_BX], *by = fields[SAMS_F_BY], *bz = fields[SAMS_F_BZ];
#pragma omp parallel for schedule(static)
    for (int64_t i = -2; i <= nx + 2; ++i)
        for (int64_t j = -2; j <= ny + 2; ++j)
            for (int64_t k = -2; k <= nz + 2; ++k) {
                int64_t o = sams_box_index(ny, nz, i, j, k);
                bx[o] = (A[2][AIX(i, j, k)] - A[2][AIX(i, j - 1, k)]) / dy -
                        (A[1][AIX(i, j, k)] - A[1][AIX(i, j, k - 1)]) / dz;
                by[o] = (A[0][AIX(i, j, k)] - A[0][AIX(i, j, k - 1)]) / dz -
                        (A[2][AIX(i, j, k)] - A[2][AIX(i - 1, j, k)]) / dx;
                bz[o] = (A[1][AIX(i, j, k)] - A[1][AIX(i - 1, j, k)]) / dx -
                        (A[0][AIX(i, j, k)] - A[0][AIX(i, j - 1, k)]) / dy;
            }
#undef AIX
    for (int c = 0; c < 3; ++c) free(A[c]);

    /* Normalise: mean over interior indices 1..n of bx^2 + by^2 + bz^2,
     * summed in a fixed order. */
    double sb = 0.0;
    for (int64_t i = 1; i <= nx; ++i) {
        double si = 0.0;
        for (int64_t j = 1; j <= ny; ++j)
            for (int64_t k = 1; k <= nz; ++k) {
                int64_t o = sams_box_index(ny, nz, i, j, k);
                si += bx[o] * bx[o] + by[o] * by[o] + bz[o] * bz[o];
            }
        sb += si;
    }
    double ncell = (double)nx * (double)ny * (double)nz;
    double bscale = sb > 0.0 ? b_rms / sqrt(sb / ncell) : 0.0;

    /* Centred fields are defined on -1..n+2; staggered B components keep
     * their -2 layer along their own axis only. */
    const double e0 = p0 / ((gamma - 1.0) * rho0) / 2.0;
    for (int64_t i = -2; i <= nx + 2; ++i)
        for (int64_t j = -2; j <= ny + 2; ++j)
            for (int64_t k = -2; k <= nz + 2; ++k) {
                int64_t o = sams_box_index(ny, nz, i, j, k);
                int inc = (i >= -1) && (j >= -1) && (k >= -1);
                bx[o] = ((j >= -1) && (k >= -1)) ? bx[o] * bscale : 0.0;
                by[o] = ((i >= -1) && (k >= -1)) ? by[o] * bscale : 0.0;
                bz[o] = ((i >= -1) && (j >= -1)) ? bz[o] * bscale : 0.0;
                if (inc) {
                    fields[SAMS_F_RHO][o] = rho0;
                    fields[SAMS_F_ENERGY_ELECTRON][o] = e0;
                    fields[SAMS_F_ENERGY_ION][o] = e0;
                }
            }

    /* Node velocity. */
    double *v[3] = {fields[SAMS_F_VX], fields[SAMS_F_VY], fields[SAMS_F_VZ]};
#pragma omp parallel for schedule(static)
    for (int64_t i = -2; i <= nx + 2; ++i)
        for (int64_t j = -2; j <= ny + 2; ++j)
            for (int64_t k = -2; k <= nz + 2; ++k) {
                int64_t o = sams_box_index(ny, nz, i, j, k);
                for (int c = 0; c < 3; ++c)
                    v[c][o] = mode_sum(nv, vm, c, &vx_t, 1, i, &vy_t, 1, j, &vz_t, 1, k);
            }
    double sv = 0.0;
    for (int64_t i = 1; i <= nx; ++i) {
        double si = 0.0;
        for (int64_t j = 1; j <= ny; ++j)
            for (int64_t k = 1; k <= nz; ++k) {
                int64_t o = sams_box_index(ny, nz, i, j, k);
                si += v[0][o] * v[0][o] + v[1][o] * v[1][o] + v[2][o] * v[2][o];
            }
        sv += si;
    }
    double vscale = sv > 0.0 ? v_rms / sqrt(sv / ncell) : 0.0;
    int64_t n = sams_box_elems(nx, ny, nz);
    for (int c = 0; c < 3; ++c)
        for (int64_t o = 0; o < n; ++o) v[c][o] *= vscale;

    axis_tab_free(&ax); axis_tab_free(&ay); axis_tab_free(&az);
    axis_tab_free(&vx_t); axis_tab_free(&vy_t); axis_tab_free(&vz_t);
    free(am); free(vm);
    return 0;
}

int sams_ic_harris(const sams_lare_grid *g, double gamma, double lambda,
                   double beta, double pert, uint64_t seed,
                   double *const fields[SAMS_NFIELDS])
{
    if (check_grid(g, fields) || !(lambda > 0.0)) return -1;
    zero_all(g, fields);
    const int64_t nx = g->nx, ny = g->ny, nz = g->nz;
    const double pinf = 0.5 * beta;
    for (int64_t i = -2; i <= nx + 2; ++i)
        for (int64_t j = -1; j <= ny + 2; ++j) {
            double yc = sams_axis_centre(g->y_min, g->y_max, ny, j);
            double ch = cosh(yc / lambda);
            double sech2 = 1.0 / (ch * ch);
            double rho = 1.0 + sech2;
            double p = pinf + 0.5 * sech2;
            double e = p / ((gamma - 1.0) * rho) / 2.0;
            double b = tanh(yc / lambda);
            for (int64_t k = -1; k <= nz + 2; ++k) {
                int64_t o = sams_box_index(ny, nz, i, j, k);
                fields[SAMS_F_BX][o] = b;
                if (i >= -1) {
                    fields[SAMS_F_RHO][o] = rho;
                    fields[SAMS_F_ENERGY_ELECTRON][o] = e;
                    fields[SAMS_F_ENERGY_ION][o] = e;
                }
            }
        }
    /* Node velocities: periodic images in x and z share a draw. */
    for (int64_t i = -2; i <= nx + 2; ++i) {
        int64_t iw = ((i % nx) + nx) % nx;
        for (int64_t j = -2; j <= ny + 2; ++j) {
            int wall = (j <= 0) || (j >= ny);
            for (int64_t k = -2; k <= nz + 2; ++k) {
                int64_t kw = ((k % nz) + nz) % nz;
                uint64_t ctr = ((uint64_t)iw * (uint64_t)(ny + 5) + (uint64_t)(j + 2)) * (uint64_t)nz + (uint64_t)kw;
                int64_t o = sams_box_index(ny, nz, i, j, k);
                for (int c = 0; c < 3; ++c) {
                    double u = sams_ic_uniform(seed, (uint64_t)(3 + c), ctr);
                    fields[SAMS_F_VX + c][o] = wall ? 0.0 : pert * (2.0 * u - 1.0);
                }
            }
        }
    }
    return 0;
}

static void set_all_bcs(sams_lare_bcs *bcs, int kind)
{
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 2; ++e) {
                bcs->kind[f][d][e] = kind;
                bcs->value[f][d][e] = 0.0;
            }
}

int sams_lare_case_setup(int case_id, int64_t nx, int64_t ny, int64_t nz,
                         double b0, sams_lare_params *p, sams_lare_bcs *bcs)
{
    (void)b0;
    if (!p || !bcs || nx < 1 || ny < 1 || nz < 1) return -1;
    memset(p, 0, sizeof(*p));
    p->nx = nx; p->ny = ny; p->nz = nz;
    p->gas_gamma = 5.0 / 3.0;
    p->mu0 = 1.0;
    p->visc1 = 0.1;
    p->visc2 = 0.5;
    p->dt_multiplier = 0.8;
    p->rke = 0;
    p->geometry = 0;
    p->j_max = 1.7976931348623157e308; /* never exceeded */
    set_all_bcs(bcs, SAMS_BC_PERIODIC);
    switch (case_id) {
    case SAMS_CASE_ORSZAG_TANG:
        p->x_min = 0.0; p->x_max = 1.0;
        p->y_min = 0.0; p->y_max = 1.0;
        p->z_min = 0.0; p->z_max = (double)nz / (double)nx; /* cubic cells */
        p->resistive_mhd = 0;
        p->eta_background = 0.0;
        p->eta0 = 0.0;
        return 0;
    case SAMS_CASE_RANDOM_FIELD:
        p->x_min = 0.0; p->x_max = 1.0;
        p->y_min = 0.0; p->y_max = 1.0;
        p->z_min = 0.0; p->z_max = 1.0;
        p->resistive_mhd = 1;
        p->eta_background = 1.0e-4;
        p->eta0 = 0.0;
        return 0;
    case SAMS_CASE_HARRIS: {
        const double L = 10.0;
        p->x_min = -L; p->x_max = L;
        p->y_min = -L / 2.0; p->y_max = L / 2.0;
        p->z_min = 0.0; p->z_max = L / 4.0;
        p->resistive_mhd = 1;
        p->eta_background = 1.0e-3;
        p->eta0 = 0.0;
        /* Conducting walls in y: zero-gradient thermodynamics and tangential
         * field, zero normal field and no-slip velocities. */
        for (int e = 0; e < 2; ++e) {
            bcs->kind[SAMS_F_RHO][1][e] = SAMS_BC_ZERO_GRADIENT;
            bcs->kind[SAMS_F_ENERGY_ELECTRON][1][e] = SAMS_BC_ZERO_GRADIENT;
            bcs->kind[SAMS_F_ENERGY_ION][1][e] = SAMS_BC_ZERO_GRADIENT;
            bcs->kind[SAMS_F_BX][1][e] = SAMS_BC_ZERO_GRADIENT;
            bcs->kind[SAMS_F_BZ][1][e] = SAMS_BC_ZERO_GRADIENT;
            bcs->kind[SAMS_F_BY][1][e] = SAMS_BC_CLAMP;
            bcs->kind[SAMS_F_DM][1][e] = SAMS_BC_ZERO_GRADIENT;
            for (int f = SAMS_F_VX; f <= SAMS_F_VZ1; ++f)
                bcs->kind[f][1][e] = SAMS_BC_CLAMP;
        }
        return 0;
    }
    default:
        return -1;
    }
}

int sams_lare_case_fields(int case_id, const sams_lare_params *p,
                          uint64_t seed, double b0,
                          double *const fields[SAMS_NFIELDS])
{
    if (!p) return -1;
    sams_lare_grid g = {p->nx, p->ny, p->nz, p->x_min, p->x_max,
                        p->y_min, p->y_max, p->z_min, p->z_max};
    switch (case_id) {
    case SAMS_CASE_ORSZAG_TANG:
        if (!(b0 > 0.0)) b0 = 1.0 / sqrt(4.0 * M_PI);
        return sams_ic_orszag_tang(&g, p->gas_gamma, b0, fields);
    case SAMS_CASE_RANDOM_FIELD:
        return sams_ic_random_field(&g, p->gas_gamma, seed, 8, 6, 0.1, 0.05,
                                    1.0, 0.1, fields);
    case SAMS_CASE_HARRIS:
        return sams_ic_harris(&g, p->gas_gamma, 0.5, 0.1, 0.01, seed, fields);
    default:
        return -1;
    }
}
