/*
 * sams_lare_ic.h -- initial-condition generators for the LARE3D workloads.
 *
 * In SAMS an initial-condition package implements controlVariables /
 * setDomain / initialConditions / setBoundaryConditions
 * (src/InitialConditions/OrszagTang/OrszagTang.cpp:28-156 is the pattern).
 * The functions here are the field-filling part of three such packages,
 * written once in plain C so that every consumer (the GPU package's host
 * mirrors, the C++ drop-in runner, Python tests, and the CPU checker)
 * starts from bit-identical states.  They fill box buffers
 * (sams_lare_layout.h): the nine primary fields over each field's own local
 * range, everything else zero.
 *
 * Axis construction follows the harness: edge axis b(i) = min + d*i with
 * d = (max-min)/n, centred axis c(i) = 0.5*(b(i) + b(i-1))
 * (include/harness/axisRegistry.h:393-430, 973-985).
 */
#ifndef SAMS_LARE_IC_H
#define SAMS_LARE_IC_H

#include <stdint.h>
#include "sams_lare_layout.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sams_lare_grid {
    int64_t nx, ny, nz;
    double x_min, x_max, y_min, y_max, z_min, z_max;
} sams_lare_grid;

/* Edge (half-cell) and centred coordinates of index i along one axis. */
double sams_axis_edge(double lo, double hi, int64_t n, int64_t i);
double sams_axis_centre(double lo, double hi, int64_t n, int64_t i);

/* Normalised Orszag-Tang vortex on [0,1]^2 x [0,nz/nx]:
 * rho = 25/(36 pi), p = 5/(12 pi) split equally between electrons and ions,
 * vx = -sin(2 pi yb), vy = sin(2 pi xb), bx = -B0 sin(2 pi yc),
 * by = B0 sin(4 pi xc), vz = bz = 0.  Returns 0 on success. */
int sams_ic_orszag_tang(const sams_lare_grid *g, double gamma, double B0,
                        double *const fields[SAMS_NFIELDS]);

/* Seeded random-field cube: uniform rho0, p0; B = discrete curl of a vector
 * potential held on cell edges (so the discrete div B vanishes), built from
 * modes_per_shell random integer wavevectors in each shell |k| = 1..kmax with
 * |A_k| ~ k^-2 (shell energy of B ~ k^-2), rescaled to rms |B| = b_rms; node
 * velocity from an independent set of modes with |v_k| ~ k^-1, rescaled to
 * rms |v| = v_rms.  Returns 0 on success. */
int sams_ic_random_field(const sams_lare_grid *g, double gamma, uint64_t seed,
                         int kmax, int modes_per_shell, double b_rms,
                         double v_rms, double rho0, double p0,
                         double *const fields[SAMS_NFIELDS]);

/* Harris current sheet: bx = tanh(y/lambda), rho = 1 + sech^2(y/lambda),
 * p = beta/2 + sech^2(y/lambda)/2 (total pressure balance with B0 = 1,
 * mu0 = 1), node velocities seeded uniform in [-pert, pert] per component,
 * zero on and beyond the y walls.  Returns 0 on success. */
int sams_ic_harris(const sams_lare_grid *g, double gamma, double lambda,
                   double beta, double pert, uint64_t seed,
                   double *const fields[SAMS_NFIELDS]);

/* The three workloads as complete problem set-ups: what an IC package's
 * controlVariables + setDomain + setBoundaryConditions would set. */
enum sams_lare_case {
    SAMS_CASE_ORSZAG_TANG = 0,  /* normalised OT vortex, periodic, ideal MHD */
    SAMS_CASE_RANDOM_FIELD = 1, /* random-field periodic cube, eta = 1e-4   */
    SAMS_CASE_HARRIS = 2        /* Harris sheet, y walls, eta = 1e-3        */
};

/* Fill params and boundary conditions for a case at the given size.
 * b0 is the Orszag-Tang field amplitude (ignored by other cases; pass a
 * value <= 0 for the default 1/sqrt(4 pi)).  Returns 0 on success. */
int sams_lare_case_setup(int case_id, int64_t nx, int64_t ny, int64_t nz,
                         double b0, sams_lare_params *p, sams_lare_bcs *bcs);

/* Fill the initial state of a case into box buffers. */
int sams_lare_case_fields(int case_id, const sams_lare_params *p,
                          uint64_t seed, double b0,
                          double *const fields[SAMS_NFIELDS]);

/* Counter-based uniform deviate in [0,1) (SplitMix64 finaliser). */
double sams_ic_uniform(uint64_t seed, uint64_t stream, uint64_t counter);

#ifdef __cplusplus
}
#endif

#endif /* SAMS_LARE_IC_H */
