/*
 * lare_oracle.h -- CPU restatement of the reference LARE3D timestep, used as
 * the checker for the GPU implementation.  TEST INFRASTRUCTURE ONLY: the
 * product never links or calls it.
 *
 * State is held in box buffers (sams_lare_layout.h).  One call of
 * lo_step() is one pass of the reference runner's step loop
 * (include/runner/runner.h:564-586) over LARE3D's three events:
 * startOfTimestep -> lagrangian_step, halfTimestep -> corrector_step,
 * endOfTimestep -> eulerian_remap + eta_calc
 * (src/PhysicsPackages/LARE/shared_data.h:397-419).
 */
#ifndef SAMS_LARE_ORACLE_H
#define SAMS_LARE_ORACLE_H

#include <stdint.h>
#include "sams_lare_layout.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lo_state lo_state;

lo_state *lo_create(const sams_lare_params *p, const sams_lare_bcs *bcs);
void lo_destroy(lo_state *s);
/* Copy the 13 fields in from box buffers. */
int lo_set_fields(lo_state *s, const double *const fields[SAMS_NFIELDS]);
/* Copy one field, or a named intermediate, out into a box buffer. */
int lo_get_field(lo_state *s, int field, double *out);
int lo_get_named(lo_state *s, const char *name, double *out);
/* Advance nsteps full timesteps. */
int lo_step(lo_state *s, int64_t nsteps);
/* Run only the first part of a step (phase 0: startOfTimestep,
 * 1: + halfTimestep, 2: whole step) -- for phase-by-phase comparisons. */
int lo_step_phase(lo_state *s, int phase);
double lo_dt(const lo_state *s);
double lo_time(const lo_state *s);
int64_t lo_steps(const lo_state *s);

#ifdef __cplusplus
}
#endif

#endif
