/*
 * sams_lare_layout.h -- field identifiers, staggering and the ghost-inclusive
 * "box" layout shared by every host-side buffer of the LARE3D timestep
 * (initial conditions, uploads, downloads, state dumps).
 *
 * Index convention follows the SAMS harness that LARE3D registers its
 * variables with (src/PhysicsPackages/LARE/setup.cpp:38-70): two ghost layers
 * on each side, cell-centred indices run -1..n+2 and half-cell (staggered)
 * indices run -2..n+2 (include/harness/dimension.h:552-600,
 * include/harness/staggerRegistry.h:42-59).  A box buffer covers -2..n+2 in
 * every dimension for every field, z fastest (row-major, as
 * include/pp/array.h:72-93 lays out portableArray), so one index formula
 * serves all staggerings; entries outside a field's own range are unused.
 */
#ifndef SAMS_LARE_LAYOUT_H
#define SAMS_LARE_LAYOUT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The thirteen harness variables LARE3D registers (setup.cpp:45-69), in a
 * fixed order used by every array-of-fields argument. */
enum sams_lare_field {
    SAMS_F_RHO = 0,
    SAMS_F_ENERGY_ELECTRON = 1,
    SAMS_F_ENERGY_ION = 2,
    SAMS_F_VX = 3,
    SAMS_F_VY = 4,
    SAMS_F_VZ = 5,
    SAMS_F_VX1 = 6,
    SAMS_F_VY1 = 7,
    SAMS_F_VZ1 = 8,
    SAMS_F_BX = 9,
    SAMS_F_BY = 10,
    SAMS_F_BZ = 11,
    SAMS_F_DM = 12,
    SAMS_NFIELDS = 13
};

/* Harness variable names, as passed to variableRegistry calls. */
static const char *const sams_lare_field_names[SAMS_NFIELDS] = {
    "rho", "energy_electron", "energy_ion", "vx", "vy", "vz",
    "LARE/vx1", "LARE/vy1", "LARE/vz1", "bx", "by", "bz", "LARE/dm"};

/* Staggering per field and dimension: 0 = CENTRED, 1 = HALF_CELL
 * (setup.cpp:45-69). */
static const unsigned char sams_lare_field_stagger[SAMS_NFIELDS][3] = {
    {0, 0, 0}, {0, 0, 0}, {0, 0, 0},          /* rho, e_e, e_i  */
    {1, 1, 1}, {1, 1, 1}, {1, 1, 1},          /* vx, vy, vz     */
    {1, 1, 1}, {1, 1, 1}, {1, 1, 1},          /* vx1, vy1, vz1  */
    {1, 0, 0}, {0, 1, 0}, {0, 0, 1},          /* bx, by, bz     */
    {0, 0, 0}};                                /* dm             */

/* Lower index of a field's local range in one dimension (upper is n+2). */
static inline int64_t sams_lare_field_lb(int field, int dim)
{
    return sams_lare_field_stagger[field][dim] ? -2 : -1;
}

/* Extent of the box in one dimension. */
static inline int64_t sams_box_extent(int64_t n) { return n + 5; }

/* Number of doubles in one box buffer. */
static inline int64_t sams_box_elems(int64_t nx, int64_t ny, int64_t nz)
{
    return (nx + 5) * (ny + 5) * (nz + 5);
}

/* Linear offset of (i, j, k), each in -2..n+2, in a box buffer. */
static inline int64_t sams_box_index(int64_t ny, int64_t nz,
                                     int64_t i, int64_t j, int64_t k)
{
    return ((i + 2) * (ny + 5) + (j + 2)) * (nz + 5) + (k + 2);
}

/* Boundary-condition kinds a (field, dim, edge) slot can hold.  Kinds 1-4
 * are the built-in SAMS boundary conditions
 * (include/boundaryConditions/builtInBoundaryConditions.h): simpleClamp :55,
 * simpleMirrorBC :145, simpleZeroGradientBC :224, simplePeriodicBC :252.
 * SAMS_BC_LARE_OTHER is the LARE "BC_OTHER" condition of the
 * LARE3DInitialConditions package for that field, dimension and edge
 * (src/InitialConditions/LARE/boundary.cpp; the plane copies and zeroed
 * wall planes of sams_lare_bc_other.h); its value is unused. */
enum sams_lare_bc_kind {
    SAMS_BC_NONE = 0,
    SAMS_BC_PERIODIC = 1,
    SAMS_BC_ZERO_GRADIENT = 2,
    SAMS_BC_MIRROR = 3,
    SAMS_BC_CLAMP = 4,
    SAMS_BC_LARE_OTHER = 5
};

/* Simulation parameters of one LARE3D solve: the members of
 * LARE::simulationData that controlVariables/defaultValues set
 * (src/PhysicsPackages/LARE/shared_data.h:96-131, control.cpp:6-30). */
typedef struct sams_lare_params {
    int64_t nx, ny, nz;                 /* interior cells per dimension */
    double x_min, x_max, y_min, y_max, z_min, z_max;
    double gas_gamma;                   /* ratio of specific heats */
    double mu0;                         /* vacuum permeability */
    double visc1, visc2;                /* linear / quadratic shock viscosity */
    double dt_multiplier;               /* CFL safety factor */
    double eta_background, eta0, j_max; /* resistivity model */
    int32_t resistive_mhd;              /* 1: resistive sub-steps */
    int32_t rke;                        /* remap kinetic-energy correction */
    int32_t geometry;                   /* 0 = Cartesian */
    int32_t reserved;
} sams_lare_params;

/* One boundary condition per (field, dimension, edge); edge 0 = lower. */
typedef struct sams_lare_bcs {
    int32_t kind[SAMS_NFIELDS][3][2];
    double value[SAMS_NFIELDS][3][2];
} sams_lare_bcs;

#ifdef __cplusplus
}
#endif

#endif /* SAMS_LARE_LAYOUT_H */
