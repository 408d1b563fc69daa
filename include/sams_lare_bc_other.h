/* sams_lare_bc_other.h -- the LARE "BC_OTHER" boundary conditions as plane
 * operations.
 *
 * The reference's LARE3DInitialConditions package
 * (src/InitialConditions/LARE/lareic.h:96-140, control.cpp:31-36) installs,
 * on every edge of the 13 LARE variables, a LAREBoundaryConditions object
 * (src/InitialConditions/LARE/lareBoundaryClass.h:10-33) whose apply(dim,
 * edge) calls one function per variable from
 * src/InitialConditions/LARE/boundary.cpp.  Each such function, where its
 * edge is BC_OTHER, copies whole planes of the variable onto its ghost
 * planes (pw::assign of one index in `dim`, every index in the other two
 * dimensions) or sets ghost planes to zero.  Within one (dim, edge) no plane
 * it reads is a plane it writes, so the copies are independent.
 *
 * sams_lare_other_planes lists those operations for one (field, dim, edge)
 * on a dimension of n interior cells: for q < return value, plane dst[q]
 * (an index in that dimension) receives plane src[q], or zero where
 * src[q] == SAMS_PLANE_ZERO.  The device fills (kind SAMS_BC_LARE_OTHER)
 * and the CPU checker both use this table.
 */
#ifndef SAMS_LARE_BC_OTHER_H
#define SAMS_LARE_BC_OTHER_H

#include <stdint.h>

#include "sams_lare_layout.h"

#define SAMS_PLANE_ZERO (-1000000)

#ifdef __cplusplus
extern "C" {
#endif

static inline int sams_lare_other_planes(int field, int dim, int edge, int64_t n, int32_t dst[3], int32_t src[3])
{
    const int32_t N = (int32_t)n;
#define SAMS_OP(q, d, s) (dst[q] = (d), src[q] = (s))
    switch (field) {
    case SAMS_F_RHO:               /* density_bcs :477-560 */
    case SAMS_F_ENERGY_ELECTRON:   /* energy_electron_bcs :389-470 */
    case SAMS_F_ENERGY_ION:        /* energy_ion_bcs :300-380 */
        if (edge == 0) { SAMS_OP(0, -1, 2); SAMS_OP(1, 0, 1); }
        else { SAMS_OP(0, N + 1, N - 1); SAMS_OP(1, N + 2, N - 2); }
        return 2;
    case SAMS_F_BX:   /* bx_bcs :31-115 */
    case SAMS_F_BY:   /* by_bcs :124-205 */
    case SAMS_F_BZ: { /* bz_bcs :212-293 */
        const int own = field - SAMS_F_BX;  /* the face field's staggered dimension */
        if (edge == 0) {
            if (dim == own) { SAMS_OP(0, -2, 2); SAMS_OP(1, -1, 1); }
            else { SAMS_OP(0, -1, 2); SAMS_OP(1, 0, 1); }
        } else if (dim == 0 && field == SAMS_F_BX) {
            SAMS_OP(0, N + 1, N - 1); SAMS_OP(1, N + 2, N - 2);
        } else {
            SAMS_OP(0, N + 1, N); SAMS_OP(1, N + 2, N - 1);
        }
        return 2;
    }
    case SAMS_F_VX: case SAMS_F_VY: case SAMS_F_VZ:     /* v*_bcs :570-645, :737-812, :903-978 */
    case SAMS_F_VX1: case SAMS_F_VY1: case SAMS_F_VZ1:  /* remap_v*_bcs :653-729, :820-895, :986-1061 */
        if (dim == 0) {  /* walls at the x edges: all three node planes zeroed */
            const int32_t b = edge == 0 ? -2 : N;
            SAMS_OP(0, b, SAMS_PLANE_ZERO); SAMS_OP(1, b + 1, SAMS_PLANE_ZERO); SAMS_OP(2, b + 2, SAMS_PLANE_ZERO);
            return 3;
        }
        if (edge == 0) { SAMS_OP(0, -2, 2); SAMS_OP(1, -1, 1); }
        else { SAMS_OP(0, N + 1, N - 1); SAMS_OP(1, N + 2, N - 2); }
        return 2;
    case SAMS_F_DM:  /* dm_x_bcs :1063-1081, the one dm function the package installs */
        if (dim != 0) return 0;
        if (edge == 0) SAMS_OP(0, -1, 0);
        else SAMS_OP(0, N + 1, N);
        return 1;
    default:
        return 0;
    }
#undef SAMS_OP
}

#ifdef __cplusplus
}
#endif

#endif /* SAMS_LARE_BC_OTHER_H */
