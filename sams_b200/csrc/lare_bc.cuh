// lare_bc.cuh -- one (field, dimension, edge) of a built-in boundary
// condition at one ghost point, shared by the single-solve and batched fill
// kernels.
//
// The reference applies a condition to a whole edge slab as one sliced copy
// or kernel over the slab in row-major order
// (include/boundaryConditions/builtInBoundaryConditions.h: simpleClamp :55,
// simpleMirrorBC :145, simpleZeroGradientBC :224, simplePeriodicBC :252).
// Lines of the slab along the other two dimensions are independent; along the
// condition's own dimension a copy may read points the same copy writes when
// the dimension has fewer than three interior cells (e.g. a periodic upper
// edge of a half-cell field with n = 2 reads index 2 after writing it), so
// then the ghost layers of a line are filled one after another in ascending
// order, as the reference's loop does.
#pragma once

#include <string>

#include "lare_device.cuh"
#include "sams_lare_bc_other.h"

namespace sams {

// Boundary conditions of all fields as the kernels read them.  A
// SAMS_BC_LARE_OTHER slot carries its plane operations: plane pdst[q] of the
// slot's dimension receives plane psrc[q] (or zero, SAMS_PLANE_ZERO) for
// q < nplanes.
struct BcTable {
    signed char kind[SAMS_NFIELDS][3][2];
    signed char nplanes[SAMS_NFIELDS][3][2];
    int pdst[SAMS_NFIELDS][3][2][3];
    int psrc[SAMS_NFIELDS][3][2][3];
    double value[SAMS_NFIELDS][3][2];
};

// Host: set one slot of a table for a grid of n[] interior cells.  The plane
// operations of a SAMS_BC_LARE_OTHER slot must write only the edge's ghost
// planes, read planes of the field's own range, and never read a plane the
// same slot writes (so one thread per point applies them in any order).
inline bool bc_slot_set(BcTable &t, int f, int d, int e, int kind, double value, const long long n[3],
                        std::string *err)
{
    if (kind < SAMS_BC_NONE || kind > SAMS_BC_LARE_OTHER) {
        *err = "unknown boundary-condition kind";
        return false;
    }
    t.kind[f][d][e] = (signed char)kind;
    t.value[f][d][e] = value;
    t.nplanes[f][d][e] = 0;
    if (kind != SAMS_BC_LARE_OTHER) return true;
    int32_t dst[3], src[3];
    const int np = sams_lare_other_planes(f, d, e, n[d], dst, src);
    const bool half = sams_lare_field_stagger[f][d] != 0;
    const long long lb = half ? -2 : -1, ub = n[d] + 2;
    const long long glo = e == 0 ? lb : (half ? n[d] : n[d] + 1), ghi = e == 0 ? 0 : n[d] + 2;
    for (int q = 0; q < np; ++q) {
        bool ok = dst[q] >= glo && dst[q] <= ghi && (src[q] == SAMS_PLANE_ZERO || (src[q] >= lb && src[q] <= ub));
        for (int r = 0; r < np; ++r) ok = ok && src[q] != dst[r];
        if (!ok) {
            *err = "LARE BC_OTHER planes outside the field's range for this grid size";
            return false;
        }
        t.pdst[f][d][e][q] = dst[q];
        t.psrc[f][d][e][q] = src[q];
    }
    t.nplanes[f][d][e] = (signed char)np;
    return true;
}

// Host: a whole table from the C-ABI descriptor.
inline bool bc_table_from(BcTable &t, const sams_lare_bcs &bcs, const long long n[3], std::string *err)
{
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 2; ++e)
                if (!bc_slot_set(t, f, d, e, bcs.kind[f][d][e], bcs.value[f][d][e], n, err)) return false;
    return true;
}

// Below this many interior cells in the condition's dimension an edge copy
// can read its own output: fill the ghost layers of each line in order.
constexpr int kBcSequentialBelow = 3;

struct BcEdge {
    int glo, ghi;  // ghost range of the edge in dimension d
    int dlb, dub;  // first and last domain index in dimension d
    int lo[3], hi[3];  // the slab (field range, ghost range in d)
};

__host__ __device__ inline BcEdge bc_edge_slab(const Geom &g, int f, int d, int e)
{
    const int n[3] = {g.nx, g.ny, g.nz};
    BcEdge s;
    for (int q = 0; q < 3; ++q) {
        s.lo[q] = field_half(f, q) ? -2 : -1;
        s.hi[q] = n[q] + 2;
    }
    const bool half = field_half(f, d) != 0;
    s.dlb = half ? 0 : 1;
    s.dub = n[d];
    s.glo = e == 0 ? s.lo[d] : (half ? n[d] : n[d] + 1);
    s.ghi = e == 0 ? 0 : n[d] + 2;
    s.lo[d] = s.glo;
    s.hi[d] = s.ghi;
    return s;
}

// Value the condition writes at ghost point q (q[d] in glo..ghi), from the
// array's current contents.
__device__ __forceinline__ double bc_edge_value(const double *a, const Geom &g, const BcEdge &s, int kind,
                                                double clamp_value, int d, int e, const int *q)
{
    const int gq = q[d];
    const int cnt = s.ghi - s.glo + 1;
    int p[3] = {q[0], q[1], q[2]};
    switch (kind) {
    case SAMS_BC_PERIODIC:
        p[d] = e == 0 ? s.dub - cnt + 1 + (gq - s.glo) : s.dlb + (gq - s.glo);
        return a[box_off(g, p[0], p[1], p[2])];
    case SAMS_BC_ZERO_GRADIENT:
        p[d] = e == 0 ? s.dlb : s.dub;
        return a[box_off(g, p[0], p[1], p[2])];
    case SAMS_BC_MIRROR: {
        const int last = e == 0 ? s.dlb : s.dub;
        const int first = e == 0 ? s.ghi : s.glo;
        p[d] = last;
        const double av = a[box_off(g, p[0], p[1], p[2])];
        const double bv = (av + av) / 2.0;
        p[d] = last - (gq - first);
        const double delta = a[box_off(g, p[0], p[1], p[2])] - bv;
        return bv - delta;
    }
    default:  // SAMS_BC_CLAMP
        return clamp_value;
    }
}

// Fill ghost point q, or (in a dimension with fewer than three interior
// cells) the whole ghost line through q when q is its first layer.  A LARE
// BC_OTHER slot writes q only if its plane is one the slot's operations
// write; those operations are independent, so every point is one thread.
__device__ __forceinline__ void bc_edge_apply(double *a, const Geom &g, const BcEdge &s, const BcTable &bt, int f,
                                              int d, int e, int *q)
{
    const int kind = bt.kind[f][d][e];
    const double clamp_value = bt.value[f][d][e];
    if (kind == SAMS_BC_LARE_OTHER) {
        const int np = bt.nplanes[f][d][e];
        for (int t = 0; t < np; ++t) {
            if (bt.pdst[f][d][e][t] != q[d]) continue;
            const int src = bt.psrc[f][d][e][t];
            double v = 0.0;
            if (src != SAMS_PLANE_ZERO) {
                int p[3] = {q[0], q[1], q[2]};
                p[d] = src;
                v = a[box_off(g, p[0], p[1], p[2])];
            }
            a[box_off(g, q[0], q[1], q[2])] = v;
        }
        return;
    }
    const int n = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
    if (n >= kBcSequentialBelow) {
        const double v = bc_edge_value(a, g, s, kind, clamp_value, d, e, q);
        a[box_off(g, q[0], q[1], q[2])] = v;
        return;
    }
    if (q[d] != s.glo) return;
    for (int gq = s.glo; gq <= s.ghi; ++gq) {
        q[d] = gq;
        const double v = bc_edge_value(a, g, s, kind, clamp_value, d, e, q);
        a[box_off(g, q[0], q[1], q[2])] = v;
    }
}

}  // namespace sams
