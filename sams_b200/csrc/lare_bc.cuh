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

#include "lare_device.cuh"

namespace sams {

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
// cells) the whole ghost line through q when q is its first layer.
__device__ __forceinline__ void bc_edge_apply(double *a, const Geom &g, const BcEdge &s, int kind, double clamp_value,
                                              int d, int e, int *q)
{
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
