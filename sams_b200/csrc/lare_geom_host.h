// lare_geom_host.h -- host tables of the cylindrical / spherical metric
// factors (sams::GeomF), built as LARE3D::grid builds them
// (src/PhysicsPackages/LARE/setup.cpp:277-335) from the axes of
// axisRegistry::setDomain (include/harness/axisRegistry.h:393-430), with the
// host's libm sin/tan like the reference, so the device sees the same bits.
#pragma once

#include <cfloat>
#include <cmath>
#include <vector>

#include "lare_device.cuh"
#include "sams_lare_layout.h"

namespace sams {

// Packed layout: hy, hyc, hyv, xb (nx+5 each), hz, hz1, hz2, hzc
// ((nx+5)(ny+5) each, index (i+2)(ny+5) + j+2), cot (ny+5).
inline size_t geom_table_size(const sams_lare_params &p)
{
    const size_t X = (size_t)p.nx + 5, Y = (size_t)p.ny + 5;
    return 4 * X + 4 * X * Y + Y;
}

inline std::vector<double> geom_tables(const sams_lare_params &p)
{
    const long long nx = p.nx, ny = p.ny;
    const size_t X = (size_t)nx + 5, Y = (size_t)ny + 5, P = X * Y;
    std::vector<double> t(geom_table_size(p), 0.0);
    double *hy = t.data(), *hyc = hy + X, *hyv = hyc + X, *xb = hyv + X;
    double *hz = xb + X, *hz1 = hz + P, *hz2 = hz1 + P, *hzc = hz2 + P, *cot = hzc + P;
    auto H2 = [&](long long i, long long j) { return (size_t)((i + 2) * (long long)Y + (j + 2)); };
    // axes: b(i) = lo + d i, c(i) = (b(i) + b(i-1)) / 2, c(-2) = 0
    std::vector<double> xc(X), yb(Y), yc(Y);
    const double dx = (p.x_max - p.x_min) / (double)nx, dy = (p.y_max - p.y_min) / (double)ny;
    for (long long i = -2; i <= nx + 2; ++i) xb[i + 2] = p.x_min + dx * (double)i;
    for (long long i = -1; i <= nx + 2; ++i) xc[i + 2] = 0.5 * (xb[i + 2] + xb[i + 1]);
    for (long long j = -2; j <= ny + 2; ++j) yb[j + 2] = p.y_min + dy * (double)j;
    for (long long j = -1; j <= ny + 2; ++j) yc[j + 2] = 0.5 * (yb[j + 2] + yb[j + 1]);
    // setup.cpp:277-292; the threshold is LARE::none_zero = DBL_MIN (constants.h:43)
    for (long long i = -2; i <= nx + 2; ++i) {
        hy[i + 2] = std::fabs(xb[i + 2]);
        hyc[i + 2] = std::fabs(xc[i + 2]);
        hyv[i + 2] = (std::fabs(xc[2]) < DBL_MIN && i == 1) ? std::fabs(xc[i + 2]) : 0.25 * std::fabs(xc[i + 2]);
    }
    for (size_t q = 0; q < P; ++q) hz[q] = hz1[q] = hz2[q] = hzc[q] = 1.0;
    if (p.geometry == 2) {  // setup.cpp:304-334
        for (long long j = -2; j <= ny + 2; ++j) {
            const double sn = std::fabs(std::sin(yb[j + 2]));
            hz[H2(-2, j)] = hy[0] * sn;
            for (long long i = -1; i <= nx + 2; ++i) {
                hz[H2(i, j)] = hy[i + 2] * sn;
                hz2[H2(i, j)] = hyc[i + 2] * sn;
            }
        }
        for (long long j = -1; j <= ny + 2; ++j) {
            const double sc = std::fabs(std::sin(yc[j + 2]));
            hz1[H2(-2, j)] = hy[0] * sc;
            for (long long i = -1; i <= nx + 2; ++i) {
                hz1[H2(i, j)] = hy[i + 2] * sc;
                hzc[H2(i, j)] = hyc[i + 2] * sc;
            }
        }
        for (long long j = -2; j <= ny + 2; ++j) cot[j + 2] = 1.0 / std::tan(yb[j + 2]);  // lagran.cpp:713
    }
    return t;
}

// The tables of an x slab (cells off+1 .. off+p.nx) of a grid of nx_global
// cells over p.x_min..p.x_max: the whole grid's tables from row off on.
inline std::vector<double> geom_tables_slab(const sams_lare_params &p, long long off, long long nx_global)
{
    sams_lare_params pg = p;
    pg.nx = nx_global;
    const std::vector<double> t = geom_tables(pg);
    const size_t GX = (size_t)nx_global + 5, X = (size_t)p.nx + 5, Y = (size_t)p.ny + 5;
    std::vector<double> s(geom_table_size(p));
    double *o = s.data();
    for (int a = 0; a < 4; ++a, o += X) std::copy(t.begin() + a * GX + off, t.begin() + a * GX + off + X, o);
    const double *h2 = t.data() + 4 * GX;
    for (int a = 0; a < 4; ++a, o += X * Y)
        std::copy(h2 + a * GX * Y + off * Y, h2 + a * GX * Y + (off + X) * Y, o);
    std::copy(h2 + 4 * GX * Y, h2 + 4 * GX * Y + Y, o);  // cot (per y)
    return s;
}

// Point a GeomF at a device copy of geom_tables(p).
inline void geom_bind(GeomF &gf, const double *dev, const sams_lare_params &p)
{
    const size_t X = (size_t)p.nx + 5, P = X * ((size_t)p.ny + 5);
    gf.hy = dev;
    gf.hyc = dev + X;
    gf.hyv = dev + 2 * X;
    gf.xb = dev + 3 * X;
    gf.hz = dev + 4 * X;
    gf.hz1 = gf.hz + P;
    gf.hz2 = gf.hz1 + P;
    gf.hzc = gf.hz2 + P;
    gf.cot = gf.hzc + P;
}

// True when every spacing array (as the axis builders lay them out: index
// i + 2, b over -2..n+2, c over -1..n+2) holds one value per axis, that
// value is a power of two, and so is mu0; fills the reciprocals (exact for
// powers of two).  Each of these values must lie in [2^-340, 2^340]: then
// every product of up to three of them (a face area, a cell volume) is a
// normal number and its reciprocal is finite and exact.  A subnormal spacing
// is a power of two for frexp too, but its reciprocal overflows.
inline bool pow2_grid(const std::vector<double> &dxb, const std::vector<double> &dyb, const std::vector<double> &dzb,
                      const std::vector<double> &dxc, const std::vector<double> &dyc, const std::vector<double> &dzc,
                      double mu0, Recip *rc)
{
    auto uniform = [](const std::vector<double> &d, size_t from, size_t to, double *v) {
        if (d.size() < to || from >= to) return false;
        const double x = d[from];
        int e;
        if (!(x >= 0x1p-340) || !(x <= 0x1p340) || std::frexp(x, &e) != 0.5) return false;
        for (size_t q = from; q < to; ++q)
            if (d[q] != x) return false;
        *v = x;
        return true;
    };
    double xb, yb, zb, xc, yc, zc;
    int e;
    if (!(mu0 >= 0x1p-340) || !(mu0 <= 0x1p340) || std::frexp(mu0, &e) != 0.5) return false;
    // b: array indices 0 .. n+4 (i = -2 .. n+2); c: 1 .. n+4 (i = -1 .. n+2)
    if (!uniform(dxb, 0, dxb.size() - 1, &xb) || !uniform(dyb, 0, dyb.size() - 1, &yb) ||
        !uniform(dzb, 0, dzb.size() - 1, &zb) || !uniform(dxc, 1, dxc.size() - 1, &xc) ||
        !uniform(dyc, 1, dyc.size() - 1, &yc) || !uniform(dzc, 1, dzc.size() - 1, &zc))
        return false;
    rc->xb = 1.0 / xb;
    rc->yb = 1.0 / yb;
    rc->zb = 1.0 / zb;
    rc->xc = 1.0 / xc;
    rc->yc = 1.0 / yc;
    rc->zc = 1.0 / zc;
    rc->cv = 1.0 / (xb * (yb * zb));
    rc->mu0 = 1.0 / mu0;
    return true;
}

}  // namespace sams
