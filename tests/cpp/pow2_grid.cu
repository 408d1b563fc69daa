// Host check of sams::pow2_grid, the test that lets the kernels multiply by
// reciprocals instead of dividing: it must accept exactly the uniform grids
// whose spacings (and mu0) are powers of two, and the reciprocals it returns
// must give the same bits as the divisions they replace.
#include <cstdio>
#include <random>
#include <vector>

#include "lare_geom_host.h"

// spacings laid out as the solver builds them: b(i) = lo + d i, c(i) =
// (b(i) + b(i-1)) / 2, db[i+2] = b(i) - b(i-1) (i = -1..n+2, db[0] = db[1]),
// dc[i+2] = c(i) - c(i-1) (i = 0..n+2, dc[1] = dc[2])
static void axis(double lo, double hi, long long n, std::vector<double> &db, std::vector<double> &dc)
{
    std::vector<double> b(n + 5), c(n + 5);
    const double d = (hi - lo) / (double)n;
    for (long long i = -2; i <= n + 2; ++i) b[i + 2] = lo + d * (double)i;
    for (long long i = -1; i <= n + 2; ++i) c[i + 2] = 0.5 * (b[i + 2] + b[i + 1]);
    db.assign(n + 6, 0.0);
    dc.assign(n + 6, 0.0);
    for (long long i = -1; i <= n + 2; ++i) db[i + 2] = b[i + 2] - b[i + 1];
    db[0] = db[1];
    for (long long i = 0; i <= n + 2; ++i) dc[i + 2] = c[i + 2] - c[i + 1];
    dc[1] = dc[2];
}

struct Case {
    double x0, x1, y0, y1, z0, z1;
    long long nx, ny, nz;
    double mu0;
    bool want;
};

int main()
{
    const Case cases[] = {
        {0, 1, 0, 1, 0, 1, 256, 256, 256, 1.0, true},           // the 256^3 cube
        {0, 1, 0, 1, 0, 4.0 / 128, 128, 128, 4, 1.0, true},     // Orszag-Tang 128 x 128 x 4
        {-8, 8, -4, 4, 0, 2, 16, 8, 4, 1.0, true},              // spacings 1, 1, 1/2
        {0, 1, 0, 1, 0, 1, 250, 256, 256, 1.0, false},          // 1/250
        {-10, 10, -5, 5, 0, 2.5, 512, 256, 64, 1.0, false},     // Harris: 5/128
        {0, 1, 0, 1, 0, 1, 64, 64, 64, 4e-7 * 3.141592653589793, false},  // mu0 not a power of two
        {0, 1, 0, 1, 0, 1, 64, 64, 64, 0.25, true},
        {0.1, 1.1, 0, 1, 0, 1, 64, 64, 64, 1.0, false},         // offset axis: spacings not all exact
    };
    int bad = 0;
    std::mt19937_64 rng(5);
    std::uniform_real_distribution<double> u(-1e3, 1e3);
    for (const Case &k : cases) {
        std::vector<double> dxb, dxc, dyb, dyc, dzb, dzc;
        axis(k.x0, k.x1, k.nx, dxb, dxc);
        axis(k.y0, k.y1, k.ny, dyb, dyc);
        axis(k.z0, k.z1, k.nz, dzb, dzc);
        sams::Recip r{};
        const bool got = sams::pow2_grid(dxb, dyb, dzb, dxc, dyc, dzc, k.mu0, &r);
        if (got != k.want) {
            std::printf("case nx=%lld: got %d want %d\n", k.nx, got, k.want);
            ++bad;
            continue;
        }
        if (!got) continue;
        const double d[8] = {dxb[2], dyb[2], dzb[2], dxc[2], dyc[2], dzc[2], dxb[2] * (dyb[2] * dzb[2]), k.mu0};
        const double rr[8] = {r.xb, r.yb, r.zb, r.xc, r.yc, r.zc, r.cv, r.mu0};
        for (int q = 0; q < 8; ++q)
            for (int t = 0; t < 1000; ++t) {
                const double x = u(rng) * (t % 3 == 0 ? 1e-300 : 1.0);
                if (x / d[q] != x * rr[q]) ++bad;
            }
    }
    // subnormal and tiny spacings are powers of two for frexp, but their
    // reciprocals (or those of their products) overflow: rejected
    for (double tiny : {0x1p-1060, 0x1p-400, 0x1p400}) {
        std::vector<double> db(10, tiny), dc(10, tiny), ok(10, 0.5);
        sams::Recip r{};
        if (sams::pow2_grid(db, ok, ok, dc, ok, ok, 1.0, &r)) {
            std::printf("spacing %a accepted\n", tiny);
            ++bad;
        }
        if (sams::pow2_grid(ok, ok, ok, ok, ok, ok, tiny, &r)) {
            std::printf("mu0 %a accepted\n", tiny);
            ++bad;
        }
    }
    std::printf("{\"bad\": %d}\n", bad);
    return bad ? 1 : 0;
}
