// Host setup of the reference's own Orszag-Tang initial-condition package
// (src/InitialConditions/OrszagTang/OrszagTang.cpp, compiled unchanged from
// the reference tree) through SAMS::runner<LARE::LARE3D, examples::OrszagTang>
// of include/sams/: the package's controlVariables, setDomain,
// initialConditions and setBoundaryConditions run against the C++ layer and
// the resulting parameters, boundary table and fields are checked.  No GPU.
#include <cmath>
#include <cstdio>

#include "sams/lare3d.hpp"
#include "OrszagTang.h"

int main()
{
    try {
        SAMS::runner<LARE::LARE3D, examples::OrszagTang> r;
        r.activatePackage("LARE3D");
        r.activatePackage("OrszagTang");
        r.initializePackages();
        const LARE::simulationData &d = r.getDataPack<LARE::simulationData>();
        const sams_lare_params p = LARE::LARE3D::params(r.harnessData, d);
        const sams_lare_bcs b = LARE::LARE3D::bcs(r.harnessData);
        int periodic = 0;
        for (int f = 0; f < SAMS_NFIELDS; ++f)
            for (int q = 0; q < 3; ++q)
                for (int e = 0; e < 2; ++e) periodic += b.kind[f][q][e] == SAMS_BC_PERIODIC;
        const double *rho = r.harnessData.variableRegistry.box(SAMS_F_RHO);
        const double *by = r.harnessData.variableRegistry.box(SAMS_F_BY);
        const double g = d.gas_gamma;
        const double xc5 = sams_axis_centre(p.x_min, p.x_max, p.nx, 5);
        const bool ok = rho[sams_box_index(p.ny, p.nz, 3, 4, 1)] == g * g &&
                        by[sams_box_index(p.ny, p.nz, 5, 2, 1)] == std::sin(2.0 * xc5);
        std::printf("{\"nx\": %lld, \"ny\": %lld, \"nz\": %lld, \"gamma\": %.17g, \"t_end\": %.17g, "
                    "\"periodic_slots\": %d, \"values_ok\": %s}\n",
                    (long long)p.nx, (long long)p.ny, (long long)p.nz, g, d.t_end, periodic, ok ? "true" : "false");
        return ok ? 0 : 1;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "exception: %s\n", e.what());
        return 2;
    }
}
