// The reference's own LARE-compatible initial-condition package
// (src/InitialConditions/LARE: lareic.h, lareBoundaryClass.h, control.cpp,
// boundary.cpp, compiled unchanged from the reference tree) driven through
// SAMS::runner<LARE::LARE3D, LARE::LARE3DInitialConditions, CaseState> of
// include/sams/.
//
// The package sets every edge to BC_OTHER and attaches its
// LAREBoundaryConditions (host functions) to the 13 variables; LARE::LARE3D
// translates them into device descriptors by probing them.  Its own initial
// state is uniform (nothing would move), so CaseState, after it in the
// runner, replaces the grid, parameters and fields by a seeded workload
// (sams_lare_case_setup / sams_lare_case_fields): the same state the
// reference harness starts from for the *_lare_* fixtures.
//
//   lare_ic_runner --check-setup              host only: the boundary table
//   lare_ic_runner --run CASE NX NY NZ STEPS SEED OUT
//                                             GPU: STEPS steps, then the 13
//                                             fields' boxes to OUT (float64)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "sams/lare3d.hpp"
#include "lareic.h"
#include "sams_lare_ic.h"

namespace {
struct Config {
    int case_id = SAMS_CASE_ORSZAG_TANG;
    long long nx = 12, ny = 10, nz = 6, steps = 1;
    unsigned long long seed = 1;
} cfg;
}  // namespace

struct CaseState {
    constexpr static std::string_view name = "CaseState";
    sams_lare_params p{};
    sams_lare_bcs b{};

    void controlVariables(SAMS::harness &, LARE::simulationData &d)
    {
        if (sams_lare_case_setup(cfg.case_id, cfg.nx, cfg.ny, cfg.nz, 0.0, &p, &b) != 0)
            throw std::runtime_error("case setup failed");
        d.nx = p.nx;
        d.ny = p.ny;
        d.nz = p.nz;
        d.x_min = p.x_min;
        d.x_max = p.x_max;
        d.y_min = p.y_min;
        d.y_max = p.y_max;
        d.z_min = p.z_min;
        d.z_max = p.z_max;
        d.gas_gamma = p.gas_gamma;
        d.mu0 = p.mu0;
        d.visc1 = p.visc1;
        d.visc2 = p.visc2;
        d.dt_multiplier = p.dt_multiplier;
        d.eta_background = p.eta_background;
        d.eta0 = p.eta0;
        d.j_max = p.j_max;
        d.resistiveMHD = p.resistive_mhd != 0;
        d.rke = false;
        d.geometry = LARE::geometryType::Cartesian;
        d.nsteps = cfg.steps;
    }

    void initialConditions(SAMS::harness &h, LARE::simulationData &)
    {
        double *ptrs[SAMS_NFIELDS];
        for (int f = 0; f < SAMS_NFIELDS; ++f) ptrs[f] = h.variableRegistry.box(f);
        if (sams_lare_case_fields(cfg.case_id, &p, cfg.seed, 0.0, ptrs) != 0)
            throw std::runtime_error("case fields failed");
    }
};

int main(int argc, char **argv)
{
    try {
        const bool run = argc >= 9 && std::strcmp(argv[1], "--run") == 0;
        if (run) {
            const std::string c = argv[2];
            cfg.case_id = c == "ot" ? SAMS_CASE_ORSZAG_TANG : c == "rf" ? SAMS_CASE_RANDOM_FIELD : SAMS_CASE_HARRIS;
            cfg.nx = std::atoll(argv[3]);
            cfg.ny = std::atoll(argv[4]);
            cfg.nz = std::atoll(argv[5]);
            cfg.steps = std::atoll(argv[6]);
            cfg.seed = std::strtoull(argv[7], nullptr, 10);
        }
        SAMS::runner<LARE::LARE3D, LARE::LARE3DInitialConditions, CaseState> r;
        r.activatePackage("LARE3D");
        r.activatePackage("LARE3DInitialConditions");
        r.activatePackage("CaseState");
        r.initializePackages();
        const sams_lare_bcs b = LARE::LARE3D::bcs(r.harnessData);
        int other = 0, none = 0;
        for (int f = 0; f < SAMS_NFIELDS; ++f)
            for (int q = 0; q < 3; ++q)
                for (int e = 0; e < 2; ++e) {
                    other += b.kind[f][q][e] == SAMS_BC_LARE_OTHER;
                    none += b.kind[f][q][e] == SAMS_BC_NONE;
                }
        if (!run) {
            std::printf("{\"lare_other_slots\": %d, \"none_slots\": %d, \"dm_y_z_none\": %s}\n", other, none,
                        (b.kind[SAMS_F_DM][1][0] == SAMS_BC_NONE && b.kind[SAMS_F_DM][2][1] == SAMS_BC_NONE) ? "true"
                                                                                                          : "false");
            return 0;
        }
        r.runPackages();
        r.finalize();
        FILE *fp = std::fopen(argv[8], "wb");
        if (!fp) throw std::runtime_error("cannot write the output file");
        const size_t n = (size_t)sams_box_elems(cfg.nx, cfg.ny, cfg.nz);
        for (int f = 0; f < SAMS_NFIELDS; ++f) std::fwrite(r.harnessData.variableRegistry.box(f), sizeof(double), n, fp);
        std::fclose(fp);
        const auto &t = r.tData;
        std::printf("{\"steps\": %lld, \"time\": %.17g, \"dt\": %.17g, \"lare_other_slots\": %d}\n", (long long)t.step,
                    t.time, t.dt, other);
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "exception: %s\n", e.what());
        return 2;
    }
}
