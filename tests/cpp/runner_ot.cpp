// A reference-style initial-condition package (the Orszag-Tang vortex on a
// 2*pi periodic box, shaped like src/InitialConditions/OrszagTang/) driven by
// SAMS::runner<LARE::LARE3D, ...> from include/sams/.
//
//   runner_ot --check-setup   host only: event order, variable ranges, the
//                             boundary-condition table and the IC values
//   runner_ot --run N [nx ny nz]
//                             N GPU steps through the runner, then the same
//                             N steps of the oracle from the same initial
//                             state; every field must match bit for bit
//
// Test program: links the oracle as the checker.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sams/lare3d.hpp"
#include "lare_oracle.h"

namespace pw = portableWrapper;

static std::vector<std::string> g_events;

class VortexIC {
public:
    constexpr static std::string_view name = "VortexIC";
    static inline long long n[3] = {24, 20, 4};
    static inline int64_t max_steps = 3;

    void registerVariables(SAMS::harness &) { g_events.push_back("registerVariables"); }

    void controlVariables(LARE::simulationData &d)
    {
        g_events.push_back("controlVariables");
        d.nx = n[0];
        d.ny = n[1];
        d.nz = n[2];
        const double L = 2.0 * M_PI;
        d.x_min = 0.0;
        d.x_max = L;
        d.y_min = 0.0;
        d.y_max = L;
        d.z_min = 0.0;
        d.z_max = L * double(d.nz) / double(d.nx);
        d.gas_gamma = 5.0 / 3.0;
        d.mu0 = 1.0;
        d.visc1 = 0.1;
        d.visc2 = 1.0;
        d.dt_multiplier = 0.8;
        d.resistiveMHD = false;
        d.rke = false;
    }

    void setDomain(SAMS::harness &h, LARE::simulationData &d)
    {
        g_events.push_back("setDomain");
        h.axisRegistry.setDomain("X", d.nx, d.x_min, d.x_max);
        h.axisRegistry.setDomain("Y", d.ny, d.y_min, d.y_max);
        h.axisRegistry.setDomain("Z", d.nz, d.z_min, d.z_max);
    }

    void setBoundaryConditions(SAMS::harness &h)
    {
        g_events.push_back("setBoundaryConditions");
        for (int f = 0; f < SAMS_NFIELDS; ++f) {
            SAMS::variableDef &v = h.variableRegistry.getVariable(sams_lare_field_names[f]);
            v.emplaceBoundaryCondition<SAMS::simplePeriodicBC<SAMS::T_dataType, 3>>();
        }
    }

    void initialConditions(SAMS::harness &h, LARE::simulationData &d)
    {
        g_events.push_back("initialConditions");
        pw::portableArray<double, 3> rho, ee, ei, vx, vy, vz, bx, by, bz;
        pw::portableArray<double, 1> xc, yc, xb, yb;
        auto &ax = h.axisRegistry;
        ax.fillPPLocalAxis("X", xc, SAMS::staggerType::CENTRED);
        ax.fillPPLocalAxis("Y", yc, SAMS::staggerType::CENTRED);
        ax.fillPPLocalAxis("X", xb, SAMS::staggerType::HALF_CELL);
        ax.fillPPLocalAxis("Y", yb, SAMS::staggerType::HALF_CELL);
        auto &vr = h.variableRegistry;
        vr.fillPPArray("rho", rho);
        vr.fillPPArray("energy_electron", ee);
        vr.fillPPArray("energy_ion", ei);
        vr.fillPPArray("vx", vx);
        vr.fillPPArray("vy", vy);
        vr.fillPPArray("vz", vz);
        vr.fillPPArray("bx", bx);
        vr.fillPPArray("by", by);
        vr.fillPPArray("bz", bz);
        const double g = d.gas_gamma;
        pw::applyKernel(
            LAMBDA(long long i, long long j, long long k) {
                const double density = g * g, pressure = g;
                rho(i, j, k) = density;
                const double eint = pressure / ((g - 1.0) * density) / 2.0;
                ee(i, j, k) = eint;
                ei(i, j, k) = eint;
                vx(i, j, k) = -std::sin(yb(j));
                vy(i, j, k) = std::sin(xb(i));
                vz(i, j, k) = 0.0;
                bx(i, j, k) = -std::sin(yc(j));
                by(i, j, k) = std::sin(2.0 * xc(i));
                bz(i, j, k) = 0.0;
            },
            rho.getRange(0), rho.getRange(1), rho.getRange(2));
    }

    void queryTerminate(bool &terminate, LARE::simulationData &, SAMS::timeState &t)
    {
        if (t.step >= max_steps) terminate |= true;
    }
};

using Runner = SAMS::runner<LARE::LARE3D, VortexIC>;

static int fail(const char *what)
{
    std::fprintf(stderr, "FAIL: %s\n", what);
    return 1;
}

static int check_setup()
{
    Runner r;
    r.activatePackage("LARE3D");
    r.activatePackage("VortexIC");
    try {
        r.activatePackage("NoSuchPackage");
        return fail("unknown package accepted");
    } catch (const std::runtime_error &) {
    }
    r.initializePackages();
    const char *order[] = {"registerVariables", "controlVariables", "setDomain", "initialConditions",
                           "setBoundaryConditions"};
    if (g_events.size() != 5) return fail("event count");
    for (int i = 0; i < 5; ++i)
        if (g_events[i] != order[i]) return fail("event order");

    auto &data = r.getDataPack<LARE::simulationData>();
    if (data.gas_gamma != 5.0 / 3.0 || data.visc2 != 1.0 || data.mu0 != 1.0) return fail("control variables");

    pw::portableArray<double, 3> rho, vx, bx;
    r.harnessData.variableRegistry.fillPPArray("rho", rho);
    r.harnessData.variableRegistry.fillPPArray("vx", vx);
    r.harnessData.variableRegistry.fillPPArray("bx", bx);
    const long long nx = VortexIC::n[0], ny = VortexIC::n[1], nz = VortexIC::n[2];
    if (rho.getRange(0).lower_bound != -1 || rho.getRange(0).upper_bound != nx + 2) return fail("centred range");
    if (vx.getRange(2).lower_bound != -2 || vx.getRange(2).upper_bound != nz + 2) return fail("staggered range");
    if (bx.getRange(0).lower_bound != -2 || bx.getRange(1).lower_bound != -1) return fail("bx range");

    const double g = 5.0 / 3.0;
    if (rho(3, 4, 1) != g * g) return fail("rho value");
    const double yb4 = sams_axis_edge(0.0, 2.0 * M_PI, ny, 4);
    if (vx(-1, 4, nz + 2) != -std::sin(yb4)) return fail("vx value");
    const double* box = r.harnessData.variableRegistry.box(SAMS_F_VX);
    if (box[sams_box_index(ny, nz, 5, 4, 2)] != -std::sin(yb4)) return fail("box layout");

    const sams_lare_bcs b = LARE::LARE3D::bcs(r.harnessData);
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 2; ++e)
                if (b.kind[f][d][e] != SAMS_BC_PERIODIC) return fail("bc table");
    const sams_lare_params p = LARE::LARE3D::params(r.harnessData, data);
    if (p.nx != nx || p.ny != ny || p.nz != nz || p.x_max != 2.0 * M_PI || p.resistive_mhd != 0)
        return fail("params");

    // A second condition on one edge is not representable: rejected.
    SAMS::variableDef &v = r.harnessData.variableRegistry.getVariable("rho");
    v.emplaceBoundaryCondition<SAMS::simpleClamp<double, 3>>(0, SAMS::domain::edges::lower, 1.0);
    try {
        (void)LARE::LARE3D::bcs(r.harnessData);
        return fail("two conditions on one edge accepted");
    } catch (const std::runtime_error &) {
    }
    std::printf("{\"check_setup\": \"ok\"}\n");
    return 0;
}

static int run(int64_t nsteps)
{
    VortexIC::max_steps = nsteps;
    Runner r;
    r.activatePackage("LARE3D");
    r.activatePackage("VortexIC");
    r.initializePackages();

    SAMS::harness &h = r.harnessData;
    const long long nx = VortexIC::n[0], ny = VortexIC::n[1], nz = VortexIC::n[2];
    const size_t nelem = (size_t)sams_box_elems(nx, ny, nz);
    std::vector<std::vector<double>> initial(SAMS_NFIELDS);
    for (int f = 0; f < SAMS_NFIELDS; ++f)
        initial[f].assign(h.variableRegistry.box(f), h.variableRegistry.box(f) + nelem);
    const sams_lare_params p = LARE::LARE3D::params(h, r.getDataPack<LARE::simulationData>());
    const sams_lare_bcs b = LARE::LARE3D::bcs(h);

    r.runPackages();
    r.finalize();

    lo_state *o = lo_create(&p, &b);
    if (!o) return fail("oracle create");
    const double *ic[SAMS_NFIELDS];
    for (int f = 0; f < SAMS_NFIELDS; ++f) ic[f] = initial[f].data();
    if (lo_set_fields(o, ic) != 0 || lo_step(o, nsteps) != 0) return fail("oracle step");

    // The nine state fields; vx1..vz1 and dm hold remap scratch at the end
    // of a step and are not part of the state.
    const int state[9] = {SAMS_F_RHO, SAMS_F_ENERGY_ELECTRON, SAMS_F_ENERGY_ION, SAMS_F_VX, SAMS_F_VY,
                          SAMS_F_VZ, SAMS_F_BX, SAMS_F_BY, SAMS_F_BZ};
    std::vector<double> want(nelem);
    long long mismatches = 0;
    double maxdiff = 0.0;
    for (int f : state) {
        lo_get_field(o, f, want.data());
        const double *got = h.variableRegistry.box(f);
        for (long long i = sams_lare_field_lb(f, 0); i <= nx + 2; ++i)
            for (long long j = sams_lare_field_lb(f, 1); j <= ny + 2; ++j)
                for (long long k = sams_lare_field_lb(f, 2); k <= nz + 2; ++k) {
                    const int64_t q = sams_box_index(ny, nz, i, j, k);
                    if (std::memcmp(&got[q], &want[q], sizeof(double)) != 0) {
                        ++mismatches;
                        maxdiff = std::fmax(maxdiff, std::fabs(got[q] - want[q]));
                    }
                }
    }
    const SAMS::timeState &t = r.tData;
    const bool time_ok = t.time == lo_time(o) && t.step == lo_steps(o) && t.dt == lo_dt(o);
    std::printf("{\"steps\": %lld, \"time\": %.17g, \"oracle_time\": %.17g, \"mismatches\": %lld, "
                "\"max_abs_diff\": %.3g, \"time_ok\": %s}\n",
                (long long)t.step, t.time, lo_time(o), mismatches, maxdiff, time_ok ? "true" : "false");
    lo_destroy(o);
    return (mismatches == 0 && time_ok) ? 0 : 1;
}

int main(int argc, char **argv)
{
    try {
        if (argc >= 2 && std::strcmp(argv[1], "--check-setup") == 0) return check_setup();
        if (argc >= 3 && std::strcmp(argv[1], "--run") == 0) {
            if (argc >= 6)
                for (int d = 0; d < 3; ++d) VortexIC::n[d] = std::atoll(argv[3 + d]);
            return run(std::atoll(argv[2]));
        }
    } catch (const std::exception &e) {
        std::fprintf(stderr, "exception: %s\n", e.what());
        return 2;
    }
    std::fprintf(stderr, "usage: runner_ot --check-setup | --run N [nx ny nz]\n");
    return 2;
}
