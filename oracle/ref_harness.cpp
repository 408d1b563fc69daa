/*
 * ref_harness.cpp -- drives the UNMODIFIED reference LARE3D package
 * (src/PhysicsPackages/LARE/*.cpp, compiled from the reference tree by
 * oracle/Makefile) through the reference's own SAMS::runner, with a
 * project-written initial-condition package and a state dumper.
 *
 * This is test infrastructure: it produces golden state dumps and the timed
 * reference CPU baseline.  Nothing in the product links it.
 *
 * The reference ships no tests and its simple writer writes no field data,
 * so the dumper here is the only way to observe its state.  The runner's
 * initializePackages / runPackages sequence (include/runner/runner.h:548-586)
 * is replayed event by event, minus writeOutput/queryOutput/steer, so no
 * output files are created.
 *
 * Usage:
 *   lare_ref --case ot|rf|harris --nx N --ny N --nz N --steps S
 *            [--seed S] [--b0 B] [--ic FILE] [--dump FILE]
 *            [--dump-step S --dump-phase start|half|end] [--quiet]
 *            [--rke] [--geometry G] [--domain x0 x1 y0 y1 z0 z1] [--lare-bcs]
 * Prints one JSON line with timing of the step loop.
 */
#include "shared_data.h"
#include "runner.h"
#include "builtInBoundaryConditions.h"

#include "sams_lare_ic.h"
// the reference's own LARE-compatible IC package: its BC_OTHER boundary
// functions (src/InitialConditions/LARE/boundary.cpp, compiled from the
// reference tree) and their registration (lareic.h:96-140)
#include "lareic.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>

namespace oracle
{
    struct config
    {
        int case_id = SAMS_CASE_ORSZAG_TANG;
        int64_t nx = 16, ny = 16, nz = 16;
        int64_t steps = 1;
        uint64_t seed = 1;
        double b0 = 0.0;
        std::string ic_file, dump_file;
        int64_t dump_step = -1; // 1-based step whose phase is dumped
        int dump_phase = 0;     // 0 start, 1 half, 2 end
        sams_lare_params params{};
        sams_lare_bcs bcs{};
        std::vector<double> dts, times, step_seconds;
        std::chrono::steady_clock::time_point last_mark;
        bool dumped = false;
        bool lare_bcs = false;  // BC_OTHER on every edge, from the reference's LARE IC package
    };
    config g;

    using volumeArray = LARE::volumeArray;
    using lineArray = LARE::lineArray;
    using planeArray = LARE::planeArray;

    struct dumpEntry
    {
        std::string name;
        int rank;
        int64_t lb[3], ub[3];
        std::vector<double> data;
    };

    template <int N>
    void collect(std::vector<dumpEntry> &out, const std::string &name,
                 const portableWrapper::portableArray<double, N, portableWrapper::arrayTags::accelerated> &a)
    {
        if (a.data() == nullptr) return;
        dumpEntry e;
        e.name = name;
        e.rank = N;
        for (int d = 0; d < 3; ++d) { e.lb[d] = 0; e.ub[d] = 0; }
        for (int d = 0; d < N; ++d)
        {
            auto r = a.getRange(d);
            e.lb[d] = r.lower_bound;
            e.ub[d] = r.upper_bound;
        }
        if constexpr (N == 1)
        {
            for (int64_t i = e.lb[0]; i <= e.ub[0]; ++i) e.data.push_back(a(i));
        }
        else if constexpr (N == 2)
        {
            for (int64_t i = e.lb[0]; i <= e.ub[0]; ++i)
                for (int64_t j = e.lb[1]; j <= e.ub[1]; ++j) e.data.push_back(a(i, j));
        }
        else
        {
            for (int64_t i = e.lb[0]; i <= e.ub[0]; ++i)
                for (int64_t j = e.lb[1]; j <= e.ub[1]; ++j)
                    for (int64_t k = e.lb[2]; k <= e.ub[2]; ++k) e.data.push_back(a(i, j, k));
        }
        out.push_back(std::move(e));
    }

    void writeDump(const std::string &path, LARE::simulationData &d, int64_t step, double time, const char *phase)
    {
        std::vector<dumpEntry> es;
        collect(es, "rho", d.rho);
        collect(es, "energy_electron", d.energy_electron);
        collect(es, "energy_ion", d.energy_ion);
        collect(es, "vx", d.vx);
        collect(es, "vy", d.vy);
        collect(es, "vz", d.vz);
        collect(es, "vx1", d.vx1);
        collect(es, "vy1", d.vy1);
        collect(es, "vz1", d.vz1);
        collect(es, "bx", d.bx);
        collect(es, "by", d.by);
        collect(es, "bz", d.bz);
        collect(es, "dm", d.dm);
        // Intermediates (values as the reference leaves them)
        collect(es, "p_visc", d.p_visc);
        collect(es, "visc_heat", d.visc_heat);
        collect(es, "alpha1", d.alpha1);
        collect(es, "alpha2", d.alpha2);
        collect(es, "alpha3", d.alpha3);
        collect(es, "pressure", d.pressure);
        collect(es, "p_e", d.p_e);
        collect(es, "p_i", d.p_i);
        collect(es, "rho_v", d.rho_v);
        collect(es, "cv_v", d.cv_v);
        collect(es, "fx", d.fx);
        collect(es, "fy", d.fy);
        collect(es, "fz", d.fz);
        collect(es, "fx_visc", d.fx_visc);
        collect(es, "fy_visc", d.fy_visc);
        collect(es, "fz_visc", d.fz_visc);
        collect(es, "bx1", d.bx1);
        collect(es, "by1", d.by1);
        collect(es, "bz1", d.bz1);
        collect(es, "cv1", d.cv1);
        collect(es, "eta", d.eta);
        collect(es, "flux_x", d.flux_x);
        collect(es, "flux_y", d.flux_y);
        collect(es, "flux_z", d.flux_z);
        collect(es, "curlb", d.curlb);
        // Grid and metrics
        collect(es, "cv", d.cv);
        collect(es, "cvc", d.cvc);
        collect(es, "dxab", d.dxab);
        collect(es, "dyab", d.dyab);
        collect(es, "dzab", d.dzab);
        collect(es, "dxac", d.dxac);
        collect(es, "dyac", d.dyac);
        collect(es, "dzac", d.dzac);
        collect(es, "xb", d.xb);
        collect(es, "yb", d.yb);
        collect(es, "zb", d.zb);
        collect(es, "xc", d.xc);
        collect(es, "yc", d.yc);
        collect(es, "zc", d.zc);
        collect(es, "dxb", d.dxb);
        collect(es, "dyb", d.dyb);
        collect(es, "dzb", d.dzb);
        collect(es, "dxc", d.dxc);
        collect(es, "dyc", d.dyc);
        collect(es, "dzc", d.dzc);
        collect(es, "x", d.x);
        collect(es, "y", d.y);
        collect(es, "z", d.z);

        std::ostringstream h;
        h.precision(17);
        h << "{\"nx\":" << d.nx << ",\"ny\":" << d.ny << ",\"nz\":" << d.nz
          << ",\"step\":" << step << ",\"phase\":\"" << phase << "\",\"time\":" << time
          << ",\"dt\":" << d.dt << ",\"dts\":[";
        for (size_t i = 0; i < g.dts.size(); ++i) h << (i ? "," : "") << g.dts[i];
        h << "],\"arrays\":[";
        size_t off = 0;
        for (size_t i = 0; i < es.size(); ++i)
        {
            const auto &e = es[i];
            h << (i ? "," : "") << "{\"name\":\"" << e.name << "\",\"rank\":" << e.rank
              << ",\"lb\":[" << e.lb[0] << "," << e.lb[1] << "," << e.lb[2] << "]"
              << ",\"ub\":[" << e.ub[0] << "," << e.ub[1] << "," << e.ub[2] << "]"
              << ",\"offset\":" << off << "}";
            off += e.data.size() * sizeof(double);
        }
        h << "]}";
        std::ofstream f(path, std::ios::binary);
        f << "SAMSDUMP1\n" << h.str() << "\n";
        for (const auto &e : es)
            f.write(reinterpret_cast<const char *>(e.data.data()), e.data.size() * sizeof(double));
    }

    /**
     * Initial-condition package for the three workloads, written against
     * the reference IC-package contract (OrszagTang.cpp:28-173).
     */
    class ConfigIC
    {
    public:
        constexpr static std::string_view name = "ConfigIC";
        constexpr static bool timeSimulation = false;
        int64_t localStep = 0;

        void controlVariables(LARE::simulationData &data)
        {
            const auto &p = g.params;
            data.nx = p.nx; data.ny = p.ny; data.nz = p.nz;
            data.x_min = p.x_min; data.x_max = p.x_max;
            data.y_min = p.y_min; data.y_max = p.y_max;
            data.z_min = p.z_min; data.z_max = p.z_max;
            data.t_end = 1e300;
            data.dt_snapshots = 1e300;
            data.dt_multiplier = p.dt_multiplier;
            data.geometry = static_cast<LARE::geometryType>(p.geometry);
            data.visc1 = p.visc1;
            data.visc2 = p.visc2;
            data.gas_gamma = p.gas_gamma;
            data.mf = 1.2;
            data.mu0 = p.mu0;
            data.resistiveMHD = p.resistive_mhd != 0;
            data.eta_background = p.eta_background;
            data.j_max = p.j_max;
            data.eta0 = p.eta0;
            data.rke = p.rke != 0;
        }

        void setDomain(SAMS::harness &harness, LARE::simulationData &data)
        {
            auto &axisReg = harness.axisRegistry;
            axisReg.setDomain("X", data.nx, data.x_min, data.x_max);
            axisReg.setDomain("Y", data.ny, data.y_min, data.y_max);
            axisReg.setDomain("Z", data.nz, data.z_min, data.z_max);
        }

        void initialConditions(SAMS::harness &harness, LARE::simulationData &data)
        {
            const auto &p = g.params;
            int64_t n = sams_box_elems(p.nx, p.ny, p.nz);
            std::vector<std::vector<double>> box(SAMS_NFIELDS, std::vector<double>(n, 0.0));
            double *ptrs[SAMS_NFIELDS];
            for (int f = 0; f < SAMS_NFIELDS; ++f) ptrs[f] = box[f].data();
            if (!g.ic_file.empty())
            {
                std::ifstream in(g.ic_file, std::ios::binary);
                for (int f = 0; f < SAMS_NFIELDS; ++f)
                    in.read(reinterpret_cast<char *>(ptrs[f]), n * sizeof(double));
                if (!in) throw std::runtime_error("cannot read IC file " + g.ic_file);
            }
            else if (sams_lare_case_fields(g.case_id, &p, g.seed, g.b0, ptrs) != 0)
            {
                throw std::runtime_error("IC generation failed");
            }
            auto &varReg = harness.variableRegistry;
            for (int f = 0; f < SAMS_NFIELDS; ++f)
            {
                portableWrapper::portableArray<double, 3> a;
                varReg.fillPPArray(sams_lare_field_names[f], a);
                for (int64_t i = a.getRange(0).lower_bound; i <= a.getRange(0).upper_bound; ++i)
                    for (int64_t j = a.getRange(1).lower_bound; j <= a.getRange(1).upper_bound; ++j)
                        for (int64_t k = a.getRange(2).lower_bound; k <= a.getRange(2).upper_bound; ++k)
                            a(i, j, k) = box[f][sams_box_index(p.ny, p.nz, i, j, k)];
            }
            (void)data;
        }

        void setBoundaryConditions(SAMS::harness &harness, LARE::simulationData &data, SAMS::timeState &time)
        {
            using namespace SAMS;
            if (g.lare_bcs)
            {
                // every edge BC_OTHER, registered by the reference package itself
                data.xbc_min = data.xbc_max = LARE::BCType::BC_OTHER;
                data.ybc_min = data.ybc_max = LARE::BCType::BC_OTHER;
                data.zbc_min = data.zbc_max = LARE::BCType::BC_OTHER;
                LARE::LARE3DInitialConditions lareIC;
                lareIC.setBoundaryConditions(harness, data, time);
                return;
            }
            for (int f = 0; f < SAMS_NFIELDS; ++f)
            {
                variableDef &vd = harness.variableRegistry.getVariable(sams_lare_field_names[f]);
                for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 2; ++e)
                    {
                        auto edge = e == 0 ? domain::edges::lower : domain::edges::upper;
                        std::shared_ptr<boundaryConditions> bc;
                        switch (g.bcs.kind[f][d][e])
                        {
                        case SAMS_BC_PERIODIC: bc = std::make_shared<simplePeriodicBC<T_dataType, 3>>(vd); break;
                        case SAMS_BC_ZERO_GRADIENT: bc = std::make_shared<simpleZeroGradientBC<T_dataType, 3>>(vd); break;
                        case SAMS_BC_MIRROR: bc = std::make_shared<simpleMirrorBC<T_dataType, 3>>(vd); break;
                        case SAMS_BC_CLAMP: bc = std::make_shared<simpleClamp<T_dataType, 3>>(vd, g.bcs.value[f][d][e]); break;
                        default: break;
                        }
                        if (bc) vd.addBoundaryCondition(d, edge, bc);
                    }
            }
        }

        void maybeDump(LARE::simulationData &data, int phase, double time)
        {
            static const char *names[3] = {"start", "half", "end"};
            if (!g.dump_file.empty() && g.dump_step == localStep + (phase == 2 ? 0 : 1) && g.dump_phase == phase && !g.dumped)
            {
                writeDump(g.dump_file, data, localStep, time, names[phase]);
                g.dumped = true;
            }
        }

        void startOfTimestep(LARE::simulationData &data) { maybeDump(data, 0, 0.0); }
        void halfTimestep(LARE::simulationData &data) { maybeDump(data, 1, 0.0); }
        void endOfTimestep(LARE::simulationData &data)
        {
            auto now = std::chrono::steady_clock::now();
            g.step_seconds.push_back(std::chrono::duration<double>(now - g.last_mark).count());
            g.last_mark = now;
            ++localStep;
            g.dts.push_back(data.dt);
            maybeDump(data, 2, 0.0);
        }

        void queryTerminate(bool &terminate, LARE::simulationData &, SAMS::timeState &t)
        {
            if (t.step >= g.steps) terminate |= true;
        }
    };
}

static const char *arg_value(int &i, int argc, char **argv)
{
    if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", argv[i]); std::exit(2); }
    return argv[++i];
}

int main(int argc, char *argv[])
{
    using namespace oracle;
    std::string dumpFinal;
    bool quiet = false, rke = false, set_domain = false;
    int geometry = 0;
    double domain[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 1; i < argc; ++i)
    {
        std::string a = argv[i];
        if (a == "--case")
        {
            std::string c = arg_value(i, argc, argv);
            g.case_id = c == "ot" ? SAMS_CASE_ORSZAG_TANG : c == "rf" ? SAMS_CASE_RANDOM_FIELD : c == "harris" ? SAMS_CASE_HARRIS : -1;
        }
        else if (a == "--nx") g.nx = std::atoll(arg_value(i, argc, argv));
        else if (a == "--ny") g.ny = std::atoll(arg_value(i, argc, argv));
        else if (a == "--nz") g.nz = std::atoll(arg_value(i, argc, argv));
        else if (a == "--steps") g.steps = std::atoll(arg_value(i, argc, argv));
        else if (a == "--seed") g.seed = std::strtoull(arg_value(i, argc, argv), nullptr, 10);
        else if (a == "--b0") g.b0 = std::atof(arg_value(i, argc, argv));
        else if (a == "--ic") g.ic_file = arg_value(i, argc, argv);
        else if (a == "--dump") dumpFinal = arg_value(i, argc, argv);
        else if (a == "--dump-step") g.dump_step = std::atoll(arg_value(i, argc, argv));
        else if (a == "--dump-phase")
        {
            std::string p = arg_value(i, argc, argv);
            g.dump_phase = p == "start" ? 0 : p == "half" ? 1 : 2;
        }
        else if (a == "--quiet") quiet = true;
        else if (a == "--rke") rke = true;
        else if (a == "--lare-bcs") g.lare_bcs = true;
        else if (a == "--geometry") geometry = std::atoi(arg_value(i, argc, argv));
        else if (a == "--domain")
        {
            for (int d = 0; d < 6; ++d) domain[d] = std::atof(arg_value(i, argc, argv));
            set_domain = true;
        }
        else { std::fprintf(stderr, "unknown argument %s\n", a.c_str()); return 2; }
    }
    if (g.case_id < 0 || sams_lare_case_setup(g.case_id, g.nx, g.ny, g.nz, g.b0, &g.params, &g.bcs) != 0)
    {
        std::fprintf(stderr, "bad case/size\n");
        return 2;
    }
    if (rke) g.params.rke = 1;  // remap kinetic-energy correction on
    g.params.geometry = geometry;  // 0 Cartesian, 1 cylindrical, 2 spherical
    if (set_domain)
    {
        g.params.x_min = domain[0]; g.params.x_max = domain[1];
        g.params.y_min = domain[2]; g.params.y_max = domain[3];
        g.params.z_min = domain[4]; g.params.z_max = domain[5];
    }
    if (g.dump_step >= 0) { g.dump_file = dumpFinal; dumpFinal.clear(); }
    if (quiet) std::cout.setstate(std::ios::failbit);

    int fakeArgc = 1;
    char *fakeArgv0 = argv[0];
    char **fakeArgv = &fakeArgv0;
    SAMS::MPI::initialize(fakeArgc, fakeArgv);
    portableWrapper::initialize(fakeArgc, fakeArgv);
    double loop_s = 0.0;
    int64_t steps_done = 0;
    {
        SAMS::runner<LARE::LARE3D, ConfigIC> runner;
        runner.initialize(fakeArgc, fakeArgv);
        runner.activatePackage("LARE3D");
        runner.activatePackage("ConfigIC");
        // runner::initializePackages without writeOutput (runner.h:548-562)
        runner.runnerInteraction<decltype(runner)>(runner);
        runner.pkgInit();
        runner.registerAxes();
        runner.registerVariables();
        runner.defaultValues();
        runner.controlVariables();
        runner.setDomain();
        runner.decomposeAndAllocate();
        runner.getVariables();
        runner.defaultVariables();
        runner.initialConditions();
        runner.setBoundaryConditions();

        auto &t = std::get<SAMS::timeState>(runner.runnerData);
        auto t0 = std::chrono::steady_clock::now();
        g.last_mark = t0;
        if (g.steps > 0)
        {
            // runner::runPackages step loop (runner.h:564-586) without output
            for (;;)
            {
                runner.startOfTimestep();
                runner.halfTimestep();
                t.step++;
                t.time += t.dt;
                runner.endOfTimestep();
                if (runner.queryTerminate()) break;
            }
        }
        auto t1 = std::chrono::steady_clock::now();
        loop_s = std::chrono::duration<double>(t1 - t0).count();
        steps_done = t.step;
        auto &data = std::get<LARE::simulationData>(runner.runnerData);
        if (!dumpFinal.empty()) writeDump(dumpFinal, data, t.step, t.time, "final");
        double cells = double(g.nx) * double(g.ny) * double(g.nz);
        std::cout.clear();
        std::string st;
        for (size_t i = 0; i < g.step_seconds.size(); ++i)
        {
            char buf[64];
            std::snprintf(buf, sizeof buf, "%s%.6f", i ? "," : "", g.step_seconds[i]);
            st += buf;
        }
        std::printf("{\"case\":%d,\"nx\":%lld,\"ny\":%lld,\"nz\":%lld,\"steps\":%lld,\"loop_s\":%.6f,"
                    "\"cell_updates_per_s\":%.6e,\"threads\":%d,\"time\":%.17g,\"dt\":%.17g,\"step_seconds\":[%s]}\n",
                    g.case_id, (long long)g.nx, (long long)g.ny, (long long)g.nz, (long long)steps_done, loop_s,
                    loop_s > 0 ? cells * double(steps_done) / loop_s : 0.0, omp_get_max_threads(), t.time, t.dt, st.c_str());
        runner.finalizePackages();
    }
    portableWrapper::finalize();
    return 0;
}
