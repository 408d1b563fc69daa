// lare3d.hpp -- LARE::LARE3D as a runner package whose timestep runs on the
// GPU through the C ABI of include/sams_lare.h.
//
// It keeps the reference package's name, data pack and event signatures
// (src/PhysicsPackages/LARE/shared_data.h:229-508), so a runner built as
// SAMS::runner<LARE::LARE3D, MyInitialConditions> is driven exactly as the
// reference drives it:
//   registerAxes / registerVariables   X, Y, Z and the 13 harness variables
//                                      (setup.cpp:27-70)
//   defaultValues / defaultVariables   control.cpp:6-53
//   startOfTimestep                    the whole GPU step (predictor,
//                                      corrector, remap); the new CFL dt is
//                                      read back and offered to the runner
//                                      through controlFns.calculateTimestep()
//   calculateTimestep / getTimestep    shared_data.h:428-440
//   halfTimestep / endOfTimestep       nothing left to do on the host
//   finalize                           copies the device state back into the
//                                      harness variables
// The solver is created at the first startOfTimestep, after the IC package
// has written the harness variables and attached its boundary conditions;
// from then on the state lives on the GPU and syncToHost() refreshes the host
// copy.  Cartesian, cylindrical and spherical geometry, with or without the
// remap kinetic-energy correction (rke).
#pragma once

#include <cstring>
#include <map>
#include <vector>
#include <limits>
#include <stdexcept>
#include <string>
#include <string_view>

#include "sams_runner.hpp"
#include "../sams_lare_bc_other.h"

namespace LARE {

namespace pw = portableWrapper;
using SAMS::T_dataType;
using SAMS::T_indexType;

enum class geometryType { Cartesian = 0, Cylindrical = 1, Spherical = 2 };

// LARE-style boundary types (shared_data.h:46-54); BC_OTHER edges get the
// IC package's own boundary functions, BC_EXTERNAL edges none.
enum class BCType { BC_OTHER = 0, BC_PERIODIC = 1, BC_REFLECTIVE = 2, BC_OUTFLOW = 3, BC_INFLOW = 4, BC_EXTERNAL = 5 };

// The members of the reference simulationData that initial-condition
// packages set or read (shared_data.h:60-226), including host views of the
// 13 harness variables (bound in getVariables, as LARE3D::getVariables binds
// them, setup.cpp:95-140).
struct simulationData {
    T_dataType dt = 0.0, dtr = 0.0, dt_multiplier = 0.8;
    T_dataType time = 0.0;
    int64_t step = 0;
    int64_t nsteps = -1;
    T_dataType t_end = 0.0;
    T_indexType nx = 0, ny = 0, nz = 0;
    T_dataType x_min = 0, x_max = 0, y_min = 0, y_max = 0, z_min = 0, z_max = 0;
    geometryType geometry = geometryType::Cartesian;
    bool resistiveMHD = false;
    bool rke = false;
    T_dataType visc1 = 0.1, visc2 = 1.0;
    T_dataType gas_gamma = 1.4;
    T_dataType j_max = std::numeric_limits<T_dataType>::max();
    T_dataType eta0 = 0.0;
    T_dataType eta_background = 0.0;
    T_dataType mf = 1.2;
    T_dataType mu0 = 4.0e-7 * 3.14159265358979323846;
    T_dataType dt_snapshots = 0.0;
    T_dataType lastOutputTime = 0.0;
    BCType xbc_min = BCType::BC_OTHER, xbc_max = BCType::BC_OTHER;
    BCType ybc_min = BCType::BC_OTHER, ybc_max = BCType::BC_OTHER;
    BCType zbc_min = BCType::BC_OTHER, zbc_max = BCType::BC_OTHER;
    bool x_stretch = false, y_stretch = false, z_stretch = false;
    // one process holds the whole domain, so it is on every edge
    bool isxLB = true, isxUB = true, isyLB = true, isyUB = true, iszLB = true, iszUB = true;
    using volumeArray = pw::portableArray<T_dataType, 3>;
    volumeArray rho, energy_electron, energy_ion, vx, vy, vz, vx1, vy1, vz1, bx, by, bz, dm;
    volumeArray *field(int f)
    {
        volumeArray *a[SAMS_NFIELDS] = {&rho, &energy_electron, &energy_ion, &vx, &vy, &vz, &vx1,
                                        &vy1, &vz1, &bx, &by, &bz, &dm};
        return a[f];
    }
};

// The remap's working arrays live in the solver's device scratch.
struct remapData {};

class LARE3D {
public:
    constexpr static std::string_view name = "LARE3D";
    using dataPack = SAMS::dataPacks::multiPack<simulationData, remapData>;

    explicit LARE3D(SAMS::harness &h) : harness_(&h) {}
    LARE3D(LARE3D &&o) noexcept : harness_(o.harness_), solver_(o.solver_), device_(o.device_) { o.solver_ = nullptr; }
    LARE3D(const LARE3D &) = delete;
    LARE3D &operator=(const LARE3D &) = delete;
    ~LARE3D() { sams_lare_destroy(solver_); }

    // Select the CUDA device the solver is created on (default 0).
    void setDevice(int device) { device_ = device; }
    sams_lare_solver *solver() const { return solver_; }

    void registerAxes(SAMS::harness &h)
    {
        h.axisRegistry.registerAxis("X", SAMS::MPIAxis(0));
        h.axisRegistry.registerAxis("Y", SAMS::MPIAxis(1));
        h.axisRegistry.registerAxis("Z", SAMS::MPIAxis(2));
    }

    void registerVariables(SAMS::harness &h)
    {
        static const char *const axes[3] = {"X", "Y", "Z"};
        for (int f = 0; f < SAMS_NFIELDS; ++f) {
            auto st = [&](int d) {
                return SAMS::dimension(axes[d], 2, sams_lare_field_stagger[f][d] ? SAMS::staggerType::HALF_CELL
                                                                                 : SAMS::staggerType::CENTRED);
            };
            h.variableRegistry.registerVariable<T_dataType>(sams_lare_field_names[f], pw::arrayTags::accelerated,
                                                            st(0), st(1), st(2));
        }
    }

    void defaultValues(simulationData &d)
    {
        d.dt_multiplier = 0.8;
        d.geometry = geometryType::Cartesian;
        d.visc1 = 0.1;
        d.visc2 = 1.0;
        d.gas_gamma = 1.4;
        d.mf = 1.2;
        d.rke = false;
        d.mu0 = 4.0e-7 * 3.14159265358979323846;
        d.time = 0.0;
    }

    // Host views of the harness variables (LARE3D::getVariables,
    // setup.cpp:95-140).
    void getVariables(SAMS::harness &h, simulationData &d)
    {
        for (int f = 0; f < SAMS_NFIELDS; ++f) h.variableRegistry.fillPPArray(sams_lare_field_names[f], *d.field(f));
        const auto &X = h.axisRegistry.get("X"), &Y = h.axisRegistry.get("Y"), &Z = h.axisRegistry.get("Z");
        d.nx = X.n;
        d.ny = Y.n;
        d.nz = Z.n;
    }

    void defaultVariables(simulationData &)
    {
        // Box storage is zeroed when the runner allocates it.
    }

    void startOfTimestep(simulationData &d, SAMS::controlFunctions &controlFns)
    {
        if (!solver_) create(d);
        check(sams_lare_step_graph(solver_, 1));
        check(sams_lare_get_dt(solver_, &d.dt));
        controlFns.calculateTimestep();
    }

    void calculateTimestep(SAMS::timeState &timeData, simulationData &d)
    {
        timeData.dt = d.dt < timeData.dt ? d.dt : timeData.dt;
    }

    void getTimestep(SAMS::timeState &timeData, simulationData &d) { d.dt = timeData.dt; }

    void endOfTimestep(simulationData &d, remapData &)
    {
        d.time += d.dt;
        d.step++;
    }

    void finalize(simulationData &) { syncToHost(); }

    // Copy the device state into the harness variables.
    void syncToHost()
    {
        if (!solver_) return;
        for (int f = 0; f < SAMS_NFIELDS; ++f)
            check(sams_lare_download_field(solver_, f, harness_->variableRegistry.box(f)));
    }

    // The C-ABI parameter block the solver is created from.
    static sams_lare_params params(SAMS::harness &h, const simulationData &d)
    {
        sams_lare_params p;
        std::memset(&p, 0, sizeof p);
        const auto &X = h.axisRegistry.get("X"), &Y = h.axisRegistry.get("Y"), &Z = h.axisRegistry.get("Z");
        p.nx = X.n;
        p.ny = Y.n;
        p.nz = Z.n;
        p.x_min = X.lo;
        p.x_max = X.hi;
        p.y_min = Y.lo;
        p.y_max = Y.hi;
        p.z_min = Z.lo;
        p.z_max = Z.hi;
        p.gas_gamma = d.gas_gamma;
        p.mu0 = d.mu0;
        p.visc1 = d.visc1;
        p.visc2 = d.visc2;
        p.dt_multiplier = d.dt_multiplier;
        p.eta_background = d.eta_background;
        p.eta0 = d.eta0;
        p.j_max = d.j_max;
        p.resistive_mhd = d.resistiveMHD ? 1 : 0;
        p.rke = d.rke ? 1 : 0;
        p.geometry = (int32_t)d.geometry;
        return p;
    }

    // The boundary-condition table built from what the IC package attached
    // to each harness variable (one condition per variable, dimension and
    // edge): the built-in conditions by kind; a condition defined only by
    // its host apply() (LAREBoundaryConditions) by probing it.
    static sams_lare_bcs bcs(SAMS::harness &h)
    {
        sams_lare_bcs b;
        std::memset(&b, 0, sizeof b);
        for (const auto &kv : h.variableRegistry.all()) {
            const SAMS::variableDef &v = kv.second;
            for (int d = 0; d < 3; ++d)
                for (int e = 0; e < 2; ++e) {
                    const auto &list = v.bcs[d][e];
                    if (list.empty()) continue;
                    if (list.size() > 1)
                        throw std::runtime_error("LARE3D: variable " + v.name +
                                                 " has more than one boundary condition on one edge");
                    int kind = list.front()->kind();
                    if (kind == SAMS::boundaryConditions::kHostDefined) kind = probe(h, v, *list.front(), d, e);
                    b.kind[v.field][d][e] = kind;
                    b.value[v.field][d][e] = list.front()->value();
                }
        }
        return b;
    }

    // Run a host-defined condition's apply(d, e) once on the variable's box
    // filled with distinct tags (restored afterwards) and read off what it
    // did: which ghost planes of dimension d received a copy of which plane,
    // or zero.  The result must be exactly the LARE BC_OTHER table of that
    // variable (sams_lare_bc_other.h: what the reference's
    // LARE3DInitialConditions functions do), or nothing at all; anything else
    // has no device descriptor and is refused.
    static int probe(SAMS::harness &h, const SAMS::variableDef &v, SAMS::boundaryConditions &bc, int d, int e)
    {
        const auto &X = h.axisRegistry.get("X"), &Y = h.axisRegistry.get("Y"), &Z = h.axisRegistry.get("Z");
        const long long n[3] = {X.n, Y.n, Z.n};
        const long long ext[3] = {n[0] + 5, n[1] + 5, n[2] + 5};
        const int f = v.field;
        double *box = h.variableRegistry.box(f);
        const long long ne = ext[0] * ext[1] * ext[2];
        const double base = 1048576.0;  // tags base + t are exact, distinct and nonzero
        std::vector<double> keep(box, box + ne);
        for (long long t = 0; t < ne; ++t) box[t] = base + (double)t;
        bc.apply(d, e == 0 ? SAMS::domain::edges::lower : SAMS::domain::edges::upper);
        // per destination plane: the source plane (or kZero), and how many points
        const long long kZero = -1000000, kUnset = -2000000;
        std::map<long long, std::pair<long long, long long>> planes;
        bool ok = true;
        for (long long t = 0; t < ne && ok; ++t) {
            if (box[t] == base + (double)t) continue;
            const long long q[3] = {t / (ext[1] * ext[2]) - 2, (t / ext[2]) % ext[1] - 2, t % ext[2] - 2};
            long long src = kUnset;
            if (box[t] == 0.0) {
                src = kZero;
            } else {
                const double tv = box[t] - base;
                const long long u = (long long)tv;
                if (!(tv >= 0.0) || (double)u != tv || u >= ne) { ok = false; break; }
                const long long r[3] = {u / (ext[1] * ext[2]) - 2, (u / ext[2]) % ext[1] - 2, u % ext[2] - 2};
                for (int o = 0; o < 3; ++o)
                    if (o != d && r[o] != q[o]) ok = false;
                src = r[d];
            }
            auto it = planes.find(q[d]);
            if (it == planes.end()) planes[q[d]] = {src, 1};
            else if (it->second.first != src) ok = false;
            else ++it->second.second;
        }
        std::copy(keep.begin(), keep.end(), box);
        if (planes.empty() && ok) return SAMS_BC_NONE;
        int32_t dst[3], srcs[3];
        const int np = sams_lare_other_planes(f, d, e, n[d], dst, srcs);
        long long plane = 1;  // points of one plane of the variable's own range
        for (int o = 0; o < 3; ++o)
            if (o != d) plane *= n[o] + 3 - sams_lare_field_lb(f, o);
        ok = ok && (int)planes.size() == np;
        for (int q = 0; q < np && ok; ++q) {
            auto it = planes.find(dst[q]);
            const long long want = srcs[q] == SAMS_PLANE_ZERO ? kZero : srcs[q];
            ok = it != planes.end() && it->second.first == want && it->second.second == plane;
        }
        if (!ok)
            throw std::runtime_error("LARE3D: the boundary condition of " + v.name + " (dimension " +
                                     std::to_string(d) + ", edge " + std::to_string(e) +
                                     ") is neither a built-in condition nor the LARE BC_OTHER planes");
        return SAMS_BC_LARE_OTHER;
    }

private:
    SAMS::harness *harness_;
    sams_lare_solver *solver_ = nullptr;
    int device_ = 0;

    static void check(int rc)
    {
        if (rc != SAMS_OK) throw std::runtime_error(std::string("LARE3D: ") + sams_lare_last_error());
    }

    void create(simulationData &d)
    {
        const sams_lare_params p = params(*harness_, d);
        const sams_lare_bcs b = bcs(*harness_);
        check(sams_lare_create(&p, &b, device_, &solver_));
        for (int f = 0; f < SAMS_NFIELDS; ++f)
            check(sams_lare_upload_field(solver_, f, harness_->variableRegistry.box(f)));
    }
};

}  // namespace LARE
