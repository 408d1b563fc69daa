// sams_runner.hpp -- C++ host API of the B200 LARE3D path, shaped like the
// reference's package / initial-condition / boundary-condition interface so
// that IC packages written for SAMS compile against it and drive the GPU
// timestep.
//
// What it mirrors (reference paths relative to the project root):
//   portableWrapper::portableArray / Range / applyKernel / assign / LAMBDA
//       include/pp/array.h, range.h, portableWrapperFrontend.h -- here host
//       views over the box buffers of the harness variables
//   SAMS::harness {axisRegistry, variableRegistry}
//       include/harness/harness.h:10-27, axisRegistry.h:973-985,
//       variableRegistry.h:69-420, variableDef.h:402-605
//   SAMS::simplePeriodicBC / simpleZeroGradientBC / simpleMirrorBC /
//       simpleClamp   include/boundaryConditions/builtInBoundaryConditions.h
//   SAMS::runner<Packages...> event order and parameter injection by type
//       include/runner/runner.h:108-611, runnerMacros.h
//   LARE::simulationData / LARE::LARE3D   src/PhysicsPackages/LARE/shared_data.h
// Underneath, LARE::LARE3D calls the C ABI of include/sams_lare.h: the whole
// timestep runs on the GPU; the host arrays are the IC package's view and are
// uploaded once, before the first step, and refreshed on request.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <string_view>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "../sams_lare.h"

#ifndef LAMBDA
#define LAMBDA [=]
#endif

namespace portableWrapper {

struct Range {
    long long lower_bound, upper_bound;
    bool all = false;  // Range(): every index of the dimension it slices
    Range(long long lb, long long ub) : lower_bound(lb), upper_bound(ub) {}
    explicit Range(long long n) : lower_bound(1), upper_bound(n) {}
    Range() : lower_bound(0), upper_bound(-1), all(true) {}
};

enum class arrayTags { host = 0, accelerated = 1 };

// A view over host memory with the reference's index ranges (any lower bound,
// last index fastest).  Indexing with all integers gives an element; with
// some Range arguments it gives a view of lower rank over those dimensions
// (the reference's slicing, e.g. a(-2, Range(), Range()) is the plane -2 of
// dimension 0, include/pp/array.h).
template <typename T, int N, arrayTags tag = arrayTags::accelerated>
class portableArray {
public:
    portableArray() = default;
    void bind(T *p, const long long *lb, const long long *ub, const long long *stride)
    {
        data_ = p;
        for (int d = 0; d < N; ++d) {
            lb_[d] = lb[d];
            ub_[d] = ub[d];
            st_[d] = stride[d];
        }
    }
    template <typename... I>
    decltype(auto) operator()(I... idx) const
    {
        static_assert(sizeof...(I) == N, "wrong number of indices");
        if constexpr ((std::is_integral_v<I> && ...)) {
            const long long ix[N] = {(long long)idx...};
            long long o = 0;
            for (int d = 0; d < N; ++d) o += (ix[d] - lb_[d]) * st_[d];
            return static_cast<T &>(data_[o]);
        } else {
            constexpr int M = ((std::is_same_v<I, Range> ? 1 : 0) + ...);
            static_assert(M > 0 && M <= N, "a slice keeps at least one dimension");
            portableArray<T, M, tag> v;
            long long lb[M], ub[M], st[M], off = 0;
            int d = 0, m = 0;
            auto one = [&](const auto &x) {
                if constexpr (std::is_same_v<std::decay_t<decltype(x)>, Range>) {
                    const long long a = x.all ? lb_[d] : x.lower_bound, b = x.all ? ub_[d] : x.upper_bound;
                    if (a < lb_[d] || b > ub_[d]) throw std::out_of_range("portableArray: slice outside the array");
                    lb[m] = a;
                    ub[m] = b;
                    st[m] = st_[d];
                    off += (a - lb_[d]) * st_[d];
                    ++m;
                } else {
                    if ((long long)x < lb_[d] || (long long)x > ub_[d])
                        throw std::out_of_range("portableArray: index outside the array");
                    off += ((long long)x - lb_[d]) * st_[d];
                }
                ++d;
            };
            (one(idx), ...);
            v.bind(data_ + off, lb, ub, st);
            return v;
        }
    }
    Range getRange(int d) const { return Range(lb_[d], ub_[d]); }
    T *data() const { return data_; }
    long long getElements() const
    {
        long long n = 1;
        for (int d = 0; d < N; ++d) n *= ub_[d] - lb_[d] + 1;
        return n;
    }

private:
    T *data_ = nullptr;
    long long lb_[N] = {}, ub_[N] = {}, st_[N] = {};
};

template <typename T, int N>
using acceleratedArray = portableArray<T, N, arrayTags::accelerated>;
template <typename T, int N>
using hostArray = portableArray<T, N, arrayTags::host>;

template <class F>
void applyKernel(F f, Range a)
{
    for (long long i = a.lower_bound; i <= a.upper_bound; ++i) f(i);
}
template <class F>
void applyKernel(F f, Range a, Range b)
{
    for (long long i = a.lower_bound; i <= a.upper_bound; ++i)
        for (long long j = b.lower_bound; j <= b.upper_bound; ++j) f(i, j);
}
template <class F>
void applyKernel(F f, Range a, Range b, Range c)
{
#ifdef _OPENMP
#pragma omp parallel for
#endif
    for (long long i = a.lower_bound; i <= a.upper_bound; ++i)
        for (long long j = b.lower_bound; j <= b.upper_bound; ++j)
            for (long long k = c.lower_bound; k <= c.upper_bound; ++k) f(i, j, k);
}
inline void fence() {}

namespace detail {
// Visit every element of an N-d view (last index fastest): f(offset of dst)
template <typename T, int N, arrayTags tag, typename F>
void each_index(const portableArray<T, N, tag> &a, F f)
{
    long long ix[N];
    for (int d = 0; d < N; ++d) {
        ix[d] = a.getRange(d).lower_bound;
        if (a.getRange(d).upper_bound < ix[d]) return;
    }
    for (;;) {
        f(ix);
        int d = N - 1;
        while (d >= 0 && ++ix[d] > a.getRange(d).upper_bound) {
            ix[d] = a.getRange(d).lower_bound;
            --d;
        }
        if (d < 0) return;
    }
}
template <typename T, int N, arrayTags tag>
T &at(const portableArray<T, N, tag> &a, const long long *ix)
{
    if constexpr (N == 1) return a(ix[0]);
    else if constexpr (N == 2) return a(ix[0], ix[1]);
    else return a(ix[0], ix[1], ix[2]);
}
}  // namespace detail

// pw::assign(array or slice, value) and pw::assign(array or slice, array or
// slice of the same extents) (include/pp/algorithm.h): element by element,
// the source indexed at the same offsets from its own lower bounds.
template <typename T, int N, arrayTags tag, typename V>
void assign(portableArray<T, N, tag> a, const V &v)
{
    if constexpr (std::is_same_v<V, portableArray<T, N, arrayTags::accelerated>> ||
                  std::is_same_v<V, portableArray<T, N, arrayTags::host>>) {
        for (int d = 0; d < N; ++d)
            if (a.getRange(d).upper_bound - a.getRange(d).lower_bound !=
                v.getRange(d).upper_bound - v.getRange(d).lower_bound)
                throw std::runtime_error("Error: pw::assign between arrays of different extents");
        detail::each_index(a, [&](const long long *ix) {
            long long jx[N];
            for (int d = 0; d < N; ++d) jx[d] = ix[d] - a.getRange(d).lower_bound + v.getRange(d).lower_bound;
            detail::at(a, ix) = detail::at(v, jx);
        });
    } else {
        detail::each_index(a, [&](const long long *ix) { detail::at(a, ix) = v; });
    }
}

}  // namespace portableWrapper

namespace SAMS {

namespace pw = portableWrapper;
// SAMS::cout (rank-0 output in the reference; one process here)
inline std::ostream &cout = std::cout;
using T_dataType = double;
using T_indexType = long long;
using T_sizeType = long long;

enum class staggerType { CENTRED = 0, HALF_CELL = 1 };
namespace domain {
enum class edges { lower = 0, upper = 1 };
}

struct MPIAxis {
    int axis;
    explicit MPIAxis(int a) : axis(a) {}
};

struct dimension {
    std::string axisName;
    int ghosts = 2;
    staggerType stagger = staggerType::CENTRED;
    dimension(std::string name, int g, staggerType s = staggerType::CENTRED) : axisName(std::move(name)), ghosts(g), stagger(s) {}
};

class variableDef;

// Boundary-condition objects.  On the GPU path a condition is a descriptor
// (kind, value) executed by the device fill kernels.  The built-in
// conditions name their kind.  A condition that only implements apply(dim,
// edge) on the host arrays (the reference's interface,
// include/boundaryConditions/boundaryConditions.h:9-15, as the LARE IC
// package's LAREBoundaryConditions does) reports kHostDefined; LARE::LARE3D
// then runs its apply() once on tagged host data at set-up and translates
// the plane copies it observes into a device descriptor (or refuses it).
class boundaryConditions {
public:
    static constexpr int kHostDefined = -1;
    virtual ~boundaryConditions() = default;
    virtual int kind() const { return kHostDefined; }
    virtual double value() const { return 0.0; }
    virtual void apply(int, domain::edges) {}
};

template <typename T, int rank, pw::arrayTags tag = pw::arrayTags::accelerated>
class simplePeriodicBC : public boundaryConditions {
public:
    explicit simplePeriodicBC(const variableDef &) {}
    int kind() const override { return SAMS_BC_PERIODIC; }
};
template <typename T, int rank, pw::arrayTags tag = pw::arrayTags::accelerated>
class simpleZeroGradientBC : public boundaryConditions {
public:
    explicit simpleZeroGradientBC(const variableDef &) {}
    int kind() const override { return SAMS_BC_ZERO_GRADIENT; }
};
template <typename T, int rank, pw::arrayTags tag = pw::arrayTags::accelerated>
class simpleMirrorBC : public boundaryConditions {
public:
    explicit simpleMirrorBC(const variableDef &) {}
    int kind() const override { return SAMS_BC_MIRROR; }
};
template <typename T, int rank, pw::arrayTags tag = pw::arrayTags::accelerated>
class simpleClamp : public boundaryConditions {
    T v_;
public:
    simpleClamp(const variableDef &, T v) : v_(v) {}
    int kind() const override { return SAMS_BC_CLAMP; }
    double value() const override { return (double)v_; }
};

class variableDef {
public:
    std::string name;
    int field = -1;
    std::vector<std::shared_ptr<boundaryConditions>> bcs[3][2];

    template <typename T>
    std::shared_ptr<boundaryConditions> addBoundaryCondition(int dim, domain::edges edge, std::shared_ptr<T> bc)
    {
        static_assert(std::is_base_of<boundaryConditions, T>::value, "not a boundary condition");
        if (dim < 0 || dim > 2) throw std::runtime_error("Error: variableDef addBoundaryCondition dimension out of range\n");
        bcs[dim][(int)edge].push_back(bc);
        return bc;
    }
    template <typename T>
    std::shared_ptr<boundaryConditions> addBoundaryCondition(int dim, std::shared_ptr<T> bc)
    {
        addBoundaryCondition(dim, domain::edges::lower, bc);
        return addBoundaryCondition(dim, domain::edges::upper, bc);
    }
    template <typename T>
    std::shared_ptr<boundaryConditions> addBoundaryCondition(std::shared_ptr<T> bc)
    {
        for (int d = 0; d < 3; ++d) addBoundaryCondition(d, bc);
        return bc;
    }
    template <typename T, typename... Args>
    std::shared_ptr<boundaryConditions> emplaceBoundaryCondition(int dim, domain::edges edge, Args &&...args)
    {
        return addBoundaryCondition(dim, edge, std::make_shared<T>(*this, std::forward<Args>(args)...));
    }
    template <typename T, typename... Args>
    std::shared_ptr<boundaryConditions> emplaceBoundaryCondition(int dim, Args &&...args)
    {
        auto bc = std::make_shared<T>(*this, std::forward<Args>(args)...);
        return addBoundaryCondition(dim, bc);
    }
    template <typename T, typename... Args>
    std::shared_ptr<boundaryConditions> emplaceBoundaryCondition(Args &&...args)
    {
        auto bc = std::make_shared<T>(*this, std::forward<Args>(args)...);
        return addBoundaryCondition(bc);
    }
};

class axisRegistry {
public:
    struct axis {
        long long n = 0;
        double lo = 0.0, hi = 0.0;
        bool set = false;
    };
    void registerAxis(const std::string &name, MPIAxis) { axes_[name]; }
    template <typename T_range>
    void setDomain(const std::string &name, long long elements, T_range minVal, T_range maxVal)
    {
        auto it = axes_.find(name);
        if (it == axes_.end()) throw std::runtime_error("Error: unknown axis " + name);
        it->second = axis{elements, (double)minVal, (double)maxVal, true};
    }
    const axis &get(const std::string &name) const
    {
        auto it = axes_.find(name);
        if (it == axes_.end() || !it->second.set) throw std::runtime_error("Error: axis " + name + " has no domain");
        return it->second;
    }
    // Edge (HALF_CELL, -2..n+2) or centred (-1..n+2) coordinates of an axis,
    // built as axisRegistry::setDomain builds them.
    template <typename T, int N, pw::arrayTags tag>
    void fillPPLocalAxis(const std::string &name, pw::portableArray<T, N, tag> &out, staggerType s)
    {
        static_assert(N == 1, "axes are one-dimensional");
        const axis &a = get(name);
        const long long lb = s == staggerType::HALF_CELL ? -2 : -1, ub = a.n + 2;
        auto &buf = store_[name + (s == staggerType::HALF_CELL ? "/b" : "/c")];
        buf.resize((size_t)(ub - lb + 1));
        for (long long i = lb; i <= ub; ++i)
            buf[(size_t)(i - lb)] = s == staggerType::HALF_CELL ? sams_axis_edge(a.lo, a.hi, a.n, i)
                                                                : sams_axis_centre(a.lo, a.hi, a.n, i);
        const long long st = 1;
        out.bind(buf.data(), &lb, &ub, &st);
    }

private:
    std::map<std::string, axis> axes_;
    std::map<std::string, std::vector<double>> store_;
};

class variableRegistry {
public:
    template <typename T, typename... Dims>
    void registerVariable(const std::string &name, pw::arrayTags, Dims...)
    {
        auto &v = vars_[name];
        v.name = name;
        for (int f = 0; f < SAMS_NFIELDS; ++f)
            if (name == sams_lare_field_names[f]) v.field = f;
        if (v.field < 0) throw std::runtime_error("Error: " + name + " is not a LARE3D harness variable");
    }
    variableDef &getVariable(const std::string &name)
    {
        auto it = vars_.find(name);
        if (it == vars_.end()) throw std::runtime_error("Error: variable " + name + " not registered");
        return it->second;
    }
    template <typename T>
    std::shared_ptr<boundaryConditions> addBoundaryCondition(const std::string &name, int dim, domain::edges edge,
                                                             std::shared_ptr<T> bc)
    {
        return getVariable(name).addBoundaryCondition(dim, edge, bc);
    }
    template <typename T>
    std::shared_ptr<boundaryConditions> addBoundaryCondition(const std::string &name, int dim, std::shared_ptr<T> bc)
    {
        return getVariable(name).addBoundaryCondition(dim, bc);
    }
    // Box storage of the registered variables (allocated by the runner).
    void allocate(long long nx, long long ny, long long nz)
    {
        nx_ = nx;
        ny_ = ny;
        nz_ = nz;
        const long long n = sams_box_elems(nx, ny, nz);
        for (auto &kv : vars_) store_[kv.second.field].assign((size_t)n, 0.0);
    }
    template <typename T, int N, pw::arrayTags tag>
    void fillPPArray(const std::string &name, pw::portableArray<T, N, tag> &out)
    {
        static_assert(N == 3, "LARE3D variables are three-dimensional");
        const int f = getVariable(name).field;
        long long lb[3], ub[3], st[3] = {(ny_ + 5) * (nz_ + 5), nz_ + 5, 1};
        const long long n[3] = {nx_, ny_, nz_};
        for (int d = 0; d < 3; ++d) {
            lb[d] = sams_lare_field_lb(f, d);
            ub[d] = n[d] + 2;
        }
        double *base = store_.at(f).data() + sams_box_index(ny_, nz_, lb[0], lb[1], lb[2]);
        out.bind(base, lb, ub, st);
    }
    double *box(int field) { return store_.at(field).data(); }
    const std::map<std::string, variableDef> &all() const { return vars_; }

private:
    std::map<std::string, variableDef> vars_;
    std::map<int, std::vector<double>> store_;
    long long nx_ = 0, ny_ = 0, nz_ = 0;
};

struct harness {
    SAMS::axisRegistry axisRegistry;
    SAMS::variableRegistry variableRegistry;
};

struct timeState {
    T_dataType time = 0.0;
    T_dataType dt = 0.0;
    T_indexType step = 0;
};

struct controlFunctions {
    std::function<void()> calculateTimestepFn;
    void calculateTimestep() { if (calculateTimestepFn) calculateTimestepFn(); }
};

namespace dataPacks {
template <typename... P>
struct multiPack {
    using type = std::tuple<P...>;
};
}  // namespace dataPacks

namespace detail {
template <typename P>
P make_package(harness &h)
{
    if constexpr (std::is_constructible_v<P, harness &>) return P(h);
    else return P{};
}
template <typename T, typename = void>
struct pack_of {
    using type = std::tuple<>;
};
template <typename T>
struct pack_of<T, std::void_t<typename T::dataPack>> {
    using type = typename T::dataPack::type;
};
}  // namespace detail

// The runner: packages are plain classes; an event is called on every active
// package that defines it, in template-list order, with its parameters
// supplied by type (runner.h:80-611).
template <typename... Packages>
class runner {
public:
    harness harnessData;
    timeState tData;
    controlFunctions ctrl;
    std::tuple<Packages...> packages{detail::make_package<Packages>(harnessData)...};
    using packs_t = decltype(std::tuple_cat(std::declval<typename detail::pack_of<Packages>::type>()...));
    packs_t packs{};
    bool active[sizeof...(Packages)] = {};

    runner() { ctrl.calculateTimestepFn = [this] { calculateTimestep(); }; }

    void activatePackage(const std::string &name)
    {
        bool found = false;
        size_t idx = 0;
        std::apply([&](auto &...p) { ((found |= activate_one(p, name, idx++)), ...); }, packages);
        if (!found) throw std::runtime_error("ERROR: Package with name " + name + " not found in runner.\n");
    }

#define SAMS_EVENT_AS(fn, ev)                                                                  \
    void fn()                                                                                    \
    {                                                                                            \
        size_t idx = 0;                                                                          \
        std::apply([&](auto &...p) { (call_##fn(p, idx++), ...); }, packages);                   \
    }                                                                                            \
    template <typename P>                                                                        \
    void call_##fn(P &p, size_t idx)                                                             \
    {                                                                                            \
        if constexpr (requires { &P::ev; }) {                                                    \
            if (active[idx]) invoke(p, &P::ev);                                                  \
        }                                                                                        \
    }
#define SAMS_EVENT(ev) SAMS_EVENT_AS(ev, ev)
    SAMS_EVENT(registerAxes)
    SAMS_EVENT(registerVariables)
    SAMS_EVENT(defaultValues)
    SAMS_EVENT(controlVariables)
    SAMS_EVENT(setDomain)
    SAMS_EVENT(getVariables)
    SAMS_EVENT(defaultVariables)
    SAMS_EVENT(initialConditions)
    SAMS_EVENT(setBoundaryConditions)
    SAMS_EVENT(startOfTimestep)
    SAMS_EVENT(halfTimestep)
    SAMS_EVENT(endOfTimestep)
    SAMS_EVENT_AS(calculateTimestepEvent, calculateTimestep)
    SAMS_EVENT(getTimestep)
    SAMS_EVENT(queryTerminate)
    SAMS_EVENT(finalize)
#undef SAMS_EVENT
#undef SAMS_EVENT_AS

    // runner::calculateTimestep (runner.h:158-169)
    void calculateTimestep()
    {
        tData.dt = std::numeric_limits<T_dataType>::max();
        calculateTimestepEvent();
        getTimestep();
    }

    void decomposeAndAllocate()
    {
        auto &ax = harnessData.axisRegistry;
        harnessData.variableRegistry.allocate(ax.get("X").n, ax.get("Y").n, ax.get("Z").n);
    }

    // runner::initializePackages (runner.h:548-562), without output
    void initializePackages()
    {
        registerAxes();
        registerVariables();
        defaultValues();
        controlVariables();
        setDomain();
        decomposeAndAllocate();
        getVariables();
        defaultVariables();
        initialConditions();
        setBoundaryConditions();
    }

    // runner::runPackages (runner.h:564-586), without output or steering
    void runPackages()
    {
        for (;;) {
            startOfTimestep();
            halfTimestep();
            tData.step++;
            tData.time += tData.dt;
            endOfTimestep();
            if (queryTerminateAll()) break;
        }
    }

    bool queryTerminateAll()
    {
        terminate_ = false;
        queryTerminate();
        return terminate_;
    }

    template <typename T>
    T &getDataPack() { return std::get<T>(packs); }
    harness &getHarness() { return harnessData; }

private:
    bool terminate_ = false;

    template <typename P>
    bool activate_one(P &, const std::string &name, size_t idx)
    {
        if (P::name == name) {
            active[idx] = true;
            return true;
        }
        return false;
    }

    template <typename A>
    A &arg()
    {
        using D = std::remove_cv_t<std::remove_reference_t<A>>;
        if constexpr (std::is_same_v<D, harness>) return harnessData;
        else if constexpr (std::is_same_v<D, timeState>) return tData;
        else if constexpr (std::is_same_v<D, controlFunctions>) return ctrl;
        else if constexpr (std::is_same_v<D, bool>) return terminate_;
        else return std::get<D>(packs);
    }

    template <typename P, typename C, typename R, typename... A>
    void invoke(P &p, R (C::*fn)(A...))
    {
        (p.*fn)(arg<A>()...);
    }
};

}  // namespace SAMS
