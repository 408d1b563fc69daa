// lare_dump.cu -- ghost-inclusive state dumps (checkpoint / restart).
//
// Format "SAMSDUMP1", the one the oracle's reference harness writes for the
// reference's own state (oracle/ref_harness.cpp) and oracle/dumpio.py reads:
//   line 1  SAMSDUMP1
//   line 2  one JSON object: "nx","ny","nz","step","time","dt","dts" and
//           "arrays": [{"name","rank","lb":[3],"ub":[3],"offset"}, ...]
//   then    the arrays as little-endian float64, each row-major (z fastest)
//           over its own index bounds, at "offset" bytes after line 2.
// A checkpoint holds the 13 harness variables over their local ranges
// (centred -1..n+2, half-cell -2..n+2), the step count, the time and the dt
// of the last step (which the next step's edge viscosity reads), so a
// restart continues bit for bit.  Reading accepts any SAMSDUMP1 file of the
// same grid, including the reference harness's dumps (their extra arrays are
// skipped).
#include "lare_dump.cuh"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace sams {

namespace {

// Names of the harness variables in a dump (the reference's member names).
const char *const kDumpNames[SAMS_NFIELDS] = {"rho", "energy_electron", "energy_ion", "vx", "vy", "vz",
                                              "vx1", "vy1", "vz1", "bx", "by", "bz", "dm"};

bool number_after(const std::string &s, const char *key, size_t from, double *out, size_t *end = nullptr)
{
    size_t p = s.find(key, from);
    if (p == std::string::npos) return false;
    p += std::strlen(key);
    const char *b = s.c_str() + p;
    char *e = nullptr;
    const double v = std::strtod(b, &e);
    if (e == b) return false;
    *out = v;
    if (end) *end = p + (size_t)(e - b);
    return true;
}

bool triple_after(const std::string &s, const char *key, size_t from, long long v[3], size_t *end)
{
    size_t p = s.find(key, from);
    if (p == std::string::npos) return false;
    p += std::strlen(key);
    for (int d = 0; d < 3; ++d) {
        const char *b = s.c_str() + p;
        char *e = nullptr;
        v[d] = std::strtoll(b, &e, 10);
        if (e == b) return false;
        p += (size_t)(e - b);
        if (d < 2) {
            if (s[p] != ',') return false;
            ++p;
        }
    }
    *end = p;
    return true;
}

}  // namespace

int dump_write(const char *path, const DumpState &st, const double *const box[SAMS_NFIELDS], std::string &err)
{
    const long long n[3] = {st.nx, st.ny, st.nz};
    std::ostringstream h;
    h.precision(17);
    h << "{\"nx\":" << st.nx << ",\"ny\":" << st.ny << ",\"nz\":" << st.nz << ",\"step\":" << st.step
      << ",\"phase\":\"checkpoint\",\"time\":" << st.time << ",\"dt\":" << st.dt << ",\"dts\":[" << st.dt
      << "],\"arrays\":[";
    long long off = 0;
    std::vector<long long> counts(SAMS_NFIELDS);
    for (int f = 0; f < SAMS_NFIELDS; ++f) {
        long long lb[3], cnt = 1;
        for (int d = 0; d < 3; ++d) {
            lb[d] = sams_lare_field_lb(f, d);
            cnt *= n[d] + 2 - lb[d] + 1;
        }
        counts[f] = cnt;
        h << (f ? "," : "") << "{\"name\":\"" << kDumpNames[f] << "\",\"rank\":3,\"lb\":[" << lb[0] << "," << lb[1]
          << "," << lb[2] << "],\"ub\":[" << n[0] + 2 << "," << n[1] + 2 << "," << n[2] + 2 << "],\"offset\":" << off
          << "}";
        off += cnt * (long long)sizeof(double);
    }
    h << "]}";
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out) {
        err = std::string("cannot open ") + path + " for writing";
        return SAMS_ERR_INVALID;
    }
    out << "SAMSDUMP1\n" << h.str() << "\n";
    std::vector<double> row;
    for (int f = 0; f < SAMS_NFIELDS; ++f) {
        const long long lb0 = sams_lare_field_lb(f, 0), lb1 = sams_lare_field_lb(f, 1), lb2 = sams_lare_field_lb(f, 2);
        row.resize((size_t)(n[2] + 2 - lb2 + 1));
        for (long long i = lb0; i <= n[0] + 2; ++i)
            for (long long j = lb1; j <= n[1] + 2; ++j) {
                const double *src = box[f] + sams_box_index(n[1], n[2], i, j, lb2);
                std::memcpy(row.data(), src, row.size() * sizeof(double));
                out.write(reinterpret_cast<const char *>(row.data()), (std::streamsize)(row.size() * sizeof(double)));
            }
    }
    if (!out) {
        err = std::string("write failed: ") + path;
        return SAMS_ERR_INVALID;
    }
    return SAMS_OK;
}

int dump_read(const char *path, DumpState &st, double *const box[SAMS_NFIELDS], bool present[SAMS_NFIELDS],
              std::string &err)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        err = std::string("cannot open ") + path;
        return SAMS_ERR_INVALID;
    }
    std::string magic, header;
    std::getline(in, magic);
    if (magic != "SAMSDUMP1") {
        err = std::string(path) + " is not a SAMSDUMP1 file";
        return SAMS_ERR_INVALID;
    }
    std::getline(in, header);
    const std::streamoff data0 = in.tellg();
    in.seekg(0, std::ios::end);
    const std::streamoff fsize = in.tellg();
    double nx, ny, nz, step, time, dt;
    if (!number_after(header, "\"nx\":", 0, &nx) || !number_after(header, "\"ny\":", 0, &ny) ||
        !number_after(header, "\"nz\":", 0, &nz) || !number_after(header, "\"step\":", 0, &step) ||
        !number_after(header, "\"time\":", 0, &time) || !number_after(header, "\"dt\":", 0, &dt)) {
        err = std::string(path) + ": header lacks nx/ny/nz/step/time/dt";
        return SAMS_ERR_INVALID;
    }
    if ((long long)nx != st.nx || (long long)ny != st.ny || (long long)nz != st.nz) {
        err = std::string(path) + ": grid " + std::to_string((long long)nx) + "x" + std::to_string((long long)ny) +
              "x" + std::to_string((long long)nz) + " differs from the solver's";
        return SAMS_ERR_INVALID;
    }
    st.step = (long long)step;
    st.time = time;
    st.dt = dt;
    const long long n[3] = {st.nx, st.ny, st.nz};
    for (int f = 0; f < SAMS_NFIELDS; ++f) present[f] = false;
    size_t p = header.find("\"arrays\":[");
    if (p == std::string::npos) {
        err = std::string(path) + ": header has no array directory";
        return SAMS_ERR_INVALID;
    }
    std::vector<double> row;
    while ((p = header.find("{\"name\":\"", p)) != std::string::npos) {
        p += 9;
        const size_t q = header.find('"', p);
        if (q == std::string::npos) break;
        const std::string name = header.substr(p, q - p);
        long long lb[3], ub[3];
        double rank, offset;
        size_t e;
        if (!number_after(header, "\"rank\":", q, &rank) || !triple_after(header, "\"lb\":[", q, lb, &e) ||
            !triple_after(header, "\"ub\":[", e, ub, &e) || !number_after(header, "\"offset\":", e, &offset, &e)) {
            err = std::string(path) + ": malformed entry for array " + name;
            return SAMS_ERR_INVALID;
        }
        p = e;
        int f = -1;
        for (int c = 0; c < SAMS_NFIELDS; ++c)
            if (name == kDumpNames[c]) f = c;
        if (f < 0) continue;  // an intermediate or metric array: not state
        for (int d = 0; d < 3; ++d)
            if ((int)rank != 3 || lb[d] != sams_lare_field_lb(f, d) || ub[d] != n[d] + 2) {
                err = std::string(path) + ": array " + name + " does not cover the field's local range";
                return SAMS_ERR_INVALID;
            }
        const long long cnt = (ub[0] - lb[0] + 1) * (ub[1] - lb[1] + 1) * (ub[2] - lb[2] + 1);
        if (offset < 0 || data0 + (std::streamoff)offset + (std::streamoff)(cnt * 8) > fsize) {
            err = std::string(path) + ": array " + name + " runs past the end of the file";
            return SAMS_ERR_INVALID;
        }
        in.seekg(data0 + (std::streamoff)offset);
        row.resize((size_t)(ub[2] - lb[2] + 1));
        for (long long i = lb[0]; i <= ub[0]; ++i)
            for (long long j = lb[1]; j <= ub[1]; ++j) {
                in.read(reinterpret_cast<char *>(row.data()), (std::streamsize)(row.size() * sizeof(double)));
                std::memcpy(box[f] + sams_box_index(n[1], n[2], i, j, lb[2]), row.data(), row.size() * sizeof(double));
            }
        if (!in) {
            err = std::string("read failed: ") + path;
            return SAMS_ERR_INVALID;
        }
        present[f] = true;
    }
    return SAMS_OK;
}

}  // namespace sams
