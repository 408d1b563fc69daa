// lare_dump.cuh -- SAMSDUMP1 state dumps of the 13 harness variables
// (checkpoint / restart); format described in lare_dump.cu.
#pragma once

#include <string>

#include "sams_lare.h"

namespace sams {

struct DumpState {
    long long nx, ny, nz;
    long long step;
    double time;
    double dt;  // dt of the last step taken (0 before the first)
};

// Write box buffers (-2..n+2 per dimension, z fastest) of the 13 fields.
int dump_write(const char *path, const DumpState &st, const double *const box[SAMS_NFIELDS], std::string &err);

// Read a dump of the grid st.nx x st.ny x st.nz into box buffers; present[f]
// tells which fields the file held.  Fills st.step, st.time and st.dt.
int dump_read(const char *path, DumpState &st, double *const box[SAMS_NFIELDS], bool present[SAMS_NFIELDS],
              std::string &err);

}  // namespace sams
