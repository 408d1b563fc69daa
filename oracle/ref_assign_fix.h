/*
 * ref_assign_fix.h -- force-included (g++ -include) into the reference's
 * src/PhysicsPackages/LARE/lagran.cpp only, by oracle/Makefile.
 *
 * The reference's resistive path cannot run as shipped: resistive_effects
 * (lagran.cpp:478-505) starts with pw::assign(data.bx1, data.bx) and the two
 * similar copies (lagran.cpp:482-484).  bx1 is allocated cell-centred,
 * (n+4)^3 elements (setup.cpp:191), while bx is face-staggered in x,
 * (n+5)(n+4)^2 elements (setup.cpp:63), and the array-to-array pw::assign
 * (include/pp/algorithm.h:73-79) throws "Source and destination arrays must
 * have the same number of elements" on the first resistive step.
 *
 * Those three calls are the only array-to-array assignments in lagran.cpp.
 * This non-template overload is preferred over the library template for
 * them.  When the element counts agree it copies exactly as the template
 * does (zero-based position by position); when they differ it copies element
 * by element over the index range the two arrays share, which is the data
 * bstep (lagran.cpp:537-590) reads.  No reference source file is modified.
 */
#ifndef SAMS_ORACLE_REF_ASSIGN_FIX_H
#define SAMS_ORACLE_REF_ASSIGN_FIX_H

#include "pp/parallelWrapper.h"
#include <algorithm>

namespace portableWrapper
{
    inline void assign(portableArray<double, 3, arrayTags::accelerated> dest,
                       const portableArray<double, 3, arrayTags::accelerated> &src)
    {
        if (dest.getElements() == src.getElements())
        {
            const int64_t n0 = src.getRange(0).upper_bound - src.getRange(0).lower_bound + 1;
            const int64_t n1 = src.getRange(1).upper_bound - src.getRange(1).lower_bound + 1;
            const int64_t n2 = src.getRange(2).upper_bound - src.getRange(2).lower_bound + 1;
            for (int64_t i = 0; i < n0; ++i)
                for (int64_t j = 0; j < n1; ++j)
                    for (int64_t k = 0; k < n2; ++k)
                        dest.getZB(i, j, k) = src.getZB(i, j, k);
            return;
        }
        int64_t lb[3], ub[3];
        for (int d = 0; d < 3; ++d)
        {
            lb[d] = std::max(dest.getRange(d).lower_bound, src.getRange(d).lower_bound);
            ub[d] = std::min(dest.getRange(d).upper_bound, src.getRange(d).upper_bound);
        }
        for (int64_t i = lb[0]; i <= ub[0]; ++i)
            for (int64_t j = lb[1]; j <= ub[1]; ++j)
                for (int64_t k = lb[2]; k <= ub[2]; ++k)
                    dest(i, j, k) = src(i, j, k);
    }
}

#endif
