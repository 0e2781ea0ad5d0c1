/*
 * Forced-include shim used ONLY when compiling the reference's own C++ headers
 * (test infrastructure; never part of the product).  The reference was written
 * for MSVC; these declarations let g++ accept it without editing any reference
 * file:
 *   - `min(...)` unqualified in coarse_grids_hierarchy.h:75  -> std::min
 *   - `sprintf_s(buf, fmt, ...)` in loads_calculator.h:1386 -> snprintf
 *   - <memory>/<cstring>/<algorithm> used without includes
 * Dependent-base member lookups (array.h:36, mesh_function.h:64,
 * coord_mesh_function.h:113) are accepted by g++ with -fpermissive.
 */
#ifndef LSG_REF_COMPAT_H
#define LSG_REF_COMPAT_H
#include <memory>
#include <cstring>
#include <cstdio>
#include <cmath>
#include <algorithm>
#include <string>
using std::min;
using std::max;
template <size_t Nbuf, typename... Args>
static inline int sprintf_s(char (&buf)[Nbuf], const char* fmt, Args... args)
{
    return std::snprintf(buf, Nbuf, fmt, args...);
}
#endif
