// boinc_shim.hpp -- the volunteer-computing client calls the reference's host
// makes (boinc_api.h), as a standalone shim: this build runs without a BOINC
// client, so every call behaves as boinc_is_standalone() does in the
// reference.  The host program calls them at the reference's points:
//
//   boinc_resolve_filename + boinc_fopen   my_fopen (main.cpp:93-100)
//   boinc_begin/end_critical_section       around result read-back and the
//                                           checkpoint (main.cpp:1753,1786)
//   boinc_checkpoint_completed             after a state write (main.cpp:220)
//   boinc_fraction_done                    progress, every 2 s and at the end
//                                           (main.cpp:1699-1708,1768)
//   boinc_finish                           exit (main.cpp:1549,1800)
//
// A build linked against a real client would replace these bodies; the call
// sites stay.
#pragma once

#include <stdio.h>
#include <stdlib.h>

#include <string>

namespace boinc {

struct ShimState {
    int critical_depth = 0;         // nesting of critical sections
    double fraction_done = 0.0;     // last reported progress
    unsigned checkpoints = 0;       // completed checkpoints
};

inline ShimState &shim() {
    static ShimState s;
    return s;
}

inline bool is_standalone() { return true; }

// Logical -> physical file name (identity without a client).
inline std::string resolve_filename(const std::string &name) { return name; }

inline FILE *fopen_resolved(const std::string &name, const char *mode) {
    return ::fopen(resolve_filename(name).c_str(), mode);
}

inline void begin_critical_section() { ++shim().critical_depth; }
inline void end_critical_section() {
    if (shim().critical_depth > 0) --shim().critical_depth;
}

inline void checkpoint_completed() { ++shim().checkpoints; }

inline void fraction_done(double d) { shim().fraction_done = d < 0 ? 0 : (d > 1 ? 1 : d); }

[[noreturn]] inline void finish(int status) {
    fflush(stdout);
    fflush(stderr);
    exit(status);
}

}  // namespace boinc
