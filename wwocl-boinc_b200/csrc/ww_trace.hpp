// ww_trace.hpp -- NVTX ranges around the library's host-side stages, so an
// Nsight Systems or Nsight Compute capture shows where the host queued each
// kernel (the reference's tracing was OpenCL event profiling, main.cpp:1318).
// NVTX v3 is header-only: without an attached tool the calls do nothing.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace ww {

struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

}  // namespace ww
