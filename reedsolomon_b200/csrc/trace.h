// trace.h -- NVTX ranges around the library's entry points.
//
// NVTX3 is header-only: without a profiler attached (nsys, ncu), each range
// costs a call through a no-op function pointer.  Under a profiler every
// public call shows up as a named range on the calling thread's timeline.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace rsgpu {

struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

}  // namespace rsgpu

#define RS_TRACE(name) ::rsgpu::TraceRange rs_trace_range_(name)
