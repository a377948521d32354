// trace.cuh -- NVTX ranges around the C-ABI entry points: each call shows as
// a named range in Nsight Systems and can select kernels in Nsight Compute
// (--nvtx --nvtx-include).  The reference has no tracing beyond its wall-clock
// timer (src/timer.c:8-17).  Header-only NVTX: near-zero cost without a tool.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace svof_trace {
struct Range {
  explicit Range(const char *name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range &) = delete;
  Range &operator=(const Range &) = delete;
};
}  // namespace svof_trace

// a range named after the enclosing function, closed when it returns
#define SVOF_RANGE() const svof_trace::Range svof_range_guard_(__func__)
