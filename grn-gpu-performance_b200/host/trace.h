// trace.h -- NVTX ranges around the host phases of an evaluation (compile,
// autotune, launch), of a search generation and of the surrogate's calls,
// for Nsight timelines.  NVTX 3 is header-only: without an attached tool a
// range costs a branch.
#ifndef GRN_HOST_TRACE_H_
#define GRN_HOST_TRACE_H_

#include <nvtx3/nvToolsExt.h>

namespace grn {

// Pushes a named range for the enclosing scope.
class TraceRange {
 public:
  explicit TraceRange(const char *name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange &) = delete;
  TraceRange &operator=(const TraceRange &) = delete;
};

}  // namespace grn

#endif  // GRN_HOST_TRACE_H_
