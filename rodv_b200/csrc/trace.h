// trace.h -- NVTX ranges around the host-side phases (forming, packing,
// uploading, launching and finishing batches), so that a timeline tool shows
// where host time goes next to the kernels.  NVTX v3 is header-only: without
// an attached tool each range costs a few nanoseconds and does nothing.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace rodv {

class TraceRange {
 public:
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace rodv
