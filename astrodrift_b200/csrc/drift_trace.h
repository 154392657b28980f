// drift_trace.h -- NVTX ranges around the library's host-side phases, so an
// Nsight Systems timeline shows the copy-in, the chunk launches, the
// copy-out, the server's batches and the adjoint by name.  NVTX v3 is
// header-only; without an attached tool a range costs one test of a null
// function pointer.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace drift {

class TraceRange {
public:
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

}  // namespace drift
