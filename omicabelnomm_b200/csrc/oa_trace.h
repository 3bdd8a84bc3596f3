// NVTX ranges of the engine's host-side phases (covariates, trait block, SNP
// block, per-chunk launches, stored-row sort and copy-back, file reading and
// output writing).  They name the spans that Nsight Systems and Nsight Compute
// show; without a tool attached each range costs a function call.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace oa {
struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};
}  // namespace oa

#define OA_TRACE_CAT2(a, b) a##b
#define OA_TRACE_CAT(a, b) OA_TRACE_CAT2(a, b)
#define OA_TRACE(name) ::oa::TraceRange OA_TRACE_CAT(oa_trace_, __LINE__)(name)
