// vpt_trace_delta.cu - delta tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kDelta, kDense)
VPT_DEFINE_TRACKER_TEX(kDelta)
VPT_DEFINE_TRACKER(kDelta, kNanoVdb)

cudaError_t launch_tracker_delta_iso(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s) {
    return launch_trace_t<kDeltaIso, kTrilinear, kDense, false>(P, schedule, features, pb, s);
}

}  // namespace vpt
