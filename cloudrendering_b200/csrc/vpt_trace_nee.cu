// vpt_trace_nee.cu - nee tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kNextEvent, kDense)
VPT_DEFINE_TRACKER_TEX(kNextEvent)
VPT_DEFINE_TRACKER(kNextEvent + 100, kDense)
VPT_DEFINE_TRACKER_TEX(kNextEvent + 100)
VPT_DEFINE_TRACKER(kNextEvent, kNanoVdb)

cudaError_t launch_tracker_nee_iso(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s) {
    return launch_trace_t<kNextEventIso, kTrilinear, kDense, false>(P, schedule, features, pb, s);
}

}  // namespace vpt
