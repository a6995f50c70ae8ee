// vpt_trace_spectral_delta.cu - spectral delta tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kSpectralDelta, kDense)
VPT_DEFINE_TRACKER(kSpectralDelta, kNanoVdb)

cudaError_t launch_tracker_spectral_delta_iso(const TraceParams& P, int schedule, int features, int pb,
                                              cudaStream_t s) {
    return launch_trace_t<kSpectralDeltaIso, kTrilinear, kDense, false>(P, schedule, features, pb, s);
}

}  // namespace vpt
