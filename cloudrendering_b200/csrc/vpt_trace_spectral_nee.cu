// vpt_trace_spectral_nee.cu - spectral nee tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kSpectralNextEvent, kDense)
VPT_DEFINE_TRACKER(kSpectralNextEvent + 100, kDense)
VPT_DEFINE_TRACKER(kSpectralNextEvent, kNanoVdb)

cudaError_t launch_tracker_spectral_nee_iso(const TraceParams& P, int schedule, int features, int pb,
                                            cudaStream_t s) {
    return launch_trace_t<kSpectralNextEventIso, kTrilinear, kDense, false>(P, schedule, features, pb, s);
}

}  // namespace vpt
