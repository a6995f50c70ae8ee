// vpt_trace_spectral_delta.cu - spectral delta tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kSpectralDelta, kDense)
VPT_DEFINE_TRACKER(kSpectralDelta, kNanoVdb)

}  // namespace vpt
