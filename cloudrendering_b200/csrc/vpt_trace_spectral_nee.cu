// vpt_trace_spectral_nee.cu - spectral nee tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kSpectralNextEvent, kDense)
VPT_DEFINE_TRACKER(kSpectralNextEvent + 100, kDense)
VPT_DEFINE_TRACKER(kSpectralNextEvent, kNanoVdb)

}  // namespace vpt
