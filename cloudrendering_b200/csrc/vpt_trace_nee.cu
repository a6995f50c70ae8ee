// vpt_trace_nee.cu - nee tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kNextEvent, kDense)
VPT_DEFINE_TRACKER_TEX(kNextEvent)
VPT_DEFINE_TRACKER(kNextEvent + 100, kDense)
VPT_DEFINE_TRACKER_TEX(kNextEvent + 100)
VPT_DEFINE_TRACKER(kNextEvent, kNanoVdb)

}  // namespace vpt
