// vpt_trace_ratio.cu - ratio tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kRatio, kDense)
VPT_DEFINE_TRACKER_TEX(kRatio)
VPT_DEFINE_TRACKER(kRatio, kNanoVdb)

}  // namespace vpt
