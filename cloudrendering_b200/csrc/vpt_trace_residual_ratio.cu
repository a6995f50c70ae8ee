// vpt_trace_residual_ratio.cu - residual ratio tracking kernels (the reference's estimator and the unbiased next-event form) (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kResidualRatio, kDense)
VPT_DEFINE_TRACKER(kResidualRatioNee, kDense)
VPT_DEFINE_TRACKER_TEX(kResidualRatioNee)

}  // namespace vpt
