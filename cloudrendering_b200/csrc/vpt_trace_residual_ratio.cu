// vpt_trace_residual_ratio.cu - residual ratio tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kResidualRatio, kDense)

}  // namespace vpt
