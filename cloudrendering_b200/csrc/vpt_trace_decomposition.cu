// vpt_trace_decomposition.cu - decomposition tracking kernels (instantiations of vpt_trace.cuh).
#include "vpt_trace.cuh"

namespace vpt {

VPT_DEFINE_TRACKER(kDecomposition, kDense)
VPT_DEFINE_TRACKER_TEX(kDecomposition)
VPT_DEFINE_TRACKER(kDecomposition, kNanoVdb)

}  // namespace vpt
