// vpt_trace_batch.cu - the many-scene persistent launch (trace_batch_kernel).
#include "vpt_trace.cuh"

namespace vpt {

cudaError_t launch_trace_batch(const BatchLaunch& b, cudaStream_t s) {
    return b.grid_kind == kNanoVdb ? batch_tracker<kNanoVdb>(b, s) : batch_tracker<kDense>(b, s);
}

}  // namespace vpt
