// vpt_trace_batch.cu - the many-scene persistent launch (trace_batch_kernel).
#include "vpt_trace.cuh"

namespace vpt {

cudaError_t launch_trace_batch(const BatchLaunch& b, cudaStream_t s) {
    if (b.grid_kind == kNanoVdb) return batch_tracker<kNanoVdb>(b, s);
    if (b.grid_kind == kDenseTex) return batch_tracker<kDenseTex>(b, s);  // every scene has a texture object
    return batch_tracker<kDense>(b, s);
}

}  // namespace vpt
