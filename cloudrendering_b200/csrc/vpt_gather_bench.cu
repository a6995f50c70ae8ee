// vpt_gather_bench.cu - the random 32-byte-sector gather rate that bounds the trackers.
//
// A density lookup is one 4-byte load at a data-dependent address: every lookup moves (at least)
// one 32-byte sector, and neighbouring lanes rarely share a sector.  This kernel measures the rate
// of exactly that access on this GPU: each thread issues 4-byte loads at pseudo-random
// sector-aligned offsets of a buffer (8 independent address streams per thread, so the rate is
// bound by the memory system rather than by one chain's latency).  With a buffer larger than L2 it
// is the HBM random-sector rate, with a buffer well inside L2 the L2 rate.
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/vpt_b200.h"
#include "vpt_kernels.h"

namespace {

constexpr int kStreams = 8;

__device__ __forceinline__ uint32_t xorshift32(uint32_t x) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return x;
}

__global__ void gather_bench_kernel(const float* __restrict__ buf, uint32_t sector_mask, int loads_per_stream,
                                    uint32_t seed, float* __restrict__ sink) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s[kStreams];
#pragma unroll
    for (int k = 0; k < kStreams; ++k) s[k] = xorshift32((tid * kStreams + k) * 0x9E3779B9u ^ seed) | 1u;
    float acc = 0.0f;
    for (int i = 0; i < loads_per_stream; ++i) {
#pragma unroll
        for (int k = 0; k < kStreams; ++k) {
            s[k] = xorshift32(s[k]);
            acc += __ldg(buf + (size_t)(s[k] & sector_mask) * 8);
        }
    }
    if (acc == -1.0f) sink[0] = acc;  // keeps the loads; never true for the non-negative buffers used
}

}  // namespace

extern "C" VptStatus vpt_gather_bench(const float* buffer, size_t bytes, int blocks, int loads_per_thread,
                                      uint32_t seed, float* sink, void* stream) {
    if (!buffer || !sink || bytes < 64 || (bytes & (bytes - 1)) || blocks <= 0 || loads_per_thread < kStreams ||
        bytes / 32 > (size_t)UINT32_MAX + 1)
        return VPT_ERR_ARG;
    const uint32_t mask = (uint32_t)(bytes / 32 - 1);
    gather_bench_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(buffer, mask,
                                                                              loads_per_thread / kStreams, seed, sink);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}
