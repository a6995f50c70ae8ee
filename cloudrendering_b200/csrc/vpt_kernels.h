// vpt_kernels.h - host-side declarations of the kernel launchers in vpt_kernels.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "vpt_params.h"

namespace vpt {

constexpr int kTraceBlock = 128;

enum Schedule : int { kScheduleTiles = 0, kSchedulePersistent = 1, kScheduleRefill = 2 };

struct FbmParams {
    int octaves;
    float lacunarity;
    float gain;
    float base_frequency;
    float threshold;
    float contrast;
    float inv_max_dim;
};

uint64_t padded_paths(int width, int height, uint32_t frames);
void count_launches(unsigned n);
unsigned long long launch_count();

cudaError_t launch_trace(const TraceParams& P, int tracker, int use_ess, int schedule, int features,
                         int persistent_blocks, cudaStream_t stream);
cudaError_t launch_minmax(const float* v, size_t n, float* out_minmax, cudaStream_t s);
cudaError_t launch_normalize(const float* in, float* out, size_t n, float vmin, float vmax, cudaStream_t s);
cudaError_t launch_gradient_magnitude(const float* grid, float* out, int nx, int ny, int nz, cudaStream_t s);
// Copies an x-fastest nx x ny x nz float grid into a 3D array through its surface object (ny, nz <= 65535).
cudaError_t launch_fill_density_array(const float* src, unsigned long long surface, int nx, int ny, int nz,
                                      cudaStream_t s);
cudaError_t launch_fbm(float* out, int nx, int ny, int nz, const int* perm512, const FbmParams& fp, cudaStream_t s);
cudaError_t launch_supervoxel_stats(const float* dens, int nx, int ny, int nz, int sv, int svx, int svy, int svz,
                                    int halo, float* mn, float* mx, float* avg, uint8_t* occ, cudaStream_t s);
cudaError_t launch_rrt_params(const float* mn, const float* mx, const float* avg, int total, float extinction,
                              float D, float* out_pairs, cudaStream_t s);
// Unbiased residual ratio tracking grid: per supervoxel (mu_c, mu_r_bar, 1 / max, 1 / (extinction * max)).
cudaError_t launch_rrt_local(const float* mn, const float* mx, const float* avg, int total, float extinction,
                             float D, float* out4, cudaStream_t s);
cudaError_t launch_interleave(const float* a, const float* b, int total, float* out_pairs, cudaStream_t s);
// One persistent launch over many scenes (see trace_batch_kernel).  With blocks_per_sm_out set, only
// reports the kernel's resident blocks per SM (occupancy calculator) and launches nothing.
struct BatchLaunch {
    const TraceParams* scenes;           // device array, num entries
    const unsigned long long* offsets;   // device array, num + 1 prefix sums of padded path counts
    int num;
    int tracker, interp, grid_kind;      // common to every scene of the batch
    int blocks;
    unsigned long long* work_counter;    // zeroed before the launch
    unsigned long long* counters;        // [0] paths, [1] density lookups (accumulated)
    int* error_flags;
    int* blocks_per_sm_out;
    bool counted = true;                 // add the launch to the launch counter (not while capturing)
};
cudaError_t launch_trace_batch(const BatchLaunch& b, cudaStream_t s);

// Value, get_dim and is_active of a sparse volume at `count` index-space voxels (device arrays).
cudaError_t launch_sparse_query(const SparseView& v, const int* ijk, int count, float* values, uint32_t* dims,
                                uint8_t* active, cudaStream_t s);
cudaError_t launch_occupancy(const float* dens, int nx, int ny, int nz, int bs, int gx, int gy, int gz, int halo,
                             float threshold, int ref_compat, uint8_t* out, cudaStream_t s);
cudaError_t launch_env_pyramid(const TraceParams& P, float* pyramid, const uint64_t* level_offsets_host, int levels,
                               cudaStream_t s);
cudaError_t launch_film_to_chw(const double* film, int width, int height, double inv_frames, int channels,
                               float* out, cudaStream_t s);
cudaError_t launch_film_to_rgba(const double* film, int n, double inv_frames, float* out_rgba, cudaStream_t s);
cudaError_t launch_rgba_to_chw(const float* rgba, int n, int channels, float* out, cudaStream_t s);

}  // namespace vpt
