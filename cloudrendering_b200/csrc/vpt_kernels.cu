// vpt_kernels.cu - launchers of the tracing path and the kernels around it.
//
//  * launch_trace: dispatch to the tracker families (vpt_trace_*.cu, kernels in vpt_trace.cuh).
//  * grid preparation: min/max reduction and normalisation (DensityField.cpp:136-154, 262-267),
//    seeded fBm scene generator, supervoxel and occupancy builders (SuperVoxelGrid.cpp,
//    ComputeOccupancyGrid.glsl), octahedral environment pyramid (OctahedralMapper.glsl).
//  * film readout: FP64 sums -> fp32 mean, channels x H x W.
#include <cuda_runtime.h>
#include <stdint.h>
#include "vpt_device.cuh"
#include "vpt_trace.cuh"

namespace vpt {

// Number of kernels this library has launched (all launch sites below and in vpt_denoise.cu).
static unsigned long long g_launches = 0;
void count_launches(unsigned n) { __atomic_fetch_add(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }
unsigned long long launch_count() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

uint64_t padded_paths(int width, int height, uint32_t frames) {
    uint64_t tiles = (uint64_t)((width + 15) / 16) * (uint64_t)((height + 15) / 16);
    return tiles * 256ull * frames;
}

cudaError_t launch_trace(const TraceParams& P, int tracker, int use_ess, int schedule, int features,
                         int persistent_blocks, cudaStream_t stream) {
    if (P.iso) {
        // isosurfaces: delta, spectral delta and next event tracking on dense grids, trilinear lookups,
        // no transfer function
        if ((tracker != kDelta && tracker != kSpectralDelta && tracker != kNextEvent &&
             tracker != kSpectralNextEvent) ||
            P.grid_kind != kDense || P.tf)
            return cudaErrorNotSupported;
        if (tracker == kSpectralDelta)
            return launch_tracker_spectral_delta_iso(P, schedule, features, persistent_blocks, stream);
        if (tracker == kNextEvent || tracker == kSpectralNextEvent) {
            // next event tracking: sky light samples only (no lights, no environment image, no skipping)
            if (use_ess || P.num_lights > 0 || P.env_kind == kEnvImage) return cudaErrorNotSupported;
            if (tracker == kSpectralNextEvent)
                return launch_tracker_spectral_nee_iso(P, schedule, features, persistent_blocks, stream);
            return launch_tracker_nee_iso(P, schedule, features, persistent_blocks, stream);
        }
        return launch_tracker_delta_iso(P, schedule, features, persistent_blocks, stream);
    }
    if (P.grid_kind == kNanoVdb) {
        // sparse grids: the trackers whose density access goes through sampleCloud, and the HDDA
        // decomposition tracker; residual ratio tracking and the occupancy grid are dense-only in the
        // reference (VolumetricPathTracingPass.cpp:1171-1186)
        switch (tracker) {
            case kDelta: return launch_tracker<kDelta, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kRatio: return launch_tracker<kRatio, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kDecomposition:
                return launch_tracker<kDecomposition, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kNextEvent:
                if (use_ess) return cudaErrorNotSupported;
                return launch_tracker<kNextEvent, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kSpectralDelta:
                return launch_tracker<kSpectralDelta, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kSpectralNextEvent:
                if (use_ess) return cudaErrorNotSupported;
                return launch_tracker<kSpectralNextEvent, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            default: return cudaErrorNotSupported;
        }
    }
    switch (tracker) {
        case kDelta:
            if (P.density_tex && !P.tf)
                return launch_tracker<kDelta, kDenseTex>(P, schedule, features, persistent_blocks, stream);
            return launch_tracker<kDelta, kDense>(P, schedule, features, persistent_blocks, stream);
        case kRatio:
            if (P.density_tex && !P.tf)
                return launch_tracker<kRatio, kDenseTex>(P, schedule, features, persistent_blocks, stream);
            return launch_tracker<kRatio, kDense>(P, schedule, features, persistent_blocks, stream);
        case kDecomposition:
            if (P.density_tex && !P.tf)
                return launch_tracker<kDecomposition, kDenseTex>(P, schedule, features, persistent_blocks, stream);
            return launch_tracker<kDecomposition, kDense>(P, schedule, features, persistent_blocks, stream);
        case kResidualRatio: return launch_tracker<kResidualRatio, kDense>(P, schedule, features, persistent_blocks, stream);
        case kResidualRatioNee:
            if (P.density_tex && !P.tf)
                return launch_tracker<kResidualRatioNee, kDenseTex>(P, schedule, features, persistent_blocks, stream);
            return launch_tracker<kResidualRatioNee, kDense>(P, schedule, features, persistent_blocks, stream);
        case kNextEvent:
            if (use_ess && P.density_tex && !P.tf)
                return launch_tracker<kNextEvent + 100, kDenseTex>(P, schedule, features, persistent_blocks, stream);
            if (use_ess) return launch_tracker<kNextEvent + 100, kDense>(P, schedule, features, persistent_blocks, stream);
            if (P.density_tex && !P.tf)
                return launch_tracker<kNextEvent, kDenseTex>(P, schedule, features, persistent_blocks, stream);
            return launch_tracker<kNextEvent, kDense>(P, schedule, features, persistent_blocks, stream);
        case kSpectralDelta: return launch_tracker<kSpectralDelta, kDense>(P, schedule, features, persistent_blocks, stream);
        case kSpectralNextEvent:
            if (use_ess)
                return launch_tracker<kSpectralNextEvent + 100, kDense>(P, schedule, features, persistent_blocks, stream);
            return launch_tracker<kSpectralNextEvent, kDense>(P, schedule, features, persistent_blocks, stream);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------------------------
// Sparse volume queries (accessor checks against the reference's PNanoVDB).

__global__ void sparse_query_kernel(const __grid_constant__ SparseView v, const int* __restrict__ ijk, int count,
                                    float* __restrict__ values, uint32_t* __restrict__ dims,
                                    uint8_t* __restrict__ active) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int x = ijk[3 * i], y = ijk[3 * i + 1], z = ijk[3 * i + 2];
    values[i] = sparse_value(v, x, y, z);
    dims[i] = (uint32_t)sparse_dim(v, x, y, z);
    active[i] = sparse_is_active(v, x, y, z) ? 1 : 0;
}

cudaError_t launch_sparse_query(const SparseView& v, const int* ijk, int count, float* values, uint32_t* dims,
                                uint8_t* active, cudaStream_t s) {
    sparse_query_kernel<<<(count + 255) / 256, 256, 0, s>>>(v, ijk, count, values, dims, active);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Grid preparation.

__device__ __forceinline__ void atomic_min_float(float* addr, float v) {
    int* a = reinterpret_cast<int*>(addr);
    int old = *a;
    while (__int_as_float(old) > v) {
        int assumed = old;
        old = atomicCAS(a, assumed, __float_as_int(v));
        if (old == assumed) break;
    }
}
__device__ __forceinline__ void atomic_max_float(float* addr, float v) {
    int* a = reinterpret_cast<int*>(addr);
    int old = *a;
    while (__int_as_float(old) < v) {
        int assumed = old;
        old = atomicCAS(a, assumed, __float_as_int(v));
        if (old == assumed) break;
    }
}

// min/max over the raw grid (sgl::reduceFloatArrayMinMax semantics; order-independent, exact).
__global__ void minmax_kernel(const float* __restrict__ v, size_t n, float* out_minmax) {
    float lo = INFINITY, hi = -INFINITY;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float x = v[i];
        lo = fminf(lo, x);
        hi = fmaxf(hi, x);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __shared__ float slo[32], shi[32];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        slo[warp] = lo;
        shi[warp] = hi;
    }
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        lo = lane < nw ? slo[lane] : INFINITY;
        hi = lane < nw ? shi[lane] : -INFINITY;
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            atomic_min_float(out_minmax + 0, lo);
            atomic_max_float(out_minmax + 1, hi);
        }
    }
}

// (v - min) / (max - min), IEEE division as in DensityField::getDataFloatAtNorm.
__global__ void normalize_kernel(const float* __restrict__ in, float* __restrict__ out, size_t n, float vmin,
                                 float vmax) {
    const float range = vmax - vmin;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        out[i] = (in[i] - vmin) / range;
    }
}

// Gradient magnitude of the raw grid for gradient isosurfaces (VolumetricPathTracingPass.cpp:690-727):
// central differences between the neighbours clamped to the grid, divided by their index distance
// (2 inside, 1 at a face), |g| = sqrt(dx^2 + dy^2 + dz^2) in float, x fastest.  A stencil pass at
// HBM speed: each thread owns one voxel, the six neighbour loads of a warp fall on at most a few
// cache lines of the x row and of the rows above and below it.
__global__ void gradient_magnitude_kernel(const float* __restrict__ g, float* __restrict__ out, int nx, int ny,
                                          int nz) {
    const size_t n = (size_t)nx * ny * nz;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % (size_t)nx);
        const size_t yz = i / (size_t)nx;
        const int y = (int)(yz % (size_t)ny);
        const int z = (int)(yz / (size_t)ny);
        const int xl = x > 0 ? x - 1 : 0, xu = x < nx - 1 ? x + 1 : nx - 1;
        const int yl = y > 0 ? y - 1 : 0, yu = y < ny - 1 ? y + 1 : ny - 1;
        const int zl = z > 0 ? z - 1 : 0, zu = z < nz - 1 ? z + 1 : nz - 1;
        const size_t row = (size_t)nx, plane = (size_t)nx * ny;
        const size_t base = (size_t)z * plane + (size_t)y * row;
        const float dx = (g[base + xu] - g[base + xl]) / (float)(xu - xl);
        const float dy = (g[(size_t)z * plane + (size_t)yu * row + x] - g[(size_t)z * plane + (size_t)yl * row + x]) /
                         (float)(yu - yl);
        const float dz = (g[(size_t)zu * plane + (size_t)y * row + x] - g[(size_t)zl * plane + (size_t)y * row + x]) /
                         (float)(zu - zl);
        out[i] = sqrtf(dx * dx + dy * dy + dz * dz);
    }
}

// Improved Perlin noise (K. Perlin, "Improving Noise", SIGGRAPH 2002) with a seeded permutation;
// only +, -, *, floor, so the CPU oracle reproduces every value bit for bit.
struct PermTable {
    int p[512];
};

__device__ __forceinline__ float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
__device__ __forceinline__ float lerpf(float t, float a, float b) { return a + t * (b - a); }
__device__ __forceinline__ float grad(int h, float x, float y, float z) {
    h &= 15;
    float u = h < 8 ? x : y;
    float v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}

__device__ float perlin3(const int* __restrict__ p, float x, float y, float z) {
    float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
    x -= fx;
    y -= fy;
    z -= fz;
    float u = fade(x), v = fade(y), w = fade(z);
    int A = p[X] + Y, AA = p[A] + Z, AB = p[A + 1] + Z;
    int B = p[X + 1] + Y, BA = p[B] + Z, BB = p[B + 1] + Z;
    float r0 = lerpf(v, lerpf(u, grad(p[AA], x, y, z), grad(p[BA], x - 1.0f, y, z)),
                     lerpf(u, grad(p[AB], x, y - 1.0f, z), grad(p[BB], x - 1.0f, y - 1.0f, z)));
    float r1 = lerpf(v, lerpf(u, grad(p[AA + 1], x, y, z - 1.0f), grad(p[BA + 1], x - 1.0f, y, z - 1.0f)),
                     lerpf(u, grad(p[AB + 1], x, y - 1.0f, z - 1.0f), grad(p[BB + 1], x - 1.0f, y - 1.0f, z - 1.0f)));
    return lerpf(w, r0, r1);
}

__global__ void fbm_kernel(float* __restrict__ out, int nx, int ny, int nz, const __grid_constant__ PermTable perm,
                           FbmParams fp) {
    __shared__ int p[512];
    for (int i = threadIdx.x; i < 512; i += blockDim.x) p[i] = perm.p[i];
    __syncthreads();
    const size_t n = (size_t)nx * ny * nz;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int ix = (int)(i % (size_t)nx);
        int iy = (int)((i / (size_t)nx) % (size_t)ny);
        int iz = (int)(i / ((size_t)nx * ny));
        float px = ((float)ix + 0.5f) * fp.inv_max_dim;
        float py = ((float)iy + 0.5f) * fp.inv_max_dim;
        float pz = ((float)iz + 0.5f) * fp.inv_max_dim;
        float sum = 0.0f, amp = 1.0f, freq = fp.base_frequency, norm = 0.0f;
        for (int o = 0; o < fp.octaves; o++) {
            sum += amp * perlin3(p, px * freq, py * freq, pz * freq);
            norm += amp;
            amp *= fp.gain;
            freq *= fp.lacunarity;
        }
        float v = sum / norm;
        v = fminf(fmaxf(0.5f + fp.contrast * v, 0.0f), 1.0f);
        out[i] = v < fp.threshold ? 0.0f : v;
    }
}

// ---------------------------------------------------------------------------------------------
// Supervoxel grid: min / max / mean of the normalised density over each sv^3 block, with a one
// voxel halo unless the interpolation is NEAREST; voxels outside the grid count as 0 and a
// partial boundary supervoxel has min := 0 (SuperVoxelGrid.cpp:101-211, 316-396).  One thread
// per supervoxel accumulates the mean in the reference's z-y-x loop order, so the sum is
// bit-identical; min/max are order-independent.
__global__ void supervoxel_stats_kernel(const float* __restrict__ dens, int nx, int ny, int nz, int sv, int svx,
                                        int svy, int svz, int halo, float* __restrict__ out_min,
                                        float* __restrict__ out_max, float* __restrict__ out_avg,
                                        uint8_t* __restrict__ out_occ) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    int total = svx * svy * svz;
    if (idx >= total) return;
    int bx = idx % svx, by = (idx / svx) % svy, bz = idx / (svx * svy);
    float lo = 3.402823466e+38f, hi = -3.402823466e+38f, sum = 0.0f;
    int cnt = 0;
    int o0 = halo ? -1 : 0, o1 = halo ? sv : sv - 1;
    for (int oz = o0; oz <= o1; oz++) {
        int z = bz * sv + oz;
        for (int oy = o0; oy <= o1; oy++) {
            int y = by * sv + oy;
            for (int ox = o0; ox <= o1; ox++) {
                int x = bx * sv + ox;
                float v = 0.0f;
                if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) {
                    v = __ldg(dens + ((size_t)z * ny + y) * nx + x);
                }
                lo = fminf(lo, v);
                hi = fmaxf(hi, v);
                sum += v;
                cnt++;
            }
        }
    }
    float avg = sum / (float)cnt;
    if ((nx % sv != 0 && bx == svx - 1) || (ny % sv != 0 && by == svy - 1) || (nz % sv != 0 && bz == svz - 1)) {
        lo = 0.0f;
    }
    out_min[idx] = lo;
    out_max[idx] = hi;
    if (out_avg) out_avg[idx] = avg;
    if (out_occ) out_occ[idx] = hi < 1e-5f ? 0 : 1;
}

// Residual-ratio-tracking control and residual extinctions (SuperVoxelGrid.cpp:218-256):
// mu_r_bar = max(mu_max - mu_min, 0.1), mu_c = clamp(mu_min + mu_r_bar * gamma^(1/(D mu_r_bar) - 1),
// mu_min, mu_avg) with gamma = 2, D = sqrt(3) * sv.
__global__ void rrt_params_kernel(const float* __restrict__ mn, const float* __restrict__ mx,
                                  const float* __restrict__ avg, int total, float extinction, float D,
                                  float* __restrict__ out_pairs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    float mu_min = mn[i] * extinction, mu_max = mx[i] * extinction, mu_avg = avg[i] * extinction;
    float mu_r = fmaxf(mu_max - mu_min, 0.1f);
    float mu_c = mu_min + mu_r * m_pow(2.0f, (1.0f / (D * mu_r)) - 1.0f);
    mu_c = fminf(fmaxf(mu_c, mu_min), mu_avg);
    out_pairs[2 * i + 0] = mu_c;
    out_pairs[2 * i + 1] = mu_r;
}

// Per supervoxel: the residual ratio tracking controls of rrt_params_kernel, then the free-path
// majorant's reciprocals (0 for a supervoxel whose largest density, halo included, is 0).
__global__ void rrt_local_kernel(const float* __restrict__ mn, const float* __restrict__ mx,
                                 const float* __restrict__ avg, int total, float extinction, float D,
                                 float4* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const float dmax = mx[i];
    float mu_min = mn[i] * extinction, mu_max = dmax * extinction, mu_avg = avg[i] * extinction;
    float mu_r = fmaxf(mu_max - mu_min, 0.1f);
    float mu_c = mu_min + mu_r * m_pow(2.0f, (1.0f / (D * mu_r)) - 1.0f);
    mu_c = fminf(fmaxf(mu_c, mu_min), mu_avg);
    const bool empty = !(dmax > 0.0f) || !(mu_max > 0.0f);
    out[i] = make_float4(mu_c, mu_r, empty ? 0.0f : 1.0f / dmax, empty ? 0.0f : 1.0f / mu_max);
}

__global__ void interleave_kernel(const float* __restrict__ a, const float* __restrict__ b, int total,
                                  float* __restrict__ out_pairs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    out_pairs[2 * i + 0] = a[i];
    out_pairs[2 * i + 1] = b[i];
}

// Occupancy grid for NEE empty-space skipping.  The reference shader's loop never executes
// (ComputeOccupancyGrid.glsl:108-109) so every block is marked occupied; `ref_compat` reproduces
// that.  Otherwise one warp per block votes whether any voxel of the block (plus a one-voxel halo
// for stochastic / trilinear lookups) exceeds `threshold`.
__global__ void occupancy_kernel(const float* __restrict__ dens, int nx, int ny, int nz, int bs, int gx, int gy,
                                 int gz, int halo, float threshold, int ref_compat, uint8_t* __restrict__ out) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int total = gx * gy * gz;
    if (warp >= total) return;
    if (ref_compat) {
        if (lane == 0) out[warp] = 1;
        return;
    }
    int bx = warp % gx, by = (warp / gx) % gy, bz = warp / (gx * gy);
    int ext = bs + 2 * halo;
    bool occ = false;
    if (ext <= 32) {
        // the warp reads 32 / ext rows of the block (with its halo) per step, lane (lx, lr) the voxel lx
        // of row lr; rows advance by (y, z) increments, without divisions in the loop
        const int per = 32 / ext;
        const int steps = (ext * ext + per - 1) / per;  // the same trip count on every lane
        const int lx = lane % ext, lr = lane / ext;
        int oy = lr % ext, oz = lr / ext;  // row lr of the block
        const int x = bx * bs + lx - halo;
        const bool x_in = lr < per && x >= 0 && x < nx;
        for (int k = 0; k < steps; k++) {
            if (__any_sync(0xffffffffu, occ)) break;
            const int y = by * bs + oy - halo, z = bz * bs + oz - halo;
            if (x_in && oz < ext && y >= 0 && y < ny && z >= 0 && z < nz)
                occ |= __ldg(dens + ((size_t)z * ny + y) * nx + x) > threshold;
            oy += per;
            while (oy >= ext) {
                oy -= ext;
                oz++;
            }
        }
    } else {
        const int n = ext * ext * ext;
        for (int i = lane; i < n && !__any_sync(__activemask(), occ); i += 32) {
            int ox = i % ext - halo, oy = (i / ext) % ext - halo, oz = i / (ext * ext) - halo;
            int x = bx * bs + ox, y = by * bs + oy, z = bz * bs + oz;
            if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) {
                occ |= __ldg(dens + ((size_t)z * ny + y) * nx + x) > threshold;
            }
        }
    }
    occ = __any_sync(0xffffffffu, occ);
    if (lane == 0) out[warp] = occ ? 1 : 0;
}

// ---------------------------------------------------------------------------------------------
// The grid's texture array: one thread per voxel of a row (x), rows y and slices z on the grid's y and
// z dimensions; coalesced reads, surface stores into the array's block layout.
__global__ void fill_density_array_kernel(const float* __restrict__ src, cudaSurfaceObject_t surf, int nx, int ny) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    surf3Dwrite(__ldg(src + ((size_t)z * ny + y) * nx + x), surf, x * (int)sizeof(float), y, z);
}

cudaError_t launch_fill_density_array(const float* src, unsigned long long surface, int nx, int ny, int nz,
                                      cudaStream_t s) {
    if (ny > 65535 || nz > 65535) return cudaErrorInvalidValue;
    fill_density_array_kernel<<<dim3((unsigned)((nx + 255) / 256), (unsigned)ny, (unsigned)nz), 256, 0, s>>>(
        src, (cudaSurfaceObject_t)surface, nx, ny);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Octahedral max-luminance pyramid of the environment image (OctahedralMapper.glsl:65-85, then a
// 2x2 box reduction per level like vkCmdBlitImage mip generation).
__global__ void env_octahedral_level0_kernel(const __grid_constant__ TraceParams P, float* __restrict__ out, int res) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= res || y >= res) return;
    float best = -1.0f;
    for (int i = 0; i < 5; i++) {
        float sxo = 0.1f + 0.2f * (float)i;
        for (int j = 0; j < 5; j++) {
            float syo = 0.1f + 0.2f * (float)j;
            float u = ((float)x + sxo) / (float)res;
            float v = ((float)y + syo) / (float)res;
            F3 dir = octahedral_uv_to_world(u, v);
            float tu = m_atan2(dir.z, dir.x) / (2.0f * kPi) + 0.5f;
            float tv = -m_asin(dir.y) / kPi + 0.5f;
            F3 c = env_image_fetch(P, tu, tv);
            c = f3(fminf(c.x, 100000.0f), fminf(c.y, 100000.0f), fminf(c.z, 100000.0f));
            best = fmaxf(best, length3(c));
        }
    }
    out[(size_t)y * res + x] = best;
}

__global__ void env_downsample_kernel(const float* __restrict__ in, float* __restrict__ out, int res_out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= res_out || y >= res_out) return;
    int ri = res_out * 2;
    float a = in[(size_t)(2 * y) * ri + 2 * x], b = in[(size_t)(2 * y) * ri + 2 * x + 1];
    float c = in[(size_t)(2 * y + 1) * ri + 2 * x], d = in[(size_t)(2 * y + 1) * ri + 2 * x + 1];
    out[(size_t)y * res_out + x] = ((a + b) + (c + d)) * 0.25f;
}

// ---------------------------------------------------------------------------------------------
// Film readout: mean = sum / frames as channels x H x W (alpha = 1 for 4 channels).
__global__ void film_to_chw_kernel(const double* __restrict__ film, int width, int height, double inv_frames,
                                   int channels, float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = width * height;
    if (i >= n) return;
    for (int c = 0; c < 3; c++) out[(size_t)c * n + i] = (float)(film[(size_t)i * 3 + c] * inv_frames);
    if (channels == 4) out[(size_t)3 * n + i] = 1.0f;
}

__global__ void film_to_rgba_kernel(const double* __restrict__ film, int n, double inv_frames, float4* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4((float)(film[(size_t)i * 3 + 0] * inv_frames), (float)(film[(size_t)i * 3 + 1] * inv_frames),
                         (float)(film[(size_t)i * 3 + 2] * inv_frames), 1.0f);
}

__global__ void rgba_to_chw_kernel(const float4* __restrict__ in, int n, int channels, float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = in[i];
    out[i] = v.x;
    out[(size_t)n + i] = v.y;
    out[(size_t)2 * n + i] = v.z;
    if (channels == 4) out[(size_t)3 * n + i] = v.w;
}

// ---------------------------------------------------------------------------------------------
// Launchers (declared in vpt_kernels.h).

static unsigned grid_for(size_t n, int block, unsigned cap = 148u * 32u) {
    size_t g = (n + block - 1) / block;
    if (g > cap) g = cap;
    if (g == 0) g = 1;
    return (unsigned)g;
}

cudaError_t launch_minmax(const float* v, size_t n, float* out_minmax, cudaStream_t s) {
    float init[2] = {INFINITY, -INFINITY};
    cudaMemcpyAsync(out_minmax, init, sizeof(init), cudaMemcpyHostToDevice, s);
    minmax_kernel<<<grid_for(n, 256), 256, 0, s>>>(v, n, out_minmax);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_normalize(const float* in, float* out, size_t n, float vmin, float vmax, cudaStream_t s) {
    normalize_kernel<<<grid_for(n, 256), 256, 0, s>>>(in, out, n, vmin, vmax);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gradient_magnitude(const float* grid, float* out, int nx, int ny, int nz, cudaStream_t s) {
    const size_t n = (size_t)nx * ny * nz;
    gradient_magnitude_kernel<<<grid_for(n, 256), 256, 0, s>>>(grid, out, nx, ny, nz);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fbm(float* out, int nx, int ny, int nz, const int* perm512, const FbmParams& fp, cudaStream_t s) {
    PermTable t;
    for (int i = 0; i < 512; i++) t.p[i] = perm512[i];
    size_t n = (size_t)nx * ny * nz;
    fbm_kernel<<<grid_for(n, 256), 256, 0, s>>>(out, nx, ny, nz, t, fp);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_supervoxel_stats(const float* dens, int nx, int ny, int nz, int sv, int svx, int svy, int svz,
                                    int halo, float* mn, float* mx, float* avg, uint8_t* occ, cudaStream_t s) {
    int total = svx * svy * svz;
    supervoxel_stats_kernel<<<(total + 127) / 128, 128, 0, s>>>(dens, nx, ny, nz, sv, svx, svy, svz, halo, mn, mx,
                                                                avg, occ);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_rrt_params(const float* mn, const float* mx, const float* avg, int total, float extinction,
                              float D, float* out_pairs, cudaStream_t s) {
    rrt_params_kernel<<<(total + 255) / 256, 256, 0, s>>>(mn, mx, avg, total, extinction, D, out_pairs);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_rrt_local(const float* mn, const float* mx, const float* avg, int total, float extinction,
                             float D, float* out4, cudaStream_t s) {
    rrt_local_kernel<<<(total + 255) / 256, 256, 0, s>>>(mn, mx, avg, total, extinction, D,
                                                        reinterpret_cast<float4*>(out4));
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_interleave(const float* a, const float* b, int total, float* out_pairs, cudaStream_t s) {
    interleave_kernel<<<(total + 255) / 256, 256, 0, s>>>(a, b, total, out_pairs);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_occupancy(const float* dens, int nx, int ny, int nz, int bs, int gx, int gy, int gz, int halo,
                             float threshold, int ref_compat, uint8_t* out, cudaStream_t s) {
    int total = gx * gy * gz;
    size_t threads = (size_t)total * 32;
    occupancy_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(dens, nx, ny, nz, bs, gx, gy, gz, halo,
                                                                       threshold, ref_compat, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_env_pyramid(const TraceParams& P, float* pyramid, const uint64_t* level_offsets_host, int levels,
                               cudaStream_t s) {
    int res = 1 << levels;
    dim3 b(16, 16);
    env_octahedral_level0_kernel<<<dim3((res + 15) / 16, (res + 15) / 16), b, 0, s>>>(P, pyramid, res);
    count_launches((unsigned)levels);
    for (int l = 1; l < levels; l++) {
        int r = res >> l;
        env_downsample_kernel<<<dim3((r + 15) / 16, (r + 15) / 16), b, 0, s>>>(
            pyramid + level_offsets_host[l - 1], pyramid + level_offsets_host[l], r);
    }
    return cudaGetLastError();
}

cudaError_t launch_film_to_chw(const double* film, int width, int height, double inv_frames, int channels,
                               float* out, cudaStream_t s) {
    int n = width * height;
    film_to_chw_kernel<<<(n + 255) / 256, 256, 0, s>>>(film, width, height, inv_frames, channels, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_film_to_rgba(const double* film, int n, double inv_frames, float* out_rgba, cudaStream_t s) {
    film_to_rgba_kernel<<<(n + 255) / 256, 256, 0, s>>>(film, n, inv_frames, reinterpret_cast<float4*>(out_rgba));
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_rgba_to_chw(const float* rgba, int n, int channels, float* out, cudaStream_t s) {
    rgba_to_chw_kernel<<<(n + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float4*>(rgba), n, channels, out);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace vpt
