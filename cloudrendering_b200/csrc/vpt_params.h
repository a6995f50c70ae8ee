// vpt_params.h - launch parameter block shared by the host context and the tracer kernels.
//
// This is the CUDA-side counterpart of the reference's std140 `Parameters` UBO
// (Data/Shaders/VPT/VptHeader.glsl:45-112, filled in VolumetricPathTracingPass.cpp:1981-2156) and
// `FrameInfo` (VptHeader.glsl:114-119).  Only the fields the tracing path reads are kept; the
// derived reciprocals are computed once on the host (see vpt_context.cu).  The whole block is passed
// as a __grid_constant__ kernel argument, so it lives in the constant bank and costs no loads.
#pragma once
#include <stdint.h>

namespace vpt {

enum Tracker : int {
    kDelta = 0,
    kRatio = 2,
    kDecomposition = 3,
    kResidualRatio = 4,
    kNextEvent = 5,
};

enum GridKind : int { kDense = 0, kNanoVdb = 1 };
enum Interp : int { kNearest = 0, kStochastic = 1, kTrilinear = 2 };
enum EnvKind : int { kEnvDefault = 0, kEnvBlack = 1, kEnvSingleColor = 2, kEnvConstantSun = 3, kEnvImage = 4 };

// Error bits written to TraceParams::error_flags (sticky until the host clears them).
enum ErrorBit : int { kErrIterLimit = 1 };

// Default guard on tentative collisions per camera path (all loops of one path together).  A path
// that reaches it stops, contributes what it has and raises kErrIterLimit.
constexpr uint32_t kMaxStepsPerPath = 1u << 24;

struct F3 { float x, y, z; };

struct TraceParams {
    // camera: inverse(proj * view), column-major like glm (m[col*4 + row])
    float inv_view_proj[16];
    float prev_view_proj[16];
    int width, height;
    uint32_t frame_count;      // FrameInfo::frameCount of the first frame in this launch
    uint32_t global_frame;     // FrameInfo::globalFrameNumber of the first frame in this launch
    uint32_t num_frames;       // frames traced by this launch
    uint32_t seed_offset;      // CUSTOM_SEED_OFFSET
    uint64_t num_paths;        // width * height * num_frames

    // medium
    F3 box_min, box_max;       // world-space volume box
    int nx, ny, nz;            // dense grid resolution
    F3 vox_per_unit;           // grid voxels per world unit along each axis
    float border_density;      // normalised value of the CLAMP_TO_BORDER texel (0 - min)/(max - min)
    float extinction;          // parameters.extinction.x (= global majorant)
    float inv_extinction;
    float albedo;              // parameters.scatteringAlbedo.x
    float absorb_albedo;       // 1 - albedo
    float g;                   // Henyey-Greenstein parameter
    int interp;                // Interp
    int max_bounces;           // 0 = unlimited
    uint32_t max_steps;        // guard on tentative collisions per path (kMaxStepsPerPath by default)
    int ess_ref_compat;        // reproduce the reference's empty-space-skipping shadow loop exactly

    // supervoxels (residual ratio / decomposition tracking, occupancy grid)
    int sv_size;               // voxels per supervoxel side
    int svx, svy, svz;         // supervoxel grid resolution
    F3 sv_world;               // supervoxel size in world units (superVoxelSize * boxDelta / gridResolution)

    // sky and sun
    int env_kind;              // EnvKind
    int use_linear_rgb;
    int env_is_black;          // parameters.isEnvMapBlack
    int env_image_linear;      // ENV_MAP_IMAGE_USES_LINEAR_RGB
    F3 sun_dir;
    F3 sun_intensity;
    F3 sky_color;              // constant sky of kEnvConstantSun
    F3 env_intensity;          // environmentMapIntensityFactor
    int env_w, env_h;          // equirectangular environment image
    int env_levels;            // octahedral pyramid levels (12 in the reference)
    int env_base_res;          // 1 << env_levels

    // device buffers (all owned by the context)
    const float* density;          // normalised density, x-fastest
    const float* sv_data;          // 2 floats per supervoxel: (min, max) or (mu_c, mu_r_bar)
    const uint8_t* occupancy;      // 1 byte per supervoxel
    const float* env_rgba;         // equirect RGBA fp32
    const float* env_pyramid;      // octahedral max-luminance pyramid, level 0 first
    const uint64_t* env_level_offset; // float offset of each level in env_pyramid (indexed by level)
    double* film;                  // 3 doubles per pixel: sum of radiance
    double* film_sq;               // 3 doubles per pixel: sum of squared radiance (optional)
    float* feat;                   // feature accumulators (optional), 16 floats per pixel
    unsigned long long* counters;  // [0] paths, [1] density lookups
    int* error_flags;
    unsigned int* work_counter;    // persistent-kernel path queue
};

// Offsets of the per-pixel feature accumulators (floats).
enum FeatureSlot : int {
    kFeatPos = 0,        // first event position xyz + hit count
    kFeatNormal = 4,     // xyz (finite difference of the density)
    kFeatDepth = 7,      // depth, depth^2
    kFeatDensity = 9,    // density*0.001, squared
    kFeatCloudOnly = 11, // rgb of paths with an event
    kFeatTrans = 14,     // primary-ray transmittance
    kFeatBackground = 15,// luminance proxy (unused slot kept for alignment)
    kFeatStride = 16,
};

}  // namespace vpt
