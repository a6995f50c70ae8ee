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
    kSpectralDelta = 1,
    kRatio = 2,
    kDecomposition = 3,
    kResidualRatio = 4,
    kNextEvent = 5,
    kSpectralNextEvent = 6,
    // no reference counterpart: next-event estimation with residual-ratio-tracked shadow rays and
    // supervoxel-majorant free paths (VPT_MODE_RESIDUAL_RATIO_TRACKING_UNBIASED)
    kResidualRatioNee = 9,
    // kernel variants, not VptModes: delta, spectral delta and next event tracking with isosurfaces inside
    // the volume
    kDeltaIso = 300,
    kSpectralDeltaIso = 301,
    kNextEventIso = 302,
    kSpectralNextEventIso = 303,
};

// Collision probabilities of spectral tracking (SpectralDeltaTrackingCollisionProbability,
// src/PathTracer/RenderSettings.hpp:64-69).
enum SdtProbability : int { kSdtMax = 0, kSdtAvg = 1, kSdtPathHistory = 2 };

// kDenseTex: the dense grid read through a 3D texture object (point filtering, border colour 0), a
// kernel variant chosen by the host when the border density is 0; P.grid_kind stays kDense.
enum GridKind : int { kDense = 0, kNanoVdb = 1, kDenseTex = 2 };
enum Interp : int { kNearest = 0, kStochastic = 1, kTrilinear = 2 };
// surface BRDFs of isosurface hits (SurfaceBrdf, RenderSettings.hpp:94-99, numbered in this core's
// order) and the slots of TraceParams::brdf
enum IsoBrdf : int {
    kBrdfLambertian = 0, kBrdfBlinnPhong = 1, kBrdfAmbient = 2, kBrdfCookTorrance = 3, kBrdfDisney = 4
};
enum BrdfParam : int {
    kBrdfSubsurface = 0, kBrdfMetallic, kBrdfSpecular, kBrdfSpecularTint, kBrdfRoughness,
    kBrdfAnisotropic, kBrdfSheen, kBrdfSheenTint, kBrdfClearcoat, kBrdfClearcoatGloss, kBrdfParamCount
};
enum EnvKind : int { kEnvDefault = 0, kEnvBlack = 1, kEnvSingleColor = 2, kEnvConstantSun = 3, kEnvImage = 4 };

// Error bits written to TraceParams::error_flags (sticky until the host clears them).
enum ErrorBit : int { kErrIterLimit = 1 };

// Default guard on tentative collisions per camera path (all loops of one path together).  A path
// that reaches it stops, contributes what it has and raises kErrIterLimit.
constexpr uint32_t kMaxStepsPerPath = 1u << 24;

struct F3 { float x, y, z; };

// A constant region of a sparse grid: a tile of a lower (level 1), upper (level 2) or root (level
// 3) node, or the background outside every root tile (level 4).  `box` is the index-space bounding
// box of the node that holds the tile (its active values, inclusive), which the sparse
// decomposition tracker clips against (DecompositionTracking.glsl:219-240).
struct SparseTile {
    float value;
    int active;
    int level;
    int box[6];
};

// Sparse (NanoVDB-compatible) volume as the tracer reads it.  The tree is flattened into a table
// with one 32-bit entry per 8^3 brick of the root's bounding box: bit 31 clear = index of a leaf in
// the leaf pools, bit 31 set = index into `tiles`.  Bricks outside the table are background.
constexpr uint32_t kSparseTileBit = 0x80000000u;
// Root tiles (4096^3 regions) known to the view, for voxels outside the brick table: inside a root
// tile with an upper node such a voxel lies in an inactive upper-node tile (dim 128, background
// value); inside a root tile without child it takes the tile; elsewhere it is background.
constexpr int kSparseMaxRootTiles = 8;
struct SparseView {
    float mat[9];              // index -> world (Map::mMatF, row-major as PNanoVDB applies it)
    float inv_mat[9];          // world -> index (Map::mInvMatF)
    float vec[3];              // Map::mVecF
    F3 grid_min, grid_max;     // world bounding box of the active values (float)
    int root_min[3], root_max[3];  // index bounding box of the root node (inclusive)
    int tbl_origin[3];         // first voxel of the brick table (multiple of 8)
    int tbl_dim[3];            // bricks per axis
    int lowest_level;          // HDDA cell size of the decomposition tracker: 8 (leaves) or 1 (voxels)
    int fp16;                  // leaf values stored as IEEE half
    float background;
    int root_tiles;                                  // entries used below
    int rt_origin[kSparseMaxRootTiles][3];
    int rt_child[kSparseMaxRootTiles];               // 1: the tile holds an upper node
    float rt_value[kSparseMaxRootTiles];
    int rt_active[kSparseMaxRootTiles];
    const uint32_t* table;
    const float* values;            // 512 floats per leaf, NanoVDB voxel order ((x&7)<<6 | (y&7)<<3 | (z&7))
    const unsigned short* values_h; // the same as half (fp16 variant)
    const uint32_t* masks;          // 16 words per leaf: active voxels
    const int* leaf_bbox_min;       // 3 per leaf: LeafData::mBBoxMin
    const SparseTile* tiles;
};

// A light of the reference's light editor (struct Light, VptHeader.glsl:233-248; defaults of
// LightEditorWidget.hpp:69-85), sampled by next event tracking only.
enum LightType : int { kLightPoint = 0, kLightSpot = 1, kLightDirectional = 2 };
enum LightSpace : int { kLightSpaceWorld = 0, kLightSpaceView = 1, kLightSpaceViewOrientation = 2 };
constexpr int kMaxLights = 16;
struct LightParams {
    int type;                 // LightType
    int space;                // LightSpace
    float spot_total_width;   // radians
    float spot_falloff_start; // radians
    F3 color;
    float intensity;
    F3 position;              // point / spot position; direction (times distance) of a directional light
    int use_distance;         // 1/d^2 falloff for point and spot lights
    F3 spot_direction;
};

struct TraceParams {
    // camera: inverse(proj * view), column-major like glm (m[col*4 + row])
    float inv_view_proj[16];
    float inv_view[16];        // inverse(view): view-space lights to world space
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
    float ext_rgb[3];          // parameters.extinction (spectral trackers)
    float albedo_rgb[3];       // parameters.scatteringAlbedo (spectral trackers)
    float sdt_majorant;        // maxComponent(parameters.extinction)
    float inv_sdt_majorant;
    int sdt_prob;              // SdtProbability
    float g;                   // Henyey-Greenstein parameter
    int interp;                // Interp
    int max_bounces;           // 0 = unlimited
    uint32_t max_steps;        // guard on tentative collisions per path (kMaxStepsPerPath by default)
    int grid_kind;             // GridKind: dense texture or sparse (NanoVDB) volume
    unsigned long long density_tex; // cudaTextureObject_t over `density` (0: none; kDenseTex kernels)
    int refill_min;            // per-lane refill schedule: a warp refills its empty lanes once this many wait
    float* frame_normals;      // Depth (nabla) / (fwidth): 4 floats per frame of the launch and pixel, the
                               //   first event's normal and 1 (0 0 0 0 without an event), frame-major
    int ess_ref_compat;        // reproduce the reference's empty-space-skipping shadow loop exactly

    // supervoxels (residual ratio / decomposition tracking, occupancy grid)
    int sv_size;               // voxels per supervoxel side
    int svx, svy, svz;         // supervoxel grid resolution
    F3 sv_world;               // supervoxel size in world units (superVoxelSize * boxDelta / gridResolution)
    F3 sv_inv_world;           // 1 / sv_world

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
    // USE_ENV_MAP_ROTATION (VptUtils.glsl:142-153, 303-306): environment-image lookups rotate the
    // direction by env_rot (mat3, column-major m[col * 3 + row]); importance samples by its transpose
    int env_rot;
    float env_rot_m[9];

    // device buffers (all owned by the context)
    const float* density;          // normalised density, x-fastest
    const float* sv_data;          // 2 floats per supervoxel: (min, max) or (mu_c, mu_r_bar)
    const uint8_t* occupancy;      // 1 byte per supervoxel
    const float* sv_local;         // 4 floats per supervoxel: mu_c, mu_r_bar, 1 / max density, 1 / majorant
    const float* env_rgba;         // equirect RGBA fp32
    const float* env_pyramid;      // octahedral max-luminance pyramid, level 0 first
    const uint64_t* env_level_offset; // float offset of each level in env_pyramid (indexed by level)
    double* film;                  // 3 doubles per pixel: sum of radiance
    double* film_sq;               // 3 doubles per pixel: sum of squared radiance (optional)
    float* feat;                   // feature accumulators (optional), kFeatStride floats per pixel
    int feat_background;           // accumulate the background map (requested by the user)
    int feat_depth_maps;           // bit 0: Depth Blended, bit 1: Depth Nearest Opaque (requested)

    // emission grid (USE_EMISSION): absorptions in next event tracking add sampleEmission(x)
    const float* emission;         // dense [nz][ny][nx] values, or null (no emission)
    int enx, eny, enz;
    F3 emission_box_min;
    F3 emission_vox_per_unit;
    float emission_cap, emission_strength;  // the strength also scales transfer-function emission
    int iso_brdf;              // surface BRDF of isosurface hits (IsoBrdf)
    // setBrdfParameter (VolumetricPathTracingPass.cpp:987-1011): subsurface, metallic, specular,
    // specular_tint, roughness, anisotropic, sheen, sheen_tint, clearcoat, clearcoat_gloss
    float brdf[10];
    float tf_albedo_strength;  // spectral trackers with a transfer function: scattering albedo mixed toward
                               //   the table's rgb by this weight (0: off; USE_TRANSFER_FUNCTION_SCATTERING_ALBEDO)

    // transfer function (USE_TRANSFER_FUNCTION): every density lookup becomes the table's alpha at the
    // normalised density; absorptions emit strength * its rgb
    const float* tf;               // tf_size RGBA entries, or null
    int tf_size;
    // isosurfaces inside the volume (USE_ISOSURFACES with a density field and Lambertian surfaces;
    // delta tracking with trilinear lookups): surfaces where the normalised density crosses iso_value
    int iso;
    int iso_subdivisions;          // checks per free-flight segment (NUM_ISOSURFACE_SUBDIVISIONS)
    float iso_value;
    F3 iso_color;
    // ISOSURFACE_TYPE_GRADIENT: the grid's gradient magnitudes [nz][ny][nx] (raw, not normalised), or
    // null for density isosurfaces; normals read them normalised with the density's min / range
    const float* iso_grad;
    float iso_norm_min, iso_norm_range;
    // USE_CLIP_PLANE: the volume box's ray intervals cut to the positive side of the plane
    // dot(clip_n, x) = clip_d (clip_n normalised)
    int use_clip;
    F3 clip_n;
    float clip_d;
    // CLOSE_ISOSURFACES (isosurfaces with the clip plane on): the box faces and the clip plane close the
    // isosurfaces, i.e. outside the volume counts as below the iso value on a path's first check point
    int iso_close;
    unsigned long long* counters;  // [0] paths, [1] density lookups
    int* error_flags;
    unsigned int* work_counter;    // persistent-kernel path queue

    SparseView sparse;             // valid when grid_kind == kNanoVdb

    int num_lights;                // NUM_LIGHTS of the reference (0 when lights are off)
    LightParams lights[kMaxLights];
};

// Offsets of the per-pixel feature accumulators (floats).
enum FeatureSlot : int {
    kFeatPos = 0,        // first event position xyz + hit count
    kFeatNormal = 4,     // xyz (finite difference of the density)
    kFeatDepth = 7,      // depth, depth^2
    kFeatDensity = 9,    // density*0.001, squared
    kFeatCloudOnly = 11, // rgb of paths with an event
    kFeatTrans = 14,     // primary-ray transmittance
                         // 15: unused (keeps the background float4-aligned)
    kFeatBackground = 16,// rgb: skybox of the camera ray for paths with an event, else their radiance
                         // 19: unused
    kFeatDepthBlended = 20,  // alpha-blended depth of the camera ray's march, its alpha
    kFeatDepthNearest = 22,  // depth of the last non-transparent march step times alpha, alpha
    // maps the reference overwrites every frame (not accumulated): written by the path of the last
    // frame of a launch
    kFeatFirstW = 24,        // direction after the first scatter, its phase pdf
    kFeatFlow = 28,          // pixel - the first event's pixel in the previous view (0 without an event)
    kFeatFlowReverse = 30,   // the first event's (or the camera direction's) previous pixel - pixel
    kFeatReprojUV = 32,      // two 64-bit keys (slots 32-33: u, 34-35: v), each (frame + 1) << 32 | float
                             //   bits: atomicMax keeps the uv of the latest frame with an event in the
                             //   previous view, whatever order the frames are traced in (0: none yet)
                             // 35: unused
    kFeatDerivNormal = 36,   // Depth (nabla) / (fwidth): the running-mean normal as Clouds.glsl mixes it,
    kFeatNabla = 39,         //   the nabla running mean (2)
    kFeatFwidth = 41,        //   and the fwidth running mean, advanced frame by frame by depth_deriv_kernel
    kFeatStride = 42,
};

}  // namespace vpt
