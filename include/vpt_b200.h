/*
 * vpt_b200.h - C ABI of the B200-native volumetric path-tracing core.
 *
 * Plain C, plain pointers and sizes.  No CUDA or torch types appear in the signatures: a CUDA
 * stream is passed as `void*` (a cudaStream_t, or NULL for the legacy default stream).  Every entry
 * point returns a VptStatus; no C++ exception crosses this boundary.  A context is not
 * thread-safe: use one context per host thread.
 *
 * Each declaration names the reference interface it replaces (paths inside chrismile/CloudRendering).
 * The reference reaches its tracer through the pybind11/TORCH_LIBRARY module `vpt`
 * (src/PyTorch/Module.cpp:85-182, 186+) and, below it, the VolumetricPathTracingPass setters
 * (src/PathTracer/VolumetricPathTracingPass.hpp:137-212).
 */
#ifndef VPT_B200_H
#define VPT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VPT_B200_ABI_VERSION 1

typedef struct VptContext VptContext;
typedef struct VptBatch VptBatch;

typedef enum VptStatus {
    VPT_OK = 0,
    VPT_ERR_ARG = 1,          /* bad argument (shape, range, null pointer, unknown name) */
    VPT_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    VPT_ERR_OOM = 3,          /* device allocation failed */
    VPT_ERR_ITER_LIMIT = 4,   /* a device loop hit its iteration guard (result is incomplete) */
    VPT_ERR_STATE = 5,        /* call not valid in the current state (e.g. no volume loaded) */
    VPT_ERR_UNSUPPORTED = 6   /* combination of settings not supported */
} VptStatus;

/* VptMode, same numbering as the reference enum (src/PathTracer/RenderSettings.hpp:32-36). */
enum {
    VPT_MODE_DELTA_TRACKING = 0,
    VPT_MODE_SPECTRAL_DELTA_TRACKING = 1,
    VPT_MODE_RATIO_TRACKING = 2,
    VPT_MODE_DECOMPOSITION_TRACKING = 3,
    VPT_MODE_RESIDUAL_RATIO_TRACKING = 4,
    VPT_MODE_NEXT_EVENT_TRACKING = 5,
    VPT_MODE_NEXT_EVENT_TRACKING_SPECTRAL = 6,
    VPT_MODE_ISOSURFACE_RENDERING = 7,
    VPT_MODE_RAY_MARCHING_EMISSION_ABSORPTION = 8,
    /* No counterpart in the reference, whose residual ratio mode (4) is a biased reservoir estimator
     * (ResidualRatioTracking.glsl, marked work in progress): next-event estimation with residual ratio
     * tracking (Novak et al. 2014) for the shadow rays over the supervoxel (mu_c, mu_r_bar) grid of
     * SuperVoxelGrid.cpp:218-265, and delta tracking with per-supervoxel majorants for the free paths.
     * Dense grids only. */
    VPT_MODE_RESIDUAL_RATIO_TRACKING_UNBIASED = 9
};

/* GridInterpolationType (RenderSettings.hpp:51-55). */
enum { VPT_INTERP_NEAREST = 0, VPT_INTERP_STOCHASTIC = 1, VPT_INTERP_TRILINEAR = 2 };

/* BuiltinEnvMap (RenderSettings.hpp:120-122) plus one addition: a constant sky with the
 * reference's Phong sun lobe, so that every tracker sees the sun (value 3). */
enum {
    VPT_ENV_DEFAULT = 0,
    VPT_ENV_BLACK = 1,
    VPT_ENV_SINGLE_COLOR = 2,
    VPT_ENV_CONSTANT_SUN = 3,
    VPT_ENV_IMAGE = 4          /* set by vpt_load_environment_map_rgba */
};

/* Feature maps (FeatureMapTypeVpt, VolumetricPathTracingPass.hpp:67-73) that this core writes. */
enum {
    VPT_FEATURE_RESULT = 0,
    VPT_FEATURE_FIRST_X = 1,
    VPT_FEATURE_FIRST_W = 2,       /* direction after the first scatter and its pdf, of the last frame */
    VPT_FEATURE_NORMAL = 3,
    VPT_FEATURE_NORMAL_LEN_1 = 4,  /* Normal with rgb scaled to length 1 (NormalizeNormals.glsl) */
    VPT_FEATURE_CLOUD_ONLY = 5,
    VPT_FEATURE_DEPTH = 6,
    VPT_FEATURE_DEPTH_FAR = 7,     /* mean of (event ? depth : far distance) */
    VPT_FEATURE_FLOW = 8,          /* (pixel - previous pixel of the first event, 0, 0), last frame */
    VPT_FEATURE_FLOW_REVERSE = 9,  /* (previous pixel of the first event or camera direction - pixel), last frame */
    VPT_FEATURE_DEPTH_NABLA = 10,  /* running mean over frames of (A / sqrt(1 - A^2), B / sqrt(1 - B^2)), (A, B) the
                                      view-space x, y of that frame's running-mean normal (0 without an event) */
    VPT_FEATURE_DEPTH_FWIDTH = 11, /* running mean of |nabla.x| + |nabla.y| (all channels) */
    VPT_FEATURE_DENSITY = 12,
    VPT_FEATURE_BACKGROUND = 13,
    VPT_FEATURE_REPROJ_UV = 14,    /* previous-view uv of the most recent first event, (-1, -1) before one */
    VPT_FEATURE_DEPTH_BLENDED = 15,        /* (alpha-blended depth, alpha, 0, 1) of a march along the camera ray */
    VPT_FEATURE_DEPTH_NEAREST_OPAQUE = 16, /* (depth of the last non-transparent step x alpha, alpha, 0, 1) */
    VPT_FEATURE_ALBEDO = 17,
    VPT_FEATURE_TRANSMITTANCE = 32 /* new: primary-ray transmittance (no reference counterpart) */
};

/* Denoiser types (DenoiserType, src/Denoiser/Denoiser.hpp:63-79; only these are built here). */
enum { VPT_DENOISER_NONE = 0, VPT_DENOISER_EAW = 1, VPT_DENOISER_SVGF = 2 };

typedef struct VptStats {
    uint64_t paths;            /* camera paths traced since the last reset of the counters */
    uint64_t density_lookups;  /* sampleCloud calls (trilinear = 1 call = 8 texels) */
    uint64_t frames;           /* frames accumulated in the film since the last reset */
    int32_t error_flags;       /* sticky device error bits (1 = iteration guard) */
    int32_t reserved;
} VptStats;

/* ---- life cycle: replaces vpt.initialize()/cleanup() (Module.cpp:732-813) ---- */
const char* vpt_status_string(int status);
int         vpt_abi_version(void);
/* Number of CUDA kernels this library has launched in this process (all contexts). */
uint64_t    vpt_kernel_launch_count(void);
VptStatus   vpt_create(VptContext** out_ctx, int cuda_device);
void        vpt_destroy(VptContext* ctx);
const char* vpt_last_error(const VptContext* ctx);

/* ---- volume data ----
 * Dense grid in x-fastest order (CloudData::setDensityField, src/CloudData.cpp:147-167; note the
 * reference sizes the buffer as X*Z*Z there, this core uses X*Y*Z).  The world box follows
 * CloudData::computeGridBounds (CloudData.cpp:63-78): largest side spans [-maxGridExtent, maxGridExtent].
 * Values are normalised on the device by (v - min)/(max - min) (DensityField::getDataFloatAtNorm,
 * src/DensityField.cpp:262-267; min := 0 when min == max, DensityField.cpp:146-150). */
VptStatus vpt_set_dense_grid(VptContext* ctx, const float* data, int nx, int ny, int nz, int data_on_device);
/* Emission (Module.cpp load_emission_file / set_use_emission / set_emission_cap / set_emission_strength;
 * sampleEmission, VptUtils.glsl:604-626): a dense [nz][ny][nx] grid with its own box (centred, largest
 * side 2 * max_grid_extent), looked up with the density grid's interpolation; with emission on, an
 * absorption in next event tracking (grey or spectral) ends the path with (t^2, t^4, t^8) * strength,
 * t = clamp(value * cap, 0, 1).  Defaults: off, cap 1, strength 1.  (The reference's delta-tracking
 * emission branch returns an undeclared variable and does not compile; delta tracking ignores it.) */
VptStatus vpt_set_emission_grid(VptContext* ctx, const float* data, int nx, int ny, int nz, int data_on_device);
VptStatus vpt_set_use_emission(VptContext* ctx, int use);
VptStatus vpt_set_emission_cap(VptContext* ctx, float cap);
VptStatus vpt_set_emission_strength(VptContext* ctx, float strength);
/* Transfer-function appearance (Module.cpp set_use_transfer_function; USE_TRANSFER_FUNCTION in
 * VptUtils.glsl:629-672, DeltaTracking.glsl, NextEventTracking.glsl): with it on, every density lookup
 * is the table's alpha at the normalised density (linear filtering over `entries` RGBA entries on
 * [0, 1], clamp to edge, as transferFunctionTexture), and an absorption emits emission_strength times
 * the table's rgb (delta and next event tracking, grey and spectral; other trackers and batched
 * rendering return VPT_ERR_UNSUPPORTED while a table is in use).  The table is the caller's:
 * the reference builds it in sgl's TransferFunctionWindow, which is not part of its source tree. */
VptStatus vpt_set_transfer_function(VptContext* ctx, const float* rgba, int entries);
VptStatus vpt_set_use_transfer_function(VptContext* ctx, int use);
/* setTfScatteringAlbedoStrength (Module.cpp:1352-1354, VolumetricPathTracingPass.cpp:914-925): with a
 * transfer function, spectral delta and spectral next event tracking scatter with the albedo
 * mix(scattering albedo, the table's rgb at the lookup, strength) (USE_TRANSFER_FUNCTION_SCATTERING_ALBEDO,
 * DeltaTracking.glsl:76-81) when strength > 0, as the reference enables it; 0, the default, leaves the
 * albedo alone. */
VptStatus vpt_set_tf_scattering_albedo_strength(VptContext* ctx, float strength);
/* Isosurfaces inside the volume (Module.cpp set_use_isosurfaces / set_iso_value / set_iso_surface_color /
 * set_isosurface_type / set_surface_brdf, src/PyTorch/Module.cpp:1163-1194; USE_ISOSURFACES in
 * DeltaTracking.glsl and CheckIsosurfaceHit.glsl): the surface where the normalised density crosses
 * iso_value (default 0.5) is found on every free-flight segment and reflects like an opaque surface
 * of colour iso_surface_color (default 0.4 0.4 0.4) with the selected BRDF; lookups are trilinear
 * while isosurfaces are on.  Built for delta and next event tracking, plain and spectral, on dense
 * grids (next event tracking with surface next-event estimation, USE_ISOSURFACE_NEE, for sky light
 * samples: with lights, an environment image or empty-space skipping it returns VPT_ERR_UNSUPPORTED);
 * other trackers, sparse grids, a transfer function and batched rendering return VPT_ERR_UNSUPPORTED.  Types "Density" and "Gradient"
 * (the surface where the trilinear-filtered gradient magnitude of the raw grid crosses iso_value:
 * central differences with clamped neighbours, VolumetricPathTracingPass.cpp:690-745, built on the GPU
 * at the first render after the grid or the type changed) and the BRDFs
 * "Lambertian" (Lambertian.glsl, the default), "Blinn Phong" (BlinnPhong.glsl), "Disney (2012)"
 * (Disney2012.glsl), "Cook Torrance" (CookTorrance.glsl) and "Ambient" (ConstantLighting.glsl) are
 * accepted, unknown names are ignored (as in the reference).
 * vpt_set_num_isosurface_subdivisions is the pass's own setting (VolumetricPathTracingPass.cpp:1028-1033,
 * default 2, 1..8).
 * vpt_set_brdf_parameter replaces set_brdf_parameter (src/PyTorch/Module.cpp:1196-1199,
 * VolumetricPathTracingPass.cpp:987-1014): key one of subsurface, metallic, specular, specular_tint,
 * roughness, anisotropic, sheen, sheen_tint, clearcoat, clearcoat_gloss (defaults 0, 0, 0.5, 0, 0.5, 0,
 * 0, 0.5, 0, 1), value a decimal string; unknown keys are ignored, the film restarts either way, a
 * value that is not a number returns VPT_ERR_ARG.  Cook-Torrance reads metallic, specular and
 * roughness; Disney (2012) reads all ten. */
VptStatus vpt_set_use_isosurfaces(VptContext* ctx, int use);
VptStatus vpt_set_iso_value(VptContext* ctx, double value);
VptStatus vpt_set_iso_surface_color(VptContext* ctx, double r, double g, double b);
VptStatus vpt_set_isosurface_type(VptContext* ctx, const char* name);
VptStatus vpt_set_surface_brdf(VptContext* ctx, const char* name);
VptStatus vpt_set_brdf_parameter(VptContext* ctx, const char* key, const char* value);
VptStatus vpt_set_num_isosurface_subdivisions(VptContext* ctx, int subdivisions);
/* The clip plane (set_use_clip_plane / set_clip_plane_normal / set_clip_plane_distance,
 * src/PyTorch/Module.cpp:1218-1232; USE_CLIP_PLANE in rayBoxIntersect, VptUtils.glsl:776-799): every
 * ray's interval in the volume box is cut to the side where dot(n, x) > distance, n the normalised
 * normal (default (1, 0, 0), distance 0, off).  Built for delta, ratio and next event tracking (plain
 * and spectral; with isosurfaces too); decomposition, residual ratio tracking and empty-space skipping
 * return VPT_ERR_UNSUPPORTED while it is on.  A zero or non-finite normal returns VPT_ERR_ARG. */
VptStatus vpt_set_use_clip_plane(VptContext* ctx, int use);
VptStatus vpt_set_clip_plane_normal(VptContext* ctx, double x, double y, double z);
VptStatus vpt_set_clip_plane_distance(VptContext* ctx, double distance);
/* set_close_isosurfaces (src/PyTorch/Module.cpp:1209-1211; CLOSE_ISOSURFACES, defined while isosurfaces
 * and the clip plane are both on, VolumetricPathTracingPass.cpp:1777-1779): outside the volume counts as
 * below the iso value on a path's first check point, so the box faces and the clip plane close the
 * isosurfaces, with the face's normal (rayBoxIntersectionNormal) and that normal in the normal map.
 * Off by default; traced on persistent warp batches. */
VptStatus vpt_set_close_isosurfaces(VptContext* ctx, int close);
/* Synthetic scene on the device: seeded fBm of improved Perlin noise, remapped to [0, 1], values
 * below `threshold` set to 0.  No reference counterpart (the reference loads files). */
VptStatus vpt_generate_fbm_grid(VptContext* ctx, int nx, int ny, int nz, uint32_t seed, int octaves,
                                float lacunarity, float gain, float base_frequency, float threshold);
/* Copies the device grid (raw, un-normalised values) to `out` (x-fastest, nx*ny*nz floats). */
VptStatus vpt_get_dense_grid(VptContext* ctx, float* out, int out_on_device);
/* Voxel spacing of the next grid set by vpt_set_dense_grid (CloudData voxelSizeX/Y/Z, read from
 * .xyz headers in CloudData::loadFromXyzFile, CloudData.cpp:248-258); reset to 1 after that call. */
VptStatus vpt_set_voxel_size(VptContext* ctx, double sx, double sy, double sz);
/* vpt.set_max_grid_extent (Module.cpp setMaxGridExtent); applies to the next grid that is set. */
VptStatus vpt_set_max_grid_extent(VptContext* ctx, float max_grid_extent);
/* Returns boxMin (3 floats) then boxMax (3 floats) in world space (vpt.get_render_bounding_box). */
VptStatus vpt_get_render_bounding_box(VptContext* ctx, float out_min_max[6]);
/* setGlobalWorldBoundingBox (Module.cpp:1383-1388, CloudData.cpp:1274-1349): NanoVDB grids loaded
 * afterwards are placed by this world box instead of their own (the largest side of the global box
 * spans 2 * max grid extent); box_min / box_max NULL clears it.  Grids built from dense data ignore it,
 * as in the reference. */
VptStatus vpt_set_global_world_bounding_box(VptContext* ctx, const float box_min[3], const float box_max[3]);

/* ---- settings (VolumetricPathTracingPass setters, .hpp:137-212) ---- */
VptStatus vpt_set_vpt_mode(VptContext* ctx, int mode);                     /* setVptMode */
VptStatus vpt_set_grid_interpolation(VptContext* ctx, int interpolation);  /* setSparseGridInterpolationType */
VptStatus vpt_set_extinction_scale(VptContext* ctx, float scale);          /* setExtinctionScale */
VptStatus vpt_set_extinction_base(VptContext* ctx, const float rgb[3]);    /* setExtinctionBase */
VptStatus vpt_set_scattering_albedo(VptContext* ctx, const float rgb[3]);  /* setScatteringAlbedo */
VptStatus vpt_set_phase_g(VptContext* ctx, float g);                       /* setPhaseG */
VptStatus vpt_set_seed_offset(VptContext* ctx, uint32_t offset);           /* setCustomSeedOffset */
VptStatus vpt_set_use_linear_rgb(VptContext* ctx, int use_linear_rgb);     /* setUseLinearRGB */
/* Scatter events after which a path counts as absorbed; 0 = unlimited (the reference has no cap). */
VptStatus vpt_set_max_bounces(VptContext* ctx, int max_bounces);
/* setUseBuiltinEnvironmentMap (VolumetricPathTracingPass.cpp:1194-1202) by enum value. */
VptStatus vpt_set_builtin_environment_map(VptContext* ctx, int env_kind);
VptStatus vpt_set_environment_map_intensity_rgb(VptContext* ctx, const float rgb[3]);
/* Sun direction (normalised here) and sun intensity (rgb, = sunlightIntensity * sunlightColor in
 * VolumetricPathTracingPass.cpp:2063-2064).  For VPT_ENV_SINGLE_COLOR the sky is `intensity`. */
VptStatus vpt_set_sun(VptContext* ctx, const float direction[3], const float intensity_rgb[3]);
/* Sky radiance of VPT_ENV_CONSTANT_SUN. */
VptStatus vpt_set_sky_color(VptContext* ctx, const float rgb[3]);
/* loadEnvironmentMapImageFromLinearBuffer (VolumetricPathTracingPass.cpp:1489-1556) for fp32 RGBA,
 * equirectangular, row-major; builds the 4096^2 octahedral importance pyramid on the device. */
VptStatus vpt_load_environment_map_rgba(VptContext* ctx, const float* rgba, int width, int height,
                                        int is_linear_rgb, int data_on_device);
/* Environment-image rotation (USE_ENV_MAP_ROTATION, VptUtils.glsl:142-153, 303-306;
 * VolumetricPathTracingPass.cpp:1218-1284, 2102-2113): lookups use envMapDirRot * dir, importance
 * samples invEnvMapDirRot * dir.  `rotation` is a 3x3 matrix, column-major; NULL disables the rotation
 * (disableEnvMapRot).  Applies to environment images only, as in the reference. */
VptStatus vpt_set_env_map_rotation(VptContext* ctx, const float rotation[9]);
/* setEnvMapRotCamera: the rotation follows the camera's view matrix (its upper 3x3) each frame. */
VptStatus vpt_set_env_map_rotation_camera(VptContext* ctx);

/* ---- camera (VolumetricPathTracingModuleRenderer.cpp:124-131, 303-324) ----
 * Right-handed look-at view, perspective projection with depth in [0, 1] and y flipped so that
 * image row 0 is the top of the picture.  fovy in radians. */
VptStatus vpt_set_camera(VptContext* ctx, const float position[3], const float target[3],
                         const float up[3], float fovy_radians, float near_dist, float far_dist);
/* Overwrites the view matrix (16 floats, column-major) (overwrite_camera_view_matrix). */
VptStatus vpt_set_view_matrix(VptContext* ctx, const float view[16]);
/* setViewProjectionMatrixAsPrevious (Module.cpp:1339-1341, VolumetricPathTracingModuleRenderer.cpp:339-341):
 * the previous view-projection (16 floats, column-major) that the Flow, Flow Reverse and Reprojected
 * UV feature maps reproject into; NULL stores the current camera's.  Until it is called the current
 * camera's is used (VolumetricPathTracingPass.cpp:1985-1989). */
VptStatus vpt_set_previous_view_projection(VptContext* ctx, const float view_proj[16]);
/* 16 floats each, column-major: inverse(proj * view) for the current resolution, and proj * view. */
VptStatus vpt_get_camera_matrices(VptContext* ctx, float inv_view_proj[16], float view_proj[16]);

/* ---- rendering: replaces vpt.render_frame (Module.cpp:286-317, 589-693) ---- */
VptStatus vpt_set_resolution(VptContext* ctx, int width, int height);
/* Clears the film: next frame index is 0 (onHasMoved, VolumetricPathTracingPass.cpp:1150-1162). */
VptStatus vpt_reset_accumulation(VptContext* ctx);
/* Clears the film and makes `first_frame` the frame index (seed, Clouds.glsl:80-84) that every
 * cleared film starts from, until set again (default 0; a parameter change clears the film back to
 * it).  Ranks that render disjoint frame ranges of one image this way trace exactly the paths of a
 * single run over all frames, so the sum of their FP64 films is that run's film (no counterpart in
 * the reference, which renders on one GPU). */
VptStatus vpt_set_frame_index(VptContext* ctx, uint32_t first_frame);
/* Traces `frames` 1-spp frames into the FP64 film on `stream` (enqueued, not synchronised). */
VptStatus vpt_render_frames(VptContext* ctx, int frames, void* stream);
/* Writes the accumulated mean (denoised when a denoiser is set) as channels x H x W fp32
 * (channels 3 or 4; alpha = 1).  `out` is a device pointer when out_on_device, else host
 * memory (the copy is synchronous then). */
VptStatus vpt_read_result(VptContext* ctx, float* out, int channels, int out_on_device, void* stream);
/* render_frames + read_result in one call: the reference render_frame. */
VptStatus vpt_render_frame(VptContext* ctx, int frames, float* out, int channels, int out_on_device,
                           void* stream);
/* Per-pixel sample variance of the mean (channels x H x W) when statistics are enabled. */
VptStatus vpt_set_collect_statistics(VptContext* ctx, int enabled);
VptStatus vpt_read_statistics(VptContext* ctx, double* out_sum, double* out_sum_sq, int out_on_device,
                              void* stream);
/* vpt.set_use_feature_maps / get_feature_map (Module.cpp setUseFeatureMaps, getFeatureMap). */
VptStatus vpt_set_use_feature_maps(VptContext* ctx, const int* features, int count);
VptStatus vpt_get_feature_map(VptContext* ctx, int feature, float* out, int channels, int out_on_device,
                              void* stream);
/* The feature planes a learned denoiser reads, in one launch on `stream`, into device buffers of the
 * current image size (any may be NULL): albedo [3][H][W] (medium albedo x hit fraction), normal
 * [3][H][W], depth mean [H][W], transmittance [H][W]; the first channels of vpt_get_feature_map's
 * Albedo / Normal / Depth / Transmittance maps. */
VptStatus vpt_get_denoiser_features(VptContext* ctx, float* albedo, float* normal, float* depth, float* transmittance,
                                    void* stream);
VptStatus vpt_get_stats(VptContext* ctx, VptStats* stats);
VptStatus vpt_reset_stats(VptContext* ctx);
/* Waits for the context's work on `stream`, then reports sticky device errors. */
VptStatus vpt_synchronize(VptContext* ctx, void* stream);

/* vpt.set_use_empty_space_skipping (VolumetricPathTracingPass::setUseEmptySpaceSkipping): NEE shadow
 * rays skip empty 8^3 blocks of the occupancy grid. */
VptStatus vpt_set_use_empty_space_skipping(VptContext* ctx, int enabled);
/* Tuning knobs without a reference counterpart: "schedule" (0 = one path per thread over pixel
 * tiles, 1 = persistent warps taking 32-path batches, 2 = persistent with per-lane path refill, the
 * default; trackers without a refill kernel fall back to 1),
 * "persistent_blocks_per_sm", "max_steps_per_path" (guard on tentative collisions of one path,
 * default 2^24; a path that reaches it stops and vpt_synchronize reports VPT_ERR_ITER_LIMIT),
 * "ess_ref_compat" (1 = empty-space skipping exactly as the reference runs it: every block marked
 * occupied, ComputeOccupancyGrid.glsl:108-109, and shadow samples stepped from the moving point,
 * NeeTransmittance.glsl:173-228), "sparse_fp16" (1 = leaf values of the next sparse volume stored as
 * IEEE half), "fbm_contrast" (remap clamp(0.5 + contrast * fbm, 0, 1) of vpt_generate_fbm_grid,
 * default 3.5), "density_texture" (1, the default: delta, ratio, next event, decomposition and unbiased
 * residual ratio tracking (without a transfer function) on a dense grid whose border density is 0 read the
 * density through a 3D texture object, the same texels bit for bit, for a second copy of the grid in
 * device memory; a grid beyond the 3D texture size or without memory for the copy is read directly;
 * 0 = always read directly), "refill_min_lanes" (1..32, default 4: in the per-lane refill schedule a
 * warp takes new paths for its empty lanes once this many wait, or when none holds a path; the paths
 * are the same whatever the value). */
VptStatus vpt_set_option(VptContext* ctx, const char* key, double value);

/* ---- denoisers (VolumetricPathTracingPass.cpp:2287-2311) ---- */
VptStatus vpt_set_denoiser(VptContext* ctx, int denoiser_type);
/* EAW keys: "iterations", "phi_color", "phi_position", "phi_normal", "ref_compute_quirk", "lattice_tiles"
 * (1, the default: each pass stages its taps in shared memory, 16 x 16 pixels of one residue class
 * modulo the step per block; 0: every tap read from global memory; the same arithmetic either way);
 * SVGF keys: "z_threshold", "normal_threshold" (set_denoiser_property). */
VptStatus vpt_set_denoiser_property(VptContext* ctx, const char* key, const char* value);

/* ---- stateless kernels on caller-owned device buffers (all pointers are device pointers) ---- */
/* Supervoxel min / max / mean of a normalised x-fastest grid with optional one-voxel halo and the
 * occupancy byte (max >= 1e-5) (SuperVoxelGridResidualRatioTracking::computeSuperVoxels and
 * SuperVoxelGridDecompositionTracking, src/PathTracer/SuperVoxelGrid.cpp:101-211, 316-396).
 * Outputs hold ceil(nx/sv)*ceil(ny/sv)*ceil(nz/sv) entries; avg/occ may be NULL. */
VptStatus vpt_build_supervoxel_grid(const float* density, int nx, int ny, int nz, int sv, int halo,
                                    float* out_min, float* out_max, float* out_avg, uint8_t* out_occupancy,
                                    void* stream);
/* Residual ratio tracking (mu_c, mu_r_bar) pairs from supervoxel min/max/mean and the extinction
 * (SuperVoxelGridResidualRatioTracking::recomputeSuperVoxels, SuperVoxelGrid.cpp:218-256). */
VptStatus vpt_build_rrt_params(const float* sv_min, const float* sv_max, const float* sv_avg, int count,
                               float extinction, int sv, float* out_pairs, void* stream);
/* No counterpart in the reference: the supervoxel grid of VPT_MODE_RESIDUAL_RATIO_TRACKING_UNBIASED,
 * 4 floats per supervoxel: (mu_c, mu_r_bar) as vpt_build_rrt_params, then 1 / max and
 * 1 / (extinction * max) of the supervoxel's largest normalised density (0 when that is 0). */
VptStatus vpt_build_residual_ratio_grid(const float* sv_min, const float* sv_max, const float* sv_avg, int count,
                                        float extinction, int sv, float* out4, void* stream);
/* Occupancy of block^3 blocks: 1 if any voxel (plus `halo` voxels around) exceeds `threshold`
 * (intent of OccupancyGridPass / ComputeOccupancyGrid.glsl:91-143, whose loop never runs). */
VptStatus vpt_build_occupancy_grid(const float* density, int nx, int ny, int nz, int block, int halo,
                                   float threshold, uint8_t* out, void* stream);
/* Octahedral max-luminance importance pyramid (2^levels square at level 0, levels concatenated)
 * of an equirectangular RGBA image (OctahedralMapper.glsl:65-85 + mip reduction). */
VptStatus vpt_build_environment_pyramid(const float* rgba, int width, int height, int levels, float* out_pyramid,
                                        void* stream);
/* ---- batched rendering (no counterpart in the reference; the many-scene configuration) ----
 * A batch renders several contexts in ONE persistent launch: each context keeps its own grid,
 * camera, resolution, medium, seeds and film, and frames[i] 1-spp frames are traced for context i
 * (0 skips it).  All contexts live on one device and share the tracker (delta, ratio or NEE without
 * empty space skipping), the interpolation and the grid kind; feature maps and SVGF are not
 * written.  The launch (parameter upload from pinned memory, counter reset, trace) is captured in a
 * CUDA graph on first use and replayed afterwards ("use_graph", default 1).  The first context's
 * "refill_min_lanes" and, when every context has one, the density texture apply to the launch.
 * Results are read per context with vpt_read_result / vpt_read_statistics. */
VptStatus vpt_batch_create(VptBatch** out_batch, VptContext* const* contexts, int count);
void vpt_batch_destroy(VptBatch* batch);
const char* vpt_batch_last_error(VptBatch* batch);
/* "use_graph" (0/1), "blocks_per_sm" (0 = occupancy calculator), "refill_min_lanes" (0 = the first
 * context's). */
VptStatus vpt_batch_set_option(VptBatch* batch, const char* key, double value);
VptStatus vpt_batch_render(VptBatch* batch, const int* frames, void* stream);
/* Times the batch at 1, 3/4, 1/2 and 1/4 of the resident blocks per SM and keeps the fastest, then at
 * that block count with refill thresholds of 1, 2, 4 and 8 lanes and keeps the fastest; the
 * calibration frames are rendered into the contexts' films, whose accumulation is then reset. */
VptStatus vpt_batch_autotune(VptBatch* batch, const int* frames, void* stream, int* out_blocks_per_sm);
VptStatus vpt_batch_get_stats(VptBatch* batch, VptStats* stats);
VptStatus vpt_batch_reset_stats(VptBatch* batch);

/* ---- lights (NEE only; struct Light, Data/Shaders/VPT/VptHeader.glsl:233-248) ---- */

/* vpt.set_use_lights (Module.cpp:1088-1092): NEE samples the lights (NUM_LIGHTS > 0) when set. */
VptStatus vpt_set_use_lights(VptContext* ctx, int use_lights);
/* vpt.clear_lights / add_light / remove_light (Module.cpp:1094-1113, LightEditorWidget.cpp:89-103).
 * add_light appends a light with the defaults of LightEditorWidget.hpp:69-85 (point light in view
 * space at the camera, intensity 0.5); at most 16 lights. */
VptStatus vpt_clear_lights(VptContext* ctx);
VptStatus vpt_add_light(VptContext* ctx, int* out_index);
VptStatus vpt_remove_light(VptContext* ctx, int index);
VptStatus vpt_get_light_count(VptContext* ctx, int* out_count);
/* vpt.set_light_property (LightEditorWidget::setLightProperty, LightEditorWidget.cpp:286-320): keys
 * "type" ("Point Light", "Spotlight", "Directional Light"), "space" ("World", "View",
 * "View Orientation"), "color", "position" / "direction", "spot_direction" (three numbers separated by
 * white space), "intensity", "spot_total_width", "spot_falloff_start", "use_distance" ("0"/"1"). */
VptStatus vpt_set_light_property(VptContext* ctx, int index, const char* key, const char* value);

/* ---- sparse (NanoVDB) volumes ---- */

typedef struct VptSparseInfo {
    uint64_t leaves;          /* 8^3 leaf nodes */
    uint64_t tiles;           /* distinct constant tiles referenced by the brick table */
    uint64_t device_bytes;    /* device memory of the sparse volume */
    int32_t table_origin[3];  /* first voxel of the brick table */
    int32_t table_dim[3];     /* bricks per axis */
    int32_t root_min[3];      /* index bounding box of the active values (inclusive) */
    int32_t root_max[3];
    float box_min[3];         /* render box (world) */
    float box_max[3];
    double world_min[3];      /* GridData::mWorldBBox */
    double world_max[3];
    double voxel_size[3];     /* GridData::mVoxelSize */
    int32_t fp16;             /* leaf values stored as half */
    int32_t lowest_level;     /* HDDA cell of the sparse decomposition tracker: 8 or 1 */
} VptSparseInfo;

/* Render through a sparse volume (VolumetricPathTracingPass::setUseSparseGrid,
 * src/PathTracer/VolumetricPathTracingPass.cpp:863-869).  With a dense grid loaded, the sparse
 * volume is built from it on the next render as CloudData::getSparseDensityField does
 * (src/CloudData.cpp:1385-1407: GridBuilder, background 0, voxel size boxExtent.x / nx).  Delta,
 * ratio, NEE (without empty space skipping) and HDDA decomposition tracking run on sparse grids;
 * residual ratio tracking needs the dense grid, as in the reference. */
VptStatus vpt_set_use_sparse_grid(VptContext* ctx, int use_sparse);
/* Loads a NanoVDB float grid (version 32; CloudData::loadFromNvdbFile / setNanoVdbGridHandle,
 * src/CloudData.cpp:169-172, 1360-1365) from host or device memory; it replaces the dense grid and
 * is fitted into [-maxGridExtent, maxGridExtent] (CloudData::computeSparseGridMetadata,
 * src/CloudData.cpp:1289-1357).  vpt_set_option(ctx, "sparse_fp16", 1) before loading stores the
 * leaf values as IEEE half. */
VptStatus vpt_set_nanovdb_grid(VptContext* ctx, const void* buffer, size_t bytes, int on_device);
/* Sparse volume description (builds it from the dense grid first if needed, as
 * CloudData::getVDBWorldBoundingBox does, src/CloudData.cpp:1440-1491). */
VptStatus vpt_get_sparse_grid_info(VptContext* ctx, VptSparseInfo* out);
/* Value, dim and active state of the sparse volume at `count` voxels (device arrays: 3 int32 per voxel
 * in, float / uint32 / uint8 out), as pnanovdb_readaccessor_get_value_address + read_float,
 * pnanovdb_readaccessor_get_dim and pnanovdb_readaccessor_is_active return them
 * (Data/Shaders/VPT/PNanoVDB.glsl:1800-1990). */
VptStatus vpt_sparse_query(VptContext* ctx, const int32_t* ijk, int count, float* values, uint32_t* dims,
                           uint8_t* active, void* stream);

/* ---- kernel-predicting denoiser (modules/kpn_module/src/Kernel.cu; PyTorchDenoiser.cpp:174-179,
 * 411-440).  Device arrays, NCHW float, at most 4 channels, odd kernel size up to 7. ---- */

/* perPixelKernelCuda (Kernel.cu:38-135): out[n,c,y,x] = sum over the k*k taps of
 * w[n,t,y,x] * image[n,c,y+dy,x+dx], taps outside the output size skipped; output size
 * min(image, weights).  softmax = 1 applies torch::softmax over the taps first (fused). */
VptStatus vpt_kpn_apply(const float* image, const float* weights, int n, int c, int h, int w, int weights_h,
                        int weights_w, int kernel_size, int softmax, float* out, void* stream);
/* inv_iter_kernel (PyTorchDenoiser.cpp:174-179 with getInvIterBaseKernel, Kernel.cu:138-186): the
 * sigmoid-gated blend of the low-resolution prediction, the high-frequency detail and (use_prev)
 * the reprojected previous frame, followed by the softmaxed per-pixel kernel of fused_weights'
 * first k*k channels.  fused_weights has k*k + 3 channels; x_lo / pred_lo are low_h x low_w. */
VptStatus vpt_kpn_inv_iter(const float* x_hi, const float* pred_lo, const float* x_lo, const float* prev,
                           const float* fused_weights, int n, int c, int h, int w, int low_h, int low_w, int weights_h,
                           int weights_w, int kernel_size, int use_prev, float* out, void* stream);
/* torch::avg_pool2d(x, 2, 2). */
VptStatus vpt_kpn_avg_pool2(const float* in, int n, int c, int h, int w, float* out, void* stream);
/* torch::grid_sampler_2d(prev, uv * 2 - 1, bilinear, zeros, align_corners = false), uv N x 2 x h x w. */
VptStatus vpt_kpn_reproject(const float* prev, const float* uv, int n, int c, int prev_h, int prev_w, int h, int w,
                            float* out, void* stream);

/* EAW a-trous chain (EAWBlitPass::_renderCompute, src/Denoiser/EAWDenoiser.cpp:345-391; weights of
 * EAWDenoise.glsl) on RGBA images; position/normal may be NULL.  Allocates its ping-pong images
 * on `stream` with the stream-ordered allocator and frees them before returning.  `out` must not
 * overlap color, position or normal (in-place filtering is rejected with VPT_ERR_ARG). */
VptStatus vpt_eaw_denoise_rgba(const float* color, const float* position, const float* normal, int width,
                               int height, int iterations, float phi_color, float phi_position, float phi_normal,
                               int ref_compute_quirk, float* out, void* stream);
/* No counterpart in the reference.  Same filter and arguments as vpt_eaw_denoise_rgba, for callers
 * that cannot allocate device memory while they denoise (a frame loop whose device memory is
 * already spent on the volume, the film and a framework's caching allocator; a host engine with a
 * fixed memory budget).  It allocates and frees nothing: its ping-pong image is one RGBA fp32 array
 * of at most 1024*1024 pixels (16 MiB) that the library reserves on every GPU that loads it, for the
 * life of the process.  width*height above 1048576 returns VPT_ERR_ARG.  The first call on a device
 * looks up the array's address and uploads the filter's tap weights with a synchronous copy; make
 * that first call before any stream capture.  All calls on a device share the array, so calls whose
 * work overlaps on the GPU race; nothing in it needs to start at zero.  As for vpt_eaw_denoise_rgba,
 * `out` must not overlap color, position or normal (VPT_ERR_ARG). */
VptStatus vpt_eaw_denoise_rgba_noalloc(const float* color, const float* position, const float* normal, int width,
                                       int height, int iterations, float phi_color, float phi_position,
                                       float phi_normal, int ref_compute_quirk, float* out, void* stream);

/* One frame of SVGF (Data/Shaders/Denoiser/SVGF/SVGF.glsl: reprojection, moments filter, `iterations`
 * a-trous passes, history update) on caller-prepared maps: noisy and normal rgba (normal.w unused),
 * depth, depth fwidth and screen-space motion (2 floats per pixel, previous = current - motion), and
 * the caller's history (colour rgba, moments rgba (mean, second moment, history length), normal
 * rgba, depth), updated in place.  Device arrays, width*height pixels. */
VptStatus vpt_svgf_filter(const float* noisy_rgba, const float* normal_rgba, const float* depth,
                          const float* depth_fwidth, const float* motion, float* color_history,
                          float* moments_history, float* normal_history, float* depth_history, int width, int height,
                          float z_threshold, float normal_threshold, int iterations, float* out_rgba, void* stream);

/* Random-sector gather rate (the access of a density lookup): blocks x 256 threads each issue
 * loads_per_thread (a multiple of 8) 4-byte loads at pseudo-random 32-byte-aligned offsets of
 * `buffer` (bytes a power of two, non-negative floats).  Time it on `stream`; sectors per second = 
 * blocks * 256 * (loads_per_thread / 8 * 8) / time. */
VptStatus vpt_gather_bench(const float* buffer, size_t bytes, int blocks, int loads_per_thread, uint32_t seed,
                           float* sink, void* stream);

/* ---- learned denoiser network (no reference counterpart: the reference runs a TorchScript model
 * through libtorch, src/Denoiser/PyTorchDenoiser.cpp:637-800, and has no training code).  A U-Net of
 * 3x3 convolutions predicting per-pixel 5x5 kernels, forward and backward on tcgen05 tensor cores.
 * Tensors are device arrays, NHWC bf16 ("pixels x channels", channel counts multiples of 16 for the
 * convolutions, 8 for the rest); conv weights [cout][9][cin] bf16 with tap = (dy+1)*3 + (dx+1).
 * `err` (device int, may be NULL) receives VPT_ERR_ITER_LIMIT if a kernel's bounded wait expired. ---- */

/* y[p][co] = act(bias[co] + sum_{t,ci} x[p + off(t)][ci] w[co][t][ci]) (zero padding), act = ReLU if
 * relu; then times (mask[p][co] > 0) if mask != NULL; y bf16, or fp32 if out_f32.  The input gradient
 * of a convolution is this call on the output gradient with vpt_unet_rotate_weights' weights and
 * the forward input as mask (ReLU derivative). */
VptStatus vpt_unet_conv3x3(const void* x, const void* w, const float* bias, const void* mask, void* y, int n, int h,
                           int width, int cin, int cout, int relu, int out_f32, int* err, void* stream);
/* Selects the convolution kernels: 0 (default) = by shape (the persistent row-strip kernels for images
 * at least 128 pixels wide where they are measured faster; input channels in up to 4 groups through an
 * fp32 partial allocated on the stream), 1 = the per-tile gather kernels everywhere, 2 = the row-strip
 * kernels wherever they apply. */
VptStatus vpt_unet_set_conv_path(int path);
/* Row-strip convolution kernel: 0 (default) = warp-specialised (input rows loaded by the tensor-memory-
 * access unit into a ring, one MMA warp, four epilogue warps, double TMEM accumulators; input
 * channel groups when the weights and a 4-row ring do not fit), 1 = the cp.async row-strip kernel. */
VptStatus vpt_unet_set_strip_kernel(int kind);
/* K splits of the per-tile gather convolution: 0 (default) = by grid size (grids of at most half an SM wave
 * split their K stages over up to 8 CTAs, whose fp32 sums, allocated on the stream, are added in split
 * order before the bias / ReLU / mask epilogue), 1 = never, k > 1 = always k (at most the K stages). */
VptStatus vpt_unet_set_conv_ksplit(int ksplit);
/* Shared-memory ring depth of the per-tile gather kernel: 3 or 4 stages, 0 (default) = by shape. */
VptStatus vpt_unet_set_gather_stages(int stages);
/* Weight gradient: partial[s][t*cin + ci][co] = sum over the pixels p of split s of
 * dy[p][co] x[p + off(t)][ci]; vpt_unet_wgrad_splits splits (pixels_per_split a multiple of 64 sizes
 * them for the gather kernel), vpt_unet_wgrad_rows(cin) rows each, reduced by vpt_unet_reduce_grads. */
VptStatus vpt_unet_conv3x3_wgrad(const void* x, const void* dy, float* partial, int n, int h, int width, int cin,
                                 int cout, int pixels_per_split, int* err, void* stream);
int vpt_unet_wgrad_rows(int cin);
/* Number of partial sums (splits) vpt_unet_conv3x3_wgrad writes for this shape: the row-strip kernel
 * (images at least 128 pixels wide) writes one per CTA, the gather kernel one per pixels_per_split
 * pixels. */
int vpt_unet_wgrad_splits(int n, int h, int width, int cin, int cout, int pixels_per_split);
/* wrot[ci][t][co] = w[co][8 - t][ci] */
VptStatus vpt_unet_rotate_weights(const void* w, void* wrot, int cin, int cout, void* stream);
/* 2x2 average pooling [n][h][w][c] -> [n][h/2][w/2][c] */
VptStatus vpt_unet_pool2(const void* in, void* out, int n, int h, int w, int c, void* stream);
/* out[n][y][x] = concat(lo[n][y/2][x/2] (ca channels), skip[n][y][x] (cs channels)) */
VptStatus vpt_unet_upcat(const void* lo, const void* skip, void* out, int n, int h, int w, int ca, int cs,
                         void* stream);
/* gradient at the coarse input of vpt_unet_upcat: (lo > 0) * sum over the 2x2 children of d[..][0:ca] */
VptStatus vpt_unet_upcat_grad_lo(const void* d, const void* lo, void* dlo, int n, int h, int w, int ca, int cs,
                                 void* stream);
/* (e > 0) * (d_cat[p][cat_off .. cat_off + c] + d_pool[n][y/2][x/2] / 4); d_cat / d_pool may be NULL */
VptStatus vpt_unet_encoder_grad(const void* d_cat, int cat_c, int cat_off, const void* d_pool, const void* e,
                                void* out, int n, int h, int w, int c, void* stream);
/* per-block column sums of dy [pixels][c] into partial[blocks][c] (bias gradient, first pass) */
VptStatus vpt_unet_bias_grad(const void* dy, float* partial, int pixels, int c, int blocks, void* stream);
/* grad_w[co][t][ci] = sum_s wpartial[s][t*cin+ci][co]; grad_b[co] = sum_b bpartial[b][co] (fixed order) */
VptStatus vpt_unet_reduce_grads(const float* wpartial, int splits, int cin, int cout, const float* bpartial,
                                int bblocks, float* grad_w, float* grad_b, void* stream);
/* one Adam step (Kingma & Ba 2015) on fp32 parameters; param_bf16 (may be NULL) receives the bf16 copy */
VptStatus vpt_unet_adam(float* param, void* param_bf16, float* m1, float* m2, const float* grad, long count, float lr,
                        float beta1, float beta2, float eps, int step, float grad_scale, void* stream);
VptStatus vpt_unet_to_bf16(const float* in, void* out, long count, void* stream);
/* network input [n][h][w][16] bf16 from planes [n][c][h][w]: log1p(radiance) 3, albedo 3, normal 3,
 * depth 1, transmittance 1, noise_level[n] (1/sqrt(frames) per image) 1, and from second_moment (mean
 * of the squared per-frame radiance, [n][3][h][w]) log1p of the standard error of the pixel mean
 * sqrt(max(0, m2 - mean^2)) * noise_level 3 (NULL inputs give zeros) */
VptStatus vpt_unet_pack_input(const float* radiance, const float* albedo, const float* normal, const float* depth,
                              const float* transmittance, const float* noise_level, const float* second_moment,
                              void* out, int n, int h, int w, void* stream);
int vpt_unet_head_blocks(int n, int h, int w);
/* Kernel-prediction head (perPixelKernelCuda semantics, modules/kpn_module/src/Kernel.cu:38-135, with
 * the tap softmax fused): out[n][c][y][x] = sum_j softmax(logits[p][0 .. k*k-1])_j
 * radiance[n][c][y+dy][x+dx] (k = kernel_size odd <= 15, taps outside skipped; logits [p][head_channels]
 * fp32, 16-byte aligned, head_channels >= k*k a multiple of 8, at most 512).  With target != NULL also the relative MSE
 * sum (d-t)^2/(t^2+eps)/(3*n*h*w) as per-block partial sums (vpt_unet_head_blocks of them) and its
 * gradient dlogits [p][head_channels] bf16 (0 beyond k*k).  out may be NULL. */
VptStatus vpt_unet_kpn_head(const float* logits, int head_channels, int kernel_size, const float* radiance,
                            const float* target, float* out, void* dlogits, float* loss_partial, int n, int h, int w,
                            float eps, void* stream);

/* Multi-scale reconstruction, level l (planar [n][3][h][w] fp32, h and w even):
 * c = d + sigmoid(logits[p][alpha_channel]) * (up(c_coarse) - up(pool(d))), c_coarse at h/2 x w/2. */
VptStatus vpt_unet_kpn_combine(const float* d, const float* c_coarse, const float* logits, int head_channels,
                               int alpha_channel, float* c, int n, int h, int w, void* stream);
/* Backward of one level of the reconstruction and of its kernel application (d = apply(x, logits)):
 * dlogits [p][head_channels] bf16 (tap logits, the blend logit at alpha_channel (< 0: no blend),
 * 0 elsewhere) and (with a blend) g_coarse = dL/dc_coarse.  The gradient at this level's output
 * comes from g_in, or with target != NULL from the relative MSE of c_out against the target (its
 * per-block partial sums to loss_partial, vpt_unet_head_blocks of them). */
VptStatus vpt_unet_kpn_level_grad(const float* logits, int head_channels, int kernel_size, int alpha_channel,
                                  const float* x, const float* d, const float* c_coarse, const float* g_in,
                                  const float* c_out, const float* target, float eps, void* dlogits, float* g_coarse,
                                  float* loss_partial, int n, int h, int w, void* stream);
/* out = a + b, bf16, count a multiple of 8 */
VptStatus vpt_unet_add(const void* a, const void* b, void* out, long count, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VPT_B200_H */
