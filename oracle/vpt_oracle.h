/*
 * vpt_oracle.h - CPU oracle of the volumetric path-tracing hot path (TEST INFRASTRUCTURE).
 *
 * A plain C++17 + OpenMP restatement of the reference's shader math (Data/Shaders/VPT/*.glsl,
 * src/PathTracer/SuperVoxelGrid.cpp, Data/Shaders/Denoiser/EAWDenoise.glsl).  It is the checker of
 * the CUDA core and the timed CPU baseline; nothing in the product links or calls it.
 *
 * Arithmetic follows the same conventions as the CUDA core: no FMA contraction
 * (-ffp-contract=off), IEEE division and sqrt, libm transcendentals (which may differ from CUDA's
 * by an ulp, the only source of path divergence).
 */
#ifndef VPT_ORACLE_H
#define VPT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleScene {
    float inv_view_proj[16];  /* column-major */
    int width, height;
    uint32_t frame_count;     /* first frame index (seed frame) */
    uint32_t num_frames;
    uint32_t seed_offset;
    int mode;                 /* VptMode numbering */
    int interp;               /* 0 nearest, 1 stochastic, 2 trilinear */
    int max_bounces;
    int use_ess;              /* NEE: occupancy-grid empty-space skipping */
    int ess_ref_compat;       /* reference stepping of the skipping shadow loop */
    float box_min[3], box_max[3];
    int nx, ny, nz;
    float vox_per_unit[3];
    float border_density;
    float extinction, albedo, g;
    int sv_size, svx, svy, svz;
    float sv_world[3];
    int env_kind, use_linear_rgb, env_image_linear;
    float sun_dir[3], sun_intensity[3], sky_color[3], env_intensity[3];
    int env_w, env_h, env_levels;
    const float* density;     /* normalised, x-fastest */
    const float* sv_data;     /* 2 floats per supervoxel */
    const uint8_t* occupancy;
    const float* env_rgba;
    const float* env_pyramid; /* levels concatenated, level 0 first */
    /* sparse grid: when `nanovdb` is set, densities come from this NanoVDB float grid buffer
     * (version 32) through a restatement of PNanoVDB's read accessor */
    const uint8_t* nanovdb;
    float grid_min[3], grid_max[3];  /* world box of the grid: sampleCloud maps box -> grid box */
    int sparse_lowest_level;         /* HDDA cell of sparse decomposition tracking: 8 or 1 */
    int sparse_fp16;                 /* leaf values rounded to IEEE half (fp16 variant) */
    /* lights (NEE only): 16 floats per light: type, space, spot total width, spot falloff start,
     * color rgb, intensity, position xyz, use_distance, spot direction xyz, unused */
    float inv_view[16];              /* inverse view matrix, column-major (view-space lights) */
    int num_lights;
    int env_is_black;                /* parameters.isEnvMapBlack */
    float lights[16 * 16];
    /* spectral trackers: parameters.extinction and parameters.scatteringAlbedo (rgb; zero extinction =
     * extinction on every channel), SpectralDeltaTrackingCollisionProbability (0 max, 1 avg, 2 path
     * history avg) */
    float ext_rgb[3];
    float albedo_rgb[3];
    int sdt_prob;
    /* emission grid (USE_EMISSION; next event tracking, grey and spectral): raw values x-fastest, or
     * NULL; its world box, voxels per world unit, cap and strength */
    const float* emission;
    int enx, eny, enz;
    float emission_box_min[3], emission_vox_per_unit[3];
    float emission_cap, emission_strength;
    /* transfer function (USE_TRANSFER_FUNCTION): tf_size RGBA entries, or NULL; lookups return the
     * table's alpha at the normalised density, absorptions emit emission_strength * rgb */
    const float* tf;
    int tf_size;
    /* isosurfaces (USE_ISOSURFACES with ISOSURFACE_TYPE_DENSITY and SURFACE_BRDF_LAMBERTIAN; delta
     * tracking, trilinear lookups): surfaces where the normalised density crosses iso_value, checked
     * at iso_subdivisions points of every free-flight segment, reflecting with albedo iso_color */
    int use_iso;
    float iso_value;
    float iso_color[3];
    int iso_subdivisions;
    /* unbiased residual ratio tracking (mode 9): 1 / sv_world, and 4 floats per supervoxel (mu_c,
     * mu_r_bar, 1 / max density, 1 / majorant) */
    float sv_inv_world[3];
    const float* sv_local;
    /* USE_ENV_MAP_ROTATION for environment images: envMapDirRot, 3x3 column-major */
    int env_rot;
    float env_rot_m[9];
    /* USE_TRANSFER_FUNCTION_SCATTERING_ALBEDO (spectral trackers with a transfer function): the
     * scattering albedo is mixed toward the table's rgb by this weight when it is > 0 */
    float tf_albedo_strength;
    /* surface BRDF of isosurface hits: 0 Lambertian, 1 Blinn-Phong, 2 Ambient (ConstantLighting),
     * 3 Cook-Torrance, 4 Disney (2012) */
    int iso_brdf;
    /* setBrdfParameter values: subsurface, metallic, specular, specular_tint, roughness, anisotropic,
     * sheen, sheen_tint, clearcoat, clearcoat_gloss */
    float brdf[10];
    /* ISOSURFACE_TYPE_GRADIENT: the raw grid's gradient magnitudes [nz][ny][nx], or NULL (density
     * isosurfaces); normals read them as (v - iso_norm_min) / iso_norm_range (the density's range) */
    const float* iso_grad;
    float iso_norm_min, iso_norm_range;
    /* USE_CLIP_PLANE: every ray-box interval cut to the plane's positive side; clip = normalised
     * normal (3) and distance */
    int use_clip;
    float clip[4];
    /* CLOSE_ISOSURFACES (isosurfaces with the clip plane on): outside the volume counts as below the iso
     * value on a path's first check point; the surface there takes the entered face's normal */
    int iso_close;
} OracleScene;

/* Renders width*height*num_frames paths; adds radiance (and its square) per pixel (3 doubles). */
int oracle_render(const OracleScene* s, double* film, double* film_sq, uint64_t* lookups, int threads);
/* One path per (x, y, frame) triple; writes rgb radiance per path. */
int oracle_trace_paths(const OracleScene* s, const int* xs, const int* ys, const uint32_t* frames, int n,
                       float* out_rgb, int threads);
/* Rows [row0, row1) of every frame (bounded CPU-baseline samples). */
int oracle_render_rows(const OracleScene* s, int row0, int row1, double* film, uint64_t* lookups, int threads);

/* Scene preparation (same definitions as the CUDA core). */
void oracle_fbm(float* out, int nx, int ny, int nz, uint32_t seed, int octaves, float lacunarity, float gain,
                float base_frequency, float threshold, float contrast);
void oracle_minmax(const float* v, uint64_t n, float* out_min, float* out_max);
void oracle_normalize(const float* in, float* out, uint64_t n, float vmin, float vmax);
void oracle_grid_bounds(int nx, int ny, int nz, float max_grid_extent, float* box_min, float* box_max);
void oracle_supervoxel_stats(const float* dens, int nx, int ny, int nz, int sv, int halo, float* out_min,
                             float* out_max, float* out_avg, uint8_t* out_occ);
void oracle_rrt_params(const float* mn, const float* mx, const float* avg, int total, float extinction, int sv,
                       float* out_pairs);
void oracle_rrt_local(const float* mn, const float* mx, const float* avg, int total, float extinction, int sv,
                      float* out4);
void oracle_occupancy(const float* dens, int nx, int ny, int nz, int bs, int halo, float threshold, uint8_t* out);
void oracle_env_pyramid(const float* rgba, int w, int h, int levels, float* pyramid);

/* EAW a-trous chain on RGBA images (position/normal may be NULL). */
void oracle_svgf_frame(const float* noisy, const float* normal, const float* depth, const float* fwidth,
                       const float* motion, float* color_hist, float* moments_hist, float* normal_hist,
                       float* depth_hist, int w, int h, float zt, float nt, int iterations, float* out);
void oracle_eaw(const float* color, const float* pos, const float* nrm, int w, int h, int iterations,
                float phi_c, float phi_p, float phi_n, int quirk, float* out);

/* PNanoVDB accessor restated on a NanoVDB float grid: value, dim and active state of n voxels. */
void oracle_nanovdb_query(const uint8_t* buf, int n, const int32_t* ijk, float* value, uint32_t* dim,
                          uint8_t* active);
/* The sparse decomposition tracker's node walk for a straight ray (same record layout as the
 * reference driver's refvdb_hdda_walk). */
int oracle_nanovdb_hdda_walk(const uint8_t* buf, const float world_origin[3], const float world_dir[3],
                             int lowest_level, int max_visits, int32_t* out_voxel, int32_t* out_dim,
                             uint8_t* out_active, int32_t* out_level, float* out_box, float* out_t);

/* Kernel-predicting denoiser, restated from modules/kpn_module/src/Kernel.cu and the libtorch ops it
 * is composed with (softmax over channels, avg_pool2d(2, 2), grid_sampler_2d bilinear/zeros/
 * align_corners=false).  NCHW float arrays. */
void oracle_softmax_channels(const float* in, int n, int k, int h, int w, float* out);
void oracle_kpn_apply(const float* image, const float* weights, int n, int c, int h, int w, int wh, int ww, int k,
                      float* out);
/* getInvIterBaseKernel; fused has k*k + 3 channels (batch stride (k*k + 3) * wh * ww) */
void oracle_kpn_inv_iter_base(const float* x_hi, const float* pred_lo, const float* x_lo, const float* prev,
                              const float* fused, int n, int c, int h, int w, int lh, int lw, int wh, int ww, int k,
                              int use_prev, float* out);
void oracle_avg_pool2(const float* in, int nc, int h, int w, float* out);
void oracle_grid_sample(const float* prev, const float* uv, int n, int c, int ph, int pw, int h, int w, float* out);

/* Hybrid Tausworthe stream: n floats after seeding with `seed`. */
void oracle_rng_stream(uint32_t seed, int n, float* out, uint32_t* out_state4);
/* 1: evaluate the tracer's transcendentals in double precision, rounded once to float (the mode of
 * the CUDA core's libvpt_b200_dr.so); 0 (default): the C library's float functions. */
void oracle_set_double_rounded_math(int on);

#ifdef __cplusplus
}
#endif
#endif
