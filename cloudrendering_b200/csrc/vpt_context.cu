// vpt_context.cu - the C ABI (include/vpt_b200.h): context life cycle, settings, scene data,
// camera, film and launches.  The context plays the role of the reference's
// VolumetricPathTracingModuleRenderer + VolumetricPathTracingPass pair
// (src/PyTorch/VolumetricPathTracingModuleRenderer.cpp, src/PathTracer/VolumetricPathTracingPass.cpp):
// it owns every device buffer and fills the launch parameter block before each render.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/vpt_b200.h"
#include "vpt_kernels.h"
#include "vpt_params.h"
#include "vpt_denoise.h"
#include "vpt_sparse.h"

using vpt::F3;

namespace {

F3 mk(float x, float y, float z) {
    F3 r;
    r.x = x;
    r.y = y;
    r.z = z;
    return r;
}

template <class T>
struct DevBuf {
    T* ptr = nullptr;
    size_t count = 0;
    cudaError_t alloc(size_t n) {
        if (n == count && ptr) return cudaSuccess;
        release();
        if (n == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            return e;
        }
        count = n;
        return cudaSuccess;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
};

// 32-bit PCG (RXS-M-XS output) used to shuffle the Perlin permutation.
uint32_t pcg_next(uint32_t& state) {
    state = state * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

void make_permutation(uint32_t seed, int out512[512]) {
    int p[256];
    for (int i = 0; i < 256; i++) p[i] = i;
    uint32_t st = seed;
    for (int i = 255; i > 0; i--) {
        uint32_t j = pcg_next(st) % (uint32_t)(i + 1);
        std::swap(p[i], p[j]);
    }
    for (int i = 0; i < 512; i++) out512[i] = p[i & 255];
}

// 4x4 helpers, column-major (m[col * 4 + row]) like glm, computed in double.
void mat_mul(const double* a, const double* b, double* out) {
    double r[16];
    for (int c = 0; c < 4; c++)
        for (int rr = 0; rr < 4; rr++) {
            double s = 0.0;
            for (int k = 0; k < 4; k++) s += a[k * 4 + rr] * b[c * 4 + k];
            r[c * 4 + rr] = s;
        }
    memcpy(out, r, sizeof(r));
}

bool mat_inverse(const double* m, double* out) {
    double a[4][8];
    for (int r = 0; r < 4; r++) {
        for (int c = 0; c < 4; c++) a[r][c] = m[c * 4 + r];
        for (int c = 0; c < 4; c++) a[r][4 + c] = (r == c) ? 1.0 : 0.0;
    }
    for (int col = 0; col < 4; col++) {
        int piv = col;
        for (int r = col + 1; r < 4; r++)
            if (fabs(a[r][col]) > fabs(a[piv][col])) piv = r;
        if (fabs(a[piv][col]) < 1e-300) return false;
        if (piv != col)
            for (int c = 0; c < 8; c++) std::swap(a[piv][c], a[col][c]);
        double inv = 1.0 / a[col][col];
        for (int c = 0; c < 8; c++) a[col][c] *= inv;
        for (int r = 0; r < 4; r++) {
            if (r == col) continue;
            double f = a[r][col];
            for (int c = 0; c < 8; c++) a[r][c] -= f * a[col][c];
        }
    }
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) out[c * 4 + r] = a[r][4 + c];
    return true;
}

}  // namespace

struct VptContext {
    int device = 0;
    std::string last_error;

    // settings (defaults of VolumetricPathTracingPass.hpp:247-345 and Module.cpp:797-798)
    int mode = VPT_MODE_DELTA_TRACKING;
    int interp = VPT_INTERP_STOCHASTIC;
    float extinction_scale = 1024.0f;
    float extinction_base[3] = {1.0f, 1.0f, 1.0f};
    float albedo[3] = {0.9f, 0.9f, 0.9f};
    float g = 0.5f;
    uint32_t seed_offset = 0;
    int use_linear_rgb = 1;
    int max_bounces = 0;
    int env_kind = VPT_ENV_DEFAULT;
    int env_image_loaded = 0;
    int env_image_linear = 1;
    int env_image_black = 0;
    float env_intensity[3] = {1.0f, 1.0f, 1.0f};
    int env_rot_mode = 0;         // 0 off, 1 matrix, 2 camera view (useEnvMapRot, useEnvMapRotCamera)
    float env_rot_m[9] = {1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f};
    int has_global_box = 0;       // setGlobalWorldBoundingBox
    float global_box_min[3] = {0.0f, 0.0f, 0.0f}, global_box_max[3] = {0.0f, 0.0f, 0.0f};
    float sun_dir[3] = {0.0f, 0.0f, 0.0f};
    float sun_intensity[3] = {2.6f * 1.0f, 2.6f * 0.961538462f, 2.6f * 0.884615385f};
    float sky_color[3] = {1.0f, 1.0f, 1.0f};
    float max_grid_extent = 0.25f;
    float voxel_size[3] = {1.0f, 1.0f, 1.0f};          // spacing of the current grid
    float pending_voxel_size[3] = {1.0f, 1.0f, 1.0f};  // spacing for the next grid
    int use_ess = 0;
    int ess_ref_compat = 0;
    int schedule = vpt::kScheduleRefill;
    int persistent_blocks_per_sm = 0;  // 0 = occupancy calculator (one resident wave)
    uint32_t max_steps = vpt::kMaxStepsPerPath;
    float fbm_contrast = 3.5f;  // remap of the fBm generator: clamp(0.5 + contrast * fbm, 0, 1)

    // dense grid
    int nx = 0, ny = 0, nz = 0;
    float vmin = 0.0f, vmax = 1.0f;
    float box_min[3] = {0, 0, 0}, box_max[3] = {0, 0, 0};
    DevBuf<float> raw, norm;
    DevBuf<float> grad;      // gradient magnitudes of `raw` for gradient isosurfaces, built on demand
    bool grad_valid = false;
    // emission grid (load_emission_file / set_use_emission / set_emission_cap / set_emission_strength;
    // VolumetricPathTracingPass.hpp:326-328 defaults)
    DevBuf<float> emission;
    int enx = 0, eny = 0, enz = 0;
    bool use_emission = false;
    float emission_cap = 1.0f, emission_strength = 1.0f;
    float tf_albedo_strength = 0.0f;  // setTfScatteringAlbedoStrength
    int iso_brdf = 0;                 // setSurfaceBrdf: 0 Lambertian, 1 Blinn Phong, 2 Ambient, 3 Cook Torrance,
                                      //   4 Disney (2012)
    // setBrdfParameter, in BrdfParam order; defaults of VolumetricPathTracingPass.hpp:410-419
    float brdf[vpt::kBrdfParamCount] = {0.0f, 0.0f, 0.5f, 0.0f, 0.5f, 0.0f, 0.0f, 0.5f, 0.0f, 1.0f};
    // transfer function (set_use_transfer_function; the RGBA table of transferFunctionTexture)
    DevBuf<float> tf;
    int tf_size = 0;
    bool use_tf = false;
    // isosurfaces (setUseIsosurfaces, setIsoValue, setIsoSurfaceColor; VolumetricPathTracingPass.hpp:382-395)
    bool use_iso = false;
    int iso_type = 0;  // setIsosurfaceType: 0 Density, 1 Gradient
    // setUseClipPlane / setClipPlaneNormal / setClipPlaneDistance (VolumetricPathTracingPass.hpp:403-405)
    bool use_clip = false;
    bool close_iso = false;  // setCloseIsosurfaces: CLOSE_ISOSURFACES with isosurfaces and the clip plane on
    float clip_normal[3] = {1.0f, 0.0f, 0.0f};
    float clip_distance = 0.0f;
    float iso_value = 0.5f;
    float iso_color[3] = {0.4f, 0.4f, 0.4f};
    int iso_subdivisions = 2;
    DevBuf<float> minmax;

    // sparse (NanoVDB) volume: built from the dense grid when use_sparse is set
    // (VolumetricPathTracingPass::setUseSparseGrid -> CloudData::getSparseDensityField) or loaded
    // from a NanoVDB buffer (CloudData::loadFromNvdbFile)
    bool use_sparse = false;
    bool sparse_valid = false;
    bool sparse_from_dense = true;
    bool sparse_fp16 = false;
    int sparse_grid_size[3] = {0, 0, 0};   // gridSizeX/Y/Z of the reference's CloudData
    float sparse_box_min[3] = {0, 0, 0}, sparse_box_max[3] = {0, 0, 0};
    vpt::SparseHost sparse_host;
    vpt::SparseDevice sparse_dev;

    // acceleration structures (rebuilt lazily)
    int sv_size = 8, svx = 0, svy = 0, svz = 0;
    int sv_kind = -1;            // tracker they were built for
    int sv_interp = -1;
    float sv_extinction = -1.0f;
    DevBuf<float> sv_min, sv_max, sv_avg, sv_pairs;
    DevBuf<float> sv_local;      // unbiased residual ratio tracking: 4 floats per supervoxel
    DevBuf<uint8_t> sv_occ;
    bool occ_valid = false;
    int occ_interp = -1;
    DevBuf<uint8_t> occupancy;
    // the normalised dense grid as a 3D texture (option "density_texture"): delta tracking reads it
    // through the texture unit when the border density is 0
    int density_texture = 1;
    int refill_min = 4;  // option "refill_min_lanes" (4: measured best of 1, 2, 4, 8 on the headline launch)
    cudaArray_t dens_array = nullptr;
    cudaTextureObject_t dens_tex = 0;
    cudaSurfaceObject_t dens_surf = 0;  // the same array, written by fill_density_array_kernel
    int dens_dims[3] = {0, 0, 0};
    bool dens_tex_fresh = false;   // the array holds the current grid
    bool dens_tex_failed = false;  // no texture for the current grid (size limit or memory)

    // environment image
    int env_w = 0, env_h = 0;
    int env_levels = 12;
    DevBuf<float> env_rgba, env_pyramid;
    DevBuf<uint64_t> env_offsets;
    std::vector<uint64_t> env_offsets_host;

    // lights of the light editor (LightEditorWidget), used by NEE when use_lights is set
    bool use_lights = false;
    std::vector<vpt::LightParams> lights;

    // camera (VolumetricPathTracingModuleRenderer.cpp:124-131)
    float cam_pos[3] = {0.0f, 0.0f, 0.8f};
    float cam_target[3] = {0.0f, 0.0f, 0.0f};
    float cam_up[3] = {0.0f, 1.0f, 0.0f};
    float fovy = 2.0f * atanf(0.5f);
    float near_dist = 1.0f / 512.0f, far_dist = 80.0f;
    bool view_overridden = false;
    double view[16];

    // film
    int width = 0, height = 0;
    uint32_t frame_count = 0;      // FrameInfo::frameCount: seeds and accumulation
    uint32_t frame_origin = 0;     // frame index a cleared film starts from (frame sharding)
    uint32_t film_frames = 0;      // frames held in the film (1 for SVGF, which wants 1-spp input)
    uint32_t feat_frames = 0;      // frames held in the feature accumulators
    uint32_t feature_frame_limit = 0;  // > 0: feature maps accumulate over the first this many frames only
    int sdt_prob = vpt::kSdtPathHistory;  // sdtCollisionProbability (VolumetricPathTracingPass.hpp:250-251)
    DevBuf<double> film, film_sq;
    bool collect_stats = false;
    bool features_on = false;
    bool feat_background = false;  // the Background map was requested (one more accumulator per sample)
    int feat_depth_maps = 0;       // bit 0: Depth Blended, bit 1: Depth Nearest Opaque requested (ray marches)
    int feat_depth_deriv = 0;      // bit 0: Depth (nabla), bit 1: Depth (fwidth) requested (normals replayed)
    DevBuf<float> frame_normals;   //   4 floats per pixel and frame of one feature launch
    DevBuf<float> feat;
    DevBuf<float> rgba_src, rgba_a, rgba_b;  // denoiser input and ping-pong buffers
    DevBuf<float> eaw_maps;                  // position + normal RGBA for EAW
    double prev_view_proj[16];
    bool has_prev_view_proj = false;
    // parameters.previousViewProjMatrix of the tracer (Flow, Flow Reverse, Reprojected UV): the matrix
    // stored by setViewProjectionMatrixAsPrevious, else the current camera's
    // (VolumetricPathTracingPass.cpp:1985-1989)
    float trace_prev_vp[16];
    bool has_trace_prev_vp = false;
    DevBuf<float> staging;         // CHW staging for host outputs

    DevBuf<unsigned long long> counters;
    DevBuf<int> error_flags;
    DevBuf<unsigned int> work_counter;
    uint64_t frames_total = 0;

    // denoiser
    int denoiser = VPT_DENOISER_EAW;
    vpt::EawSettings eaw;
    vpt::SvgfSettings svgf;
    vpt::SvgfState svgf_state;

    int num_sms = 148;
};

namespace {

VptStatus fail(VptContext* ctx, VptStatus st, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return st;
}

VptStatus cuda_fail(VptContext* ctx, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return fail(ctx, e == cudaErrorMemoryAllocation ? VPT_ERR_OOM : VPT_ERR_CUDA, m);
}

#define VPT_CHECK_CUDA(ctx, expr)                                   \
    do {                                                            \
        cudaError_t _e = (expr);                                    \
        if (_e != cudaSuccess) return cuda_fail((ctx), _e, #expr);  \
    } while (0)

#define VPT_CHECK_CTX(ctx) \
    do {                   \
        if (!(ctx)) return VPT_ERR_ARG; \
    } while (0)

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

bool features_needed(const VptContext* ctx);

// frames held in the feature accumulators (every film frame unless a feature frame limit applies)
uint32_t feature_frames(const VptContext* ctx) { return ctx->feat_frames > 0 ? ctx->feat_frames : 1u; }

void reset_film_state(VptContext* ctx) {
    ctx->frame_count = ctx->frame_origin;
    ctx->film_frames = 0;
    ctx->feat_frames = 0;
}

// CloudData::computeGridBounds (CloudData.cpp:63-78) with voxel size 1.
void compute_bounds(VptContext* ctx) {
    float sx = float(ctx->nx) * ctx->voxel_size[0], sy = float(ctx->ny) * ctx->voxel_size[1];
    float sz = float(ctx->nz) * ctx->voxel_size[2];
    float ms = std::max(sx, std::max(sy, sz));
    ctx->box_max[0] = sx * ctx->max_grid_extent / ms;
    ctx->box_max[1] = sy * ctx->max_grid_extent / ms;
    ctx->box_max[2] = sz * ctx->max_grid_extent / ms;
    for (int i = 0; i < 3; i++) ctx->box_min[i] = -ctx->box_max[i];
}

void release_density_texture(VptContext* ctx) {
    if (ctx->dens_tex) cudaDestroyTextureObject(ctx->dens_tex);
    if (ctx->dens_surf) cudaDestroySurfaceObject(ctx->dens_surf);
    if (ctx->dens_array) cudaFreeArray(ctx->dens_array);
    ctx->dens_tex = 0;
    ctx->dens_surf = 0;
    ctx->dens_array = nullptr;
    ctx->dens_dims[0] = ctx->dens_dims[1] = ctx->dens_dims[2] = 0;
    ctx->dens_tex_fresh = false;
}

// A new grid: the texture array is refilled on next use (kept when the dimensions stay the same).
void invalidate_accel(VptContext* ctx) {
    ctx->sv_kind = -1;
    ctx->occ_valid = false;
    ctx->dens_tex_fresh = false;
    ctx->dens_tex_failed = false;
    ctx->grad_valid = false;
}

// The texture over the normalised dense grid: a float 3D array (the driver's block layout) with a
// texture object (point filtering, unnormalised coordinates, border address mode: 0) and a surface
// object through which fill_density_array_kernel copies the grid in (one pass at HBM speed).  The
// array is kept across grids of the same size.  Returns false (and the kernels read the grid by
// global loads) when the array cannot be had: a grid beyond the 3D texture size limit, or no device
// memory left for the second copy.
bool ensure_density_texture(VptContext* ctx, cudaStream_t s) {
    if (ctx->dens_tex_fresh) return true;
    if (ctx->dens_tex_failed) return false;
    if (ctx->dens_array &&
        (ctx->dens_dims[0] != ctx->nx || ctx->dens_dims[1] != ctx->ny || ctx->dens_dims[2] != ctx->nz))
        release_density_texture(ctx);
    if (!ctx->dens_array) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess || ctx->nx > prop.maxTexture3D[0] ||
            ctx->ny > prop.maxTexture3D[1] || ctx->nz > prop.maxTexture3D[2] || ctx->ny > 65535 || ctx->nz > 65535) {
            ctx->dens_tex_failed = true;
            return false;
        }
        const cudaChannelFormatDesc fmt = cudaCreateChannelDesc<float>();
        const cudaExtent ext = make_cudaExtent((size_t)ctx->nx, (size_t)ctx->ny, (size_t)ctx->nz);
        if (cudaMalloc3DArray(&ctx->dens_array, &fmt, ext, cudaArraySurfaceLoadStore) != cudaSuccess) {
            cudaGetLastError();  // out of memory is not sticky: clear it and read the grid directly
            ctx->dens_array = nullptr;
            ctx->dens_tex_failed = true;
            return false;
        }
        cudaResourceDesc res = {};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = ctx->dens_array;
        cudaTextureDesc td = {};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        if (cudaCreateTextureObject(&ctx->dens_tex, &res, &td, nullptr) != cudaSuccess ||
            cudaCreateSurfaceObject(&ctx->dens_surf, &res) != cudaSuccess) {
            cudaGetLastError();
            release_density_texture(ctx);
            ctx->dens_tex_failed = true;
            return false;
        }
        ctx->dens_dims[0] = ctx->nx;
        ctx->dens_dims[1] = ctx->ny;
        ctx->dens_dims[2] = ctx->nz;
    }
    if (vpt::launch_fill_density_array(ctx->norm.ptr, ctx->dens_surf, ctx->nx, ctx->ny, ctx->nz, s) != cudaSuccess) {
        cudaGetLastError();
        release_density_texture(ctx);
        ctx->dens_tex_failed = true;
        return false;
    }
    ctx->dens_tex_fresh = true;
    return true;
}

VptStatus finish_grid(VptContext* ctx, cudaStream_t s) {
    size_t n = (size_t)ctx->nx * ctx->ny * ctx->nz;
    for (int i = 0; i < 3; i++) {
        ctx->voxel_size[i] = ctx->pending_voxel_size[i];
        ctx->pending_voxel_size[i] = 1.0f;
    }
    VPT_CHECK_CUDA(ctx, ctx->minmax.alloc(2));
    VPT_CHECK_CUDA(ctx, vpt::launch_minmax(ctx->raw.ptr, n, ctx->minmax.ptr, s));
    float mm[2];
    VPT_CHECK_CUDA(ctx, cudaMemcpyAsync(mm, ctx->minmax.ptr, sizeof(mm), cudaMemcpyDeviceToHost, s));
    VPT_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    ctx->vmin = mm[0];
    ctx->vmax = mm[1];
    if (ctx->vmin == ctx->vmax) ctx->vmin = 0.0f;  // DensityField.cpp:146-150
    VPT_CHECK_CUDA(ctx, ctx->norm.alloc(n));
    VPT_CHECK_CUDA(ctx, vpt::launch_normalize(ctx->raw.ptr, ctx->norm.ptr, n, ctx->vmin, ctx->vmax, s));
    VPT_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    compute_bounds(ctx);
    invalidate_accel(ctx);
    ctx->sparse_valid = false;  // a sparse volume is rebuilt from the new dense grid on demand
    ctx->sparse_from_dense = true;
    reset_film_state(ctx);
    return VPT_OK;
}

// Render box of a sparse volume (CloudData::computeSparseGridMetadata, CloudData.cpp:1289-1357):
// the grid's world box itself when it was built from the dense grid, otherwise the world box fitted
// into [-maxGridExtent, maxGridExtent] along its longest side (float arithmetic as glm::vec3).
void compute_sparse_box(VptContext* ctx) {
    const vpt::SparseHost& h = ctx->sparse_host;
    float wmin[3], wmax[3];
    for (int i = 0; i < 3; i++) {
        wmin[i] = float(h.world_min[i]);
        wmax[i] = float(h.world_max[i]);
    }
    if (ctx->sparse_from_dense) {
        for (int i = 0; i < 3; i++) {
            ctx->sparse_box_min[i] = wmin[i];
            ctx->sparse_box_max[i] = wmax[i];
        }
        return;
    }
    // the global world box, when set, replaces the grid's own box in the normalisation
    // (CloudData::computeSparseGridMetadata, CloudData.cpp:1320-1344)
    float gmin[3], gmax[3];
    for (int i = 0; i < 3; i++) {
        gmin[i] = ctx->has_global_box ? ctx->global_box_min[i] : wmin[i];
        gmax[i] = ctx->has_global_box ? ctx->global_box_max[i] : wmax[i];
    }
    float diff[3] = {gmax[0] - gmin[0], gmax[1] - gmin[1], gmax[2] - gmin[2]};
    float max_dim = std::max(diff[0], std::max(diff[1], diff[2]));
    float A = 2.0f * ctx->max_grid_extent / max_dim;
    for (int i = 0; i < 3; i++) {
        float L = diff[i] / max_dim;
        float B = ctx->max_grid_extent * L - gmax[i] * A;
        ctx->sparse_box_min[i] = A * wmin[i] + B;
        ctx->sparse_box_max[i] = A * wmax[i] + B;
    }
}

// Builds the sparse volume from the normalised dense grid as CloudData::getSparseDensityField does
// (CloudData.cpp:1385-1407): voxel size (boxMax.x - boxMin.x) / gridSizeX, origin boxMin.
VptStatus ensure_sparse(VptContext* ctx, cudaStream_t s) {
    if (ctx->sparse_valid) return VPT_OK;
    if (!ctx->norm.ptr) return fail(ctx, VPT_ERR_STATE, "no volume loaded");
    const double dx = double(ctx->box_max[0] - ctx->box_min[0]) / double(ctx->nx);
    const double origin[3] = {ctx->box_min[0], ctx->box_min[1], ctx->box_min[2]};
    std::string err;
    cudaError_t e = vpt::build_sparse_from_dense(ctx->norm.ptr, ctx->nx, ctx->ny, ctx->nz, dx, origin,
                                                 ctx->sparse_fp16, ctx->sparse_host, ctx->sparse_dev, s, err);
    if (e != cudaSuccess) {
        if (!err.empty()) return fail(ctx, VPT_ERR_UNSUPPORTED, err);
        return cuda_fail(ctx, e, "build_sparse_from_dense");
    }
    ctx->sparse_valid = true;
    ctx->sparse_from_dense = true;
    ctx->sparse_grid_size[0] = ctx->nx;
    ctx->sparse_grid_size[1] = ctx->ny;
    ctx->sparse_grid_size[2] = ctx->nz;
    compute_sparse_box(ctx);
    return VPT_OK;
}

int tracker_of(int mode) {
    switch (mode) {
        case VPT_MODE_DELTA_TRACKING: return vpt::kDelta;
        case VPT_MODE_RATIO_TRACKING: return vpt::kRatio;
        case VPT_MODE_DECOMPOSITION_TRACKING: return vpt::kDecomposition;
        case VPT_MODE_RESIDUAL_RATIO_TRACKING: return vpt::kResidualRatio;
        case VPT_MODE_NEXT_EVENT_TRACKING: return vpt::kNextEvent;
        case VPT_MODE_SPECTRAL_DELTA_TRACKING: return vpt::kSpectralDelta;
        case VPT_MODE_NEXT_EVENT_TRACKING_SPECTRAL: return vpt::kSpectralNextEvent;
        case VPT_MODE_RESIDUAL_RATIO_TRACKING_UNBIASED: return vpt::kResidualRatioNee;
        default: return -1;
    }
}

// SuperVoxelGrid constructors (SuperVoxelGrid.cpp:46-65, 275-294): halve the supervoxel size until
// it divides the grid when the grid is smaller than one supervoxel.
void supervoxel_dims(VptContext* ctx) {
    int s = 8;
    if (ctx->nx < s || ctx->ny < s || ctx->nz < s) {
        while (!(ctx->nx % s == 0 && ctx->ny % s == 0 && ctx->nz % s == 0)) s /= 2;
    }
    ctx->sv_size = s;
    ctx->svx = (ctx->nx + s - 1) / s;
    ctx->svy = (ctx->ny + s - 1) / s;
    ctx->svz = (ctx->nz + s - 1) / s;
}

float extinction_x(const VptContext* ctx) { return ctx->extinction_base[0] * ctx->extinction_scale; }

VptStatus ensure_accel(VptContext* ctx, int tracker, cudaStream_t s) {
    if (ctx->use_sparse) {
        if (tracker == vpt::kResidualRatio || tracker == vpt::kResidualRatioNee ||
            ((tracker == vpt::kNextEvent || tracker == vpt::kSpectralNextEvent) && ctx->use_ess))
            return fail(ctx, VPT_ERR_UNSUPPORTED,
                        "residual ratio tracking and empty space skipping need a dense grid (as in the reference)");
        return ensure_sparse(ctx, s);
    }
    const bool need_sv =
        tracker == vpt::kDecomposition || tracker == vpt::kResidualRatio || tracker == vpt::kResidualRatioNee;
    const bool need_occ = (tracker == vpt::kNextEvent || tracker == vpt::kSpectralNextEvent) && ctx->use_ess;
    if (need_sv) {
        // setExtinctionScale does not rebuild the RRT grid in the reference
        // (VolumetricPathTracingPass.cpp:1289-1291); here the grid follows the current extinction.
        bool stale = ctx->sv_kind != tracker || ctx->sv_interp != ctx->interp ||
                     ((tracker == vpt::kResidualRatio || tracker == vpt::kResidualRatioNee) &&
                      ctx->sv_extinction != extinction_x(ctx));
        if (stale) {
            supervoxel_dims(ctx);
            int total = ctx->svx * ctx->svy * ctx->svz;
            VPT_CHECK_CUDA(ctx, ctx->sv_min.alloc(total));
            VPT_CHECK_CUDA(ctx, ctx->sv_max.alloc(total));
            VPT_CHECK_CUDA(ctx, ctx->sv_avg.alloc(total));
            VPT_CHECK_CUDA(ctx, ctx->sv_occ.alloc(total));
            VPT_CHECK_CUDA(ctx, ctx->sv_pairs.alloc((size_t)total * 2));
            // the unbiased tracker's majorants always include the one-voxel halo (a bound for every
            // lookup of the supervoxel, whatever the interpolation)
            int halo = (ctx->interp == VPT_INTERP_NEAREST && tracker != vpt::kResidualRatioNee) ? 0 : 1;
            VPT_CHECK_CUDA(ctx, vpt::launch_supervoxel_stats(ctx->norm.ptr, ctx->nx, ctx->ny, ctx->nz, ctx->sv_size,
                                                             ctx->svx, ctx->svy, ctx->svz, halo, ctx->sv_min.ptr,
                                                             ctx->sv_max.ptr, ctx->sv_avg.ptr, ctx->sv_occ.ptr, s));
            if (tracker == vpt::kResidualRatioNee) {
                float D = sqrtf(3.0f) * float(ctx->sv_size);
                VPT_CHECK_CUDA(ctx, ctx->sv_local.alloc((size_t)total * 4));
                VPT_CHECK_CUDA(ctx, vpt::launch_rrt_local(ctx->sv_min.ptr, ctx->sv_max.ptr, ctx->sv_avg.ptr, total,
                                                          extinction_x(ctx), D, ctx->sv_local.ptr, s));
            } else if (tracker == vpt::kResidualRatio) {
                float D = sqrtf(3.0f) * float(ctx->sv_size);
                VPT_CHECK_CUDA(ctx, vpt::launch_rrt_params(ctx->sv_min.ptr, ctx->sv_max.ptr, ctx->sv_avg.ptr, total,
                                                           extinction_x(ctx), D, ctx->sv_pairs.ptr, s));
            } else {
                VPT_CHECK_CUDA(ctx, vpt::launch_interleave(ctx->sv_min.ptr, ctx->sv_max.ptr, total, ctx->sv_pairs.ptr, s));
            }
            ctx->sv_kind = tracker;
            ctx->sv_interp = ctx->interp;
            ctx->sv_extinction = extinction_x(ctx);
        }
    }
    if (need_occ && (!ctx->occ_valid || ctx->occ_interp != ctx->interp)) {
        int bs = 8;
        ctx->sv_size = bs;
        int gx = (ctx->nx + bs - 1) / bs, gy = (ctx->ny + bs - 1) / bs, gz = (ctx->nz + bs - 1) / bs;
        VPT_CHECK_CUDA(ctx, ctx->occupancy.alloc((size_t)gx * gy * gz));
        int halo = ctx->interp == VPT_INTERP_NEAREST ? 0 : 1;
        VPT_CHECK_CUDA(ctx, vpt::launch_occupancy(ctx->norm.ptr, ctx->nx, ctx->ny, ctx->nz, bs, gx, gy, gz, halo, 0.0f,
                                                  ctx->ess_ref_compat, ctx->occupancy.ptr, s));
        ctx->occ_valid = true;
        ctx->occ_interp = ctx->interp;
        ctx->sv_kind = -1;  // sv_size now refers to the occupancy grid
    }
    return VPT_OK;
}

void compute_view(const VptContext* ctx, double* view) {
    if (ctx->view_overridden) {
        memcpy(view, ctx->view, sizeof(ctx->view));
    } else {
        double e[3] = {ctx->cam_pos[0], ctx->cam_pos[1], ctx->cam_pos[2]};
        double f[3] = {ctx->cam_target[0] - e[0], ctx->cam_target[1] - e[1], ctx->cam_target[2] - e[2]};
        double fl = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
        for (double& v : f) v /= fl;
        double u0[3] = {ctx->cam_up[0], ctx->cam_up[1], ctx->cam_up[2]};
        double s[3] = {f[1] * u0[2] - f[2] * u0[1], f[2] * u0[0] - f[0] * u0[2], f[0] * u0[1] - f[1] * u0[0]};
        double sl = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
        for (double& v : s) v /= sl;
        double u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
        double m[16] = {s[0], u[0], -f[0], 0.0, s[1], u[1], -f[1], 0.0, s[2], u[2], -f[2], 0.0,
                        -(s[0] * e[0] + s[1] * e[1] + s[2] * e[2]), -(u[0] * e[0] + u[1] * e[1] + u[2] * e[2]),
                        (f[0] * e[0] + f[1] * e[1] + f[2] * e[2]), 1.0};
        memcpy(view, m, sizeof(m));
    }
}

void compute_camera(const VptContext* ctx, double* vp_out, double* inv_out) {
    double view[16];
    compute_view(ctx, view);
    double aspect = (ctx->width > 0 && ctx->height > 0) ? double(ctx->width) / double(ctx->height) : 1.0;
    double th = tan(double(ctx->fovy) / 2.0);
    double n = ctx->near_dist, fa = ctx->far_dist;
    double proj[16] = {0};
    proj[0] = 1.0 / (aspect * th);
    proj[5] = -1.0 / th;  // y flipped: image row 0 is the top of the picture
    proj[10] = fa / (n - fa);
    proj[11] = -1.0;
    proj[14] = -(fa * n) / (fa - n);
    mat_mul(proj, view, vp_out);
    mat_inverse(vp_out, inv_out);
}

VptStatus fill_params(VptContext* ctx, int tracker, int frames, vpt::TraceParams& P) {
    memset(&P, 0, sizeof(P));
    double vp[16], inv[16];
    compute_camera(ctx, vp, inv);
    for (int i = 0; i < 16; i++) {
        P.inv_view_proj[i] = float(inv[i]);
        P.prev_view_proj[i] = ctx->has_trace_prev_vp ? ctx->trace_prev_vp[i] : float(vp[i]);
    }
    P.width = ctx->width;
    P.height = ctx->height;
    P.frame_count = ctx->frame_count;
    P.global_frame = ctx->frame_count;
    P.num_frames = (uint32_t)frames;
    P.seed_offset = ctx->seed_offset;
    P.num_paths = (uint64_t)ctx->width * ctx->height * (uint64_t)frames;
    P.box_min = mk(ctx->box_min[0], ctx->box_min[1], ctx->box_min[2]);
    P.box_max = mk(ctx->box_max[0], ctx->box_max[1], ctx->box_max[2]);
    P.nx = ctx->nx;
    P.ny = ctx->ny;
    P.nz = ctx->nz;
    P.vox_per_unit = mk(float(double(ctx->nx) / (double(ctx->box_max[0]) - double(ctx->box_min[0]))),
                        float(double(ctx->ny) / (double(ctx->box_max[1]) - double(ctx->box_min[1]))),
                        float(double(ctx->nz) / (double(ctx->box_max[2]) - double(ctx->box_min[2]))));
    P.border_density = (0.0f - ctx->vmin) / (ctx->vmax - ctx->vmin);
    P.emission = nullptr;
    P.emission_strength = ctx->emission_strength;
    P.tf_albedo_strength = ctx->tf_albedo_strength;
    P.iso_brdf = ctx->iso_brdf;
    for (int i = 0; i < vpt::kBrdfParamCount; ++i) P.brdf[i] = ctx->brdf[i];
    P.tf = (ctx->use_tf && ctx->tf.ptr && ctx->tf_size > 0) ? ctx->tf.ptr : nullptr;
    P.tf_size = ctx->tf_size;
    if (ctx->use_emission && ctx->emission.ptr) {
        // the emission grid's own box (CloudData::computeGridBounds with voxel size 1, centred)
        const float sx = float(ctx->enx), sy = float(ctx->eny), sz = float(ctx->enz);
        const float ms = std::max(sx, std::max(sy, sz));
        const float hx = sx * ctx->max_grid_extent / ms, hy = sy * ctx->max_grid_extent / ms,
                    hz = sz * ctx->max_grid_extent / ms;
        P.emission = ctx->emission.ptr;
        P.enx = ctx->enx;
        P.eny = ctx->eny;
        P.enz = ctx->enz;
        P.emission_box_min = mk(-hx, -hy, -hz);
        P.emission_vox_per_unit = mk(float(double(ctx->enx) / (2.0 * double(hx))),
                                     float(double(ctx->eny) / (2.0 * double(hy))),
                                     float(double(ctx->enz) / (2.0 * double(hz))));
        P.emission_cap = ctx->emission_cap;
    }
    P.extinction = extinction_x(ctx);
    P.inv_extinction = 1.0f / P.extinction;
    P.albedo = ctx->albedo[0];
    P.absorb_albedo = 1.0f - ctx->albedo[0];
    for (int c = 0; c < 3; ++c) {
        P.ext_rgb[c] = ctx->extinction_base[c] * ctx->extinction_scale;
        P.albedo_rgb[c] = ctx->albedo[c];
    }
    P.sdt_majorant = std::max(P.ext_rgb[0], std::max(P.ext_rgb[1], P.ext_rgb[2]));
    P.inv_sdt_majorant = 1.0f / P.sdt_majorant;
    P.sdt_prob = ctx->sdt_prob;
    P.g = ctx->g;
    // isosurfaces force trilinear lookups (VolumetricPathTracingPass.cpp:117-120)
    P.interp = ctx->use_iso ? vpt::kTrilinear : ctx->interp;
    P.iso = ctx->use_iso ? 1 : 0;
    P.iso_subdivisions = ctx->iso_subdivisions;
    P.iso_value = ctx->iso_value;
    P.iso_color = mk(ctx->iso_color[0], ctx->iso_color[1], ctx->iso_color[2]);
    P.iso_grad = (ctx->use_iso && ctx->iso_type == 1) ? ctx->grad.ptr : nullptr;
    P.use_clip = ctx->use_clip ? 1 : 0;
    P.iso_close = (ctx->use_clip && ctx->use_iso && ctx->close_iso) ? 1 : 0;  // VolumetricPathTracingPass.cpp:1777
    {  // the uniform holds glm::normalize(clipPlaneNormal): v * inversesqrt(dot(v, v)) in float
        const float* v = ctx->clip_normal;
        const float inv = 1.0f / std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
        P.clip_n = mk(v[0] * inv, v[1] * inv, v[2] * inv);
    }
    P.clip_d = ctx->clip_distance;
    P.iso_norm_min = ctx->vmin;
    P.iso_norm_range = ctx->vmax - ctx->vmin;
    P.max_bounces = ctx->max_bounces;
    P.max_steps = ctx->max_steps;
    P.ess_ref_compat = ctx->ess_ref_compat;
    P.sv_size = ctx->sv_size;
    P.svx = (ctx->nx + ctx->sv_size - 1) / ctx->sv_size;
    P.svy = (ctx->ny + ctx->sv_size - 1) / ctx->sv_size;
    P.svz = (ctx->nz + ctx->sv_size - 1) / ctx->sv_size;
    for (int a = 0; a < 3; a++) {
        float delta = ctx->box_max[a] - ctx->box_min[a];
        int n = a == 0 ? ctx->nx : (a == 1 ? ctx->ny : ctx->nz);
        float v = (float(ctx->sv_size) * delta) / float(n);
        if (a == 0) P.sv_world.x = v;
        if (a == 1) P.sv_world.y = v;
        if (a == 2) P.sv_world.z = v;
    }
    P.sv_inv_world = mk(1.0f / P.sv_world.x, 1.0f / P.sv_world.y, 1.0f / P.sv_world.z);
    P.env_kind = ctx->env_kind;
    P.use_linear_rgb = ctx->use_linear_rgb;
    P.env_image_linear = ctx->env_image_linear;
    P.sun_dir = mk(ctx->sun_dir[0], ctx->sun_dir[1], ctx->sun_dir[2]);
    P.sun_intensity = mk(ctx->sun_intensity[0], ctx->sun_intensity[1], ctx->sun_intensity[2]);
    P.sky_color = mk(ctx->sky_color[0], ctx->sky_color[1], ctx->sky_color[2]);
    P.env_intensity = mk(ctx->env_intensity[0], ctx->env_intensity[1], ctx->env_intensity[2]);
    P.env_is_black = ctx->env_kind == VPT_ENV_BLACK || (ctx->env_kind == VPT_ENV_IMAGE && ctx->env_image_black);
    P.env_w = ctx->env_w;
    P.env_h = ctx->env_h;
    P.env_levels = ctx->env_levels;
    P.env_base_res = 1 << ctx->env_levels;
    P.env_rot = ctx->env_rot_mode != 0 && ctx->env_kind == VPT_ENV_IMAGE;
    if (ctx->env_rot_mode == 2) {
        // useEnvMapRotCamera: envMapRot = camera->getViewMatrix() (its upper 3x3, column-major)
        double view[16];
        compute_view(ctx, view);
        for (int c = 0; c < 3; c++)
            for (int r = 0; r < 3; r++) P.env_rot_m[c * 3 + r] = float(view[c * 4 + r]);
    } else {
        for (int i = 0; i < 9; i++) P.env_rot_m[i] = ctx->env_rot_m[i];
    }
    P.density = ctx->norm.ptr;
    P.refill_min = ctx->refill_min;
    P.sv_data = ctx->sv_pairs.ptr;
    P.sv_local = ctx->sv_local.ptr;
    P.occupancy = ctx->occupancy.ptr;
    P.env_rgba = ctx->env_rgba.ptr;
    P.env_pyramid = ctx->env_pyramid.ptr;
    P.env_level_offset = ctx->env_offsets.ptr;
    P.film = ctx->film.ptr;
    P.film_sq = ctx->collect_stats ? ctx->film_sq.ptr : nullptr;
    P.feat = features_needed(ctx) ? ctx->feat.ptr : nullptr;
    P.feat_background = ctx->feat_background ? 1 : 0;
    P.feat_depth_maps = ctx->feat_depth_maps;
    P.counters = ctx->counters.ptr;
    P.error_flags = ctx->error_flags.ptr;
    P.work_counter = ctx->work_counter.ptr;
    {
        double view[16], iv[16];
        compute_view(ctx, view);
        mat_inverse(view, iv);
        for (int i = 0; i < 16; i++) P.inv_view[i] = float(iv[i]);
    }
    P.num_lights = ctx->use_lights ? (int)ctx->lights.size() : 0;
    for (int i = 0; i < P.num_lights; i++) P.lights[i] = ctx->lights[i];
    P.grid_kind = vpt::kDense;
    if (ctx->use_sparse && ctx->sparse_valid) {
        // superVoxelSize 8 (leaf level) unless the grid is smaller than a leaf
        // (VolumetricPathTracingPass.cpp:2071-2076)
        const int* gs = ctx->sparse_grid_size;
        const int lowest = (gs[0] >= 8 && gs[1] >= 8 && gs[2] >= 8) ? 8 : 1;
        P.grid_kind = vpt::kNanoVdb;
        P.sparse = vpt::make_sparse_view(ctx->sparse_host, ctx->sparse_dev, lowest);
        P.box_min = mk(ctx->sparse_box_min[0], ctx->sparse_box_min[1], ctx->sparse_box_min[2]);
        P.box_max = mk(ctx->sparse_box_max[0], ctx->sparse_box_max[1], ctx->sparse_box_max[2]);
    }
    (void)tracker;
    return VPT_OK;
}

// Feature accumulators are written when the user asked for feature maps or a denoiser needs them
// (the reference creates the maps a denoiser requests, VolumetricPathTracingPass.cpp:231-293).
bool features_needed(const VptContext* ctx) {
    return ctx->features_on || ctx->denoiser == VPT_DENOISER_SVGF ||
           (ctx->denoiser == VPT_DENOISER_EAW && ctx->eaw.iterations > 0);
}

VptStatus ensure_film(VptContext* ctx, cudaStream_t s) {
    size_t n = (size_t)ctx->width * ctx->height;
    if (ctx->film.count != n * 3) {
        VPT_CHECK_CUDA(ctx, ctx->film.alloc(n * 3));
        reset_film_state(ctx);
    }
    if (ctx->collect_stats && ctx->film_sq.count != n * 3) {
        VPT_CHECK_CUDA(ctx, ctx->film_sq.alloc(n * 3));
        reset_film_state(ctx);
    }
    if (features_needed(ctx) && ctx->feat.count != n * vpt::kFeatStride) {
        VPT_CHECK_CUDA(ctx, ctx->feat.alloc(n * vpt::kFeatStride));
        reset_film_state(ctx);
    }
    if (ctx->film_frames == 0) {
        VPT_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->film.ptr, 0, n * 3 * sizeof(double), s));
        if (ctx->collect_stats) VPT_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->film_sq.ptr, 0, n * 3 * sizeof(double), s));
        if (features_needed(ctx))
            VPT_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->feat.ptr, 0, n * vpt::kFeatStride * sizeof(float), s));
    }
    return VPT_OK;
}

bool parse_float(const char* v, float& out) {
    char* end = nullptr;
    out = strtof(v, &end);
    return end && end != v;
}

}  // namespace

namespace {

vpt::LightParams default_light() {
    // struct Light defaults (LightEditorWidget.hpp:69-85)
    vpt::LightParams l{};
    l.type = vpt::kLightPoint;
    l.space = vpt::kLightSpaceView;
    l.spot_total_width = 0.0981747704f;
    l.spot_falloff_start = 0.0245436926f;
    l.color = mk(1.0f, 0.961538462f, 0.884615385f);
    l.intensity = 0.5f;
    l.position = mk(0.0f, 0.0f, 0.0f);
    l.use_distance = 1;
    l.spot_direction = mk(0.0f, 0.0f, -1.0f);
    return l;
}

bool parse_vec3(const char* v, F3& out) {
    float a[3];
    const char* p = v;
    for (int i = 0; i < 3; i++) {
        char* end = nullptr;
        a[i] = strtof(p, &end);
        if (end == p) return false;
        p = end;
    }
    while (*p == ' ' || *p == '\t' || *p == '\n') p++;
    if (*p != '\0') return false;
    out = mk(a[0], a[1], a[2]);
    return true;
}

}  // namespace

struct VptBatch {
    std::vector<VptContext*> ctxs;
    int device = 0;
    int num_sms = 148;
    vpt::TraceParams* h_params = nullptr;     // pinned staging, read by the launch's first copy
    unsigned long long* h_offsets = nullptr;  // pinned staging
    vpt::TraceParams* d_params = nullptr;
    unsigned long long* d_offsets = nullptr;
    unsigned long long* d_counters = nullptr; // [0] work counter, [1] paths, [2] lookups
    int* d_err = nullptr;
    int blocks_per_sm = 0;                    // 0: occupancy calculator; set by vpt_batch_autotune
    int refill_min = 0;                       // 0: the first context's refill threshold; set by vpt_batch_autotune
    bool use_graph = true;
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    int exec_key[4] = {-1, -1, -1, -1};       // tracker, interp, grid kind, blocks of the captured launch
    cudaEvent_t done = nullptr;               // after the last launch (guards the pinned staging)
    bool launched = false;
    std::string last_error;
};

namespace {

VptStatus batch_fail(VptBatch* b, VptStatus st, const std::string& msg) {
    if (b) b->last_error = msg;
    return st;
}

void batch_release(VptBatch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    if (b->done) cudaEventDestroy(b->done);
    cudaFreeHost(b->h_params);
    cudaFreeHost(b->h_offsets);
    cudaFree(b->d_params);
    cudaFree(b->d_offsets);
    cudaFree(b->d_counters);
    cudaFree(b->d_err);
}

// Prepares every context (acceleration structures, film) and stages the launch parameters.
VptStatus batch_prepare(VptBatch* b, const int* frames, cudaStream_t s, vpt::BatchLaunch& L) {
    const int n = (int)b->ctxs.size();
    if (b->launched && cudaEventSynchronize(b->done) != cudaSuccess)
        return batch_fail(b, VPT_ERR_CUDA, "previous batch launch failed");
    int tracker = -1, interp = -1, grid_kind = -1;
    b->h_offsets[0] = 0;
    for (int i = 0; i < n; i++) {
        VptContext* ctx = b->ctxs[i];
        if (frames[i] < 0) return batch_fail(b, VPT_ERR_ARG, "frames must be >= 0");
        if (!ctx->norm.ptr && !(ctx->use_sparse && ctx->sparse_valid))
            return batch_fail(b, VPT_ERR_STATE, "a context has no volume loaded");
        if (ctx->width <= 0) return batch_fail(b, VPT_ERR_STATE, "a context has no resolution");
        const int t = tracker_of(ctx->mode);
        const int gk = ctx->use_sparse ? vpt::kNanoVdb : vpt::kDense;
        if (i == 0) {
            tracker = t;
            interp = ctx->interp;
            grid_kind = gk;
        } else if (t != tracker || ctx->interp != interp || gk != grid_kind) {
            return batch_fail(b, VPT_ERR_UNSUPPORTED,
                              "all contexts of a batch need the same tracker, interpolation and grid kind");
        }
        if (!(t == vpt::kDelta || t == vpt::kRatio || (t == vpt::kNextEvent && !ctx->use_ess)))
            return batch_fail(b, VPT_ERR_UNSUPPORTED,
                              "batched rendering supports delta, ratio and NEE (without empty space skipping)");
        if (features_needed(ctx)) return batch_fail(b, VPT_ERR_UNSUPPORTED, "batched rendering writes no feature maps");
        if (ctx->use_tf && ctx->tf.ptr)
            return batch_fail(b, VPT_ERR_UNSUPPORTED, "batched rendering has no transfer-function variant");
        if (ctx->use_iso) return batch_fail(b, VPT_ERR_UNSUPPORTED, "batched rendering has no isosurface variant");
        if (ctx->env_kind == VPT_ENV_IMAGE && !ctx->env_pyramid.ptr)
            return batch_fail(b, VPT_ERR_STATE, "environment image not loaded");
        VptStatus st = ensure_accel(ctx, t, s);
        if (st == VPT_OK) st = ensure_film(ctx, s);
        if (st != VPT_OK) return batch_fail(b, st, ctx->last_error);
        fill_params(ctx, t, frames[i], b->h_params[i]);
        b->h_offsets[i + 1] = b->h_offsets[i] + vpt::padded_paths(ctx->width, ctx->height, (uint32_t)frames[i]);
        // the density through each scene's texture object when every scene has one
        if (gk == vpt::kDense && ctx->density_texture && b->h_params[i].border_density == 0.0f &&
            ensure_density_texture(ctx, s))
            b->h_params[i].density_tex = ctx->dens_tex;
    }
    if (b->refill_min > 0)
        for (int i = 0; i < n; i++) b->h_params[i].refill_min = b->refill_min;
    if (grid_kind == vpt::kDense) {
        bool all_tex = true;
        for (int i = 0; i < n; i++) all_tex = all_tex && b->h_params[i].density_tex != 0;
        if (all_tex) grid_kind = vpt::kDenseTex;
    }
    int per_sm = b->blocks_per_sm;
    if (per_sm <= 0) {
        vpt::BatchLaunch q{};
        q.tracker = tracker;
        q.interp = interp;
        q.grid_kind = grid_kind;
        q.blocks_per_sm_out = &per_sm;
        if (vpt::launch_trace_batch(q, s) != cudaSuccess) return batch_fail(b, VPT_ERR_CUDA, "occupancy query failed");
    }
    L = vpt::BatchLaunch{};
    L.scenes = b->d_params;
    L.offsets = b->d_offsets;
    L.num = n;
    L.tracker = tracker;
    L.interp = interp;
    L.grid_kind = grid_kind;
    L.blocks = per_sm * b->num_sms;
    L.work_counter = b->d_counters;
    L.counters = b->d_counters + 1;
    L.error_flags = b->d_err;
    return VPT_OK;
}

// copy parameters -> zero the work counter -> trace, on stream s
cudaError_t batch_enqueue(VptBatch* b, const vpt::BatchLaunch& L, cudaStream_t s) {
    const int n = (int)b->ctxs.size();
    cudaError_t e = cudaMemcpyAsync(b->d_params, b->h_params, sizeof(vpt::TraceParams) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_offsets, b->h_offsets, sizeof(unsigned long long) * (n + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = vpt::launch_trace_batch(L, s);
    return e;
}

void batch_commit(VptBatch* b, const int* frames) {
    for (size_t i = 0; i < b->ctxs.size(); i++) {
        VptContext* ctx = b->ctxs[i];
        ctx->frame_count += (uint32_t)frames[i];
        ctx->film_frames += (uint32_t)frames[i];
        ctx->frames_total += (uint64_t)frames[i];
    }
}

}  // namespace

extern "C" {

const char* vpt_status_string(int status) {
    switch (status) {
        case VPT_OK: return "ok";
        case VPT_ERR_ARG: return "invalid argument";
        case VPT_ERR_CUDA: return "CUDA error";
        case VPT_ERR_OOM: return "out of device memory";
        case VPT_ERR_ITER_LIMIT: return "iteration guard reached";
        case VPT_ERR_STATE: return "invalid state";
        case VPT_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

int vpt_abi_version(void) { return VPT_B200_ABI_VERSION; }

uint64_t vpt_kernel_launch_count(void) { return vpt::launch_count(); }

VptStatus vpt_create(VptContext** out_ctx, int cuda_device) {
    if (!out_ctx) return VPT_ERR_ARG;
    *out_ctx = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return VPT_ERR_CUDA;
    if (cuda_device < 0 || cuda_device >= count) return VPT_ERR_ARG;
    if (cudaSetDevice(cuda_device) != cudaSuccess) return VPT_ERR_CUDA;
    VptContext* ctx = new VptContext();
    ctx->device = cuda_device;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, cuda_device);
    // sunlightDirection = normalize(0.5826, 0.7660, 0.2717) (VolumetricPathTracingPass.hpp:319)
    float d[3] = {0.5826f, 0.7660f, 0.2717f};
    float l = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int i = 0; i < 3; i++) ctx->sun_dir[i] = d[i] / l;
    if (ctx->counters.alloc(4) != cudaSuccess || ctx->error_flags.alloc(1) != cudaSuccess ||
        ctx->work_counter.alloc(2) != cudaSuccess) {
        delete ctx;
        return VPT_ERR_OOM;
    }
    cudaMemset(ctx->counters.ptr, 0, 4 * sizeof(unsigned long long));
    cudaMemset(ctx->error_flags.ptr, 0, sizeof(int));
    *out_ctx = ctx;
    return VPT_OK;
}

void vpt_destroy(VptContext* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    ctx->raw.release();
    ctx->norm.release();
    release_density_texture(ctx);
    ctx->sparse_dev.release();
    ctx->minmax.release();
    ctx->sv_min.release();
    ctx->sv_max.release();
    ctx->sv_avg.release();
    ctx->sv_pairs.release();
    ctx->sv_local.release();
    ctx->sv_occ.release();
    ctx->occupancy.release();
    ctx->env_rgba.release();
    ctx->env_pyramid.release();
    ctx->env_offsets.release();
    ctx->film.release();
    ctx->film_sq.release();
    ctx->feat.release();
    ctx->rgba_src.release();
    ctx->eaw_maps.release();
    ctx->rgba_a.release();
    ctx->rgba_b.release();
    ctx->staging.release();
    ctx->counters.release();
    ctx->error_flags.release();
    ctx->work_counter.release();
    vpt::svgf_release(ctx->svgf_state);
    delete ctx;
}

const char* vpt_last_error(const VptContext* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

VptStatus vpt_set_dense_grid(VptContext* ctx, const float* data, int nx, int ny, int nz, int data_on_device) {
    VPT_CHECK_CTX(ctx);
    if (!data || nx <= 0 || ny <= 0 || nz <= 0) return fail(ctx, VPT_ERR_ARG, "vpt_set_dense_grid: bad grid");
    cudaSetDevice(ctx->device);
    size_t n = (size_t)nx * ny * nz;
    VPT_CHECK_CUDA(ctx, ctx->raw.alloc(n));
    VPT_CHECK_CUDA(ctx, cudaMemcpy(ctx->raw.ptr, data, n * sizeof(float),
                                   data_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    ctx->nx = nx;
    ctx->ny = ny;
    ctx->nz = nz;
    return finish_grid(ctx, 0);
}

VptStatus vpt_set_emission_grid(VptContext* ctx, const float* data, int nx, int ny, int nz, int data_on_device) {
    VPT_CHECK_CTX(ctx);
    if (!data || nx <= 0 || ny <= 0 || nz <= 0) return fail(ctx, VPT_ERR_ARG, "vpt_set_emission_grid: bad grid");
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)nx * ny * nz;
    VPT_CHECK_CUDA(ctx, ctx->emission.alloc(n));
    VPT_CHECK_CUDA(ctx, cudaMemcpy(ctx->emission.ptr, data, n * sizeof(float),
                                   data_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    ctx->enx = nx;
    ctx->eny = ny;
    ctx->enz = nz;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_transfer_function(VptContext* ctx, const float* rgba, int entries) {
    VPT_CHECK_CTX(ctx);
    if (!rgba || entries <= 0 || entries > 65536) return fail(ctx, VPT_ERR_ARG, "vpt_set_transfer_function: bad table");
    cudaSetDevice(ctx->device);
    VPT_CHECK_CUDA(ctx, ctx->tf.alloc((size_t)entries * 4));
    VPT_CHECK_CUDA(ctx, cudaMemcpy(ctx->tf.ptr, rgba, (size_t)entries * 4 * sizeof(float), cudaMemcpyHostToDevice));
    ctx->tf_size = entries;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_tf_scattering_albedo_strength(VptContext* ctx, float strength) {
    VPT_CHECK_CTX(ctx);
    if (!std::isfinite(strength)) return fail(ctx, VPT_ERR_ARG, "vpt_set_tf_scattering_albedo_strength: not finite");
    if (strength != ctx->tf_albedo_strength) reset_film_state(ctx);
    ctx->tf_albedo_strength = strength;
    return VPT_OK;
}

VptStatus vpt_set_use_transfer_function(VptContext* ctx, int use) {
    VPT_CHECK_CTX(ctx);
    if ((use != 0) != ctx->use_tf) reset_film_state(ctx);
    ctx->use_tf = use != 0;
    return VPT_OK;
}

VptStatus vpt_set_use_isosurfaces(VptContext* ctx, int use) {
    VPT_CHECK_CTX(ctx);
    if ((use != 0) != ctx->use_iso) reset_film_state(ctx);
    ctx->use_iso = use != 0;
    return VPT_OK;
}

VptStatus vpt_set_iso_value(VptContext* ctx, double value) {
    VPT_CHECK_CTX(ctx);
    if (float(value) != ctx->iso_value) reset_film_state(ctx);
    ctx->iso_value = float(value);
    return VPT_OK;
}

VptStatus vpt_set_iso_surface_color(VptContext* ctx, double r, double g, double b) {
    VPT_CHECK_CTX(ctx);
    const float c[3] = {float(r), float(g), float(b)};
    if (c[0] != ctx->iso_color[0] || c[1] != ctx->iso_color[1] || c[2] != ctx->iso_color[2]) reset_film_state(ctx);
    for (int i = 0; i < 3; ++i) ctx->iso_color[i] = c[i];
    return VPT_OK;
}

VptStatus vpt_set_isosurface_type(VptContext* ctx, const char* name) {
    VPT_CHECK_CTX(ctx);
    if (!name) return fail(ctx, VPT_ERR_ARG, "null isosurface type");
    int type = -1;
    if (strcmp(name, "Density") == 0) type = 0;
    if (strcmp(name, "Gradient") == 0) type = 1;
    if (type < 0) return VPT_OK;  // unknown names are ignored, as in the reference
    if (type != ctx->iso_type) reset_film_state(ctx);
    ctx->iso_type = type;
    return VPT_OK;
}

VptStatus vpt_set_surface_brdf(VptContext* ctx, const char* name) {
    VPT_CHECK_CTX(ctx);
    if (!name) return fail(ctx, VPT_ERR_ARG, "null surface BRDF");
    int brdf = -1;
    if (strcmp(name, "Lambertian") == 0) brdf = 0;
    if (strcmp(name, "Blinn Phong") == 0) brdf = 1;
    if (strcmp(name, "Ambient") == 0) brdf = 2;
    if (strcmp(name, "Cook Torrance") == 0) brdf = 3;
    if (strcmp(name, "Disney (2012)") == 0) brdf = 4;
    if (brdf < 0) return VPT_OK;  // unknown names are ignored, as in the reference
    if (brdf != ctx->iso_brdf) reset_film_state(ctx);
    ctx->iso_brdf = brdf;
    return VPT_OK;
}

VptStatus vpt_set_brdf_parameter(VptContext* ctx, const char* key, const char* value) {
    VPT_CHECK_CTX(ctx);
    if (!key || !value) return fail(ctx, VPT_ERR_ARG, "null BRDF parameter key or value");
    static const char* const kKeys[vpt::kBrdfParamCount] = {"subsurface", "metallic", "specular", "specular_tint",
                                                        "roughness", "anisotropic", "sheen", "sheen_tint",
                                                        "clearcoat", "clearcoat_gloss"};
    for (int i = 0; i < vpt::kBrdfParamCount; ++i) {
        if (strcmp(key, kKeys[i]) != 0) continue;
        char* end = nullptr;
        const float v = strtof(value, &end);
        if (end == value) return fail(ctx, VPT_ERR_ARG, "BRDF parameter value is not a number");
        ctx->brdf[i] = v;
        break;
    }
    // unknown keys are logged and ignored by the reference; the film restarts either way
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_use_clip_plane(VptContext* ctx, int use) {
    VPT_CHECK_CTX(ctx);
    if ((use != 0) != ctx->use_clip) reset_film_state(ctx);
    ctx->use_clip = use != 0;
    return VPT_OK;
}

VptStatus vpt_set_clip_plane_normal(VptContext* ctx, double x, double y, double z) {
    VPT_CHECK_CTX(ctx);
    const float v[3] = {(float)x, (float)y, (float)z};
    if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2]) ||
        (v[0] == 0.0f && v[1] == 0.0f && v[2] == 0.0f))
        return fail(ctx, VPT_ERR_ARG, "vpt_set_clip_plane_normal: the normal must be finite and non-zero");
    if (v[0] != ctx->clip_normal[0] || v[1] != ctx->clip_normal[1] || v[2] != ctx->clip_normal[2])
        reset_film_state(ctx);
    for (int i = 0; i < 3; ++i) ctx->clip_normal[i] = v[i];
    return VPT_OK;
}

VptStatus vpt_set_close_isosurfaces(VptContext* ctx, int close) {
    VPT_CHECK_CTX(ctx);
    if ((close != 0) != ctx->close_iso) reset_film_state(ctx);
    ctx->close_iso = close != 0;
    return VPT_OK;
}

VptStatus vpt_set_clip_plane_distance(VptContext* ctx, double distance) {
    VPT_CHECK_CTX(ctx);
    const float d = (float)distance;
    if (!std::isfinite(d)) return fail(ctx, VPT_ERR_ARG, "vpt_set_clip_plane_distance: not finite");
    if (d != ctx->clip_distance) reset_film_state(ctx);
    ctx->clip_distance = d;
    return VPT_OK;
}

VptStatus vpt_set_num_isosurface_subdivisions(VptContext* ctx, int subdivisions) {
    VPT_CHECK_CTX(ctx);
    if (subdivisions < 1 || subdivisions > 8) return fail(ctx, VPT_ERR_ARG, "isosurface subdivisions must be in [1, 8]");
    if (subdivisions != ctx->iso_subdivisions) reset_film_state(ctx);
    ctx->iso_subdivisions = subdivisions;
    return VPT_OK;
}

VptStatus vpt_set_use_emission(VptContext* ctx, int use) {
    VPT_CHECK_CTX(ctx);
    if ((use != 0) != ctx->use_emission) reset_film_state(ctx);
    ctx->use_emission = use != 0;
    return VPT_OK;
}

VptStatus vpt_set_emission_cap(VptContext* ctx, float cap) {
    VPT_CHECK_CTX(ctx);
    ctx->emission_cap = cap;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_emission_strength(VptContext* ctx, float strength) {
    VPT_CHECK_CTX(ctx);
    ctx->emission_strength = strength;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_generate_fbm_grid(VptContext* ctx, int nx, int ny, int nz, uint32_t seed, int octaves, float lacunarity,
                                float gain, float base_frequency, float threshold) {
    VPT_CHECK_CTX(ctx);
    if (nx <= 0 || ny <= 0 || nz <= 0 || octaves <= 0 || octaves > 16)
        return fail(ctx, VPT_ERR_ARG, "vpt_generate_fbm_grid: bad size or octave count");
    cudaSetDevice(ctx->device);
    size_t n = (size_t)nx * ny * nz;
    VPT_CHECK_CUDA(ctx, ctx->raw.alloc(n));
    int perm[512];
    make_permutation(seed, perm);
    vpt::FbmParams fp;
    fp.octaves = octaves;
    fp.lacunarity = lacunarity;
    fp.gain = gain;
    fp.base_frequency = base_frequency;
    fp.threshold = threshold;
    fp.contrast = ctx->fbm_contrast;  // 0.5 + 3.5 * fbm by default: ~35% of voxels below 0.3 at frequency 3
    fp.inv_max_dim = 1.0f / float(std::max(nx, std::max(ny, nz)));
    VPT_CHECK_CUDA(ctx, vpt::launch_fbm(ctx->raw.ptr, nx, ny, nz, perm, fp, 0));
    ctx->nx = nx;
    ctx->ny = ny;
    ctx->nz = nz;
    return finish_grid(ctx, 0);
}

VptStatus vpt_get_dense_grid(VptContext* ctx, float* out, int out_on_device) {
    VPT_CHECK_CTX(ctx);
    if (!ctx->raw.ptr) return fail(ctx, VPT_ERR_STATE, "no dense grid");
    if (!out) return fail(ctx, VPT_ERR_ARG, "null output");
    size_t n = (size_t)ctx->nx * ctx->ny * ctx->nz;
    VPT_CHECK_CUDA(ctx, cudaMemcpy(out, ctx->raw.ptr, n * sizeof(float),
                                   out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
    return VPT_OK;
}

VptStatus vpt_set_voxel_size(VptContext* ctx, double sx, double sy, double sz) {
    VPT_CHECK_CTX(ctx);
    if (!(sx > 0.0 && sy > 0.0 && sz > 0.0)) return fail(ctx, VPT_ERR_ARG, "voxel sizes must be > 0");
    ctx->pending_voxel_size[0] = float(sx);
    ctx->pending_voxel_size[1] = float(sy);
    ctx->pending_voxel_size[2] = float(sz);
    return VPT_OK;
}

VptStatus vpt_set_max_grid_extent(VptContext* ctx, float e) {
    VPT_CHECK_CTX(ctx);
    if (!(e > 0.0f)) return fail(ctx, VPT_ERR_ARG, "max grid extent must be > 0");
    ctx->max_grid_extent = e;
    return VPT_OK;
}

VptStatus vpt_get_render_bounding_box(VptContext* ctx, float out[6]) {
    VPT_CHECK_CTX(ctx);
    if (!out) return VPT_ERR_ARG;
    if (ctx->use_sparse) {
        VptStatus st = ensure_sparse(ctx, nullptr);
        if (st != VPT_OK) return st;
    }
    for (int i = 0; i < 3; i++) {
        out[i] = ctx->use_sparse ? ctx->sparse_box_min[i] : ctx->box_min[i];
        out[3 + i] = ctx->use_sparse ? ctx->sparse_box_max[i] : ctx->box_max[i];
    }
    return VPT_OK;
}

VptStatus vpt_set_use_sparse_grid(VptContext* ctx, int use_sparse) {
    VPT_CHECK_CTX(ctx);
    bool u = use_sparse != 0;
    if (!u && ctx->use_sparse && !ctx->norm.ptr)
        return fail(ctx, VPT_ERR_UNSUPPORTED, "the loaded NanoVDB grid has no dense counterpart in this core");
    if (u != ctx->use_sparse) reset_film_state(ctx);
    ctx->use_sparse = u;
    return VPT_OK;
}

VptStatus vpt_set_nanovdb_grid(VptContext* ctx, const void* buffer, size_t bytes, int on_device) {
    VPT_CHECK_CTX(ctx);
    if (!buffer || bytes == 0) return fail(ctx, VPT_ERR_ARG, "vpt_set_nanovdb_grid: empty buffer");
    cudaSetDevice(ctx->device);
    cudaStream_t s = nullptr;
    std::vector<uint8_t> host;
    const uint8_t* hb = static_cast<const uint8_t*>(buffer);
    if (on_device) {
        host.resize(bytes);
        VPT_CHECK_CUDA(ctx, cudaMemcpy(host.data(), buffer, bytes, cudaMemcpyDeviceToHost));
        hb = host.data();
    }
    vpt::SparseHost h;
    std::string err;
    if (!vpt::parse_nanovdb(hb, bytes, h, err)) return fail(ctx, VPT_ERR_ARG, "vpt_set_nanovdb_grid: " + err);
    const uint8_t* db = static_cast<const uint8_t*>(buffer);
    uint8_t* tmp = nullptr;
    if (!on_device) {
        VPT_CHECK_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&tmp), bytes));
        cudaError_t e = cudaMemcpy(tmp, buffer, bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(tmp);
            return cuda_fail(ctx, e, "vpt_set_nanovdb_grid upload");
        }
        db = tmp;
    }
    cudaError_t e = vpt::upload_sparse_from_nanovdb(h, db, ctx->sparse_fp16, ctx->sparse_dev, s);
    if (tmp) cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "upload_sparse_from_nanovdb");
    ctx->sparse_host = std::move(h);
    // the NanoVDB grid replaces the dense grid (CloudData::setNanoVdbGridHandle)
    ctx->raw.release();
    ctx->norm.release();
    release_density_texture(ctx);
    invalidate_accel(ctx);
    ctx->use_sparse = true;
    ctx->sparse_valid = true;
    ctx->sparse_from_dense = false;
    for (int i = 0; i < 3; i++) {
        const int lo = ctx->sparse_host.root_min[i], hi = ctx->sparse_host.root_max[i];
        ctx->sparse_grid_size[i] = hi >= lo ? hi - lo + 1 : 0;
    }
    compute_sparse_box(ctx);
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_get_sparse_grid_info(VptContext* ctx, VptSparseInfo* out) {
    VPT_CHECK_CTX(ctx);
    if (!out) return VPT_ERR_ARG;
    cudaSetDevice(ctx->device);
    VptStatus st = ensure_sparse(ctx, nullptr);
    if (st != VPT_OK) return st;
    const vpt::SparseHost& h = ctx->sparse_host;
    memset(out, 0, sizeof(*out));
    out->leaves = h.leaf_count();
    out->tiles = h.tiles.size();
    out->device_bytes = ctx->sparse_dev.bytes;
    for (int i = 0; i < 3; i++) {
        out->table_origin[i] = h.tbl_origin[i];
        out->table_dim[i] = h.tbl_dim[i];
        out->root_min[i] = h.root_min[i];
        out->root_max[i] = h.root_max[i];
        out->box_min[i] = ctx->sparse_box_min[i];
        out->box_max[i] = ctx->sparse_box_max[i];
        out->world_min[i] = h.world_min[i];
        out->world_max[i] = h.world_max[i];
        out->voxel_size[i] = h.voxel_size[i];
    }
    out->fp16 = ctx->sparse_dev.values_h ? 1 : 0;
    const int* gs = ctx->sparse_grid_size;
    out->lowest_level = (gs[0] >= 8 && gs[1] >= 8 && gs[2] >= 8) ? 8 : 1;
    return VPT_OK;
}

VptStatus vpt_sparse_query(VptContext* ctx, const int32_t* ijk, int count, float* values, uint32_t* dims,
                           uint8_t* active, void* stream) {
    VPT_CHECK_CTX(ctx);
    if (!ijk || count < 0 || !values || !dims || !active) return VPT_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStream_t s = as_stream(stream);
    VptStatus st = ensure_sparse(ctx, s);
    if (st != VPT_OK) return st;
    if (count == 0) return VPT_OK;
    vpt::SparseView v = vpt::make_sparse_view(ctx->sparse_host, ctx->sparse_dev, 8);
    VPT_CHECK_CUDA(ctx, vpt::launch_sparse_query(v, ijk, count, values, dims, active, s));
    return VPT_OK;
}

VptStatus vpt_set_vpt_mode(VptContext* ctx, int mode) {
    VPT_CHECK_CTX(ctx);
    if (mode < 0 || mode > VPT_MODE_RESIDUAL_RATIO_TRACKING_UNBIASED)
        return fail(ctx, VPT_ERR_ARG, "unknown VptMode");
    if (tracker_of(mode) < 0) return fail(ctx, VPT_ERR_UNSUPPORTED, "VptMode not built in this core");
    if (mode != ctx->mode) reset_film_state(ctx);
    ctx->mode = mode;
    return VPT_OK;
}

VptStatus vpt_set_grid_interpolation(VptContext* ctx, int interpolation) {
    VPT_CHECK_CTX(ctx);
    if (interpolation < 0 || interpolation > 2) return fail(ctx, VPT_ERR_ARG, "unknown interpolation");
    if (interpolation != ctx->interp) reset_film_state(ctx);
    ctx->interp = interpolation;
    return VPT_OK;
}

VptStatus vpt_set_extinction_scale(VptContext* ctx, float scale) {
    VPT_CHECK_CTX(ctx);
    ctx->extinction_scale = scale;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_extinction_base(VptContext* ctx, const float rgb[3]) {
    VPT_CHECK_CTX(ctx);
    if (!rgb) return VPT_ERR_ARG;
    memcpy(ctx->extinction_base, rgb, sizeof(float) * 3);
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_scattering_albedo(VptContext* ctx, const float rgb[3]) {
    VPT_CHECK_CTX(ctx);
    if (!rgb) return VPT_ERR_ARG;
    memcpy(ctx->albedo, rgb, sizeof(float) * 3);
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_phase_g(VptContext* ctx, float g) {
    VPT_CHECK_CTX(ctx);
    ctx->g = g;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_seed_offset(VptContext* ctx, uint32_t offset) {
    VPT_CHECK_CTX(ctx);
    ctx->seed_offset = offset;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_use_linear_rgb(VptContext* ctx, int v) {
    VPT_CHECK_CTX(ctx);
    ctx->use_linear_rgb = v ? 1 : 0;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_max_bounces(VptContext* ctx, int max_bounces) {
    VPT_CHECK_CTX(ctx);
    if (max_bounces < 0) return fail(ctx, VPT_ERR_ARG, "max_bounces must be >= 0");
    ctx->max_bounces = max_bounces;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_builtin_environment_map(VptContext* ctx, int env_kind) {
    VPT_CHECK_CTX(ctx);
    if (env_kind < 0 || env_kind > VPT_ENV_CONSTANT_SUN) return fail(ctx, VPT_ERR_ARG, "unknown builtin environment map");
    ctx->env_kind = env_kind;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_environment_map_intensity_rgb(VptContext* ctx, const float rgb[3]) {
    VPT_CHECK_CTX(ctx);
    if (!rgb) return VPT_ERR_ARG;
    memcpy(ctx->env_intensity, rgb, sizeof(float) * 3);
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_sun(VptContext* ctx, const float direction[3], const float intensity_rgb[3]) {
    VPT_CHECK_CTX(ctx);
    if (direction) {
        float l = sqrtf(direction[0] * direction[0] + direction[1] * direction[1] + direction[2] * direction[2]);
        if (!(l > 0.0f)) return fail(ctx, VPT_ERR_ARG, "sun direction must be non-zero");
        for (int i = 0; i < 3; i++) ctx->sun_dir[i] = direction[i] / l;
    }
    if (intensity_rgb) memcpy(ctx->sun_intensity, intensity_rgb, sizeof(float) * 3);
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_sky_color(VptContext* ctx, const float rgb[3]) {
    VPT_CHECK_CTX(ctx);
    if (!rgb) return VPT_ERR_ARG;
    memcpy(ctx->sky_color, rgb, sizeof(float) * 3);
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_load_environment_map_rgba(VptContext* ctx, const float* rgba, int width, int height, int is_linear_rgb,
                                        int data_on_device) {
    VPT_CHECK_CTX(ctx);
    if (!rgba || width <= 0 || height <= 0) return fail(ctx, VPT_ERR_ARG, "bad environment image");
    cudaSetDevice(ctx->device);
    size_t n = (size_t)width * height * 4;
    VPT_CHECK_CUDA(ctx, ctx->env_rgba.alloc(n));
    VPT_CHECK_CUDA(ctx, cudaMemcpy(ctx->env_rgba.ptr, rgba, n * sizeof(float),
                                   data_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    // computeIsImageBlack (VolumetricPathTracingPass.cpp:1358-1374)
    std::vector<float> host(n);
    VPT_CHECK_CUDA(ctx, cudaMemcpy(host.data(), ctx->env_rgba.ptr, n * sizeof(float), cudaMemcpyDeviceToHost));
    bool black = true;
    for (size_t i = 0; i < (size_t)width * height && black; i++)
        if (host[i * 4] != 0.0f || host[i * 4 + 1] != 0.0f || host[i * 4 + 2] != 0.0f) black = false;
    ctx->env_image_black = black ? 1 : 0;
    ctx->env_w = width;
    ctx->env_h = height;
    ctx->env_image_linear = is_linear_rgb ? 1 : 0;
    const int levels = ctx->env_levels;  // createEnvironmentMapOctahedralTexture(12)
    ctx->env_offsets_host.assign(levels, 0);
    uint64_t off = 0;
    for (int l = 0; l < levels; l++) {
        ctx->env_offsets_host[l] = off;
        uint64_t r = (uint64_t)1 << (levels - l);
        off += r * r;
    }
    VPT_CHECK_CUDA(ctx, ctx->env_pyramid.alloc(off));
    VPT_CHECK_CUDA(ctx, ctx->env_offsets.alloc(levels));
    VPT_CHECK_CUDA(ctx, cudaMemcpy(ctx->env_offsets.ptr, ctx->env_offsets_host.data(), levels * sizeof(uint64_t),
                                   cudaMemcpyHostToDevice));
    ctx->env_kind = VPT_ENV_IMAGE;
    vpt::TraceParams P;
    fill_params(ctx, 0, 1, P);
    VPT_CHECK_CUDA(ctx, vpt::launch_env_pyramid(P, ctx->env_pyramid.ptr, ctx->env_offsets_host.data(), levels, 0));
    VPT_CHECK_CUDA(ctx, cudaDeviceSynchronize());
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_previous_view_projection(VptContext* ctx, const float view_proj[16]) {
    VPT_CHECK_CTX(ctx);
    if (view_proj) {
        for (int i = 0; i < 16; i++) ctx->trace_prev_vp[i] = view_proj[i];
    } else {
        double vp[16], inv[16];
        compute_camera(ctx, vp, inv);
        for (int i = 0; i < 16; i++) ctx->trace_prev_vp[i] = float(vp[i]);
    }
    ctx->has_trace_prev_vp = true;
    return VPT_OK;
}

VptStatus vpt_set_env_map_rotation(VptContext* ctx, const float rotation[9]) {
    VPT_CHECK_CTX(ctx);
    if (rotation) {
        for (int i = 0; i < 9; i++) {
            if (!std::isfinite(rotation[i])) return fail(ctx, VPT_ERR_ARG, "rotation must be finite");
            ctx->env_rot_m[i] = rotation[i];
        }
        ctx->env_rot_mode = 1;
    } else {
        ctx->env_rot_mode = 0;
    }
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_env_map_rotation_camera(VptContext* ctx) {
    VPT_CHECK_CTX(ctx);
    ctx->env_rot_mode = 2;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_global_world_bounding_box(VptContext* ctx, const float box_min[3], const float box_max[3]) {
    VPT_CHECK_CTX(ctx);
    if (!box_min || !box_max) {
        ctx->has_global_box = 0;
        return VPT_OK;
    }
    for (int i = 0; i < 3; i++) {
        if (!(box_max[i] > box_min[i])) return fail(ctx, VPT_ERR_ARG, "global bounding box must have max > min");
        ctx->global_box_min[i] = box_min[i];
        ctx->global_box_max[i] = box_max[i];
    }
    ctx->has_global_box = 1;
    return VPT_OK;
}

VptStatus vpt_set_camera(VptContext* ctx, const float position[3], const float target[3], const float up[3],
                         float fovy_radians, float near_dist, float far_dist) {
    VPT_CHECK_CTX(ctx);
    if (!position || !target || !up || !(fovy_radians > 0.0f) || !(near_dist > 0.0f) || !(far_dist > near_dist))
        return fail(ctx, VPT_ERR_ARG, "bad camera");
    memcpy(ctx->cam_pos, position, sizeof(float) * 3);
    memcpy(ctx->cam_target, target, sizeof(float) * 3);
    memcpy(ctx->cam_up, up, sizeof(float) * 3);
    ctx->fovy = fovy_radians;
    ctx->near_dist = near_dist;
    ctx->far_dist = far_dist;
    ctx->view_overridden = false;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_view_matrix(VptContext* ctx, const float view[16]) {
    VPT_CHECK_CTX(ctx);
    if (!view) return VPT_ERR_ARG;
    for (int i = 0; i < 16; i++) ctx->view[i] = view[i];
    ctx->view_overridden = true;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_get_camera_matrices(VptContext* ctx, float inv_view_proj[16], float view_proj[16]) {
    VPT_CHECK_CTX(ctx);
    double vp[16], inv[16];
    compute_camera(ctx, vp, inv);
    for (int i = 0; i < 16; i++) {
        if (inv_view_proj) inv_view_proj[i] = float(inv[i]);
        if (view_proj) view_proj[i] = float(vp[i]);
    }
    return VPT_OK;
}

VptStatus vpt_set_resolution(VptContext* ctx, int width, int height) {
    VPT_CHECK_CTX(ctx);
    if (width <= 0 || height <= 0 || width > 16384 || height > 16384)
        return fail(ctx, VPT_ERR_ARG, "resolution out of range");
    if (width != ctx->width || height != ctx->height) {
        ctx->width = width;
        ctx->height = height;
        reset_film_state(ctx);
        vpt::svgf_release(ctx->svgf_state);
    }
    return VPT_OK;
}

VptStatus vpt_reset_accumulation(VptContext* ctx) {
    VPT_CHECK_CTX(ctx);
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_frame_index(VptContext* ctx, uint32_t first_frame) {
    VPT_CHECK_CTX(ctx);
    ctx->frame_origin = first_frame;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_render_frames(VptContext* ctx, int frames, void* stream) {
    VPT_CHECK_CTX(ctx);
    if (frames <= 0) return fail(ctx, VPT_ERR_ARG, "frames must be > 0");
    if (!ctx->norm.ptr && !(ctx->use_sparse && ctx->sparse_valid)) return fail(ctx, VPT_ERR_STATE, "no volume loaded");
    if (ctx->width <= 0) return fail(ctx, VPT_ERR_STATE, "resolution not set");
    int tracker = tracker_of(ctx->mode);
    if (tracker < 0) return fail(ctx, VPT_ERR_UNSUPPORTED, "VptMode not built in this core");
    if (ctx->use_tf && ctx->tf.ptr && tracker != vpt::kDelta && tracker != vpt::kNextEvent &&
        tracker != vpt::kSpectralDelta && tracker != vpt::kSpectralNextEvent)
        return fail(ctx, VPT_ERR_UNSUPPORTED,
                    "the transfer function applies to delta, next event and spectral tracking (as in the reference)");
    if (ctx->use_iso && ((tracker != vpt::kDelta && tracker != vpt::kSpectralDelta && tracker != vpt::kNextEvent &&
                          tracker != vpt::kSpectralNextEvent) ||
                         ctx->use_sparse || (ctx->use_tf && ctx->tf.ptr)))
        return fail(ctx, VPT_ERR_UNSUPPORTED,
                    "isosurfaces are built for delta and next event tracking (plain and spectral) on dense grids "
                    "without a transfer function");
    if (ctx->use_iso && (tracker == vpt::kNextEvent || tracker == vpt::kSpectralNextEvent) &&
        (ctx->use_ess || (ctx->use_lights && !ctx->lights.empty()) || ctx->env_kind == VPT_ENV_IMAGE))
        return fail(ctx, VPT_ERR_UNSUPPORTED,
                    "next event tracking with isosurfaces is built for sky light samples: no lights, no environment "
                    "image, no empty-space skipping");
    if (ctx->use_clip && (tracker == vpt::kDecomposition || tracker == vpt::kResidualRatio ||
                          tracker == vpt::kResidualRatioNee || ctx->use_ess))
        return fail(ctx, VPT_ERR_UNSUPPORTED,
                    "the clip plane is built for delta, ratio and next event tracking (plain and spectral) without "
                    "empty-space skipping");
    if (ctx->env_kind == VPT_ENV_IMAGE && !ctx->env_pyramid.ptr)
        return fail(ctx, VPT_ERR_STATE, "environment image not loaded");
    cudaSetDevice(ctx->device);
    cudaStream_t s = as_stream(stream);
    VptStatus st = ensure_accel(ctx, tracker, s);
    if (st != VPT_OK) return st;
    if (ctx->use_iso && ctx->iso_type == 1 && !ctx->grad_valid) {  // VolumetricPathTracingPass.cpp:690-745
        VPT_CHECK_CUDA(ctx, ctx->grad.alloc((size_t)ctx->nx * ctx->ny * ctx->nz));
        VPT_CHECK_CUDA(ctx, vpt::launch_gradient_magnitude(ctx->raw.ptr, ctx->grad.ptr, ctx->nx, ctx->ny, ctx->nz, s));
        ctx->grad_valid = true;
    }
    // SVGF wants the last 1-spp frame (DISABLE_ACCUMULATION, VolumetricPathTracingPass.cpp:1665-1667):
    // earlier frames of the call only advance the frame counter, so only the last one is traced.
    const bool single = ctx->denoiser == VPT_DENOISER_SVGF;
    if (single) ctx->film_frames = 0;
    st = ensure_film(ctx, s);
    if (st != VPT_OK) return st;
    vpt::TraceParams P;
    fill_params(ctx, tracker, single ? 1 : frames, P);
    if (ctx->density_texture &&
        (tracker == vpt::kDelta || tracker == vpt::kRatio || tracker == vpt::kNextEvent ||
         tracker == vpt::kDecomposition || tracker == vpt::kResidualRatioNee) &&
        !ctx->use_sparse && !P.tf && !P.iso && P.border_density == 0.0f && ensure_density_texture(ctx, s)) {
        P.density_tex = ctx->dens_tex;
    }
    if (single) {
        P.frame_count = ctx->frame_count + (uint32_t)frames - 1u;
        P.global_frame = P.frame_count;
    }
    if (tracker == vpt::kDecomposition || tracker == vpt::kResidualRatio || tracker == vpt::kResidualRatioNee) {
        P.sv_size = ctx->sv_size;
        P.svx = ctx->svx;
        P.svy = ctx->svy;
        P.svz = ctx->svz;
    }
    int pb = 0;  // 0: persistent grid sized by the occupancy calculator
    if (ctx->schedule != vpt::kScheduleTiles && ctx->persistent_blocks_per_sm > 0) {
        pb = ctx->persistent_blocks_per_sm * ctx->num_sms;
    }
    // With a feature frame limit, the frames beyond it are traced without the feature pass (same
    // paths: the feature accumulation draws no random numbers).
    int feat_n = P.feat ? (single ? 1 : frames) : 0;
    if (P.feat && !single && ctx->feature_frame_limit > 0) {
        const uint32_t left = ctx->feat_frames < ctx->feature_frame_limit ? ctx->feature_frame_limit - ctx->feat_frames
                                                                           : 0u;
        feat_n = (int)std::min<uint32_t>(left, (uint32_t)frames);
    }
    const int plain_n = (single ? 1 : frames) - feat_n;
    if (feat_n > 0 && !ctx->feat_depth_deriv) {
        vpt::TraceParams Pf = P;
        Pf.num_frames = feat_n;
        Pf.num_paths = (uint64_t)ctx->width * ctx->height * (uint64_t)feat_n;
        VPT_CHECK_CUDA(ctx, vpt::launch_trace(Pf, tracker, ctx->use_ess, ctx->schedule, 1, pb, s));
    } else if (feat_n > 0) {
        // Depth (nabla) / (fwidth): the feature frames in chunks whose per-frame normals fit 256 MiB, each
        // followed by the in-order replay of its frames per pixel
        const size_t npix = (size_t)ctx->width * ctx->height;
        const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)feat_n, (256u << 20) / (npix * 16)));
        VPT_CHECK_CUDA(ctx, ctx->frame_normals.alloc(npix * 4 * (size_t)chunk));
        double view[16], iv[16];
        compute_view(ctx, view);
        mat_inverse(view, iv);
        float itv[16];  // transpose(inverse(view)), column-major
        for (int r = 0; r < 4; r++)
            for (int c = 0; c < 4; c++) itv[c * 4 + r] = float(iv[r * 4 + c]);
        const uint32_t film0 = single ? 0u : ctx->film_frames;  // accumulation frame of the call's first frame
        for (int done = 0; done < feat_n; done += chunk) {
            const int k = std::min(chunk, feat_n - done);
            vpt::TraceParams Pf = P;
            Pf.num_frames = (uint32_t)k;
            Pf.num_paths = (uint64_t)npix * (uint64_t)k;
            Pf.frame_count = P.frame_count + (uint32_t)done;
            Pf.global_frame = P.global_frame + (uint32_t)done;
            Pf.frame_normals = ctx->frame_normals.ptr;
            VPT_CHECK_CUDA(ctx, vpt::launch_trace(Pf, tracker, ctx->use_ess, ctx->schedule, 1, pb, s));
            VPT_CHECK_CUDA(ctx, vpt::launch_depth_deriv(ctx->frame_normals.ptr, k, (int)npix, film0 + (uint32_t)done,
                                                        itv, ctx->feat_depth_deriv & 1, ctx->feat.ptr, s));
        }
    }
    if (plain_n > 0) {
        vpt::TraceParams Pp = P;
        Pp.feat = nullptr;
        Pp.num_frames = plain_n;
        Pp.num_paths = (uint64_t)ctx->width * ctx->height * (uint64_t)plain_n;
        Pp.frame_count = P.frame_count + (uint32_t)feat_n;
        Pp.global_frame = P.global_frame + (uint32_t)feat_n;
        VPT_CHECK_CUDA(ctx, vpt::launch_trace(Pp, tracker, ctx->use_ess, ctx->schedule, 0, pb, s));
    }
    ctx->frame_count += (uint32_t)frames;
    ctx->film_frames += single ? 1u : (uint32_t)frames;
    ctx->feat_frames = single ? 1u : ctx->feat_frames + (uint32_t)feat_n;
    ctx->frames_total += (uint64_t)frames;
    return VPT_OK;
}

VptStatus vpt_read_result(VptContext* ctx, float* out, int channels, int out_on_device, void* stream) {
    VPT_CHECK_CTX(ctx);
    if (!out || (channels != 3 && channels != 4)) return fail(ctx, VPT_ERR_ARG, "channels must be 3 or 4");
    if (ctx->film_frames == 0 || !ctx->film.ptr) return fail(ctx, VPT_ERR_STATE, "nothing rendered yet");
    cudaSetDevice(ctx->device);
    cudaStream_t s = as_stream(stream);
    int n = ctx->width * ctx->height;
    float* dst = out;
    if (!out_on_device) {
        VPT_CHECK_CUDA(ctx, ctx->staging.alloc((size_t)n * 4));
        dst = ctx->staging.ptr;
    }
    double inv = 1.0 / double(ctx->film_frames);
    bool denoise = (ctx->denoiser == VPT_DENOISER_EAW && ctx->eaw.iterations > 0) ||
                   ctx->denoiser == VPT_DENOISER_SVGF;
    if (!denoise) {
        VPT_CHECK_CUDA(ctx, vpt::launch_film_to_chw(ctx->film.ptr, ctx->width, ctx->height, inv, channels, dst, s));
    } else {
        VPT_CHECK_CUDA(ctx, ctx->rgba_src.alloc((size_t)n * 4));
        VPT_CHECK_CUDA(ctx, ctx->rgba_a.alloc((size_t)n * 4));
        VPT_CHECK_CUDA(ctx, ctx->rgba_b.alloc((size_t)n * 4));
        VPT_CHECK_CUDA(ctx, vpt::launch_film_to_rgba(ctx->film.ptr, n, inv, ctx->rgba_src.ptr, s));
        const float* feat = ctx->feat.count ? ctx->feat.ptr : nullptr;
        float* result = nullptr;
        cudaError_t e;
        if (ctx->denoiser == VPT_DENOISER_EAW) {
            VPT_CHECK_CUDA(ctx, ctx->eaw_maps.alloc((size_t)n * 8));
            e = vpt::eaw_denoise_features(ctx->rgba_src.ptr, feat, feature_frames(ctx), ctx->width, ctx->height, ctx->eaw,
                                          ctx->eaw_maps.ptr, ctx->rgba_a.ptr, ctx->rgba_b.ptr, &result, s);
        } else {
            double vp[16], inv_vp[16];
            compute_camera(ctx, vp, inv_vp);
            double view[16], iv[16];
            compute_view(ctx, view);
            mat_inverse(view, iv);
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) ctx->svgf.inv_transposed_view[c * 4 + r] = float(iv[r * 4 + c]);
            for (int i = 0; i < 16; i++)
                ctx->svgf.prev_view_proj[i] = float(ctx->has_prev_view_proj ? ctx->prev_view_proj[i] : vp[i]);
            ctx->svgf.far_dist = ctx->far_dist;
            e = vpt::svgf_denoise_features(ctx->rgba_src.ptr, feat, feature_frames(ctx), ctx->width, ctx->height, ctx->svgf,
                                           ctx->svgf_state, ctx->rgba_b.ptr, &result, s);
            // setPreviousViewProjMatrix(current) at the end of _render (VolumetricPathTracingPass.cpp:2421)
            memcpy(ctx->prev_view_proj, vp, sizeof(vp));
            ctx->has_prev_view_proj = true;
        }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "denoise");
        VPT_CHECK_CUDA(ctx, vpt::launch_rgba_to_chw(result, n, channels, dst, s));
    }
    if (!out_on_device) {
        VPT_CHECK_CUDA(ctx, cudaMemcpyAsync(out, dst, (size_t)n * channels * sizeof(float), cudaMemcpyDeviceToHost, s));
        VPT_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    }
    return VPT_OK;
}

VptStatus vpt_render_frame(VptContext* ctx, int frames, float* out, int channels, int out_on_device, void* stream) {
    VptStatus st = vpt_render_frames(ctx, frames, stream);
    if (st != VPT_OK) return st;
    return vpt_read_result(ctx, out, channels, out_on_device, stream);
}

VptStatus vpt_set_collect_statistics(VptContext* ctx, int enabled) {
    VPT_CHECK_CTX(ctx);
    bool e = enabled != 0;
    if (e != ctx->collect_stats) reset_film_state(ctx);
    ctx->collect_stats = e;
    return VPT_OK;
}

VptStatus vpt_read_statistics(VptContext* ctx, double* out_sum, double* out_sum_sq, int out_on_device, void* stream) {
    VPT_CHECK_CTX(ctx);
    if (!ctx->film.ptr || ctx->film_frames == 0) return fail(ctx, VPT_ERR_STATE, "nothing rendered yet");
    cudaStream_t s = as_stream(stream);
    size_t n = (size_t)ctx->width * ctx->height * 3;
    cudaMemcpyKind k = out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (out_sum) VPT_CHECK_CUDA(ctx, cudaMemcpyAsync(out_sum, ctx->film.ptr, n * sizeof(double), k, s));
    if (out_sum_sq) {
        if (!ctx->collect_stats) return fail(ctx, VPT_ERR_STATE, "statistics collection is off");
        VPT_CHECK_CUDA(ctx, cudaMemcpyAsync(out_sum_sq, ctx->film_sq.ptr, n * sizeof(double), k, s));
    }
    VPT_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    return VPT_OK;
}

VptStatus vpt_set_use_feature_maps(VptContext* ctx, const int* features, int count) {
    VPT_CHECK_CTX(ctx);
    bool on = false, background = false;
    int deriv = 0;
    int depth_maps = 0;
    for (int i = 0; i < count; i++) {
        if (features && features[i] != VPT_FEATURE_RESULT) on = true;
        if (features && features[i] == VPT_FEATURE_BACKGROUND) background = true;
        if (features && features[i] == VPT_FEATURE_DEPTH_BLENDED) depth_maps |= 1;
        if (features && features[i] == VPT_FEATURE_DEPTH_NEAREST_OPAQUE) depth_maps |= 2;
        if (features && features[i] == VPT_FEATURE_DEPTH_NABLA) deriv |= 1;
        if (features && features[i] == VPT_FEATURE_DEPTH_FWIDTH) deriv |= 2;
    }
    if (on != ctx->features_on || background != ctx->feat_background || depth_maps != ctx->feat_depth_maps ||
        deriv != ctx->feat_depth_deriv)
        reset_film_state(ctx);
    ctx->features_on = on;
    ctx->feat_background = background;
    ctx->feat_depth_maps = depth_maps;
    ctx->feat_depth_deriv = deriv;
    if (!deriv) ctx->frame_normals.release();
    return VPT_OK;
}

VptStatus vpt_get_feature_map(VptContext* ctx, int feature, float* out, int channels, int out_on_device, void* stream) {
    VPT_CHECK_CTX(ctx);
    if (feature == VPT_FEATURE_RESULT) return vpt_read_result(ctx, out, channels, out_on_device, stream);
    if (!features_needed(ctx) || !ctx->feat.ptr || ctx->film_frames == 0)
        return fail(ctx, VPT_ERR_STATE, "feature maps are not enabled or nothing rendered");
    if (!out || channels < 1 || channels > 4) return fail(ctx, VPT_ERR_ARG, "bad output");
    if (feature == VPT_FEATURE_BACKGROUND && !ctx->feat_background)
        return fail(ctx, VPT_ERR_STATE, "the Background map was not requested in set_use_feature_maps");
    if ((feature == VPT_FEATURE_DEPTH_BLENDED && !(ctx->feat_depth_maps & 1)) ||
        (feature == VPT_FEATURE_DEPTH_NEAREST_OPAQUE && !(ctx->feat_depth_maps & 2)) ||
        (feature == VPT_FEATURE_DEPTH_NABLA && !(ctx->feat_depth_deriv & 1)) ||
        (feature == VPT_FEATURE_DEPTH_FWIDTH && !(ctx->feat_depth_deriv & 2)))
        return fail(ctx, VPT_ERR_STATE, "the depth map was not requested in set_use_feature_maps");
    cudaStream_t s = as_stream(stream);
    int n = ctx->width * ctx->height;
    float* dst = out;
    if (!out_on_device) {
        VPT_CHECK_CUDA(ctx, ctx->staging.alloc((size_t)n * 4));
        dst = ctx->staging.ptr;
    }
    cudaError_t e = vpt::feature_to_chw(ctx->feat.ptr, n, feature_frames(ctx), feature, channels, ctx->albedo,
                                        ctx->far_dist, dst, s);
    if (e == cudaErrorInvalidValue) return fail(ctx, VPT_ERR_ARG, "feature map not supported");
    VPT_CHECK_CUDA(ctx, e);
    if (!out_on_device) {
        VPT_CHECK_CUDA(ctx, cudaMemcpyAsync(out, dst, (size_t)n * channels * sizeof(float), cudaMemcpyDeviceToHost, s));
        VPT_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    }
    return VPT_OK;
}

VptStatus vpt_get_denoiser_features(VptContext* ctx, float* albedo, float* normal, float* depth, float* transmittance,
                                    void* stream) {
    VPT_CHECK_CTX(ctx);
    if (!features_needed(ctx) || !ctx->feat.ptr || ctx->film_frames == 0)
        return fail(ctx, VPT_ERR_STATE, "feature maps are not enabled or nothing rendered");
    if (!albedo && !normal && !depth && !transmittance) return fail(ctx, VPT_ERR_ARG, "no output");
    VPT_CHECK_CUDA(ctx, vpt::denoiser_features(ctx->feat.ptr, ctx->width * ctx->height, feature_frames(ctx),
                                               ctx->albedo, albedo, normal, depth, transmittance, as_stream(stream)));
    return VPT_OK;
}

VptStatus vpt_get_stats(VptContext* ctx, VptStats* stats) {
    VPT_CHECK_CTX(ctx);
    if (!stats) return VPT_ERR_ARG;
    unsigned long long c[4];
    int flags = 0;
    VPT_CHECK_CUDA(ctx, cudaMemcpy(c, ctx->counters.ptr, sizeof(c), cudaMemcpyDeviceToHost));
    VPT_CHECK_CUDA(ctx, cudaMemcpy(&flags, ctx->error_flags.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    stats->paths = c[0];
    stats->density_lookups = c[1];
    stats->frames = ctx->film_frames;
    stats->error_flags = flags;
    stats->reserved = 0;
    return VPT_OK;
}

VptStatus vpt_reset_stats(VptContext* ctx) {
    VPT_CHECK_CTX(ctx);
    VPT_CHECK_CUDA(ctx, cudaMemset(ctx->counters.ptr, 0, 4 * sizeof(unsigned long long)));
    VPT_CHECK_CUDA(ctx, cudaMemset(ctx->error_flags.ptr, 0, sizeof(int)));
    return VPT_OK;
}

VptStatus vpt_synchronize(VptContext* ctx, void* stream) {
    VPT_CHECK_CTX(ctx);
    VPT_CHECK_CUDA(ctx, cudaStreamSynchronize(as_stream(stream)));
    int flags = 0;
    VPT_CHECK_CUDA(ctx, cudaMemcpy(&flags, ctx->error_flags.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if (flags & vpt::kErrIterLimit) return fail(ctx, VPT_ERR_ITER_LIMIT, "a path reached the iteration guard");
    return VPT_OK;
}

VptStatus vpt_set_denoiser(VptContext* ctx, int denoiser_type) {
    VPT_CHECK_CTX(ctx);
    if (denoiser_type < VPT_DENOISER_NONE || denoiser_type > VPT_DENOISER_SVGF)
        return fail(ctx, VPT_ERR_ARG, "unknown denoiser");
    ctx->denoiser = denoiser_type;
    // setDenoiserType clears the settings (VolumetricPathTracingModuleRenderer.cpp:255-261).
    ctx->eaw = vpt::EawSettings();
    ctx->svgf = vpt::SvgfSettings();
    vpt::svgf_release(ctx->svgf_state);
    return VPT_OK;
}

VptStatus vpt_set_denoiser_property(VptContext* ctx, const char* key, const char* value) {
    VPT_CHECK_CTX(ctx);
    if (!key || !value) return VPT_ERR_ARG;
    float f;
    if (!parse_float(value, f)) return fail(ctx, VPT_ERR_ARG, std::string("not a number: ") + value);
    std::string k(key);
    if (k == "iterations" || k == "maxNumIterations") ctx->eaw.iterations = int(f);
    else if (k == "phi_color" || k == "phiColor") ctx->eaw.phi_color = f;
    else if (k == "phi_position" || k == "phiPosition") ctx->eaw.phi_position = f;
    else if (k == "phi_normal" || k == "phiNormal") ctx->eaw.phi_normal = f;
    else if (k == "ref_compute_quirk") ctx->eaw.ref_compute_quirk = int(f);
    else if (k == "lattice_tiles") ctx->eaw.lattice_tiles = int(f) ? 1 : 0;
    else if (k == "z_threshold") ctx->svgf.z_threshold = f;
    else if (k == "normal_threshold") ctx->svgf.normal_threshold = f;
    else return fail(ctx, VPT_ERR_ARG, std::string("unknown denoiser property: ") + key);
    return VPT_OK;
}

VptStatus vpt_set_use_empty_space_skipping(VptContext* ctx, int enabled) {
    VPT_CHECK_CTX(ctx);
    ctx->use_ess = enabled ? 1 : 0;
    reset_film_state(ctx);
    return VPT_OK;
}

// ---- batched rendering: many contexts in one persistent launch ----

VptStatus vpt_batch_create(VptBatch** out, VptContext* const* ctxs, int count) {
    if (!out || !ctxs || count <= 0) return VPT_ERR_ARG;
    *out = nullptr;
    for (int i = 0; i < count; i++) {
        if (!ctxs[i]) return VPT_ERR_ARG;
        if (ctxs[i]->device != ctxs[0]->device) return VPT_ERR_ARG;
    }
    VptBatch* b = new VptBatch();
    b->ctxs.assign(ctxs, ctxs + count);
    b->device = ctxs[0]->device;
    b->num_sms = ctxs[0]->num_sms;
    cudaSetDevice(b->device);
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&b->h_params), sizeof(vpt::TraceParams) * count);
    if (e == cudaSuccess)
        e = cudaMallocHost(reinterpret_cast<void**>(&b->h_offsets), sizeof(unsigned long long) * (count + 1));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_params), sizeof(vpt::TraceParams) * count);
    if (e == cudaSuccess)
        e = cudaMalloc(reinterpret_cast<void**>(&b->d_offsets), sizeof(unsigned long long) * (count + 1));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_counters), sizeof(unsigned long long) * 3);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_err), sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_counters, 0, sizeof(unsigned long long) * 3);
    if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        batch_release(b);
        delete b;
        return e == cudaErrorMemoryAllocation ? VPT_ERR_OOM : VPT_ERR_CUDA;
    }
    *out = b;
    return VPT_OK;
}

void vpt_batch_destroy(VptBatch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    batch_release(b);
    delete b;
}

const char* vpt_batch_last_error(VptBatch* b) { return b ? b->last_error.c_str() : ""; }

VptStatus vpt_batch_set_option(VptBatch* b, const char* key, double value) {
    if (!b || !key) return VPT_ERR_ARG;
    std::string k(key);
    if (k == "use_graph") {
        b->use_graph = value != 0.0;
    } else if (k == "blocks_per_sm") {
        if (value < 0 || value > 64) return batch_fail(b, VPT_ERR_ARG, "blocks_per_sm out of range");
        b->blocks_per_sm = int(value);
    } else if (k == "refill_min_lanes") {
        if (value < 0 || value > 32) return batch_fail(b, VPT_ERR_ARG, "refill_min_lanes out of range");
        b->refill_min = int(value);
    } else {
        return batch_fail(b, VPT_ERR_ARG, "unknown batch option " + k);
    }
    return VPT_OK;
}

VptStatus vpt_batch_render(VptBatch* b, const int* frames, void* stream) {
    if (!b || !frames) return VPT_ERR_ARG;
    cudaSetDevice(b->device);
    cudaStream_t s = as_stream(stream);
    vpt::BatchLaunch L;
    VptStatus st = batch_prepare(b, frames, s, L);
    if (st != VPT_OK) return st;
    cudaError_t e = cudaSuccess;
    if (b->use_graph) {
        const int key[4] = {L.tracker, L.interp, L.grid_kind, L.blocks};
        if (!b->exec || memcmp(key, b->exec_key, sizeof(key)) != 0) {
            if (b->exec) {
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
            }
            cudaGraph_t g = nullptr;
            e = cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                vpt::BatchLaunch Lc = L;
                Lc.counted = false;  // counted when the graph is launched
                cudaError_t e2 = batch_enqueue(b, Lc, b->capture_stream);
                e = cudaStreamEndCapture(b->capture_stream, &g);
                if (e == cudaSuccess) e = e2;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess)
                return batch_fail(b, VPT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            memcpy(b->exec_key, key, sizeof(key));
        }
        e = cudaGraphLaunch(b->exec, s);
        if (e == cudaSuccess) vpt::count_launches(1);
    } else {
        e = batch_enqueue(b, L, s);
    }
    if (e == cudaSuccess) e = cudaEventRecord(b->done, s);
    if (e != cudaSuccess) return batch_fail(b, VPT_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    b->launched = true;
    batch_commit(b, frames);
    return VPT_OK;
}

VptStatus vpt_batch_autotune(VptBatch* b, const int* frames, void* stream, int* out_blocks_per_sm) {
    if (!b || !frames) return VPT_ERR_ARG;
    cudaSetDevice(b->device);
    cudaStream_t s = as_stream(stream);
    const int saved = b->blocks_per_sm;
    const bool saved_graph = b->use_graph;
    b->blocks_per_sm = 0;
    b->use_graph = false;
    vpt::BatchLaunch L;
    VptStatus st = batch_prepare(b, frames, s, L);  // occupancy limit
    if (st != VPT_OK) {
        b->blocks_per_sm = saved;
        b->use_graph = saved_graph;
        return st;
    }
    const int max_per_sm = L.blocks / b->num_sms;
    const int cands[4] = {max_per_sm, (3 * max_per_sm) / 4, max_per_sm / 2, max_per_sm / 4};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best_ms = 1e30f;
    int best = max_per_sm;
    for (int c = 0; c < 5 && st == VPT_OK; c++) {
        const int per_sm = c == 0 ? max_per_sm : cands[c - 1];  // the first run warms up
        if (per_sm <= 0) continue;
        b->blocks_per_sm = per_sm;
        cudaEventRecord(e0, s);
        st = vpt_batch_render(b, frames, stream);
        cudaEventRecord(e1, s);
        if (st != VPT_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            st = batch_fail(b, VPT_ERR_CUDA, "autotune launch failed");
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (c > 0 && ms < best_ms) {
            best_ms = ms;
            best = per_sm;
        }
    }
    // then the refill threshold at that block count
    const int saved_refill = b->refill_min;
    int best_refill = saved_refill;
    best_ms = 1e30f;
    const int refills[4] = {1, 2, 4, 8};
    for (int c = 0; c < 4 && st == VPT_OK; c++) {
        b->blocks_per_sm = best;
        b->refill_min = refills[c];
        cudaEventRecord(e0, s);
        st = vpt_batch_render(b, frames, stream);
        cudaEventRecord(e1, s);
        if (st != VPT_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            st = batch_fail(b, VPT_ERR_CUDA, "autotune launch failed");
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
            best_ms = ms;
            best_refill = refills[c];
        }
    }
    b->refill_min = st == VPT_OK ? best_refill : saved_refill;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // the calibration renders went into the films: start the accumulation over
    for (VptContext* ctx : b->ctxs) reset_film_state(ctx);
    b->use_graph = saved_graph;
    b->blocks_per_sm = st == VPT_OK ? best : saved;
    if (out_blocks_per_sm) *out_blocks_per_sm = b->blocks_per_sm;
    return st;
}

VptStatus vpt_batch_get_stats(VptBatch* b, VptStats* out) {
    if (!b || !out) return VPT_ERR_ARG;
    cudaSetDevice(b->device);
    unsigned long long c[3];
    int err = 0;
    if (cudaMemcpy(c, b->d_counters, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return batch_fail(b, VPT_ERR_CUDA, "reading batch counters failed");
    memset(out, 0, sizeof(*out));
    out->paths = c[1];
    out->density_lookups = c[2];
    out->error_flags = err;
    return VPT_OK;
}

VptStatus vpt_batch_reset_stats(VptBatch* b) {
    if (!b) return VPT_ERR_ARG;
    cudaSetDevice(b->device);
    if (cudaMemset(b->d_counters, 0, sizeof(unsigned long long) * 3) != cudaSuccess ||
        cudaMemset(b->d_err, 0, sizeof(int)) != cudaSuccess)
        return batch_fail(b, VPT_ERR_CUDA, "resetting batch counters failed");
    return VPT_OK;
}

// ---- lights (LightEditorWidget, src/PathTracer/LightEditorWidget.cpp:89-103, 286-320) ----

VptStatus vpt_set_use_lights(VptContext* ctx, int use_lights) {
    VPT_CHECK_CTX(ctx);
    if ((use_lights != 0) != ctx->use_lights) reset_film_state(ctx);
    ctx->use_lights = use_lights != 0;
    return VPT_OK;
}

VptStatus vpt_clear_lights(VptContext* ctx) {
    VPT_CHECK_CTX(ctx);
    ctx->lights.clear();
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_add_light(VptContext* ctx, int* out_index) {
    VPT_CHECK_CTX(ctx);
    if ((int)ctx->lights.size() >= vpt::kMaxLights)
        return fail(ctx, VPT_ERR_UNSUPPORTED, "too many lights (at most 16)");
    ctx->lights.push_back(default_light());
    if (out_index) *out_index = (int)ctx->lights.size() - 1;
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_remove_light(VptContext* ctx, int index) {
    VPT_CHECK_CTX(ctx);
    if (index >= 0 && index < (int)ctx->lights.size()) ctx->lights.erase(ctx->lights.begin() + index);
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_get_light_count(VptContext* ctx, int* out_count) {
    VPT_CHECK_CTX(ctx);
    if (!out_count) return VPT_ERR_ARG;
    *out_count = (int)ctx->lights.size();
    return VPT_OK;
}

VptStatus vpt_set_light_property(VptContext* ctx, int index, const char* key, const char* value) {
    VPT_CHECK_CTX(ctx);
    if (!key || !value) return VPT_ERR_ARG;
    if (index < 0 || index >= (int)ctx->lights.size())
        return fail(ctx, VPT_ERR_ARG, "Error in LightEditorWidget::setLightProperty: Invalid light index.");
    vpt::LightParams& l = ctx->lights[index];
    std::string k(key), v(value);
    static const char* kTypes[] = {"Point Light", "Spotlight", "Directional Light"};
    static const char* kSpaces[] = {"World", "View", "View Orientation"};
    F3 vec;
    float f;
    if (k == "type") {
        for (int i = 0; i < 3; i++)
            if (v == kTypes[i]) l.type = i;
    } else if (k == "space") {
        for (int i = 0; i < 3; i++)
            if (v == kSpaces[i]) l.space = i;
    } else if (k == "color" || k == "position" || k == "direction" || k == "spot_direction") {
        if (!parse_vec3(value, vec)) return fail(ctx, VPT_ERR_ARG, "Error in stringToVec3: Invalid number of entries.");
        if (k == "color") l.color = vec;
        else if (k == "spot_direction") l.spot_direction = vec;
        else l.position = vec;
    } else if (k == "intensity" || k == "spot_total_width" || k == "spot_falloff_start") {
        if (!parse_float(value, f)) return fail(ctx, VPT_ERR_ARG, "invalid number for light property " + k);
        if (k == "intensity") l.intensity = f;
        else if (k == "spot_total_width") l.spot_total_width = f;
        else l.spot_falloff_start = f;
    } else if (k == "use_distance") {
        // the reference writes this flag into the intensity (LightEditorWidget.cpp:305-306); here it
        // sets the distance falloff, as the property's name says
        l.use_distance = (v == "1" || v == "true" || v == "True") ? 1 : 0;
    }
    reset_film_state(ctx);
    return VPT_OK;
}

VptStatus vpt_set_option(VptContext* ctx, const char* key, double value) {
    VPT_CHECK_CTX(ctx);
    if (!key) return VPT_ERR_ARG;
    std::string k(key);
    if (k == "sdt_collision_probability") {
        if (value != 0.0 && value != 1.0 && value != 2.0)
            return fail(ctx, VPT_ERR_ARG, "sdt_collision_probability: 0 (max), 1 (avg) or 2 (path history avg)");
        ctx->sdt_prob = (int)value;
        reset_film_state(ctx);
    } else if (k == "feature_frames") {
        if (value < 0 || value > 1e9) return fail(ctx, VPT_ERR_ARG, "feature_frames out of range");
        ctx->feature_frame_limit = (uint32_t)value;
        reset_film_state(ctx);
    } else if (k == "schedule") {
        int v = int(value);
        if (v < 0 || v > 2) return fail(ctx, VPT_ERR_ARG, "schedule must be 0 (tiles), 1 (persistent) or 2 (refill)");
        ctx->schedule = v;
    } else if (k == "refill_min_lanes") {
        if (value < 1 || value > 32) return fail(ctx, VPT_ERR_ARG, "refill_min_lanes must be in 1..32");
        ctx->refill_min = int(value);
    } else if (k == "density_texture") {
        ctx->density_texture = int(value) ? 1 : 0;
    } else if (k == "persistent_blocks_per_sm") {
        if (value < 0 || value > 64) return fail(ctx, VPT_ERR_ARG, "persistent_blocks_per_sm out of range");
        ctx->persistent_blocks_per_sm = int(value);
    } else if (k == "max_steps_per_path") {
        if (value < 1 || value > 4294967295.0) return fail(ctx, VPT_ERR_ARG, "max_steps_per_path out of range");
        ctx->max_steps = (uint32_t)value;
    } else if (k == "fbm_contrast") {
        if (!(value > 0.0)) return fail(ctx, VPT_ERR_ARG, "fbm_contrast must be > 0");
        ctx->fbm_contrast = float(value);
    } else if (k == "sparse_fp16") {
        bool v = int(value) != 0;
        if (v != ctx->sparse_fp16 && ctx->sparse_from_dense) ctx->sparse_valid = false;
        ctx->sparse_fp16 = v;
        reset_film_state(ctx);
    } else if (k == "ess_ref_compat") {
        ctx->ess_ref_compat = int(value) ? 1 : 0;
        ctx->occ_valid = false;
        reset_film_state(ctx);
    } else {
        return fail(ctx, VPT_ERR_ARG, std::string("unknown option: ") + key);
    }
    return VPT_OK;
}

VptStatus vpt_build_supervoxel_grid(const float* density, int nx, int ny, int nz, int sv, int halo, float* out_min,
                                    float* out_max, float* out_avg, uint8_t* out_occ, void* stream) {
    if (!density || !out_min || !out_max || nx <= 0 || ny <= 0 || nz <= 0 || sv <= 0) return VPT_ERR_ARG;
    int gx = (nx + sv - 1) / sv, gy = (ny + sv - 1) / sv, gz = (nz + sv - 1) / sv;
    cudaError_t e = vpt::launch_supervoxel_stats(density, nx, ny, nz, sv, gx, gy, gz, halo ? 1 : 0, out_min, out_max,
                                                 out_avg, out_occ, as_stream(stream));
    return e == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_build_rrt_params(const float* sv_min, const float* sv_max, const float* sv_avg, int count,
                               float extinction, int sv, float* out_pairs, void* stream) {
    if (!sv_min || !sv_max || !sv_avg || !out_pairs || count <= 0 || sv <= 0) return VPT_ERR_ARG;
    float D = sqrtf(3.0f) * float(sv);
    cudaError_t e = vpt::launch_rrt_params(sv_min, sv_max, sv_avg, count, extinction, D, out_pairs, as_stream(stream));
    return e == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_build_residual_ratio_grid(const float* sv_min, const float* sv_max, const float* sv_avg, int count,
                                        float extinction, int sv, float* out4, void* stream) {
    if (!sv_min || !sv_max || !sv_avg || !out4 || count <= 0 || sv <= 0) return VPT_ERR_ARG;
    float D = sqrtf(3.0f) * float(sv);
    cudaError_t e = vpt::launch_rrt_local(sv_min, sv_max, sv_avg, count, extinction, D, out4, as_stream(stream));
    return e == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_build_occupancy_grid(const float* density, int nx, int ny, int nz, int block, int halo, float threshold,
                                   uint8_t* out, void* stream) {
    if (!density || !out || nx <= 0 || ny <= 0 || nz <= 0 || block <= 0 || halo < 0) return VPT_ERR_ARG;
    int gx = (nx + block - 1) / block, gy = (ny + block - 1) / block, gz = (nz + block - 1) / block;
    cudaError_t e =
        vpt::launch_occupancy(density, nx, ny, nz, block, gx, gy, gz, halo, threshold, 0, out, as_stream(stream));
    return e == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_build_environment_pyramid(const float* rgba, int width, int height, int levels, float* out_pyramid,
                                        void* stream) {
    if (!rgba || !out_pyramid || width <= 0 || height <= 0 || levels <= 0 || levels > 14) return VPT_ERR_ARG;
    std::vector<uint64_t> off(levels);
    uint64_t o = 0;
    for (int l = 0; l < levels; l++) {
        off[l] = o;
        uint64_t r = (uint64_t)1 << (levels - l);
        o += r * r;
    }
    vpt::TraceParams P;
    memset(&P, 0, sizeof(P));
    P.env_rgba = rgba;
    P.env_w = width;
    P.env_h = height;
    cudaError_t e = vpt::launch_env_pyramid(P, out_pyramid, off.data(), levels, as_stream(stream));
    return e == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_eaw_denoise_rgba(const float* color, const float* position, const float* normal, int width, int height,
                               int iterations, float phi_color, float phi_position, float phi_normal,
                               int ref_compute_quirk, float* out, void* stream) {
    if (!color || !out || width <= 0 || height <= 0 || iterations < 0) return VPT_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    size_t bytes = (size_t)width * height * 4 * sizeof(float);
    if (vpt::image_ranges_overlap(out, color, bytes) || vpt::image_ranges_overlap(out, position, bytes) ||
        vpt::image_ranges_overlap(out, normal, bytes))
        return VPT_ERR_ARG;
    if (iterations == 0) {
        return cudaMemcpyAsync(out, color, bytes, cudaMemcpyDeviceToDevice, s) == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
    }
    float* scratch = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void**>(&scratch), bytes, s) != cudaSuccess) return VPT_ERR_OOM;
    vpt::EawSettings st;
    st.iterations = iterations;
    st.phi_color = phi_color;
    st.phi_position = phi_position;
    st.phi_normal = phi_normal;
    st.ref_compute_quirk = ref_compute_quirk;
    // Ping-pong between `out` and the scratch image so that the last iteration lands in `out`.
    float* ping = (iterations % 2 == 1) ? out : scratch;
    float* pong = (iterations % 2 == 1) ? scratch : out;
    float* result = nullptr;
    cudaError_t e = vpt::eaw_denoise(color, position, normal, width, height, st, ping, pong, &result, s);
    cudaFreeAsync(scratch, s);
    return e == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

}  // extern "C"
