// ref_driver.cpp - runs the reference's tracer shader (Clouds.glsl compiled as C++) on the CPU
// (TEST INFRASTRUCTURE ONLY).  Compiled once per define set (REF_VARIANT_BODY: one namespace per
// variant holding the shader) and once as the common part (REF_DRIVER_COMMON: shared state and the
// C entry points).  Per frame the driver sets FrameInfo and invokes the shader's main() for every
// pixel, exactly like one compute dispatch; accImage keeps the reference's fp32 running mean.
#include <stdint.h>
#include <string.h>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "ref_driver_api.h"

#ifdef REF_VARIANT_BODY
namespace glslref {
namespace REF_VARIANT_NS {
static Parameters& parameters = g_ref.params;
static FrameInfo& frameInfo = g_ref.frame;
static sampler3D& gridImage = g_ref.grid;
static sampler3D& gradientImage = g_ref.gradient;
static sampler3D& emissionImage = g_ref.emission;
static sampler1DArray& transferFunctionTexture = g_ref.tf;
static sampler3D& superVoxelGridImage = g_ref.sv;
static usampler3D& superVoxelGridOccupancyImage = g_ref.svocc;
static sampler2D& environmentMapTexture = g_ref.env;
static sampler2D& environmentMapOctahedralTexture = g_ref.envocta;
static uimage3D& occupancyGridImage = g_ref.occ;
static image2D& resultImage = g_ref.result;
static image2D& accImage = g_ref.acc;
static image2D& depthBlendedImage = g_ref.dblend;
static image2D& depthNearestOpaqueImage = g_ref.dnear;
static image2D& firstW = g_ref.firstw;
static image2D& flowImage = g_ref.flow;
static image2D& flowReverseImage = g_ref.flowrev;
static image2D& reprojUVImage = g_ref.reproj;
static image2D& normalImage = g_ref.normal;
static image2D& depthNablaImage = g_ref.dnabla;
static image2D& depthFwidthImage = g_ref.dfwidth;
static Light* const lights = g_ref.lights;
#define gl_GlobalInvocationID gl_global_invocation_id
#define main glsl_main
#include "Clouds.glsl.inc"
#undef main
void run_pixel(int x, int y) {
    gl_global_invocation_id = uvec3((uint)x, (uint)y, 0u);
    glsl_main();
}
}  // namespace REF_VARIANT_NS
}  // namespace glslref
#endif

#ifdef REF_DRIVER_COMMON
namespace glslref {
RefState g_ref;
thread_local uvec3 gl_global_invocation_id;
uint ref_seed_offset = 0;
static std::vector<float> g_dblend, g_dnear;  // the depth feature images of the last ref_render
static std::vector<float> g_last[7];  // firstW, flow, flow reverse, reprojected uv, normal, depth nabla, fwidth
}  // namespace glslref

using namespace glslref;

extern "C" {

typedef struct RefScene {
    float inv_view_proj[16];
    int width, height;
    uint32_t frame_start, num_frames, seed_offset;
    float box_min[3], box_max[3];
    const float* grid;
    int nx, ny, nz;
    int linear_filter;
    float voxel_value_min, voxel_value_max;
    float extinction[3], albedo[3], g;
    float sun_dir[3], sun_intensity[3], env_intensity[3];
    const float* sv_data;
    int svx, svy, svz, sv_size;
    const uint8_t* occupancy;
    int ox, oy, oz, occ_block;
    const float* env_rgba;
    int env_w, env_h;
    const float* env_pyramid;
    int env_levels;
    int is_env_black;
    float far_dist;
    float inv_view[16];       /* parameters.inverseViewMatrix, column-major */
    float lights[16 * 16];    /* 16 floats per light (see oracle/vpt_oracle.h) */
    const float* emission;    /* emissionImage values [nz][ny][nx] (USE_EMISSION variants) */
    int enx, eny, enz;
    float emission_box_min[3], emission_box_max[3], emission_cap, emission_strength;
    const float* tf;          /* transferFunctionTexture: tf_size RGBA entries (USE_TRANSFER_FUNCTION variants) */
    int tf_size;
    float iso_value;          /* parameters.isoValue (USE_ISOSURFACES variants) */
    float iso_color[3];       /* parameters.isoSurfaceColor */
    float env_rot[9];         /* parameters.envMapDirRot, column-major (USE_ENV_MAP_ROTATION variants) */
    float prev_view_proj[16]; /* parameters.previousViewProjMatrix, column-major */
    float tf_albedo_strength; /* parameters.tfScatteringAlbedoStrength */
    float brdf[10];           /* parameters.subsurface, metallic, specular, specularTint, roughness,
                                 anisotropic, sheen, sheenTint, clearcoat, clearcoatGloss */
    const float* gradient;    /* gradientImage values [nz][ny][nx] (ISOSURFACE_TYPE_GRADIENT variants) */
    int use_clip;             /* parameters.useClipPlane (USE_CLIP_PLANE variants) */
    float clip[4];            /* parameters.clipPlaneNormal (normalised), clipPlaneDistance */
} RefScene;

int ref_variant_count(void) { return ref_num_variants; }
const char* ref_variant_name(int i) { return (i >= 0 && i < ref_num_variants) ? ref_variants[i].name : ""; }
int ref_find_variant(const char* name) {
    for (int i = 0; i < ref_num_variants; i++)
        if (strcmp(ref_variants[i].name, name) == 0) return i;
    return -1;
}

// Renders num_frames frames from a cleared accumulation image; out_rgba gets accImage (W*H*4).
int ref_render(int variant, const RefScene* s, float* out_rgba, int threads) {
    if (variant < 0 || variant >= ref_num_variants || !s || !out_rgba) return 1;
    Parameters& p = g_ref.params;
    memset(&p, 0, sizeof(p));
    for (int c = 0; c < 4; c++)
        p.inverseViewProjMatrix.c[c] = vec4(s->inv_view_proj[c * 4 + 0], s->inv_view_proj[c * 4 + 1],
                                            s->inv_view_proj[c * 4 + 2], s->inv_view_proj[c * 4 + 3]);
    p.boxMin = vec3(s->box_min[0], s->box_min[1], s->box_min[2]);
    p.boxMax = vec3(s->box_max[0], s->box_max[1], s->box_max[2]);
    p.voxelValueMin = s->voxel_value_min;
    p.voxelValueMax = s->voxel_value_max;
    p.gridMin = vec3(0.0f);
    p.gridMax = vec3(1.0f);
    p.extinction = vec3(s->extinction[0], s->extinction[1], s->extinction[2]);
    p.scatteringAlbedo = vec3(s->albedo[0], s->albedo[1], s->albedo[2]);
    p.phaseG = s->g;
    p.sunDirection = vec3(s->sun_dir[0], s->sun_dir[1], s->sun_dir[2]);
    p.sunIntensity = vec3(s->sun_intensity[0], s->sun_intensity[1], s->sun_intensity[2]);
    p.environmentMapIntensityFactor = vec3(s->env_intensity[0], s->env_intensity[1], s->env_intensity[2]);
    p.numFeatureMapSamplesPerFrame = 1;
    p.useLinearRGB = 1;
    if (s->occupancy) {
        p.superVoxelSize = ivec3(s->occ_block);
        p.superVoxelGridSize = ivec3(s->ox, s->oy, s->oz);
    } else {
        p.superVoxelSize = ivec3(s->sv_size);
        p.superVoxelGridSize = ivec3(s->svx, s->svy, s->svz);
    }
    p.gridResolution = ivec3(s->nx, s->ny, s->nz);
    p.isEnvMapBlack = (uint)s->is_env_black;
    p.voxelTexelSize = vec3(1.0f / float(s->nx - 1), 1.0f / float(s->ny - 1), 1.0f / float(s->nz - 1));
    p.farDistance = s->far_dist;
    for (int c = 0; c < 4; c++)
        p.inverseViewMatrix.c[c] = vec4(s->inv_view[c * 4 + 0], s->inv_view[c * 4 + 1], s->inv_view[c * 4 + 2],
                                        s->inv_view[c * 4 + 3]);
    // inverseTransposedViewMatrix = transpose(inverse(view)) (VolumetricPathTracingPass.cpp)
    for (int c = 0; c < 4; c++)
        p.inverseTransposedViewMatrix.c[c] = vec4(s->inv_view[0 * 4 + c], s->inv_view[1 * 4 + c],
                                                  s->inv_view[2 * 4 + c], s->inv_view[3 * 4 + c]);
    // envMapDirRot and its transpose invEnvMapDirRot (VolumetricPathTracingPass.cpp:2108-2113)
    for (int c = 0; c < 3; c++) {
        p.envMapDirRot.c[c] = vec3(s->env_rot[c * 3 + 0], s->env_rot[c * 3 + 1], s->env_rot[c * 3 + 2]);
        p.invEnvMapDirRot.c[c] = vec3(s->env_rot[0 * 3 + c], s->env_rot[1 * 3 + c], s->env_rot[2 * 3 + c]);
    }
    for (int i = 0; i < 16; i++) {
        const float* L = s->lights + 16 * i;
        Light& l = g_ref.lights[i];
        l.lightType = (uint)L[0];
        l.lightSpace = (uint)L[1];
        l.spotTotalWidth = L[2];
        l.spotFalloffStart = L[3];
        l.color = vec3(L[4], L[5], L[6]);
        l.intensity = L[7];
        l.position = vec3(L[8], L[9], L[10]);
        l.useDistance = (uint)L[11];
        l.spotDirection = vec3(L[12], L[13], L[14]);
        l.padding = 0.0f;
    }

    p.emissionBoxMin = vec3(s->emission_box_min[0], s->emission_box_min[1], s->emission_box_min[2]);
    p.emissionBoxMax = vec3(s->emission_box_max[0], s->emission_box_max[1], s->emission_box_max[2]);
    p.emissionCap = s->emission_cap;
    p.emissionStrength = s->emission_strength;
    p.tfScatteringAlbedoStrength = s->tf_albedo_strength;
    p.useClipPlane = s->use_clip;
    p.clipPlaneNormal = vec3(s->clip[0], s->clip[1], s->clip[2]);
    p.clipPlaneDistance = s->clip[3];
    p.subsurface = s->brdf[0];
    p.metallic = s->brdf[1];
    p.specular = s->brdf[2];
    p.specularTint = s->brdf[3];
    p.roughness = s->brdf[4];
    p.anisotropic = s->brdf[5];
    p.sheen = s->brdf[6];
    p.sheenTint = s->brdf[7];
    p.clearcoat = s->brdf[8];
    p.clearcoatGloss = s->brdf[9];
    p.isoValue = s->iso_value;
    p.isoSurfaceColor = vec3(s->iso_color[0], s->iso_color[1], s->iso_color[2]);
    g_ref.tf.data = s->tf;
    g_ref.tf.w = s->tf_size;
    g_ref.tf.layers = 1;
    g_ref.emission.data = s->emission;
    g_ref.emission.w = s->enx;
    g_ref.emission.h = s->eny;
    g_ref.emission.d = s->enz;
    g_ref.emission.channels = 1;
    g_ref.emission.filter = s->linear_filter ? FILTER_LINEAR : FILTER_NEAREST;
    g_ref.grid.data = s->grid;
    g_ref.grid.w = s->nx;
    g_ref.grid.h = s->ny;
    g_ref.grid.d = s->nz;
    g_ref.grid.channels = 1;
    g_ref.grid.filter = s->linear_filter ? FILTER_LINEAR : FILTER_NEAREST;
    g_ref.gradient = g_ref.grid;
    g_ref.gradient.data = s->gradient;
    g_ref.sv.data = s->sv_data;
    g_ref.sv.w = s->svx;
    g_ref.sv.h = s->svy;
    g_ref.sv.d = s->svz;
    g_ref.sv.channels = 2;
    g_ref.sv.filter = FILTER_NEAREST;
    g_ref.occ.data = s->occupancy;
    g_ref.occ.w = s->ox;
    g_ref.occ.h = s->oy;
    g_ref.occ.d = s->oz;
    g_ref.env.levels.clear();
    g_ref.envocta.levels.clear();
    if (s->env_rgba) {
        g_ref.env.levels.push_back(s->env_rgba);
        g_ref.env.w = s->env_w;
        g_ref.env.h = s->env_h;
        g_ref.env.channels = 4;
        g_ref.env.filter = FILTER_LINEAR;
        g_ref.env.address = ADDRESS_REPEAT;
        size_t off = 0;
        for (int l = 0; l < s->env_levels; l++) {
            g_ref.envocta.levels.push_back(s->env_pyramid + off);
            size_t r = (size_t)1 << (s->env_levels - l);
            off += r * r;
        }
        g_ref.envocta.w = g_ref.envocta.h = 1 << s->env_levels;
        g_ref.envocta.channels = 1;
        g_ref.envocta.address = ADDRESS_CLAMP_TO_EDGE;
    }
    std::vector<float> result((size_t)s->width * s->height * 4, 0.0f), acc((size_t)s->width * s->height * 4, 0.0f);
    g_ref.result.data = result.data();
    g_ref.result.w = s->width;
    g_ref.result.h = s->height;
    g_ref.acc.data = acc.data();
    g_ref.acc.w = s->width;
    g_ref.acc.h = s->height;
    g_dblend.assign((size_t)s->width * s->height * 4, 0.0f);
    g_dnear.assign((size_t)s->width * s->height * 4, 0.0f);
    g_ref.dblend.data = g_dblend.data();
    g_ref.dblend.w = s->width;
    g_ref.dblend.h = s->height;
    g_ref.dnear.data = g_dnear.data();
    g_ref.dnear.w = s->width;
    g_ref.dnear.h = s->height;
    image2D* last[7] = {&g_ref.firstw, &g_ref.flow, &g_ref.flowrev, &g_ref.reproj,
                        &g_ref.normal, &g_ref.dnabla, &g_ref.dfwidth};
    for (int k = 0; k < 7; k++) {
        g_last[k].assign((size_t)s->width * s->height * 4, 0.0f);
        last[k]->data = g_last[k].data();
        last[k]->w = s->width;
        last[k]->h = s->height;
    }
    for (int c = 0; c < 4; c++)
        p.previousViewProjMatrix.c[c] = vec4(s->prev_view_proj[c * 4 + 0], s->prev_view_proj[c * 4 + 1],
                                             s->prev_view_proj[c * 4 + 2], s->prev_view_proj[c * 4 + 3]);
    ref_seed_offset = s->seed_offset;
    int nt = threads;
#ifdef _OPENMP
    if (nt <= 0) nt = omp_get_max_threads();
#else
    nt = 1;
#endif
    void (*run)(int, int) = ref_variants[variant].run_pixel;
    for (uint32_t f = 0; f < s->num_frames; f++) {
        g_ref.frame.frameCount = s->frame_start + f;
        g_ref.frame.globalFrameNumber = s->frame_start + f;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
        for (int y = 0; y < s->height; y++)
            for (int x = 0; x < s->width; x++) run(x, y);
    }
    memcpy(out_rgba, acc.data(), acc.size() * sizeof(float));
    return 0;
}

// The images of the last ref_render (which: 0 firstW, 1 flowImage, 2 flowReverseImage, 3
// reprojUVImage, 4 normalImage, 5 depthNablaImage, 6 depthFwidthImage; W*H*4), for the variants with
// WRITE_FIRST_W_MAP, WRITE_FLOW_MAP, WRITE_FLOW_REVERSE_MAP, WRITE_REPROJ_UV_MAP, WRITE_NORMAL_MAP,
// WRITE_DEPTH_NABLA_MAP and WRITE_DEPTH_FWIDTH_MAP.
int ref_read_last_frame_feature(int which, float* out_rgba) {
    if (!out_rgba || which < 0 || which > 6 || g_last[which].empty()) return 1;
    memcpy(out_rgba, g_last[which].data(), g_last[which].size() * sizeof(float));
    return 0;
}

// The depth feature images of the last ref_render (which: 0 = depthBlendedImage, 1 =
// depthNearestOpaqueImage; W*H*4, the reference's running means), for WRITE_DEPTH_*_MAP variants.
int ref_read_depth_feature(int which, float* out_rgba) {
    const std::vector<float>& v = which == 0 ? g_dblend : g_dnear;
    if (!out_rgba || (which != 0 && which != 1) || v.empty()) return 1;
    memcpy(out_rgba, v.data(), v.size() * sizeof(float));
    return 0;
}

}  // extern "C"
#endif
