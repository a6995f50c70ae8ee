// ref_image_driver.cpp - the reference's image compute shaders run on the CPU (TEST INFRASTRUCTURE
// ONLY): Data/Shaders/VPT/OctahedralMapper.glsl (environment importance map), the compute path of
// Data/Shaders/Denoiser/EAWDenoise.glsl and the three compute stages of SVGF.glsl, rewritten mechanically by oracle/ref_build.py (uniform blocks
// become namespace globals that this driver sets, images and samplers likewise) and compiled on top of
// ref_shim.h.  Work groups run one after another; EAW's shared-memory tile is filled by running the
// group's invocations once before the pass that produces the output (every invocation writes only its
// own entry, before the barrier).
#include <stdint.h>
#include <string.h>

#include <vector>

#include "ref_shim.h"

namespace glslref {
thread_local uvec3 img_global_id, img_local_id;
inline void barrier() {}
inline void memoryBarrierShared() {}
inline ivec2 textureSize(const sampler2D& s, int) { return ivec2(s.w, s.h); }
}  // namespace glslref

#define gl_GlobalInvocationID img_global_id
#define gl_LocalInvocationID img_local_id

namespace glslref {
namespace octa {
#define main glsl_main
#include "OctahedralMapper.compute.inc"
#undef main
}  // namespace octa

namespace eaw {
#define BLOCK_SIZE 16
#define USE_POSITION_TEXTURE
#define USE_NORMAL_TEXTURE
#define main glsl_main
#include "EAWDenoise.compute.inc"
#undef main
#undef USE_POSITION_TEXTURE
#undef USE_NORMAL_TEXTURE
#undef BLOCK_SIZE
}  // namespace eaw

// SVGF (Data/Shaders/Denoiser/SVGF/SVGF.glsl): one namespace per compute stage
namespace svgf_rp {
#define main glsl_main
#include "SVGF.reproject.inc"
#undef main
}  // namespace svgf_rp

// The moments filter reads its neighbours from temp_accum_texture and writes the same image
// (SVGF.glsl:286-347), so on a GPU the result depends on the order of the invocations.  Here loads
// see the image as it was before the pass (this project's reading of the shader) and stores go to
// the output: the stage's image type is replaced by one with separate load and store buffers.
struct image2D_split {
    const float* load = nullptr;
    float* store = nullptr;
    int w = 0, h = 0;
};
inline vec4 imageLoad(const image2D_split& im, const ivec2& p) {
    const float* q = im.load + ((size_t)p.y * im.w + p.x) * 4;
    return vec4(q[0], q[1], q[2], q[3]);
}
inline void imageStore(image2D_split& im, const ivec2& p, const vec4& v) {
    float* q = im.store + ((size_t)p.y * im.w + p.x) * 4;
    q[0] = v.x;
    q[1] = v.y;
    q[2] = v.z;
    q[3] = v.w;
}
namespace svgf_fm {
#define image2D image2D_split
#define main glsl_main
#include "SVGF.filter_moments.inc"
#undef main
#undef image2D
}  // namespace svgf_fm

namespace svgf_at {
#define main glsl_main
#include "SVGF.atrous.inc"
#undef main
}  // namespace svgf_at
}  // namespace glslref

using namespace glslref;

namespace {
sampler2D rgba_sampler(const float* rgba, int w, int h, int address) {
    sampler2D s;
    s.levels = {rgba};
    s.w = w;
    s.h = h;
    s.channels = 4;
    s.filter = FILTER_LINEAR;
    s.address = address;
    return s;
}
}  // namespace

extern "C" {

// OctahedralMapper.glsl: res x res max-brightness map of an equirectangular RGBA image (the
// environment texture is sampled with linear filtering and repeat addressing, as the tracer's).
int ref_octahedral_map(const float* env_rgba, int w, int h, int res, float* out) {
    octa::environmentMapTexture = rgba_sampler(env_rgba, w, h, ADDRESS_REPEAT);
    std::vector<float> img((size_t)res * res * 4, 0.0f);
    octa::outputImage.data = img.data();
    octa::outputImage.w = res;
    octa::outputImage.h = res;
    for (int y = 0; y < res; y++)
        for (int x = 0; x < res; x++) {
            img_global_id = uvec3((uint)x, (uint)y, 0u);
            octa::glsl_main();
        }
    for (size_t i = 0; i < (size_t)res * res; i++) out[i] = img[i * 4];
    return 0;
}

// EAWBlitPass::_renderCompute (EAWDenoiser.cpp:345-391): `iterations` passes with step widths 1, 2,
// 4, ... ping-ponging between two images; colour, position and normal RGBA images sampled with linear
// filtering and clamp to edge (the pass's default sampler).  Writes the last pass's image.
int ref_eaw_compute(const float* color, const float* position, const float* normal, int w, int h, int iterations,
                    float phi_color, float phi_position, float phi_normal, float* out) {
    const size_t n = (size_t)w * h * 4;
    std::vector<float> ping(color, color + n), pong(n, 0.0f);
    eaw::phiColor = phi_color;
    eaw::phiPosition = phi_position;
    eaw::phiNormal = phi_normal;
    eaw::useColor = 1;
    eaw::usePosition = 1;
    eaw::useNormal = 1;
    eaw::positionTexture = rgba_sampler(position, w, h, ADDRESS_CLAMP_TO_EDGE);
    eaw::normalTexture = rgba_sampler(normal, w, h, ADDRESS_CLAMP_TO_EDGE);
    const int B = 16, gx = (w + B - 1) / B, gy = (h + B - 1) / B;
    for (int it = 0; it < iterations; it++) {
        eaw::stepWidth = 1 << it;
        eaw::colorTexture = rgba_sampler(ping.data(), w, h, ADDRESS_CLAMP_TO_EDGE);
        eaw::outputImage.data = pong.data();
        eaw::outputImage.w = w;
        eaw::outputImage.h = h;
        for (int by = 0; by < gy; by++)
            for (int bx = 0; bx < gx; bx++)
                for (int pass = 0; pass < 2; pass++)  // pass 0 fills the group's shared tile
                    for (int ly = 0; ly < B; ly++)
                        for (int lx = 0; lx < B; lx++) {
                            img_local_id = uvec3((uint)lx, (uint)ly, 0u);
                            img_global_id = uvec3((uint)(bx * B + lx), (uint)(by * B + ly), 0u);
                            eaw::glsl_main();
                        }
        std::swap(ping, pong);
    }
    memcpy(out, ping.data(), n * sizeof(float));
    return 0;
}

// One SVGF frame (SVGFDenoiser::denoise, SVGF.cpp:118-180, 340-500): reprojection, moments filter,
// `iterations` a-trous passes (the first writes the colour history; with none, the reprojected image
// is blitted to the output and the colour history), then the frame's normal, depth and moments become
// the history.  Maps as in the core's vpt_svgf_filter: RGBA colour / normal, one-channel depth and
// depth fwidth, two-channel motion; textures are read with texelFetch clamped to the image.
int ref_svgf_frame(const float* noisy, const float* normal, const float* depth, const float* fwidth,
                   const float* motion, float* color_hist, float* moments_hist, float* normal_hist, float* depth_hist,
                   int w, int h, float z_threshold, float normal_threshold, int iterations, float* out) {
    const size_t n = (size_t)w * h;
    auto tex = [&](const float* data, int channels) {
        sampler2D s;
        s.levels = {data};
        s.w = w;
        s.h = h;
        s.channels = channels;
        s.filter = FILTER_NEAREST;
        s.address = ADDRESS_CLAMP_TO_EDGE;
        return s;
    };
    std::vector<float> accum(n * 4, 0.0f), temp(n * 4, 0.0f), filt(n * 4, 0.0f), ping(n * 4, 0.0f), pong(n * 4, 0.0f);
    std::vector<float> hist_color(color_hist, color_hist + n * 4), hist_moments(moments_hist, moments_hist + n * 4);
    std::vector<float> hist_normal(normal_hist, normal_hist + n * 4), hist_depth(depth_hist, depth_hist + n);
    auto run = [&](void (*fn)()) {
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                img_global_id = uvec3((uint)x, (uint)y, 0u);
                fn();
            }
    };
    // reprojection
    svgf_rp::noisy_texture = tex(noisy, 4);
    svgf_rp::color_history = tex(hist_color.data(), 4);
    svgf_rp::motion_texture = tex(motion, 2);
    svgf_rp::normal_texture = tex(normal, 4);
    svgf_rp::depth_texture = tex(depth, 1);
    svgf_rp::normal_history_texture = tex(hist_normal.data(), 4);
    svgf_rp::depth_history_texture = tex(hist_depth.data(), 1);
    svgf_rp::moments_history_texture = tex(hist_moments.data(), 4);
    svgf_rp::depth_fwidth_texture = tex(fwidth, 1);
    svgf_rp::accum_moments_texture = image2D{accum.data(), w, h};
    svgf_rp::temp_accum_texture = image2D{temp.data(), w, h};
    svgf_rp::allowed_z_dist = z_threshold;
    svgf_rp::allowed_normal_dist = normal_threshold;
    run(svgf_rp::glsl_main);
    // moments filter: loads from the reprojected image, stores into a copy of it
    filt = temp;
    svgf_fm::accum_moments_texture = tex(accum.data(), 4);
    svgf_fm::normal_texture = tex(normal, 4);
    svgf_fm::depth_texture = tex(depth, 1);
    svgf_fm::depth_fwidth_texture = tex(fwidth, 1);
    svgf_fm::temp_accum_texture = image2D_split{temp.data(), filt.data(), w, h};
    run(svgf_fm::glsl_main);
    // a-trous
    const float* src = filt.data();
    if (iterations < 1) {
        memcpy(out, filt.data(), n * 16);
        memcpy(color_hist, filt.data(), n * 16);
    } else {
        svgf_at::normal_texture = tex(normal, 4);
        svgf_at::depth_texture = tex(depth, 1);
        svgf_at::depth_fwidth_texture = tex(fwidth, 1);
        svgf_at::color_history_texture = image2D{color_hist, w, h};
        for (int it = 0; it < iterations; it++) {
            float* dst = (it & 1) ? pong.data() : ping.data();
            svgf_at::iteration = it;
            svgf_at::color_texture = tex(src, 4);
            svgf_at::outputImage = image2D{dst, w, h};
            run(svgf_at::glsl_main);
            src = dst;
        }
        memcpy(out, src, n * 16);
    }
    // history of this frame
    memcpy(moments_hist, accum.data(), n * 16);
    memcpy(normal_hist, normal, n * 16);
    memcpy(depth_hist, depth, n * 4);
    return 0;
}

}  // extern "C"
