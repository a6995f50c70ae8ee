// vpt_denoise.h - image-space denoisers applied to the accumulated film (EAW, SVGF) and the
// feature-map readout they share.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vpt {

// EAWBlitPass settings (src/Denoiser/EAWDenoiser.hpp:104-119).  `iterations` defaults to 0 like
// the reference (the denoiser is then a pass-through).
struct EawSettings {
    int iterations = 0;
    float phi_color = 5.0f;
    float phi_position = 0.1f;
    float phi_normal = 0.1f;
    int use_color = 1;
    int use_position = 1;
    int use_normal = 1;
    int ref_compute_quirk = 0;  // EAWDenoise.glsl:269 uses exp(-1/phiColor) instead of exp(-dist/phiColor)
    int lattice_tiles = 1;      // taps staged in shared memory per residue-class lattice (eaw_lattice_kernel)
};

// SVGF settings (src/Denoiser/SVGF.hpp:111-112, 159).
struct SvgfSettings {
    float z_threshold = 0.002f;
    float normal_threshold = 0.02f;
    int atrous_iterations = 5;
    // filled by the context for each frame
    float inv_transposed_view[16] = {0};  // column-major
    float prev_view_proj[16] = {0};       // column-major
    float far_dist = 80.0f;
};

// History buffers of the temporal filter (previous_frame textures of SVGF_Texture_Pack).
struct SvgfState {
    int width = 0, height = 0;
    bool valid = false;
    float* color_history = nullptr;    // rgba
    float* moments_history = nullptr;  // (m1, m2, history length, 0)
    float* normal_history = nullptr;   // rgba
    float* depth_history = nullptr;    // 1 float
    float* cur = nullptr;              // scratch for current-frame maps (see vpt_denoise.cu)
};

void svgf_release(SvgfState& s);

// True when the byte ranges [a, a + bytes) and [b, b + bytes) overlap (b may be nullptr).  The EAW
// entry points reject an output image that overlaps one of their inputs: an odd iteration count
// writes the first pass into the output while the same launch still reads the inputs.
inline bool image_ranges_overlap(const void* a, const void* b, size_t bytes) {
    if (!a || !b) return false;
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x < y + bytes && y < x + bytes;
}

// One EAW pass chain on an RGBA image.  position/normal are RGBA images or nullptr (weights off).
cudaError_t eaw_denoise(const float* color_rgba, const float* position_rgba, const float* normal_rgba, int width,
                        int height, const EawSettings& s, float* ping, float* pong, float** result,
                        cudaStream_t stream);

// EAW on the film mean, with position/normal taken from the feature accumulators when present.
// `maps` holds 8 floats per pixel (position and normal RGBA); color_rgba must not alias ping/pong.
cudaError_t eaw_denoise_features(const float* color_rgba, const float* feat, uint32_t frames, int width, int height,
                                 const EawSettings& s, float* maps, float* ping, float* pong, float** result,
                                 cudaStream_t stream);

// SVGF on a 1-spp frame whose features are in `feat` (one frame accumulated).
cudaError_t svgf_denoise_features(const float* color_rgba, const float* feat, uint32_t frames, int width, int height,
                                  const SvgfSettings& s, SvgfState& state, float* out_rgba, float** result,
                                  cudaStream_t stream);

// Feature accumulators -> channels x H x W mean (VPT_FEATURE_* numbering).
// albedo / normal [3][n], depth / transmittance [n] planes of the feature accumulation (NULL = skip)
cudaError_t denoiser_features(const float* feat, int n, uint32_t frames, const float* albedo_rgb, float* albedo,
                              float* normal, float* depth, float* trans, cudaStream_t stream);
// Depth (nabla) / Depth (fwidth): advances each pixel's running-mean normal, nabla and fwidth over the
// `frames` frames of one feature launch (per-frame normals from the trace, frame-major float4), the
// first of which is accumulation frame f0; inv_transposed_view is column-major 4 x 4; nabla_map: the
// Depth (nabla) map is requested (the fwidth map then follows the running-mean nabla, as in the shader).
cudaError_t launch_depth_deriv(const float* frame_normals, int frames, int n, uint32_t f0,
                               const float inv_transposed_view[16], int nabla_map, float* feat, cudaStream_t s);
cudaError_t feature_to_chw(const float* feat, int n, uint32_t frames, int feature, int channels, const float* albedo,
                           float far_distance, float* out, cudaStream_t stream);

}  // namespace vpt
