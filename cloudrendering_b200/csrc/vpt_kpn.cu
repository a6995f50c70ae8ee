// vpt_kpn.cu - kernel-predicting denoiser kernels: per-pixel kernel application and the
// "inv_iter" multi-scale reconstruction of the reference's PyTorch denoiser
// (modules/kpn_module/src/Kernel.cu:38-261; composed in src/Denoiser/PyTorchDenoiser.cpp:174-179,
// 411-440), plus the average pooling and previous-frame reprojection the composition needs
// (torch::avg_pool2d, torch::grid_sampler_2d).
//
// All images are N x C x H x W float (C <= 4), weights N x K x Hw x Ww.  Compared with the reference:
//  * the softmax over the K = k*k kernel taps (torch::softmax(l, 1) before perPixelKernelCuda) is
//    fused into the application kernel: each thread reads its pixel's logits once;
//  * the inv_iter base (sigmoid-gated low/high-frequency split and previous-frame blend) is fused
//    with the tap softmax and the kernel application: the base of each of the k*k neighbours is
//    recomputed from the inputs (all reads stay in L1/L2), so no base image round-trips through HBM;
//  * the fused weights' batch stride is (k*k + 3) * Hw * Ww (the reference uses k*k * Hw * Ww,
//    Kernel.cu:166-168, which is wrong for N > 1).
// Neighbours are tested against the output size (h, w) = min(image, weights), as Kernel.cu:68 does.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include "../../include/vpt_b200.h"
#include "vpt_kernels.h"

namespace vpt {

namespace {

constexpr int kMaxKpnChannels = 4;
constexpr int kMaxTaps = 49;  // kernels up to 7 x 7

// softmax over the K logits of pixel (y, x): torch's definition exp(l - max) / sum exp(l - max).
// K is a compile-time constant so that the K values live in registers.
template <int K>
__device__ __forceinline__ void tap_softmax(const float* __restrict__ wbase, size_t plane, float* p) {
    float m = -INFINITY;
#pragma unroll
    for (int k = 0; k < K; k++) {
        p[k] = __ldg(wbase + (size_t)k * plane);
        m = fmaxf(m, p[k]);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < K; k++) {
        p[k] = expf(p[k] - m);
        s += p[k];
    }
#pragma unroll
    for (int k = 0; k < K; k++) p[k] = p[k] / s;
}

template <int KS>
__global__ void kpn_apply_kernel(const float* __restrict__ image, const float* __restrict__ weights,
                                 float* __restrict__ out, int N, int C, int H, int W, int Hw, int Ww, int h, int w,
                                 int softmax) {
    constexpr int K = KS * KS;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int n = blockIdx.z;
    if (x >= w || y >= h || n >= N) return;
    const size_t plane = (size_t)Hw * Ww;
    const float* wb = weights + (size_t)n * K * plane + (size_t)y * Ww + x;
    float p[K];
    if (softmax) {
        tap_softmax<K>(wb, plane, p);
    } else {
#pragma unroll
        for (int t = 0; t < K; t++) p[t] = __ldg(wb + (size_t)t * plane);
    }
    float acc[kMaxKpnChannels] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int dy = -KS / 2; dy <= KS / 2; dy++) {
        const int ky = y + dy;
#pragma unroll
        for (int dx = -KS / 2; dx <= KS / 2; dx++) {
            const int t = (dy + KS / 2) * KS + (dx + KS / 2);
            const int kx = x + dx;
            if (kx < 0 || kx >= w || ky < 0 || ky >= h) continue;
#pragma unroll
            for (int c = 0; c < kMaxKpnChannels; c++)
                if (c < C) acc[c] += p[t] * __ldg(image + (((size_t)n * C + c) * H + ky) * W + kx);
        }
    }
    for (int c = 0; c < C; c++) out[(((size_t)n * C + c) * h + y) * w + x] = acc[c];
}

__device__ __forceinline__ float sigmoidf(float v) { return 1.0f / (1.0f + expf(-v)); }

struct InvIterArgs {
    const float* x_hi;     // N x C x H x W
    const float* pred_lo;  // N x C x Hl x Wl
    const float* x_lo;     // N x C x Hl x Wl
    const float* prev;     // N x C x H x W (used when use_prev)
    const float* fused;    // N x (K + 3) x Hw x Ww
    float* out;            // N x C x h x w
    int N, C, H, W, Hl, Wl, Hw, Ww, h, w, k, use_prev;
};

// getInvIterBaseKernel (Kernel.cu:138-186) for one pixel and channel; false where the reference
// writes nothing (the low-resolution pixel is out of range; the output keeps its zero).
__device__ __forceinline__ bool inv_iter_base(const InvIterArgs& a, int n, int c, int x, int y, float& base) {
    const int lx = x / 2, ly = y / 2;
    if (lx >= a.Wl || ly >= a.Hl) return false;
    const int K = a.k * a.k;
    const size_t plane = (size_t)a.Hw * a.Ww;
    const float* wb = a.fused + (size_t)n * (K + 3) * plane + (size_t)y * a.Ww + x;
    const float lf_w = sigmoidf(__ldg(wb + (size_t)K * plane));
    const float hf_w = sigmoidf(__ldg(wb + (size_t)(K + 1) * plane));
    const float pv_w = sigmoidf(__ldg(wb + (size_t)(K + 2) * plane));
    const float xh = __ldg(a.x_hi + (((size_t)n * a.C + c) * a.H + y) * a.W + x);
    const float xl = __ldg(a.x_lo + (((size_t)n * a.C + c) * a.Hl + ly) * a.Wl + lx);
    const float pl = __ldg(a.pred_lo + (((size_t)n * a.C + c) * a.Hl + ly) * a.Wl + lx);
    float lf = lf_w * pl + (1.0f - lf_w) * xl;
    if (a.use_prev) {
        const float pr = __ldg(a.prev + (((size_t)n * a.C + c) * a.H + y) * a.W + x);
        // the reference computes this line with a double literal: lf * (1.0 - w) + prev * w
        lf = (float)((double)lf * (1.0 - (double)pv_w) + (double)(pr * pv_w));
    }
    base = hf_w * (xh - xl + lf) + (1.0f - hf_w) * lf;
    return true;
}

template <int KS>
__global__ void kpn_inv_iter_kernel(const InvIterArgs a) {
    constexpr int K = KS * KS;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int n = blockIdx.z;
    if (x >= a.w || y >= a.h || n >= a.N) return;
    const size_t plane = (size_t)a.Hw * a.Ww;
    float p[K];
    tap_softmax<K>(a.fused + (size_t)n * (K + 3) * plane + (size_t)y * a.Ww + x, plane, p);
    float acc[kMaxKpnChannels] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int dy = -KS / 2; dy <= KS / 2; dy++) {
        const int ky = y + dy;
#pragma unroll
        for (int dx = -KS / 2; dx <= KS / 2; dx++) {
            const int t = (dy + KS / 2) * KS + (dx + KS / 2);
            const int kx = x + dx;
            if (kx < 0 || kx >= a.w || ky < 0 || ky >= a.h) continue;
            for (int c = 0; c < a.C; c++) {
                float b = 0.0f;
                inv_iter_base(a, n, c, kx, ky, b);
                acc[c] += p[t] * b;
            }
        }
    }
    for (int c = 0; c < a.C; c++) a.out[(((size_t)n * a.C + c) * a.h + y) * a.w + x] = acc[c];
}

// torch::avg_pool2d(x, 2, 2): floor(H/2) x floor(W/2), mean of each 2 x 2 block
__global__ void kpn_avg_pool2_kernel(const float* __restrict__ in, float* __restrict__ out, int NC, int H, int W) {
    const int Ho = H / 2, Wo = W / 2;
    const size_t total = (size_t)NC * Ho * Wo;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % Wo);
        const int y = (int)((i / Wo) % Ho);
        const size_t nc = i / ((size_t)Wo * Ho);
        const float* b = in + (nc * H + 2 * y) * W + 2 * x;
        out[i] = (((__ldg(b) + __ldg(b + 1)) + __ldg(b + W)) + __ldg(b + W + 1)) / 4.0f;
    }
}

// torch::grid_sampler_2d(prev, uv * 2 - 1, bilinear, zeros, align_corners = false) with uv the
// 2-channel reprojection map (N x 2 x H x W, texture coordinates in [0, 1]).
__global__ void kpn_reproject_kernel(const float* __restrict__ prev, const float* __restrict__ uv,
                                     float* __restrict__ out, int N, int C, int Hp, int Wp, int H, int W) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int n = blockIdx.z;
    if (x >= W || y >= H || n >= N) return;
    const size_t plane = (size_t)H * W;
    const float gx = __ldg(uv + ((size_t)n * 2 + 0) * plane + (size_t)y * W + x) * 2.0f - 1.0f;
    const float gy = __ldg(uv + ((size_t)n * 2 + 1) * plane + (size_t)y * W + x) * 2.0f - 1.0f;
    // unnormalise (align_corners = false): ((g + 1) * size - 1) / 2
    const float ix = ((gx + 1.0f) * (float)Wp - 1.0f) / 2.0f;
    const float iy = ((gy + 1.0f) * (float)Hp - 1.0f) / 2.0f;
    const float fx0 = floorf(ix), fy0 = floorf(iy);
    const int x0 = (int)fx0, y0 = (int)fy0, x1 = x0 + 1, y1 = y0 + 1;
    // bilinear weights as grid_sampler_2d forms them (north-west, north-east, south-west, south-east)
    const float fx1 = fx0 + 1.0f, fy1 = fy0 + 1.0f;
    const float w00 = (fx1 - ix) * (fy1 - iy), w10 = (ix - fx0) * (fy1 - iy);
    const float w01 = (fx1 - ix) * (iy - fy0), w11 = (ix - fx0) * (iy - fy0);
    const bool in00 = x0 >= 0 && x0 < Wp && y0 >= 0 && y0 < Hp;
    const bool in10 = x1 >= 0 && x1 < Wp && y0 >= 0 && y0 < Hp;
    const bool in01 = x0 >= 0 && x0 < Wp && y1 >= 0 && y1 < Hp;
    const bool in11 = x1 >= 0 && x1 < Wp && y1 >= 0 && y1 < Hp;
    for (int c = 0; c < C; c++) {
        const float* src = prev + ((size_t)n * C + c) * Hp * Wp;
        float v = 0.0f;
        if (in00) v += __ldg(src + (size_t)y0 * Wp + x0) * w00;
        if (in10) v += __ldg(src + (size_t)y0 * Wp + x1) * w10;
        if (in01) v += __ldg(src + (size_t)y1 * Wp + x0) * w01;
        if (in11) v += __ldg(src + (size_t)y1 * Wp + x1) * w11;
        out[((size_t)n * C + c) * plane + (size_t)y * W + x] = v;
    }
}

dim3 grid2d(int w, int h, int n) { return dim3((w + 15) / 16, (h + 15) / 16, n); }

}  // namespace

}  // namespace vpt

extern "C" {

VptStatus vpt_kpn_apply(const float* image, const float* weights, int n, int c, int h, int w, int weights_h,
                        int weights_w, int kernel_size, int softmax, float* out, void* stream) {
    if (!image || !weights || !out || n <= 0 || c <= 0 || c > vpt::kMaxKpnChannels || h <= 0 || w <= 0 ||
        weights_h <= 0 || weights_w <= 0 || kernel_size <= 0 || kernel_size % 2 == 0 ||
        kernel_size * kernel_size > vpt::kMaxTaps)
        return VPT_ERR_ARG;
    const int ho = h < weights_h ? h : weights_h, wo = w < weights_w ? w : weights_w;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const dim3 g = vpt::grid2d(wo, ho, n), b(16, 16);
    switch (kernel_size) {
        case 1: vpt::kpn_apply_kernel<1><<<g, b, 0, s>>>(image, weights, out, n, c, h, w, weights_h, weights_w, ho, wo, softmax); break;
        case 3: vpt::kpn_apply_kernel<3><<<g, b, 0, s>>>(image, weights, out, n, c, h, w, weights_h, weights_w, ho, wo, softmax); break;
        case 5: vpt::kpn_apply_kernel<5><<<g, b, 0, s>>>(image, weights, out, n, c, h, w, weights_h, weights_w, ho, wo, softmax); break;
        default: vpt::kpn_apply_kernel<7><<<g, b, 0, s>>>(image, weights, out, n, c, h, w, weights_h, weights_w, ho, wo, softmax); break;
    }
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_kpn_inv_iter(const float* x_hi, const float* pred_lo, const float* x_lo, const float* prev,
                           const float* fused_weights, int n, int c, int h, int w, int low_h, int low_w, int weights_h,
                           int weights_w, int kernel_size, int use_prev, float* out, void* stream) {
    if (!x_hi || !pred_lo || !x_lo || !fused_weights || !out || (use_prev && !prev) || n <= 0 || c <= 0 ||
        c > vpt::kMaxKpnChannels || h <= 0 || w <= 0 || low_h <= 0 || low_w <= 0 || weights_h <= 0 ||
        weights_w <= 0 || kernel_size <= 0 || kernel_size % 2 == 0 || kernel_size * kernel_size > vpt::kMaxTaps)
        return VPT_ERR_ARG;
    vpt::InvIterArgs a;
    a.x_hi = x_hi;
    a.pred_lo = pred_lo;
    a.x_lo = x_lo;
    a.prev = prev;
    a.fused = fused_weights;
    a.out = out;
    a.N = n;
    a.C = c;
    a.H = h;
    a.W = w;
    a.Hl = low_h;
    a.Wl = low_w;
    a.Hw = weights_h;
    a.Ww = weights_w;
    a.h = h < weights_h ? h : weights_h;
    a.w = w < weights_w ? w : weights_w;
    a.k = kernel_size;
    a.use_prev = use_prev ? 1 : 0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const dim3 g = vpt::grid2d(a.w, a.h, n), b(16, 16);
    switch (kernel_size) {  // odd and at most 7 (checked above)
        case 1: vpt::kpn_inv_iter_kernel<1><<<g, b, 0, s>>>(a); break;
        case 3: vpt::kpn_inv_iter_kernel<3><<<g, b, 0, s>>>(a); break;
        case 5: vpt::kpn_inv_iter_kernel<5><<<g, b, 0, s>>>(a); break;
        default: vpt::kpn_inv_iter_kernel<7><<<g, b, 0, s>>>(a); break;
    }
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_kpn_avg_pool2(const float* in, int n, int c, int h, int w, float* out, void* stream) {
    if (!in || !out || n <= 0 || c <= 0 || h < 2 || w < 2) return VPT_ERR_ARG;
    const size_t total = (size_t)n * c * (h / 2) * (w / 2);
    unsigned blocks = (unsigned)((total + 255) / 256);
    if (blocks > 148u * 32u) blocks = 148u * 32u;
    vpt::kpn_avg_pool2_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(in, out, n * c, h, w);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_kpn_reproject(const float* prev, const float* uv, int n, int c, int prev_h, int prev_w, int h, int w,
                            float* out, void* stream) {
    if (!prev || !uv || !out || n <= 0 || c <= 0 || prev_h <= 0 || prev_w <= 0 || h <= 0 || w <= 0)
        return VPT_ERR_ARG;
    vpt::kpn_reproject_kernel<<<vpt::grid2d(w, h, n), dim3(16, 16), 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        prev, uv, out, n, c, prev_h, prev_w, h, w);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

}  // extern "C"
