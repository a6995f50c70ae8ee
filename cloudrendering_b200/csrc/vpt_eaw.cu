// vpt_eaw.cu - the EAW a-trous passes (Data/Shaders/Denoiser/EAWDenoise.glsl): 5x5 taps at step 2^i
// with Gaussian weights exp(-(x^2+y^2)/2), colour / position / normal edge stops
// min(exp(-|d|^2/phi), 1), taps outside the image clamped to the edge.  A unit of its own so that its
// multiply-adds are contracted (the other denoiser kernels are compiled without contraction): the
// passes are bound by instruction issue.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <mutex>
#include "vpt_denoise.h"
#include "vpt_kernels.h"

namespace vpt {

constexpr int kMaxEawDevices = 64;
__constant__ float c_eaw_kernel[25];

__device__ __forceinline__ float4 ld4(const float* img, int x, int y, int w, int h) {
    x = min(max(x, 0), w - 1);
    y = min(max(y, 0), h - 1);
    return __ldg(reinterpret_cast<const float4*>(img) + (size_t)y * w + x);
}

__device__ __forceinline__ float dot4(float4 a, float4 b) {
    return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w;
}
__device__ __forceinline__ float4 sub4(float4 a, float4 b) {
    return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}

// Edge-stopping weight min(exp(-|d|^2 / phi), 1) with the special-function unit's exponential and
// the reciprocal of phi computed once (a few ulp from the IEEE form; the filter is a normalised
// weighted mean, so its output moves by about as much).
__device__ __forceinline__ float eaw_stop(float4 d, float inv_phi) {
    return fminf(__expf(-dot4(d, d) * inv_phi), 1.0f);
}

__global__ void eaw_iteration_kernel(const float* __restrict__ color, const float* __restrict__ pos,
                                     const float* __restrict__ nrm, float* __restrict__ out, int w, int h, int step,
                                     float phi_c, float phi_p, float phi_n, int use_c, int use_p, int use_n,
                                     int quirk) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    float4 cc = ld4(color, x, y, w, h);
    float4 cp = pos ? ld4(pos, x, y, w, h) : make_float4(0, 0, 0, 0);
    float4 cn = nrm ? ld4(nrm, x, y, w, h) : make_float4(0, 0, 0, 0);
    float4 sum = make_float4(0, 0, 0, 0);
    float acc = 0.0f;
    const float quirk_wc = fminf(expf(-1.0f / phi_c), 1.0f);
    const float inv_c = 1.0f / phi_c, inv_p = 1.0f / phi_p, inv_n = 1.0f / phi_n;
#pragma unroll
    for (int i = 0; i < 25; i++) {
        int ox = i % 5 - 2, oy = i / 5 - 2;
        float kv = c_eaw_kernel[i];
        int sx = x + ox * step, sy = y + oy * step;
        float4 oc = ld4(color, sx, sy, w, h);
        float weight = 1.0f;
        if (use_c) {
            float4 d = sub4(cc, oc);
            weight *= quirk ? quirk_wc : eaw_stop(d, inv_c);
        }
        if (use_p && pos) {
            float4 d = sub4(cp, ld4(pos, sx, sy, w, h));
            weight *= eaw_stop(d, inv_p);
        }
        if (use_n && nrm) {
            float4 d = sub4(cn, ld4(nrm, sx, sy, w, h));
            weight *= eaw_stop(d, inv_n);
        }
        float wk = weight * kv;
        sum.x += oc.x * wk;
        sum.y += oc.y * wk;
        sum.z += oc.z * wk;
        sum.w += oc.w * wk;
        acc += wk;
    }
    const float ia = 1.0f / acc;
    reinterpret_cast<float4*>(out)[(size_t)y * w + x] = make_float4(sum.x * ia, sum.y * ia, sum.z * ia, sum.w * ia);
}

// The same iteration with the taps staged in shared memory.  The 25 taps of pixel (x, y) at step s lie
// on the lattice (x + i s, y + j s), so a block takes 16 x 16 pixels of ONE residue class (x mod s,
// y mod s) spaced s apart: their taps all fall on a 20 x 20 patch of that class's lattice, loaded
// once (16x reuse at every step, where a dense 16 x 16 tile would share few taps at large steps).
// Lattice points beyond the image are clamped to the edge pixel, as the taps are.  Same arithmetic,
// tap for tap, as eaw_iteration_kernel.
constexpr int kEawTile = 16;
constexpr int kEawPatch = kEawTile + 4;

__global__ void __launch_bounds__(kEawTile* kEawTile)
    eaw_lattice_kernel(const float* __restrict__ color, const float* __restrict__ pos, const float* __restrict__ nrm,
                       float* __restrict__ out, int w, int h, int step, int tiles_x, int tiles_y, float phi_c,
                       float phi_p, float phi_n, int use_c, int use_p, int use_n, int quirk) {
    __shared__ float4 sc[kEawPatch][kEawPatch];
    __shared__ float4 sp[kEawPatch][kEawPatch];
    __shared__ float4 sn[kEawPatch][kEawPatch];
    // block -> (residue rx, ry; tile tx, ty)
    int b = blockIdx.x;
    const int tx = b % tiles_x;
    b /= tiles_x;
    const int ty = b % tiles_y;
    b /= tiles_y;
    const int rx = b % step, ry = b / step;
    const int t = threadIdx.y * kEawTile + threadIdx.x;
    const bool use_pos = use_p && pos, use_nrm = use_n && nrm;
    for (int k = t; k < kEawPatch * kEawPatch; k += kEawTile * kEawTile) {
        const int a = k % kEawPatch, c = k / kEawPatch;
        const int px = min(max((tx * kEawTile + a - 2) * step + rx, 0), w - 1);
        const int py = min(max((ty * kEawTile + c - 2) * step + ry, 0), h - 1);
        const size_t o = (size_t)py * w + px;
        sc[c][a] = __ldg(reinterpret_cast<const float4*>(color) + o);
        if (use_pos) sp[c][a] = __ldg(reinterpret_cast<const float4*>(pos) + o);
        if (use_nrm) sn[c][a] = __ldg(reinterpret_cast<const float4*>(nrm) + o);
    }
    __syncthreads();
    const int x = (tx * kEawTile + threadIdx.x) * step + rx;
    const int y = (ty * kEawTile + threadIdx.y) * step + ry;
    if (x >= w || y >= h) return;
    const int cx = threadIdx.x + 2, cy = threadIdx.y + 2;
    const float4 cc = sc[cy][cx];
    const float4 cp = use_pos ? sp[cy][cx] : make_float4(0, 0, 0, 0);
    const float4 cn = use_nrm ? sn[cy][cx] : make_float4(0, 0, 0, 0);
    float4 sum = make_float4(0, 0, 0, 0);
    float acc = 0.0f;
    const float quirk_wc = fminf(expf(-1.0f / phi_c), 1.0f);
    const float inv_c = 1.0f / phi_c, inv_p = 1.0f / phi_p, inv_n = 1.0f / phi_n;
#pragma unroll
    for (int i = 0; i < 25; i++) {
        const int ox = i % 5 - 2, oy = i / 5 - 2;
        const float kv = c_eaw_kernel[i];
        const float4 oc = sc[cy + oy][cx + ox];
        float weight = 1.0f;
        if (use_c) {
            float4 d = sub4(cc, oc);
            weight *= quirk ? quirk_wc : eaw_stop(d, inv_c);
        }
        if (use_pos) {
            float4 d = sub4(cp, sp[cy + oy][cx + ox]);
            weight *= eaw_stop(d, inv_p);
        }
        if (use_nrm) {
            float4 d = sub4(cn, sn[cy + oy][cx + ox]);
            weight *= eaw_stop(d, inv_n);
        }
        float wk = weight * kv;
        sum.x += oc.x * wk;
        sum.y += oc.y * wk;
        sum.z += oc.z * wk;
        sum.w += oc.w * wk;
        acc += wk;
    }
    const float ia = 1.0f / acc;
    reinterpret_cast<float4*>(out)[(size_t)y * w + x] = make_float4(sum.x * ia, sum.y * ia, sum.z * ia, sum.w * ia);
}

// The 25 Gaussian tap weights live in constant memory, which is per device: upload once per device.
static cudaError_t upload_eaw_kernel(cudaStream_t s) {
    static std::mutex mu;
    static bool done[kMaxEawDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxEawDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return cudaSuccess;
    float k[25];
    for (int i = 0; i < 25; i++) {
        int x = i % 5 - 2, y = i / 5 - 2;
        k[i] = expf(-float(x * x + y * y) / 2.0f);
    }
    e = cudaMemcpyToSymbolAsync(c_eaw_kernel, k, sizeof(k), 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) done[dev] = true;
    return e;
}

cudaError_t eaw_denoise(const float* color, const float* pos, const float* nrm, int w, int h, const EawSettings& s,
                        float* ping, float* pong, float** result, cudaStream_t stream) {
    cudaError_t e = upload_eaw_kernel(stream);
    if (e != cudaSuccess) return e;
    dim3 b(16, 16), g((w + 15) / 16, (h + 15) / 16);
    const float* src = color;
    float* bufs[2] = {ping, pong};
    int step = 1;
    float* dst = nullptr;
    for (int i = 0; i < s.iterations; i++) {
        dst = bufs[i & 1];
        if (s.lattice_tiles) {
            // per residue class: ceil(ceil(w / step) / 16) x ceil(ceil(h / step) / 16) tiles
            const int tiles_x = ((w + step - 1) / step + kEawTile - 1) / kEawTile;
            const int tiles_y = ((h + step - 1) / step + kEawTile - 1) / kEawTile;
            const long long blocks = (long long)tiles_x * tiles_y * step * step;
            if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
            eaw_lattice_kernel<<<(unsigned)blocks, dim3(kEawTile, kEawTile), 0, stream>>>(
                src, pos, nrm, dst, w, h, step, tiles_x, tiles_y, s.phi_color, s.phi_position, s.phi_normal,
                s.use_color, s.use_position, s.use_normal, s.ref_compute_quirk);
        } else {
            eaw_iteration_kernel<<<g, b, 0, stream>>>(src, pos, nrm, dst, w, h, step, s.phi_color, s.phi_position,
                                                      s.phi_normal, s.use_color, s.use_position, s.use_normal,
                                                      s.ref_compute_quirk);
        }
        count_launches(1);
        src = dst;
        step *= 2;
    }
    *result = const_cast<float*>(src);
    return cudaGetLastError();
}

}  // namespace vpt
