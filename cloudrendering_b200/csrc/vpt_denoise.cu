// vpt_denoise.cu - EAW feature inputs and entry points, SVGF, and feature-map readout.
//
// EAW: edge-avoiding a-trous wavelet filter (Dammertz et al. 2010) as in
// Data/Shaders/Denoiser/EAWDenoise.glsl; its passes are in vpt_eaw.cu (one launch per iteration, each
// thread one pixel; by default a block stages the taps of 16 x 16 pixels of one residue class modulo
// the step in shared memory, eaw_lattice_kernel; the direct kernel reads every tap through L1).
//
// SVGF: Data/Shaders/Denoiser/SVGF/SVGF.glsl (reproject 210-267, filter moments 286-347, a-trous
// 401-495) with compute_weight from svgf_common.glsl:29-41.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <mutex>
#include "vpt_denoise.h"
#include "vpt_params.h"
#include "vpt_kernels.h"
#include "../../include/vpt_b200.h"

namespace vpt {

constexpr int kMaxDevices = 64;


// Position map (Clouds.glsl:195-202: mean of (x, 1) over hits, (0) otherwise) and normal map
// (Clouds.glsl:266-312: mean of the finite-difference normal, alpha 1) from the accumulators.
__global__ void features_to_eaw_maps_kernel(const float* __restrict__ feat, int n, float inv_frames,
                                            float4* __restrict__ pos, float4* __restrict__ nrm) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* f = feat + (size_t)i * kFeatStride;
    pos[i] = make_float4(f[kFeatPos] * inv_frames, f[kFeatPos + 1] * inv_frames, f[kFeatPos + 2] * inv_frames,
                         f[kFeatPos + 3] * inv_frames);
    nrm[i] = make_float4(f[kFeatNormal] * inv_frames, f[kFeatNormal + 1] * inv_frames, f[kFeatNormal + 2] * inv_frames,
                         1.0f);
}

cudaError_t eaw_denoise_features(const float* color, const float* feat, uint32_t frames, int w, int h,
                                 const EawSettings& s, float* maps, float* ping, float* pong, float** result,
                                 cudaStream_t stream) {
    const int n = w * h;
    const float* pos = nullptr;
    const float* nrm = nullptr;
    if (feat) {
        features_to_eaw_maps_kernel<<<(n + 255) / 256, 256, 0, stream>>>(
            feat, n, 1.0f / float(frames), reinterpret_cast<float4*>(maps), reinterpret_cast<float4*>(maps + (size_t)n * 4));
        count_launches(1);
        pos = maps;
        nrm = maps + (size_t)n * 4;
    }
    return eaw_denoise(color, pos, nrm, w, h, s, ping, pong, result, stream);
}

// ---------------------------------------------------------------------------------------------
// SVGF

void svgf_release(SvgfState& s) {
    if (s.color_history) cudaFree(s.color_history);
    if (s.moments_history) cudaFree(s.moments_history);
    if (s.normal_history) cudaFree(s.normal_history);
    if (s.depth_history) cudaFree(s.depth_history);
    if (s.cur) cudaFree(s.cur);
    s = SvgfState();
}

__device__ __forceinline__ float svgf_weight(float cd, float od, float phi_d, float3 cn, float3 on, float cc, float oc,
                                             float phi_c) {
    float wn = powf(fmaxf(0.0f, (cn.x * on.x + cn.y * on.y) + cn.z * on.z), 128.0f);
    float wz = (phi_d == 0.0f) ? 0.0f : fabsf(cd - od) / phi_d;
    float wc = fabsf(cc - oc) * 2.0f / phi_c;
    return expf(0.0f - fmaxf(wc, 0.0f) - fmaxf(wz, 0.0f)) * wn;
}

struct SvgfCur {
    float4* noisy;     // rgba
    float2* motion;    // flow
    float4* normal;    // rgba
    float* depth;
    float* fwidth;
    float4* moments;   // accum moments
    float4* temp;      // temp accum (rgb, variance)
    float4* ping;
    float4* pong;
};

static SvgfCur svgf_cur(float* base, int n) {
    SvgfCur c;
    c.noisy = reinterpret_cast<float4*>(base);
    c.normal = reinterpret_cast<float4*>(base + (size_t)n * 4);
    c.moments = reinterpret_cast<float4*>(base + (size_t)n * 8);
    c.temp = reinterpret_cast<float4*>(base + (size_t)n * 12);
    c.ping = reinterpret_cast<float4*>(base + (size_t)n * 16);
    c.pong = reinterpret_cast<float4*>(base + (size_t)n * 20);
    c.motion = reinterpret_cast<float2*>(base + (size_t)n * 24);
    c.depth = base + (size_t)n * 26;
    c.fwidth = base + (size_t)n * 27;
    return c;
}
constexpr int kSvgfCurFloats = 28;

struct Mat4 {
    float m[16];
};

// Current-frame maps from one frame of feature accumulators (DISABLE_ACCUMULATION semantics,
// Clouds.glsl:204-216, 266-328, 356-365).
__global__ void svgf_prepare_kernel(const float4* __restrict__ color, const float* __restrict__ feat, int w, int h,
                                    Mat4 itv, Mat4 pvp, float far_dist, SvgfCur c) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const float* f = feat + (size_t)i * kFeatStride;
    bool hit = f[kFeatPos + 3] > 0.0f;
    c.noisy[i] = color[i];
    float3 n = make_float3(f[kFeatNormal], f[kFeatNormal + 1], f[kFeatNormal + 2]);
    c.normal[i] = make_float4(n.x, n.y, n.z, hit ? 1.0f : 0.0f);
    c.depth[i] = hit ? f[kFeatDepth] : far_dist;
    float fw = 0.0f;
    float2 flow = make_float2(0.0f, 0.0f);
    if (hit) {
        float A = (itv.m[0] * n.x + itv.m[4] * n.y) + itv.m[8] * n.z;
        float B = (itv.m[1] * n.x + itv.m[5] * n.y) + itv.m[9] * n.z;
        float nx = A / sqrtf(1.0f - A * A), ny = B / sqrtf(1.0f - B * B);
        fw = fabsf(nx) + fabsf(ny);
        float px = f[kFeatPos], py = f[kFeatPos + 1], pz = f[kFeatPos + 2];
        float cx = ((pvp.m[0] * px + pvp.m[4] * py) + pvp.m[8] * pz) + pvp.m[12];
        float cy = ((pvp.m[1] * px + pvp.m[5] * py) + pvp.m[9] * pz) + pvp.m[13];
        float cw = ((pvp.m[3] * px + pvp.m[7] * py) + pvp.m[11] * pz) + pvp.m[15];
        float lx = (0.5f * (cx / cw) + 0.5f) * (float)w - 0.5f;
        float ly = (0.5f * (cy / cw) + 0.5f) * (float)h - 0.5f;
        flow = make_float2((float)(i % w) - lx, (float)(i / w) - ly);
    }
    c.fwidth[i] = fw;
    c.motion[i] = flow;
}

__device__ __forceinline__ bool svgf_valid(int x, int y, int w, int h, float z, float zp, float3 n, float3 np,
                                           float zt, float nt) {
    if (x < 1 || y < 1 || x > w - 1 || y > h - 1) return false;
    if (fabsf(zp - z) > zt) return false;
    float dx = np.x - n.x, dy = np.y - n.y, dz = np.z - n.z;
    if (sqrtf((dx * dx + dy * dy) + dz * dz) > nt) return false;
    return true;
}

__global__ void svgf_reproject_kernel(SvgfCur c, const float4* __restrict__ color_hist,
                                      const float4* __restrict__ moments_hist, const float4* __restrict__ normal_hist,
                                      const float* __restrict__ depth_hist, int w, int h, float zt, float nt) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float2 mv = c.motion[i];
    int pxp = (int)(0.5f + ((float)x - mv.x)), pyp = (int)(0.5f + ((float)y - mv.y));
    float2 prev_m = make_float2(0.0f, 0.0f);
    float hist_len = 0.0f;
    bool ok = !(pxp < 0 || pyp < 0 || pxp >= w || pyp >= h);
    if (ok) {
        float4 r = moments_hist[pyp * w + pxp];
        prev_m = make_float2(r.x, r.y);
        hist_len = r.z;
    }
    float4 col4 = c.noisy[i];
    float3 col = make_float3(col4.x, col4.y, col4.z);
    float4 lf = color_hist[i];
    float3 last = make_float3(lf.x, lf.y, lf.z);
    if (ok) {
        float fx = 0.01f + ((float)x - mv.x), fy = 0.01f + ((float)y - mv.y);
        int ix = (int)fx, iy = (int)fy;
        float depth = c.depth[i];
        float4 nn = c.normal[i];
        float3 n = make_float3(nn.x, nn.y, nn.z);
        const int ox[4] = {0, 0, 1, 1}, oy[4] = {0, 1, 0, 1};
        bool valids[4];
        bool found = false;
        for (int k = 0; k < 4; k++) {
            int qx = ix + ox[k], qy = iy + oy[k];
            bool inside = qx >= 0 && qy >= 0 && qx < w && qy < h;
            float4 on = inside ? normal_hist[qy * w + qx] : make_float4(0, 0, 0, 0);
            float od = inside ? depth_hist[qy * w + qx] : 0.0f;
            valids[k] = inside && svgf_valid(qx, qy, w, h, depth, od, n, make_float3(on.x, on.y, on.z), zt, nt);
            found = found || valids[k];
        }
        if (found) {
            float ax = fx - floorf(fx), ay = fy - floorf(fy);
            const float wk[4] = {(1 - ax) * (1 - ay), ax * (1 - ay), (1 - ax) * ay, ax * ay};
            float3 cb = make_float3(0, 0, 0);
            float2 mb = make_float2(0, 0);
            float sw = 0.0f;
            for (int k = 0; k < 4; k++) {
                if (!valids[k]) continue;
                int qx = ix + ox[k], qy = iy + oy[k];
                float4 oc = color_hist[qy * w + qx];
                float4 om = moments_hist[qy * w + qx];
                mb.x += wk[k] * om.x;
                mb.y += wk[k] * om.y;
                cb.x += wk[k] * oc.x;
                cb.y += wk[k] * oc.y;
                cb.z += wk[k] * oc.z;
                sw += wk[k];
            }
            found = sw >= 0.001f;
            if (found) {
                last = make_float3(cb.x / sw, cb.y / sw, cb.z / sw);
                prev_m = make_float2(mb.x / sw, mb.y / sw);
            }
        }
        if (!found) {
            float nv = 0.0f;
            float3 fc = make_float3(0, 0, 0);
            float2 fm = make_float2(0, 0);
            for (int yy = -1; yy <= 1; yy++)
                for (int xx = -1; xx <= 1; xx++) {
                    int qx = ix + xx, qy = iy + yy;
                    if (qx < 1 || qy < 1 || qx >= w || qy >= h) continue;
                    float4 on = normal_hist[qy * w + qx];
                    float od = depth_hist[qy * w + qx];
                    if (svgf_valid(qx, qy, w, h, depth, od, n, make_float3(on.x, on.y, on.z), zt, nt)) {
                        float4 oc = color_hist[qy * w + qx];
                        float4 om = moments_hist[qy * w + qx];
                        fc.x += oc.x;
                        fc.y += oc.y;
                        fc.z += oc.z;
                        fm.x += om.x;
                        fm.y += om.y;
                        nv += 1.0f;
                    }
                }
            if (nv > 0.0f) {
                last = make_float3(fc.x / nv, fc.y / nv, fc.z / nv);
                prev_m = make_float2(fm.x / nv, fm.y / nv);
                found = true;
            }
        }
        ok = found;
    }
    hist_len = fminf(ok ? hist_len + 1.0f : 1.0f, 32.0f);
    float a_c = ok ? fmaxf(0.01f, 1.0f / hist_len) : 1.0f;
    float a_m = ok ? fmaxf(0.2f, 1.0f / hist_len) : 1.0f;
    float m1 = col.x, m2 = m1 * m1;
    m1 = prev_m.x * (1.0f - a_m) + m1 * a_m;
    m2 = prev_m.y * (1.0f - a_m) + m2 * a_m;
    float var = fmaxf(0.0f, m2 - m1 * m1);
    c.moments[i] = make_float4(m1, m2, hist_len, 0.0f);
    c.temp[i] = make_float4(last.x * (1.0f - a_c) + col.x * a_c, last.y * (1.0f - a_c) + col.y * a_c,
                            last.z * (1.0f - a_c) + col.z * a_c, var);
}

__global__ void svgf_filter_moments_kernel(SvgfCur c, float4* __restrict__ temp_out, int w, int h) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float hl = c.moments[i].z;
    float4 center = c.temp[i];
    if (hl >= 4.0f) {
        temp_out[i] = center;
        return;
    }
    float cd = c.depth[i], cfw = c.fwidth[i];
    float4 cn4 = c.normal[i];
    float3 cn = make_float3(cn4.x, cn4.y, cn4.z);
    float sw = 0.0f;
    float3 sc = make_float3(0, 0, 0);
    float2 sm = make_float2(0, 0);
    for (int yy = -3; yy <= 3; yy++)
        for (int xx = -3; xx <= 3; xx++) {
            int qx = x + xx, qy = y + yy;
            if (qx < 0 || qy < 0 || qx >= w || qy >= h) continue;
            int q = qy * w + qx;
            float4 oc = c.temp[q];
            float4 om = c.moments[q];
            float4 on = c.normal[q];
            float wt = svgf_weight(cd, c.depth[q], fabsf(cfw) + 0.0001f, cn, make_float3(on.x, on.y, on.z), center.x,
                                   oc.x, 10.0f);
            sw += wt;
            sc.x += wt * oc.x;
            sc.y += wt * oc.y;
            sc.z += wt * oc.z;
            sm.x += wt * om.x;
            sm.y += wt * om.y;
        }
    sw = fmaxf(sw, 1e-6f);
    sc = make_float3(sc.x / sw, sc.y / sw, sc.z / sw);
    sm = make_float2(sm.x / sw, sm.y / sw);
    float var = sm.y - sm.x * sm.x;
    var *= 4.0f / hl;
    temp_out[i] = make_float4(sc.x, sc.y, sc.z, var);
}

__global__ void svgf_atrous_kernel(const float4* __restrict__ in, SvgfCur c, float4* __restrict__ out,
                                   float4* __restrict__ color_hist, int w, int h, int iteration) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    int step = 1 << iteration;
    float4 cc = in[i];
    const float kv2[2][2] = {{1.0f / 4.0f, 1.0f / 8.0f}, {1.0f / 8.0f, 1.0f / 16.0f}};
    float fv = 0.0f;
    for (int yy = -1; yy <= 1; yy++)
        for (int xx = -1; xx <= 1; xx++) {
            int qx = min(max(x + xx, 0), w - 1), qy = min(max(y + yy, 0), h - 1);
            fv += in[qy * w + qx].w * kv2[abs(xx)][abs(yy)];
        }
    float4 cn4 = c.normal[i];
    float3 cn = make_float3(cn4.x, cn4.y, cn4.z);
    float cz = c.depth[i], cfw = c.fwidth[i];
    float phi_c = sqrtf(fmaxf(0.0f, 1e-10f + fv));
    const float kvals[3] = {1.0f, 2.0f / 3.0f, 1.0f / 6.0f};
    float accw = kvals[0] * kvals[0];
    float4 sum = make_float4(cc.x * accw, cc.y * accw, cc.z * accw, cc.w * accw);
    for (int yy = -2; yy <= 2; yy++)
        for (int xx = -2; xx <= 2; xx++) {
            int qx = x + xx * step, qy = y + yy * step;
            bool inside = qx >= 0 && qy >= 0 && qx < w && qy < h;
            if (!inside || (xx == 0 && yy == 0)) continue;
            float kval = kvals[abs(xx)] * kvals[abs(yy)];
            int q = qy * w + qx;
            float4 oc = in[q];
            float4 on = c.normal[q];
            float len = sqrtf((float)(xx * xx + yy * yy));
            float wt = svgf_weight(cz, c.depth[q], fabsf(cfw * len * (float)step) + 0.0001f, cn,
                                   make_float3(on.x, on.y, on.z), cc.x, oc.x, phi_c) *
                       kval;
            sum.x += wt * oc.x;
            sum.y += wt * oc.y;
            sum.z += wt * oc.z;
            sum.w += wt * wt * oc.w;
            accw += wt;
        }
    float4 r = make_float4(sum.x / accw, sum.y / accw, sum.z / accw, sum.w / (accw * accw));
    if (iteration == 0) color_hist[i] = r;
    out[i] = r;
}

__global__ void svgf_update_history_kernel(SvgfCur c, float4* __restrict__ moments_hist,
                                           float4* __restrict__ normal_hist, float* __restrict__ depth_hist, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    moments_hist[i] = c.moments[i];
    normal_hist[i] = c.normal[i];
    depth_hist[i] = c.depth[i];
}

cudaError_t svgf_filter_passes(SvgfCur c, float4* color_history, float4* moments_history, float4* normal_history,
                               float* depth_history, int w, int h, const SvgfSettings& s, cudaStream_t stream,
                               const float4** result);

cudaError_t svgf_denoise_features(const float* color, const float* feat, uint32_t frames, int w, int h,
                                  const SvgfSettings& s, SvgfState& st, float* out_rgba, float** result,
                                  cudaStream_t stream) {
    (void)frames;
    (void)out_rgba;
    if (!feat) return cudaErrorInvalidValue;
    const int n = w * h;
    if (!st.valid || st.width != w || st.height != h) {
        svgf_release(st);
        cudaError_t e;
        if ((e = cudaMalloc(&st.color_history, (size_t)n * 16)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&st.moments_history, (size_t)n * 16)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&st.normal_history, (size_t)n * 16)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&st.depth_history, (size_t)n * 4)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&st.cur, (size_t)n * kSvgfCurFloats * 4)) != cudaSuccess) return e;
        cudaMemsetAsync(st.color_history, 0, (size_t)n * 16, stream);
        cudaMemsetAsync(st.moments_history, 0, (size_t)n * 16, stream);
        cudaMemsetAsync(st.normal_history, 0, (size_t)n * 16, stream);
        cudaMemsetAsync(st.depth_history, 0, (size_t)n * 4, stream);
        st.width = w;
        st.height = h;
        st.valid = true;
    }
    SvgfCur c = svgf_cur(st.cur, n);
    Mat4 itv, pvp;
    for (int k = 0; k < 16; k++) {
        itv.m[k] = s.inv_transposed_view[k];
        pvp.m[k] = s.prev_view_proj[k];
    }
    svgf_prepare_kernel<<<(n + 255) / 256, 256, 0, stream>>>(reinterpret_cast<const float4*>(color), feat, w, h, itv, pvp,
                                                             s.far_dist, c);
    count_launches(1);
    const float4* src = nullptr;
    cudaError_t e = svgf_filter_passes(c, reinterpret_cast<float4*>(st.color_history),
                                       reinterpret_cast<float4*>(st.moments_history),
                                       reinterpret_cast<float4*>(st.normal_history), st.depth_history, w, h, s, stream,
                                       &src);
    *result = reinterpret_cast<float*>(const_cast<float4*>(src));
    return e;
}

// The filter passes of one SVGF frame on prepared maps (c.noisy / normal / depth / fwidth / motion)
// and scratch (c.moments / temp / ping / pong); the result is c.temp, c.ping or c.pong.
cudaError_t svgf_filter_passes(SvgfCur c, float4* color_history, float4* moments_history, float4* normal_history,
                               float* depth_history, int w, int h, const SvgfSettings& s, cudaStream_t stream,
                               const float4** result) {
    const int n = w * h;
    dim3 b(16, 16), g((w + 15) / 16, (h + 15) / 16);
    svgf_reproject_kernel<<<g, b, 0, stream>>>(c, color_history, moments_history, normal_history, depth_history, w, h,
                                               s.z_threshold, s.normal_threshold);
    svgf_filter_moments_kernel<<<g, b, 0, stream>>>(c, c.ping, w, h);
    cudaMemcpyAsync(c.temp, c.ping, (size_t)n * 16, cudaMemcpyDeviceToDevice, stream);
    const float4* src = c.temp;
    float4* bufs[2] = {c.ping, c.pong};
    if (s.atrous_iterations < 1) {
        cudaMemcpyAsync(color_history, c.temp, (size_t)n * 16, cudaMemcpyDeviceToDevice, stream);
    }
    for (int it = 0; it < s.atrous_iterations; it++) {
        float4* dst = bufs[it & 1];
        svgf_atrous_kernel<<<g, b, 0, stream>>>(src, c, dst, color_history, w, h, it);
        src = dst;
    }
    svgf_update_history_kernel<<<(n + 255) / 256, 256, 0, stream>>>(c, moments_history, normal_history, depth_history,
                                                                     n);
    count_launches(4 + (unsigned)s.atrous_iterations);
    *result = src;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Depth (nabla) and Depth (fwidth) (Clouds.glsl:258-297, 344-364).  Each frame f of the reference
// mixes the normal map (running mean; frames without an event scale it by f / (f + 1)), then, for a
// frame with an event, projects that running-mean normal with inverseTransposedViewMatrix and takes
// nabla = (A / sqrt(1 - A^2), B / sqrt(1 - B^2)) of its x and y (0 without an event), whose running
// means are the two maps (fwidth = |nabla.x| + |nabla.y|).  The frames of a launch run concurrently
// here, so the trace stores each frame's normal and this kernel replays the frames in order per pixel.

__global__ void depth_deriv_kernel(const float4* __restrict__ frame_normals, int frames, int n, uint32_t f0, Mat4 M,
                                   int nabla_map, float* __restrict__ feat) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* f = feat + (size_t)i * kFeatStride;
    float nx = f[kFeatDerivNormal + 0], ny = f[kFeatDerivNormal + 1], nz = f[kFeatDerivNormal + 2];
    float ax = f[kFeatNabla + 0], ay = f[kFeatNabla + 1], fw = f[kFeatFwidth];
    for (int j = 0; j < frames; j++) {
        const uint32_t frame = f0 + (uint32_t)j;
        const float4 v = frame_normals[(size_t)j * n + i];
        const float t = 1.0f / float(frame + 1u);
        float bx = 0.0f, by = 0.0f;
        if (v.w != 0.0f) {
            float dx = v.x, dy = v.y, dz = v.z;
            if (frame != 0u) {  // mix(diffOld, diff, 1 / (frame + 1)); diffOld = 0 at frame 0
                dx = nx * (1.0f - t) + dx * t;
                dy = ny * (1.0f - t) + dy * t;
                dz = nz * (1.0f - t) + dz * t;
            } else {
                dx = 0.0f * (1.0f - t) + dx * t;
                dy = 0.0f * (1.0f - t) + dy * t;
                dz = 0.0f * (1.0f - t) + dz * t;
            }
            nx = dx;
            ny = dy;
            nz = dz;
            // (inverseTransposedViewMatrix * vec4(diff, 0)).xy
            const float A = ((M.m[0] * dx + M.m[4] * dy) + M.m[8] * dz) + M.m[12] * 0.0f;
            const float B = ((M.m[1] * dx + M.m[5] * dy) + M.m[9] * dz) + M.m[13] * 0.0f;
            bx = A / sqrtf(1.0f - A * A);
            by = B / sqrtf(1.0f - B * B);
        } else {
            const float s = frame == 0u ? 0.0f : float(frame) / float(frame + 1u);
            nx = frame == 0u ? 0.0f : nx * s;
            ny = frame == 0u ? 0.0f : ny * s;
            nz = frame == 0u ? 0.0f : nz * s;
        }
        if (frame != 0u) {
            ax = ax * (1.0f - t) + bx * t;
            ay = ay * (1.0f - t) + by * t;
        } else {
            ax = bx;
            ay = by;
        }
        // with the nabla map written, the shader's `nabla` already holds its running mean when the
        // fwidth block reads it (Clouds.glsl:344-357); without it, this frame's nabla
        const float fv = nabla_map ? fabsf(ax) + fabsf(ay) : fabsf(bx) + fabsf(by);
        fw = frame != 0u ? fw * (1.0f - t) + fv * t : fv;
    }
    f[kFeatDerivNormal + 0] = nx;
    f[kFeatDerivNormal + 1] = ny;
    f[kFeatDerivNormal + 2] = nz;
    f[kFeatNabla + 0] = ax;
    f[kFeatNabla + 1] = ay;
    f[kFeatFwidth] = fw;
}

cudaError_t launch_depth_deriv(const float* frame_normals, int frames, int n, uint32_t f0,
                               const float inv_transposed_view[16], int nabla_map, float* feat, cudaStream_t s) {
    Mat4 M;
    for (int k = 0; k < 16; k++) M.m[k] = inv_transposed_view[k];
    depth_deriv_kernel<<<(n + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float4*>(frame_normals), frames, n, f0,
                                                       M, nabla_map, feat);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
__global__ void feature_to_chw_kernel(const float* __restrict__ feat, int n, float inv_frames, int feature,
                                      int channels, float a0, float a1, float a2, float far_distance,
                                      float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* f = feat + (size_t)i * kFeatStride;
    float v[4] = {0, 0, 0, 0};
    float hit = f[kFeatPos + 3] * inv_frames;
    switch (feature) {
        case VPT_FEATURE_FIRST_X:
            v[0] = f[kFeatPos] * inv_frames;
            v[1] = f[kFeatPos + 1] * inv_frames;
            v[2] = f[kFeatPos + 2] * inv_frames;
            v[3] = hit;
            break;
        case VPT_FEATURE_NORMAL:
            v[0] = f[kFeatNormal] * inv_frames;
            v[1] = f[kFeatNormal + 1] * inv_frames;
            v[2] = f[kFeatNormal + 2] * inv_frames;
            v[3] = 1.0f;
            break;
        case VPT_FEATURE_NORMAL_LEN_1: {  // NormalizeNormals.glsl: rgb / length when length > 1e-5
            v[0] = f[kFeatNormal] * inv_frames;
            v[1] = f[kFeatNormal + 1] * inv_frames;
            v[2] = f[kFeatNormal + 2] * inv_frames;
            const float len = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            if (len > 1e-5f) {
                v[0] /= len;
                v[1] /= len;
                v[2] /= len;
            }
            v[3] = 1.0f;
            break;
        }
        case VPT_FEATURE_DEPTH_FAR:  // Clouds.glsl:219-227: mean of (event ? depth : far distance)
            v[0] = f[kFeatDepth] * inv_frames + (1.0f - hit) * far_distance;
            break;
        case VPT_FEATURE_DEPTH_BLENDED:  // Clouds.glsl:367-374: (depth, alpha, 0, 1)
            v[0] = f[kFeatDepthBlended] * inv_frames;
            v[1] = f[kFeatDepthBlended + 1] * inv_frames;
            v[3] = 1.0f;
            break;
        case VPT_FEATURE_DEPTH_NEAREST_OPAQUE:  // Clouds.glsl:376-383
            v[0] = f[kFeatDepthNearest] * inv_frames;
            v[1] = f[kFeatDepthNearest + 1] * inv_frames;
            v[3] = 1.0f;
            break;
        case VPT_FEATURE_BACKGROUND:  // Clouds.glsl:162-170 (alpha 1 for every sample)
            v[0] = f[kFeatBackground] * inv_frames;
            v[1] = f[kFeatBackground + 1] * inv_frames;
            v[2] = f[kFeatBackground + 2] * inv_frames;
            v[3] = 1.0f;
            break;
        case VPT_FEATURE_DEPTH: {
            float m = f[kFeatDepth] * inv_frames, m2 = f[kFeatDepth + 1] * inv_frames;
            v[0] = m;
            v[1] = sqrtf(fmaxf(0.0f, m2 - m * m));
            break;
        }
        case VPT_FEATURE_DENSITY: {
            float m = f[kFeatDensity] * inv_frames, m2 = f[kFeatDensity + 1] * inv_frames;
            v[0] = m;
            v[1] = sqrtf(fmaxf(0.0f, m2 - m * m));
            break;
        }
        case VPT_FEATURE_CLOUD_ONLY:
            v[0] = f[kFeatCloudOnly] * inv_frames;
            v[1] = f[kFeatCloudOnly + 1] * inv_frames;
            v[2] = f[kFeatCloudOnly + 2] * inv_frames;
            v[3] = hit;
            break;
        case VPT_FEATURE_ALBEDO:
            v[0] = a0 * hit;
            v[1] = a1 * hit;
            v[2] = a2 * hit;
            v[3] = hit;
            break;
        case VPT_FEATURE_FIRST_W:  // the last frame's values (not accumulated in the reference)
            v[0] = f[kFeatFirstW];
            v[1] = f[kFeatFirstW + 1];
            v[2] = f[kFeatFirstW + 2];
            v[3] = f[kFeatFirstW + 3];
            break;
        case VPT_FEATURE_FLOW:
            v[0] = f[kFeatFlow];
            v[1] = f[kFeatFlow + 1];
            break;
        case VPT_FEATURE_FLOW_REVERSE:
            v[0] = f[kFeatFlowReverse];
            v[1] = f[kFeatFlowReverse + 1];
            break;
        case VPT_FEATURE_DEPTH_NABLA:  // running means written by depth_deriv_kernel (imageStore(vec4(nabla, 0, 0)))
            v[0] = f[kFeatNabla];
            v[1] = f[kFeatNabla + 1];
            break;
        case VPT_FEATURE_DEPTH_FWIDTH:  // imageStore(depthFwidthImage, vec4(fwidthValue))
            v[0] = v[1] = v[2] = v[3] = f[kFeatFwidth];
            break;
        case VPT_FEATURE_REPROJ_UV: {  // (-1, -1) until a frame had an event (Clouds.glsl:240)
            const unsigned long long* key = reinterpret_cast<const unsigned long long*>(f + kFeatReprojUV);
            v[0] = (key[0] >> 32) != 0 ? __uint_as_float((uint32_t)key[0]) : -1.0f;
            v[1] = (key[1] >> 32) != 0 ? __uint_as_float((uint32_t)key[1]) : -1.0f;
            break;
        }
        default:  // VPT_FEATURE_TRANSMITTANCE
            v[0] = f[kFeatTrans] * inv_frames;
            break;
    }
    for (int c = 0; c < channels; c++) out[(size_t)c * n + i] = v[c];
}

cudaError_t feature_to_chw(const float* feat, int n, uint32_t frames, int feature, int channels, const float* albedo,
                           float far_distance, float* out, cudaStream_t stream) {
    switch (feature) {
        case VPT_FEATURE_FIRST_X:
        case VPT_FEATURE_NORMAL:
        case VPT_FEATURE_NORMAL_LEN_1:
        case VPT_FEATURE_DEPTH_FAR:
        case VPT_FEATURE_BACKGROUND:
        case VPT_FEATURE_DEPTH_BLENDED:
        case VPT_FEATURE_DEPTH_NEAREST_OPAQUE:
        case VPT_FEATURE_DEPTH:
        case VPT_FEATURE_DENSITY:
        case VPT_FEATURE_CLOUD_ONLY:
        case VPT_FEATURE_ALBEDO:
        case VPT_FEATURE_TRANSMITTANCE:
        case VPT_FEATURE_FIRST_W:
        case VPT_FEATURE_FLOW:
        case VPT_FEATURE_FLOW_REVERSE:
        case VPT_FEATURE_REPROJ_UV:
        case VPT_FEATURE_DEPTH_NABLA:
        case VPT_FEATURE_DEPTH_FWIDTH:
            break;
        default:
            return cudaErrorInvalidValue;
    }
    feature_to_chw_kernel<<<(n + 255) / 256, 256, 0, stream>>>(feat, n, 1.0f / float(frames), feature, channels,
                                                               albedo[0], albedo[1], albedo[2], far_distance, out);
    count_launches(1);
    return cudaGetLastError();
}

// The four feature planes a learned denoiser reads, in one pass over the feature accumulation:
// albedo (3 planes: the medium albedo times the hit fraction), normal (3), depth mean (1),
// transmittance (1), each output optional; the same values as feature_to_chw's first channels.
__global__ void denoiser_features_kernel(const float* __restrict__ feat, int n, float inv_frames, float a0, float a1,
                                         float a2, float* __restrict__ albedo, float* __restrict__ normal,
                                         float* __restrict__ depth, float* __restrict__ trans) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* f = feat + (size_t)i * kFeatStride;
    if (albedo) {
        const float hit = f[kFeatPos + 3] * inv_frames;
        albedo[i] = a0 * hit;
        albedo[(size_t)n + i] = a1 * hit;
        albedo[2 * (size_t)n + i] = a2 * hit;
    }
    if (normal) {
        normal[i] = f[kFeatNormal] * inv_frames;
        normal[(size_t)n + i] = f[kFeatNormal + 1] * inv_frames;
        normal[2 * (size_t)n + i] = f[kFeatNormal + 2] * inv_frames;
    }
    if (depth) depth[i] = f[kFeatDepth] * inv_frames;
    if (trans) trans[i] = f[kFeatTrans] * inv_frames;
}

cudaError_t denoiser_features(const float* feat, int n, uint32_t frames, const float* albedo_rgb, float* albedo,
                              float* normal, float* depth, float* trans, cudaStream_t stream) {
    denoiser_features_kernel<<<(n + 255) / 256, 256, 0, stream>>>(feat, n, 1.0f / float(frames), albedo_rgb[0],
                                                                  albedo_rgb[1], albedo_rgb[2], albedo, normal, depth,
                                                                  trans);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// EAW without allocation.
//
// vpt_eaw_denoise_rgba takes its ping-pong image from the stream-ordered allocator.  Some callers
// cannot allocate at that point: a frame loop that has already given nearly all device memory to
// the volume, the film and a framework's caching allocator (an allocation there fails mid-frame or
// makes the caching allocator release blocks and synchronise), and host engines that keep a fixed
// device-memory budget and do not let a library touch the allocator inside their render loop.
// For them, the ping-pong image lives in the fixed array below, which the library reserves on
// every GPU that loads it, for the life of the process.
//
// The array holds one RGBA fp32 image of at most kEawNoAllocMaxPixels pixels (16 MiB).  Every call
// on a device shares it and it keeps the previous call's contents.  Nothing in it has to start at
// zero: each a-trous iteration writes every pixel of its target image before the next iteration
// reads it.  Calls whose work overlaps on the GPU (other streams, other host threads) race on the
// array.
constexpr long long kEawNoAllocMaxPixels = 1024LL * 1024LL;
static __device__ __align__(256) float4 g_eaw_noalloc_scratch[kEawNoAllocMaxPixels];

// Device address of the array on the current device.  In host code the array's name only stands
// in for the symbol; the address comes from the runtime, once per device.  The first call on a
// device also uploads the tap weights (a synchronous copy), so it should come before any stream
// capture.
static cudaError_t eaw_noalloc_scratch(float** ptr) {
    static std::mutex mu;
    static float* addr[kMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_eaw_noalloc_scratch);
        if (e != cudaSuccess) return e;
        addr[dev] = static_cast<float*>(p);
    }
    *ptr = addr[dev];
    return cudaSuccess;
}

}  // namespace vpt

extern "C" VptStatus vpt_eaw_denoise_rgba_noalloc(const float* color, const float* position, const float* normal,
                                                  int width, int height, int iterations, float phi_color,
                                                  float phi_position, float phi_normal, int ref_compute_quirk,
                                                  float* out, void* stream) {
    if (!color || !out || width <= 0 || height <= 0 || iterations < 0) return VPT_ERR_ARG;
    if ((long long)width * (long long)height > vpt::kEawNoAllocMaxPixels) return VPT_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t bytes = (size_t)width * height * 4 * sizeof(float);
    if (vpt::image_ranges_overlap(out, color, bytes) || vpt::image_ranges_overlap(out, position, bytes) ||
        vpt::image_ranges_overlap(out, normal, bytes))
        return VPT_ERR_ARG;
    if (iterations == 0) {
        return cudaMemcpyAsync(out, color, bytes, cudaMemcpyDeviceToDevice, s) == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
    }
    float* scratch = nullptr;
    if (vpt::eaw_noalloc_scratch(&scratch) != cudaSuccess) return VPT_ERR_CUDA;
    vpt::EawSettings st;
    st.iterations = iterations;
    st.phi_color = phi_color;
    st.phi_position = phi_position;
    st.phi_normal = phi_normal;
    st.ref_compute_quirk = ref_compute_quirk;
    // The last iteration lands in `out`: odd counts start there, even counts start in the array.
    float* ping = (iterations % 2 == 1) ? out : scratch;
    float* pong = (iterations % 2 == 1) ? scratch : out;
    float* result = nullptr;
    cudaError_t e = vpt::eaw_denoise(color, position, normal, width, height, st, ping, pong, &result, s);
    return e == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

// One SVGF frame on caller-prepared maps and history (see include/vpt_b200.h).
extern "C" VptStatus vpt_svgf_filter(const float* noisy_rgba, const float* normal_rgba, const float* depth,
                                     const float* depth_fwidth, const float* motion, float* color_history,
                                     float* moments_history, float* normal_history, float* depth_history, int width,
                                     int height, float z_threshold, float normal_threshold, int iterations,
                                     float* out_rgba, void* stream) {
    if (!noisy_rgba || !normal_rgba || !depth || !depth_fwidth || !motion || !color_history || !moments_history ||
        !normal_history || !depth_history || !out_rgba || width <= 0 || height <= 0 || iterations < 0 ||
        iterations > 10)
        return VPT_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)width * height;
    float* scratch = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void**>(&scratch), n * 16 * 4, s) != cudaSuccess) return VPT_ERR_OOM;
    vpt::SvgfCur c;
    c.noisy = reinterpret_cast<float4*>(const_cast<float*>(noisy_rgba));
    c.normal = reinterpret_cast<float4*>(const_cast<float*>(normal_rgba));
    c.depth = const_cast<float*>(depth);
    c.fwidth = const_cast<float*>(depth_fwidth);
    c.motion = reinterpret_cast<float2*>(const_cast<float*>(motion));
    c.moments = reinterpret_cast<float4*>(scratch);
    c.temp = reinterpret_cast<float4*>(scratch + n * 4);
    c.ping = reinterpret_cast<float4*>(scratch + n * 8);
    c.pong = reinterpret_cast<float4*>(scratch + n * 12);
    vpt::SvgfSettings st;
    st.z_threshold = z_threshold;
    st.normal_threshold = normal_threshold;
    st.atrous_iterations = iterations;
    const float4* res = nullptr;
    cudaError_t e = vpt::svgf_filter_passes(c, reinterpret_cast<float4*>(color_history),
                                            reinterpret_cast<float4*>(moments_history),
                                            reinterpret_cast<float4*>(normal_history), depth_history, width, height, st,
                                            s, &res);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_rgba, res, n * 16, cudaMemcpyDeviceToDevice, s);
    cudaFreeAsync(scratch, s);
    return e == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}
