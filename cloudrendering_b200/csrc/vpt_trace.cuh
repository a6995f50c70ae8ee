// vpt_trace.cuh - the tracer kernels and their launch templates, shared by the vpt_trace_*.cu
// units.  Each unit instantiates the kernels of one tracker family (launch_tracker below), so
// that the families compile in parallel; vpt_kernels.cu dispatches to them (launch_trace).
//
//  * trace kernels: one camera path per thread; TRACKER x INTERP x GRID x TF are template
//    parameters (the reference selects them with shader #defines, VolumetricPathTracingPass.cpp:
//    1558-1782).  Three schedules: a plain grid over 16x16 pixel tiles, a persistent grid whose
//    warps pull 32-path batches from a global counter, and the per-lane refill loop.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "vpt_device.cuh"
#include "vpt_trackers.cuh"
#include "vpt_kernels.h"

namespace vpt {


// Density access of the trackers: the dense texture or the sparse (NanoVDB) volume.
// TF: transfer-function variant (density = the table's alpha); compiled only where a table is in
// use, so that the ordinary lookup carries no check of its own
template <int INTERP, int GRID, bool TF = false>
struct Sampler {
    const TraceParams& P;
    F3 tf_rgb = {0.0f, 0.0f, 0.0f};  // transfer-function colour of the last lookup
    static constexpr bool kSparse = GRID == kNanoVdb;
    // a lookup that draws no random number and reads the density itself (trilinear, dense, no
    // transfer function): two lookups at one point return the same value
    static constexpr bool kRepeatable = INTERP == kTrilinear && GRID != kNanoVdb && !TF;
    VPT_DEV float operator()(F3 pos, Rng& rng) {
        float v;
        if constexpr (GRID == kNanoVdb) v = sample_sparse<INTERP>(P, pos, rng);
        else if constexpr (GRID == kDenseTex) v = sample_dense_tex<INTERP>(P, pos, rng);
        else v = sample_dense<INTERP>(P, pos, rng);
        if constexpr (TF) {  // sampleCloud with USE_TRANSFER_FUNCTION: the table's alpha at the density
            float a;
            tf_lookup(P, v, tf_rgb, a);
            return a;
        }
        return v;
    }
    // transfer-function emission of the last lookup (parameters.emissionStrength * densityEmission.rgb)
    VPT_DEV F3 tf_emission() const {
        return f3(P.emission_strength * tf_rgb.x, P.emission_strength * tf_rgb.y, P.emission_strength * tf_rgb.z);
    }
    // the emission grid is dense whatever the density grid is
    VPT_DEV F3 emission(F3 pos, Rng& rng) const { return sample_emission<INTERP>(P, pos, rng); }
    VPT_DEV F3 normal(F3 pos, Rng& rng, const FirstEvent* fe = nullptr) const {
        // getCloudFiniteDifference returns 0 for NanoVDB grids (VptUtils.glsl:726-729)
        if constexpr (GRID == kNanoVdb) return f3(0.0f, 0.0f, 0.0f);
        // CLOSE_ISOSURFACES: a surface hit as the first event writes its own normal (Clouds.glsl:266-272)
        else if (P.iso && P.iso_close && fe && fe->iso) return fe->n;
        // with isosurfaces the normal map is -computeGradient at the first event (Clouds.glsl:274-275)
        else if (P.iso) return -iso_normal(P, pos);
        else return density_normal<INTERP>(P, pos, rng);
    }
};

// Depth Blended (DepthBlended.glsl) / Depth Nearest Opaque (DepthNearestOpaque.glsl): a march along
// the camera ray in steps of 0.25 / the largest grid dimension (0.001 for NanoVDB grids) with
// alpha = 1 - exp(-density * extinction * step), stopping past the box or above 0.999 accumulated
// alpha A.  Blended: (sum of (1 - A) alpha t / max(A, 1e-5), A); nearest: (t of the last step with
// alpha > 1e-5, times A; A).  Lookups continue the path's random stream (stochastic interpolation).
template <bool NEAREST, class S>
VPT_DEV void depth_march(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, float& depth_out, float& alpha_out) {
    const float step = S::kSparse ? 0.001f : 0.25f / (float)max(P.nx, max(P.ny, P.nz));
    const float atten = P.extinction * step;
    float acc_depth = 0.0f, acc_alpha = 0.0f, nearest = 0.0f;
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        float t = tmin;
        while (true) {
            t += step;
            if (t > tmax || acc_alpha > 0.999f) break;
            const float density = sample(x + w * t, rng);
            const float alpha = 1.0f - expf(-density * atten);
            if (!NEAREST) acc_depth = acc_depth + (1.0f - acc_alpha) * alpha * t;
            acc_alpha = acc_alpha + (1.0f - acc_alpha) * alpha;
            if (NEAREST && alpha > 1e-5f) nearest = t;
        }
    }
    depth_out = NEAREST ? nearest * acc_alpha : acc_depth / fmaxf(acc_alpha, 1e-5f);
    alpha_out = acc_alpha;
}

// Per-path feature accumulation (Clouds.glsl:148-256): position of the first event, depth,
// density, albedo-weighted hit flag, primary-ray transmittance proxy and, when requested, the
// background (Clouds.glsl:162-170: sampleSkybox of the camera ray for paths with an event, the
// path's radiance otherwise).
// previousViewProjMatrix * (v, vw), column-major, columns summed in order
VPT_DEV void prev_clip(const TraceParams& P, F3 v, float vw, float out[4]) {
    const float* m = P.prev_view_proj;
#pragma unroll
    for (int r = 0; r < 4; r++) out[r] = ((m[r] * v.x + m[4 + r] * v.y) + m[8 + r] * v.z) + m[12 + r] * vw;
}

// The maps the reference overwrites every frame (Clouds.glsl:239-246, 300-343), from the path of the
// frame that is traced last: First W (the direction after the first scatter and its pdf), Flow, Flow
// Reverse and Reprojected UV (which keeps an earlier frame's value when this frame has no event).
VPT_DEV void write_last_frame_features(const TraceParams& P, float* f, const FirstEvent& fe, int px, int py,
                                       F3 w_camera) {
    f[kFeatFirstW + 0] = fe.has ? fe.w.x : 0.0f;
    f[kFeatFirstW + 1] = fe.has ? fe.w.y : 0.0f;
    f[kFeatFirstW + 2] = fe.has ? fe.w.z : 0.0f;
    f[kFeatFirstW + 3] = fe.has ? fe.pdf_w : 0.0f;
    const float dw = (float)P.width, dh = (float)P.height;
    float c[4];
    float flow_x = 0.0f, flow_y = 0.0f;
    if (fe.has) {
        prev_clip(P, fe.x, 1.0f, c);
        const float nx = c[0] / c[3], ny = c[1] / c[3];
        flow_x = (float)px - ((0.5f * nx + 0.5f) * dw - 0.5f);
        flow_y = (float)py - ((0.5f * ny + 0.5f) * dh - 0.5f);
    }
    f[kFeatFlow + 0] = flow_x;
    f[kFeatFlow + 1] = flow_y;
    if (fe.has) prev_clip(P, fe.x, 1.0f, c);
    else prev_clip(P, w_camera, 0.0f, c);
    const float rx = c[0] / c[3], ry = c[1] / c[3];
    f[kFeatFlowReverse + 0] = ((0.5f * rx + 0.5f) * dw - 0.5f) - (float)px;
    f[kFeatFlowReverse + 1] = ((0.5f * ry + 0.5f) * dh - 0.5f) - (float)py;
}

// Reprojected UV (Clouds.glsl:240-246): prevClip.xy / prevClip.w * 0.5 + 0.5 of every frame's first
// event; the reference keeps the last frame's value, or an earlier one when the last frame has none.
// Frames of one pixel may run concurrently here, so each coordinate is a 64-bit key whose high word is
// the frame (+1) and whose low word the coordinate's bits, and atomicMax keeps the latest frame's.
VPT_DEV void update_reproj_uv(const TraceParams& P, float* f, const FirstEvent& fe, uint32_t global_frame) {
    float c[4];
    prev_clip(P, fe.x, 1.0f, c);
    const float u = (c[0] / c[3]) * 0.5f + 0.5f;
    const float v = (c[1] / c[3]) * 0.5f + 0.5f;
    const unsigned long long stamp = (unsigned long long)(global_frame + 1u) << 32;
    unsigned long long* key = reinterpret_cast<unsigned long long*>(f + kFeatReprojUV);
    atomicMax(key + 0, stamp | __float_as_uint(u));
    atomicMax(key + 1, stamp | __float_as_uint(v));
}

template <class S>
VPT_DEV void accumulate_features(const TraceParams& P, S& sample, Rng& rng, size_t pix, uint32_t frame,
                                 const FirstEvent& fe, F3 result, F3 x_camera, F3 w_camera) {
    float* f = P.feat + pix * kFeatStride;
    float4 frame_normal = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (P.feat_background) {
        const F3 bg = fe.has ? sky_only(P, w_camera) : result;
        atomicAdd(f + kFeatBackground + 0, bg.x);
        atomicAdd(f + kFeatBackground + 1, bg.y);
        atomicAdd(f + kFeatBackground + 2, bg.z);
    }
    if (fe.has) {
        F3 n = sample.normal(fe.x, rng, &fe);
        frame_normal = make_float4(n.x, n.y, n.z, 1.0f);
        atomicAdd(f + kFeatNormal + 0, n.x);
        atomicAdd(f + kFeatNormal + 1, n.y);
        atomicAdd(f + kFeatNormal + 2, n.z);
        atomicAdd(f + kFeatPos + 0, fe.x.x);
        atomicAdd(f + kFeatPos + 1, fe.x.y);
        atomicAdd(f + kFeatPos + 2, fe.x.z);
        atomicAdd(f + kFeatPos + 3, 1.0f);
        atomicAdd(f + kFeatDepth + 0, fe.depth);
        atomicAdd(f + kFeatDepth + 1, fe.depth * fe.depth);
        atomicAdd(f + kFeatDensity + 0, fe.density * 0.001f);
        atomicAdd(f + kFeatDensity + 1, (fe.density * fe.density * 0.001f) * 0.001f);
        atomicAdd(f + kFeatCloudOnly + 0, result.x);
        atomicAdd(f + kFeatCloudOnly + 1, result.y);
        atomicAdd(f + kFeatCloudOnly + 2, result.z);
    } else {
        atomicAdd(f + kFeatTrans, 1.0f);
    }
    if (P.frame_normals) {
        const size_t npix = (size_t)P.width * P.height;
        reinterpret_cast<float4*>(P.frame_normals)[(size_t)frame * npix + pix] = frame_normal;
    }
    // after the normal, in the reference's order (Clouds.glsl:367-383)
    if (P.feat_depth_maps & 1) {
        float d, a;
        depth_march<false>(P, sample, rng, x_camera, w_camera, d, a);
        atomicAdd(f + kFeatDepthBlended + 0, d);
        atomicAdd(f + kFeatDepthBlended + 1, a);
    }
    if (P.feat_depth_maps & 2) {
        float d, a;
        depth_march<true>(P, sample, rng, x_camera, w_camera, d, a);
        atomicAdd(f + kFeatDepthNearest + 0, d);
        atomicAdd(f + kFeatDepthNearest + 1, a);
    }
}

template <int TRACKER, class S>
VPT_DEV F3 run_tracker(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe, PathCtx& pc) {
    if constexpr (TRACKER == kDeltaIso) return track_delta_iso(P, sample, rng, x, w, fe, pc);
    if (TRACKER == kDelta) return track_delta(P, sample, rng, x, w, fe, pc);
    if (TRACKER == kRatio) return track_ratio(P, sample, rng, x, w, fe, pc);
    if constexpr (TRACKER == kDecomposition) {
        if constexpr (S::kSparse) return track_decomposition_sparse(P, sample, rng, x, w, fe, pc);
        else return track_decomposition(P, sample, rng, x, w, fe, pc);
    }
    if (TRACKER == kResidualRatio) return track_residual_ratio(P, sample, rng, x, w, fe, pc);
    if constexpr (TRACKER == kResidualRatioNee) return track_residual_ratio_nee(P, sample, rng, x, w, fe, pc);
    if constexpr (TRACKER == kSpectralDelta) return track_delta_spectral<false>(P, sample, rng, x, w, fe, pc);
    if constexpr (TRACKER == kSpectralDeltaIso) return track_delta_spectral<true>(P, sample, rng, x, w, fe, pc);
    if constexpr (TRACKER == kNextEventIso) return track_nee_iso(P, sample, rng, x, w, fe, pc);
    if constexpr (TRACKER == kSpectralNextEventIso) return track_nee_spectral<false, true>(P, sample, rng, x, w, fe, pc);
    if constexpr (TRACKER == kSpectralNextEvent) return track_nee_spectral<false>(P, sample, rng, x, w, fe, pc);
    if constexpr (TRACKER == kSpectralNextEvent + 100) return track_nee_spectral<true>(P, sample, rng, x, w, fe, pc);
    if (TRACKER == kNextEvent + 100) return track_nee<true>(P, sample, rng, x, w, fe, pc);
    return track_nee<false>(P, sample, rng, x, w, fe, pc);
}

// Maps a path index to (frame, x, y): 16x16 pixel tiles, tiles row-major, frames outermost, so a
// warp traces a 16x2 pixel strip of one frame (coherent primary rays).
VPT_DEV bool decode_path(const TraceParams& P, uint64_t p, uint32_t& frame, int& x, int& y) {
    const uint32_t tiles_x = (uint32_t)(P.width + 15) >> 4;
    const uint32_t tiles_y = (uint32_t)(P.height + 15) >> 4;
    const uint64_t per_frame = (uint64_t)tiles_x * tiles_y * 256u;
    uint32_t q;
    if ((p | per_frame) < 0x100000000ull) {  // 32-bit division (a 64-bit one is a long software routine)
        const uint32_t p32 = (uint32_t)p, pf = (uint32_t)per_frame;
        frame = p32 / pf;
        q = p32 - frame * pf;
    } else {
        frame = (uint32_t)(p / per_frame);
        q = (uint32_t)(p - (uint64_t)frame * per_frame);
    }
    const uint32_t tile = q >> 8, within = q & 255u;
    const uint32_t ty = tile / tiles_x, tx = tile - ty * tiles_x;
    x = (int)(tx * 16u + (within & 15u));
    y = (int)(ty * 16u + (within >> 4));
    return frame < P.num_frames && x < P.width && y < P.height;
}

// One camera path: seed (Clouds.glsl:80-84), jittered NDC (Clouds.glsl:86), tracker, film.
template <int TRACKER, class S>
VPT_DEV void trace_one(const TraceParams& P, S& sample, uint32_t frame, int px, int py, bool features,
                       uint32_t& lookups, bool& guard_hit) {
    const uint32_t w_u = (uint32_t)P.width, h_u = (uint32_t)P.height;
    uint32_t seed = (P.global_frame + frame) * w_u * h_u + (uint32_t)px + (uint32_t)py * w_u;
    seed += P.seed_offset;
    Rng rng = rng_init(seed);
    float rx = rng_next(rng);
    float ry = rng_next(rng);
    float sx = (2.0f * ((float)px + rx)) / (float)P.width - 1.0f;
    float sy = (2.0f * ((float)py + ry)) / (float)P.height - 1.0f;
    F3 x, w;
    camera_ray(P, sx, sy, x, w);
    FirstEvent fe;
    fe.has = false;
    fe.iso = false;
    PathCtx pc;
    pc.steps = 0;
    pc.max_steps = P.max_steps;
    pc.lookups = 0;
    pc.guard_hit = false;
    F3 L = run_tracker<TRACKER>(P, sample, rng, x, w, fe, pc);
    const size_t pix = (size_t)py * P.width + px;
    atomicAdd(P.film + pix * 3 + 0, (double)L.x);
    atomicAdd(P.film + pix * 3 + 1, (double)L.y);
    atomicAdd(P.film + pix * 3 + 2, (double)L.z);
    if (P.film_sq) {
        atomicAdd(P.film_sq + pix * 3 + 0, (double)L.x * (double)L.x);
        atomicAdd(P.film_sq + pix * 3 + 1, (double)L.y * (double)L.y);
        atomicAdd(P.film_sq + pix * 3 + 2, (double)L.z * (double)L.z);
    }
    if (features) {
        accumulate_features(P, sample, rng, pix, frame, fe, L, x, w);
        if (fe.has) update_reproj_uv(P, P.feat + pix * kFeatStride, fe, P.global_frame + frame);
        if (frame + 1 == P.num_frames) write_last_frame_features(P, P.feat + pix * kFeatStride, fe, px, py, w);
    }
    lookups += pc.lookups;
    guard_hit |= pc.guard_hit;
}

VPT_DEV void flush_counters(const TraceParams& P, uint32_t paths, uint32_t lookups, bool guard_hit) {
    unsigned long long l = lookups;
    unsigned long long n = paths;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        l += __shfl_xor_sync(0xffffffffu, l, o);
        n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(P.counters + 0, n);
        atomicAdd(P.counters + 1, l);
    }
    if (guard_hit) atomicOr(P.error_flags, kErrIterLimit);
}

template <int TRACKER, int INTERP, int GRID, bool TF>
__global__ void __launch_bounds__(kTraceBlock) trace_tiles_kernel(const __grid_constant__ TraceParams P, int features) {
    Sampler<INTERP, GRID, TF> sample{P};
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t frame;
    int px, py;
    uint32_t lookups = 0, paths = 0;
    bool guard_hit = false;
    if (decode_path(P, p, frame, px, py)) {
        trace_one<TRACKER>(P, sample, frame, px, py, features != 0, lookups, guard_hit);
        paths = 1;
    }
    __syncwarp();
    flush_counters(P, paths, lookups, guard_hit);
}

template <int TRACKER, int INTERP, int GRID, bool TF>
__global__ void __launch_bounds__(kTraceBlock) trace_persistent_kernel(const __grid_constant__ TraceParams P,
                                                                       int features, uint64_t total) {
    Sampler<INTERP, GRID, TF> sample{P};
    const int lane = threadIdx.x & 31;
    uint32_t lookups = 0, paths = 0;
    bool guard_hit = false;
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(reinterpret_cast<unsigned long long*>(P.work_counter), 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        uint64_t p = base + lane;
        uint32_t frame;
        int px, py;
        if (p < total && decode_path(P, p, frame, px, py)) {
            trace_one<TRACKER>(P, sample, frame, px, py, features != 0, lookups, guard_hit);
            paths++;
        }
        __syncwarp();
    }
    flush_counters(P, paths, lookups, guard_hit);
}


// ---------------------------------------------------------------------------------------------
// Per-lane path refill schedule (delta, ratio and NEE trackers).
//
// Each loop iteration advances every live lane by ONE tentative collision.  A lane whose path ends
// (escape, absorption, bounce cap) writes the film and takes the next path id at the top of the
// next iteration, so the 32 lanes of a warp keep executing the same step code instead of waiting
// for the warp's longest path.  NEE shadow rays are a second mode of the same step: the free-path
// sample and the density lookup are shared code for primary and shadow lanes.  Random numbers are
// drawn in exactly the order of the recursive trackers (vpt_trackers.cuh), so every path is the same
// path.  Path ids come from a global counter in warp batches of 64 (one atomic per 64 paths).
enum : int { kModePrimary = 0, kModeShadow = 1, kModeShadowEss = 2 };

// Block walk of shadow_transmittance_ess (NeeTransmittance.glsl:173-228): the block of the entry
// point, and the next block from the exit point (the axis of the largest offset from the block centre).
VPT_DEV void ess_first_block(const TraceParams& P, F3 x, int& bx, int& by, int& bz) {
    const F3 delta = P.box_max - P.box_min;
    const F3 sp = (((x - P.box_min) / delta) * f3((float)P.nx, (float)P.ny, (float)P.nz)) /
                  f3((float)P.sv_size, (float)P.sv_size, (float)P.sv_size);
    bx = (int)floorf(sp.x);
    by = (int)floorf(sp.y);
    bz = (int)floorf(sp.z);
}

VPT_DEV void ess_next_block(const TraceParams& P, F3 x, F3 w, int& bx, int& by, int& bz) {
    const F3 smin = P.box_min + f3((float)bx, (float)by, (float)bz) * P.sv_world;
    const F3 smax = smin + P.sv_world;
    const F3 center = (smin + smax) * 0.5f;
    F3 mov = (x + w * 0.00001f) - center;
    const float sx = signf(mov.x), sy = signf(mov.y), sz = signf(mov.z);
    mov = f3(mov.x * sx, mov.y * sy, mov.z * sz);
    const int dx = (mov.x >= mov.y && mov.x >= mov.z) ? 1 : 0;
    const int dy = (mov.y >= mov.x && mov.y >= mov.z) ? 1 : 0;
    const int dz = (mov.z >= mov.x && mov.z >= mov.y) ? 1 : 0;
    bx += dx * (int)sx;
    by += dy * (int)sy;
    bz += dz * (int)sz;
}
constexpr int kRefillBatch = 64;

template <int TRACKER>
VPT_DEV void refill_finish(const TraceParams& P, size_t pix, F3 L, bool& has) {
    atomicAdd(P.film + pix * 3 + 0, (double)L.x);
    atomicAdd(P.film + pix * 3 + 1, (double)L.y);
    atomicAdd(P.film + pix * 3 + 2, (double)L.z);
    if (P.film_sq) {
        atomicAdd(P.film_sq + pix * 3 + 0, (double)L.x * (double)L.x);
        atomicAdd(P.film_sq + pix * 3 + 1, (double)L.y * (double)L.y);
        atomicAdd(P.film_sq + pix * 3 + 2, (double)L.z * (double)L.z);
    }
    has = false;
}

// Shadow ray done: add the light sample (f = weight * T with weight = pdf_phase / pdf_light for the
// sky, or the light probability factor times pdf_phase for a light; NextEventTracking.glsl:348-369)
// and resume the primary path at the scatter point with the sampled direction.
VPT_DEV void end_shadow(const TraceParams& P, F3& color, F3& x, F3& w, float& d, F3 xp, F3 nw, float dp,
                        float weight, float ts, int light, int& mode) {
    const float f = weight * ts;
    const F3 l = light >= 0 ? light_radiance(P, xp, light) : sky_and_sun(P, w);
    color = color + f3(f * l.x, f * l.y, f * l.z);
    x = xp;
    w = nw;
    d = dp;
    mode = kModePrimary;
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        d = tmax - tmin;
    }
}

// Where the parameters of a path come from: one scene (the kernel's constant parameter block) or a
// batch of scenes in global memory whose path ids are concatenated scene after scene.
struct OneScene {
    const TraceParams& P;
    VPT_DEV const TraceParams& scene(int) const { return P; }
    VPT_DEV int locate(unsigned long long&) const { return 0; }
};
struct SceneBatch {
    const TraceParams* scenes;
    const unsigned long long* offsets;  // num + 1 prefix sums of the scenes' path counts
    int num;
    VPT_DEV const TraceParams& scene(int s) const { return scenes[s]; }
    // scene of global path id p (binary search); p becomes the scene-local id
    VPT_DEV int locate(unsigned long long& p) const {
        int lo = 0, hi = num - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(offsets + mid) <= p) lo = mid;
            else hi = mid - 1;
        }
        p -= __ldg(offsets + lo);
        return lo;
    }
};

VPT_DEV void flush_counters_to(unsigned long long* counters, int* error_flags, uint32_t paths, uint32_t lookups,
                               bool guard_hit) {
    unsigned long long l = lookups;
    unsigned long long n = paths;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        l += __shfl_xor_sync(0xffffffffu, l, o);
        n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counters + 0, n);
        atomicAdd(counters + 1, l);
    }
    if (guard_hit) atomicOr(error_flags, kErrIterLimit);
}

template <int TRACKER, int INTERP, int GRID, bool TF, class SRC>
VPT_DEV void refill_loop(const SRC& src, uint64_t total, unsigned long long* work_counter,
                         unsigned long long* counters, int* error_flags, int refill_min) {
    // next event tracking; kNextEvent + 100: its sky shadow rays skip the occupancy grid's empty blocks
    constexpr bool kNee = TRACKER == kNextEvent || TRACKER == kNextEvent + 100;
    constexpr bool kEss = TRACKER == kNextEvent + 100;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const F3 zero = f3(0.0f, 0.0f, 0.0f);

    // warp-uniform local batch of path ids
    unsigned long long q_base = 0;
    int q_left = 0;

    bool has = false, exhausted = false;
    Rng rng;
    F3 x = zero, w = zero, color = zero, xp = zero, nw = zero;
    float d = 0.0f, dp = 0.0f, trans = 1.0f, ts = 1.0f, weight = 0.0f;
    float shadow_dist = 0.0f, shadow_max = 0.0f;  // distance walked / light distance (light shadow rays)
    int mode = kModePrimary, bounces = 0, light = -1;
    bool ev = false;
    // isosurface state (kDeltaIso): surface throughput, sign at the first point after the last event,
    // loop iterations of the path
    F3 iw = f3(1.0f, 1.0f, 1.0f);
    float iso_last = 0.0f;
    bool iso_first = true;
    int iso_it = 0;
    // empty-space-skipping shadow ray (kEss), the walk of shadow_transmittance_ess one step per
    // iteration: current block, the block whose occupancy `empty` holds, inside an occupied block or
    // at a block boundary, distance sampled so far from the block entry x0, the block's length
    int bx = 0, by = 0, bz = 0, ox = 0, oy = 0, oz = 0;
    bool empty = false, in_block = false;
    float bt = 0.0f, bd = 0.0f;
    F3 bx0 = zero;
    // decomposition tracking (the same block walk): the block's normalised min / max density, its
    // control and residual extinctions and the control clock (bt is the residual clock)
    float dc_min = 0.0f, dc_max = 0.0f, mu_c = 1.0f, mu_r = 1.0f, t_c = 0.0f;
    // unbiased residual ratio tracking: the Amanatides-Woo supervoxel walk of the current free flight
    // or shadow ray (started lazily), its axis and cell, the distance reached, the walk's length
    SvWalk sw;
    bool walking = false;
    int wa = 0;
    float4 wc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float wt0 = 0.0f, wt1 = 0.0f, wlen = 0.0f;
    int scene = 0;
    uint32_t steps = 0;
    size_t pix = 0;
    uint32_t lookups = 0, paths = 0;
    bool guard_hit = false;

    while (true) {
        // ---- refill lanes without a path ----
        const bool need = !has && !exhausted;
        const unsigned m = __ballot_sync(FULL, need);
        // refill once `refill_min` lanes wait (the refill step is the loop's longest and most divergent
        // code), or when no lane of the warp holds a path
        if (m && (refill_min <= 1 || __popc(m) >= refill_min || !__any_sync(FULL, has))) {
            const int n = __popc(m);
            const int r = __popc(m & lt_mask);
            unsigned long long fresh = 0;
            if (n > q_left) {
                unsigned long long b = 0;
                if (lane == 0) b = atomicAdd(work_counter, (unsigned long long)kRefillBatch);
                fresh = __shfl_sync(FULL, b, 0);
            }
            if (need) {
                unsigned long long p = r < q_left ? q_base + (unsigned long long)r
                                                  : fresh + (unsigned long long)(r - q_left);
                uint32_t frame;
                int px, py;
                const bool done = p >= total;
                int s = 0;
                if (!done) s = src.locate(p);
                const TraceParams& P = src.scene(s);
                if (done) {
                    exhausted = true;
                } else if (decode_path(P, p, frame, px, py)) {
                    scene = s;
                    const uint32_t w_u = (uint32_t)P.width, h_u = (uint32_t)P.height;
                    uint32_t seed = (P.global_frame + frame) * w_u * h_u + (uint32_t)px + (uint32_t)py * w_u;
                    seed += P.seed_offset;
                    rng = rng_init(seed);
                    float rx = rng_next(rng);
                    float ry = rng_next(rng);
                    float sx = (2.0f * ((float)px + rx)) / (float)P.width - 1.0f;
                    float sy = (2.0f * ((float)py + ry)) / (float)P.height - 1.0f;
                    camera_ray(P, sx, sy, x, w);
                    pix = (size_t)py * P.width + px;
                    paths++;
                    steps = 0;
                    bounces = 0;
                    trans = 1.0f;
                    color = zero;
                    ev = false;
                    mode = kModePrimary;
                    walking = false;
                    in_block = false;
                    iw = f3(1.0f, 1.0f, 1.0f);
                    iso_first = true;
                    iso_it = 0;
                    float tmin, tmax;
                    has = true;
                    if constexpr (TRACKER == kDecomposition) {
                        // analogDecompositionTracking: entry through the box shrunk by 1e-6, then the
                        // supervoxel walk (its first block's bounds are read)
                        const F3 eps = f3(1e-6f, 1e-6f, 1e-6f);
                        if (ray_box(P.box_min + eps, P.box_max - eps, x, w, tmin, tmax)) {
                            x = x + w * tmin;
                            ess_first_block(P, x, bx, by, bz);
                            ox = oy = oz = -1;
                            in_block = false;
                        } else {
                            F3 L = sky_and_sun(P, w);
                            refill_finish<TRACKER>(P, pix, L, has);
                        }
                    } else if (ray_box_p(P, x, w, tmin, tmax)) {
                        x = x + w * tmin;
                        d = tmax - tmin;
                    } else {
                        F3 L = sky_and_sun(P, w);
                        refill_finish<TRACKER>(P, pix, L, has);
                    }
                }
            }
            if (n > q_left) {
                q_base = fresh + (unsigned long long)(n - q_left);
                q_left = kRefillBatch - (n - q_left);
            } else {
                q_base += (unsigned long long)n;
                q_left -= n;
            }
        }
        if (!__any_sync(FULL, has)) {
            if (__all_sync(FULL, exhausted)) break;
            continue;
        }
        if (!has) continue;

        // ---- one tentative collision ----
        const TraceParams& P = src.scene(scene);
        Sampler<INTERP, GRID, TF> sample{P};
        if (TRACKER == kDeltaIso && ++iso_it == 1000) {
            refill_finish<TRACKER>(P, pix, zero, has);
            continue;
        }
        if (++steps > P.max_steps) {
            guard_hit = true;
            refill_finish<TRACKER>(P, pix, (kNee || TRACKER == kResidualRatioNee) ? color : zero, has);
            continue;
        }
        if constexpr (kEss) {
            if (mode == kModeShadowEss) {
                if (!in_block) {  // at a block boundary (or the entry point)
                    if (bx < 0 || by < 0 || bz < 0 || bx >= P.svx || by >= P.svy || bz >= P.svz) {
                        end_shadow(P, color, x, w, d, xp, nw, dp, weight, ts, light, mode);
                        continue;
                    }
                    const F3 smin = P.box_min + f3((float)bx, (float)by, (float)bz) * P.sv_world;
                    const F3 smax = smin + P.sv_world;
                    float tmin_sv = 0.0f, tmax_sv = 0.0f;
                    ray_box(smin, smax, x, w, tmin_sv, tmax_sv);
                    bd = tmax_sv - tmin_sv;
                    x = x + w * tmin_sv;
                    if (ox != bx || oy != by || oz != bz) {
                        empty = __ldg(P.occupancy + ((size_t)bz * P.svy + by) * P.svx + bx) == 0;
                        ox = bx;
                        oy = by;
                        oz = bz;
                    }
                    if (empty) {
                        x = x + w * bd;
                        ess_next_block(P, x, w, bx, by, bz);
                    } else {
                        bx0 = x;
                        bt = 0.0f;
                        in_block = true;
                    }
                    continue;
                }
                bt -= m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) * P.inv_extinction;
                if (bt >= bd) {
                    x = (P.ess_ref_compat ? x : bx0) + w * bd;
                    in_block = false;
                    ess_next_block(P, x, w, bx, by, bz);
                    continue;
                }
                const F3 xn = (P.ess_ref_compat ? x : bx0) + w * bt;
                const float dens = sample(xn, rng);
                lookups++;
                x = xn;
                ts *= 1.0f - dens;
                continue;
            }
        }
        if constexpr (TRACKER == kResidualRatioNee) {
            // track_residual_ratio_nee one step per iteration: a free flight by delta tracking with each
            // supervoxel's majorant, then at a scatter a shadow ray whose transmittance is residual
            // ratio tracking over the same walk (shadow_residual_ratio); a cell boundary or one
            // tentative collision per iteration
            if (!walking) {
                if (mode == kModePrimary) {
                    wlen = d;
                } else {  // shadow ray from xp along w (x == xp here), up to the light or the box exit
                    float tmin_s, tmax_s;
                    float len = -1.0f;
                    if (ray_box_p(P, x, w, tmin_s, tmax_s)) len = fminf(tmax_s, shadow_max) - tmin_s;
                    if (!(len > 0.0f)) {  // transmittance 1, no random numbers
                        goto rrt_shadow_done;
                    }
                    x = x + w * tmin_s;
                    wlen = len;
                }
                sv_walk_begin(P, x, w, sw);
                wt0 = 0.0f;
                in_block = false;
                walking = true;
            }
            if (!in_block) {  // entering a cell
                wa = sv_walk_axis(sw);
                wt1 = fminf(sw.next[wa], wlen);
                wc = sv_local_cell(P, sw);
                if (wc.w > 0.0f && wt1 > wt0) {
                    if (mode != kModePrimary) ts *= m_exp(-wc.x * (wt1 - wt0));
                    bt = wt0;
                    in_block = true;
                    continue;
                }
            } else {
                if (mode == kModePrimary) {
                    bt += free_path(rng, wc.w);
                    if (bt < wt1) {
                        const float dens = sample(x + w * bt, rng);
                        lookups++;
                        const float r = dens * wc.z;  // density / majorant density
                        const float xi = rng_next(rng);
                        if (xi < P.absorb_albedo * r) {
                            refill_finish<TRACKER>(P, pix, P.emission ? color + sample.emission(x + w * bt, rng) : color,
                                                   has);
                            continue;
                        }
                        if (xi < r) {  // scatter: next event estimate, then the next free flight
                            x = x + w * bt;
                            walking = false;
                            in_block = false;
                            if (P.max_bounces > 0 && ++bounces > P.max_bounces) {
                                refill_finish<TRACKER>(P, pix, color, has);
                                continue;
                            }
                            nw = sample_phase(rng, P.g, w);
                            ev = true;
                            bool to_light = false;
                            float prob_factor = 1.0f, pdf_light = 0.0f, light_dist = 0.0f;
                            int light_idx = 0;
                            if (P.num_lights > 0) {
                                to_light = P.env_is_black ? true : (rng_next(rng) > 0.5f);
                                prob_factor = P.env_is_black ? 1.0f : 2.0f;
                            }
                            F3 dir;
                            if (to_light) dir = light_direction(P, x, rng, light_idx, prob_factor, light_dist);
                            else dir = importance_sample_sky(P, rng, pdf_light);
                            const float pdf_phase = evaluate_phase(P.g, w, dir);
                            weight = to_light ? prob_factor * pdf_phase : (prob_factor * pdf_phase) / pdf_light;
                            light = to_light ? light_idx : -1;
                            shadow_max = to_light ? light_dist : INFINITY;
                            xp = x;
                            w = dir;
                            ts = 1.0f;
                            mode = kModeShadow;
                        }
                        continue;
                    }
                } else {
                    bt += free_path(rng, 1.0f / wc.y);
                    if (bt < wt1) {
                        const float dens = sample(x + w * bt, rng);
                        lookups++;
                        ts *= 1.0f - (P.extinction * dens - wc.x) * (1.0f / wc.y);
                        continue;
                    }
                }
                in_block = false;
            }
            // leaving the cell [wt0, wt1)
            if (wt1 < wlen) {
                wt0 = fmaxf(wt0, wt1);
                if (sv_walk_advance(P, sw, wa)) continue;
            }
            walking = false;
            if (mode == kModePrimary) {  // the flight left the box without a collision
                refill_finish<TRACKER>(P, pix, ev ? color : color + sky_and_sun(P, w), has);
                continue;
            }
        rrt_shadow_done:
            {
                const float f = weight * ts;
                const F3 l = light >= 0 ? light_radiance(P, xp, light) : sky_and_sun(P, w);
                color = color + f3(f * l.x, f * l.y, f * l.z);
                x = xp;
                w = nw;
                mode = kModePrimary;
                walking = false;
                in_block = false;
                float tmin_b, tmax_b;
                if (!ray_box_p(P, x, w, tmin_b, tmax_b)) {
                    refill_finish<TRACKER>(P, pix, color, has);
                    continue;
                }
                x = x + w * tmin_b;
                d = tmax_b - tmin_b;
            }
            continue;
        }
        if constexpr (TRACKER == kDecomposition) {
            // the supervoxel walk of track_decomposition, one block boundary or one step of the two
            // competing exponential clocks (control t_c, residual t_r) per iteration
            if (!in_block) {
                if (bx < 0 || by < 0 || bz < 0 || bx >= P.svx || by >= P.svy || bz >= P.svz) {
                    refill_finish<TRACKER>(P, pix, sky_and_sun(P, w), has);
                    continue;
                }
                const F3 smin = P.box_min + f3((float)bx, (float)by, (float)bz) * P.sv_world;
                const F3 smax = smin + P.sv_world;
                float tmin_sv = 0.0f, tmax_sv = 0.0f;
                ray_box(smin, smax, x, w, tmin_sv, tmax_sv);
                bd = tmax_sv - tmin_sv;
                x = x + w * tmin_sv;
                if (ox != bx || oy != by || oz != bz) {
                    const float2 mm = __ldg(reinterpret_cast<const float2*>(P.sv_data) +
                                            ((size_t)bz * P.svy + by) * P.svx + bx);
                    dc_min = mm.x;
                    dc_max = mm.y;
                    ox = bx;
                    oy = by;
                    oz = bz;
                }
                if (dc_max < 1e-5f) {
                    x = x + w * bd;
                    sv_step(smin, smax, x, w, bx, by, bz);
                } else {
                    mu_c = fmaxf(0.0000000001f, P.extinction * dc_min);
                    mu_r = fmaxf(0.0000000001f, P.extinction * dc_max - mu_c);
                    t_c = -m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_c;
                    bt = 0.0f;  // t_r
                    in_block = true;
                }
                continue;
            }
            bt -= m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_r;
            if (t_c >= bd && bt >= bd) {
                x = x + w * bd;
                in_block = false;
                const F3 smin = P.box_min + f3((float)bx, (float)by, (float)bz) * P.sv_world;
                sv_step(smin, smin + P.sv_world, x, w, bx, by, bz);
                continue;
            }
            const F3 xs = x + w * fminf(t_c, bt);
            bool collision;
            if (t_c <= bt) {
                collision = true;
            } else {
                const float dens = sample(xs, rng);
                lookups++;
                collision = rng_next(rng) * mu_r < P.extinction * dens - mu_c;
            }
            if (collision) {
                x = xs;
                if (rng_next(rng) < P.absorb_albedo) {
                    refill_finish<TRACKER>(P, pix, zero, has);
                    continue;
                }
                if (P.max_bounces > 0 && ++bounces > P.max_bounces) {
                    refill_finish<TRACKER>(P, pix, zero, has);
                    continue;
                }
                w = sample_phase(rng, P.g, w);
                bt = 0.0f;
                t_c = -m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_c;
                const F3 smin = P.box_min + f3((float)bx, (float)by, (float)bz) * P.sv_world;
                float tmin_sv = 0.0f, tmax_sv = 0.0f;
                ray_box(smin, smin + P.sv_world, x, w, tmin_sv, tmax_sv);
                bd = tmax_sv - tmin_sv;
            }
            continue;
        }
        const float t = free_path(rng, P.inv_extinction);
        bool escape = t > d;
        if (kNee && mode == kModeShadow && light >= 0) {
            shadow_dist += t;
            escape = escape || shadow_dist > shadow_max;
        }
        float density = 0.0f;
        if (!escape) {
            F3 xn = x + w * t;
            density = sample(xn, rng);
            lookups++;
            if constexpr (TRACKER == kDeltaIso) {
                float tmax_unused = 0.0f;
                if (iso_segment(P, sample, rng, x, xn, density, w, d, tmax_unused, iw, iso_last, iso_first, lookups,
                                nullptr)) {
                    if (iw.x < 1e-3f && iw.y < 1e-3f && iw.z < 1e-3f) refill_finish<TRACKER>(P, pix, zero, has);
                    continue;
                }
            }
            x = xn;
        }
        if (kNee && mode == kModeShadow) {
            if (!escape) {
                ts *= 1.0f - density;
                d -= t;
                continue;
            }
            end_shadow(P, color, x, w, d, xp, nw, dp, weight, ts, light, mode);
            continue;
        }
        if (escape) {
            F3 L;
            if (kNee) L = ev ? color : color + sky_and_sun(P, w);
            else if (TRACKER == kRatio) L = sky_and_sun(P, w) * trans;
            else if (TRACKER == kDeltaIso) L = iw * sky_and_sun(P, w);
            else L = sky_and_sun(P, w);
            refill_finish<TRACKER>(P, pix, L, has);
            continue;
        }
        const float xi = rng_next(rng);
        if (TRACKER != kRatio && xi < P.absorb_albedo * density) {
            // USE_EMISSION (NextEventTracking.glsl:296-301): the absorbed NEE path ends with the emission
            F3 L = zero;
            if (kNee) {
                L = P.emission ? color + sample.emission(x, rng) : (P.tf ? color + sample.tf_emission() : color);
            } else if (P.tf) {  // delta tracking (DeltaTracking.glsl:293-301)
                L = sample.tf_emission();
            }
            refill_finish<TRACKER>(P, pix, L, has);
            continue;
        }
        if (xi < density) {
            if (P.max_bounces > 0 && ++bounces > P.max_bounces) {
                refill_finish<TRACKER>(P, pix, kNee ? color : zero, has);
                continue;
            }
            float tmin, tmax;
            if (kNee) {
                nw = sample_phase(rng, P.g, w);
                ev = true;
                bool to_light = false;
                float prob_factor = 1.0f, pdf_light = 0.0f, light_dist = 0.0f;
                int light_idx = 0;
                if (P.num_lights > 0) {
                    to_light = P.env_is_black ? true : (rng_next(rng) > 0.5f);
                    prob_factor = P.env_is_black ? 1.0f : 2.0f;
                }
                F3 dir;
                if (to_light) dir = light_direction(P, x, rng, light_idx, prob_factor, light_dist);
                else dir = importance_sample_sky(P, rng, pdf_light);
                const float pdf_phase = evaluate_phase(P.g, w, dir);
                if (P.num_lights > 0) weight = to_light ? prob_factor * pdf_phase : (prob_factor * pdf_phase) / pdf_light;
                else weight = pdf_phase / pdf_light;
                light = to_light ? light_idx : -1;
                shadow_max = light_dist;
                xp = x;
                dp = d;
                w = dir;
                ts = 1.0f;
                mode = kModeShadow;
                if (kEss && !to_light) {
                    // shadow_transmittance_ess: entry through the box shrunk by 1e-6, the entry block is
                    // walked as occupied
                    const F3 eps = f3(1e-6f, 1e-6f, 1e-6f);
                    if (ray_box(P.box_min + eps, P.box_max - eps, x, w, tmin, tmax)) {
                        x = x + w * tmin;
                        ess_first_block(P, x, bx, by, bz);
                        ox = bx;
                        oy = by;
                        oz = bz;
                        empty = false;
                        in_block = false;
                        mode = kModeShadowEss;
                    } else {
                        end_shadow(P, color, x, w, d, xp, nw, dp, weight, ts, light, mode);
                    }
                    continue;
                }
                if (ray_box_p(P, x, w, tmin, tmax)) {
                    x = x + w * tmin;
                    d = tmax - tmin;
                    shadow_dist = tmin;
                } else {
                    // no shadow steps (and no random numbers), like calculateTransmittance
                    end_shadow(P, color, x, w, d, xp, nw, dp, weight, ts, light, mode);
                }
                continue;
            }
            if (TRACKER == kRatio) {
                float pa = P.absorb_albedo * density;
                float ps = P.albedo * density;
                trans *= 1.0f - pa / (pa + ps);
            }
            w = sample_phase(rng, P.g, w);
            if (ray_box_p(P, x, w, tmin, tmax)) {
                x = x + w * tmin;
                d = tmax - tmin;
            }
        } else {
            d -= t;
        }
    }
    flush_counters_to(counters, error_flags, paths, lookups, guard_hit);
}

template <int TRACKER, int INTERP, int GRID, bool TF>
__global__ void __launch_bounds__(kTraceBlock) trace_refill_kernel(const __grid_constant__ TraceParams P, uint64_t total) {
    refill_loop<TRACKER, INTERP, GRID, TF>(OneScene{P}, total, reinterpret_cast<unsigned long long*>(P.work_counter),
                                       P.counters, P.error_flags, P.refill_min);
}

// Many independent scenes (own grid, camera, image size, spp, medium) traced by one persistent
// launch: lanes refill from one id space that concatenates the scenes' paths.  The total path count
// is read from offsets[num], so a captured launch serves any frame counts.
template <int TRACKER, int INTERP, int GRID>
__global__ void __launch_bounds__(kTraceBlock) trace_batch_kernel(const TraceParams* __restrict__ scenes,
                                                                  const unsigned long long* __restrict__ offsets,
                                                                  int num, unsigned long long* work_counter,
                                                                  unsigned long long* counters, int* error_flags) {
    refill_loop<TRACKER, INTERP, GRID, false>(SceneBatch{scenes, offsets, num}, __ldg(offsets + num), work_counter, counters,
                                       error_flags, scenes[0].refill_min);
}


template <int TRACKER, int INTERP, int GRID>
static cudaError_t batch_t(const BatchLaunch& b, cudaStream_t s) {
    if (b.blocks_per_sm_out) {
        int per_sm = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_batch_kernel<TRACKER, INTERP, GRID>,
                                                                      kTraceBlock, 0);
        *b.blocks_per_sm_out = per_sm > 0 ? per_sm : 1;
        return e;
    }
    trace_batch_kernel<TRACKER, INTERP, GRID><<<b.blocks, kTraceBlock, 0, s>>>(b.scenes, b.offsets, b.num,
                                                                              b.work_counter, b.counters,
                                                                              b.error_flags);
    if (b.counted) count_launches(1);
    return cudaGetLastError();
}

template <int TRACKER, int GRID>
static cudaError_t batch_interp(const BatchLaunch& b, cudaStream_t s) {
    switch (b.interp) {
        case kNearest: return batch_t<TRACKER, kNearest, GRID>(b, s);
        case kStochastic: return batch_t<TRACKER, kStochastic, GRID>(b, s);
        default: return batch_t<TRACKER, kTrilinear, GRID>(b, s);
    }
}

template <int GRID>
static cudaError_t batch_tracker(const BatchLaunch& b, cudaStream_t s) {
    switch (b.tracker) {
        case kDelta: return batch_interp<kDelta, GRID>(b, s);
        case kRatio: return batch_interp<kRatio, GRID>(b, s);
        case kNextEvent: return batch_interp<kNextEvent, GRID>(b, s);
        default: return cudaErrorNotSupported;
    }
}
template <int TRACKER, int INTERP, int GRID, bool TF>
static int refill_blocks(int requested) {
    if (requested > 0) return requested;
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_refill_kernel<TRACKER, INTERP, GRID, TF>, kTraceBlock,
                                                      0);
        if (per_sm <= 0) per_sm = 1;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return per_sm * sms;
}

template <int TRACKER, int INTERP, int GRID, bool TF>
static cudaError_t launch_trace_t(const TraceParams& P, int schedule, int features, int persistent_blocks,
                                  cudaStream_t stream) {
    uint64_t total = padded_paths(P.width, P.height, P.num_frames);
    constexpr bool kRefillable = TRACKER == kDelta || TRACKER == kRatio || TRACKER == kNextEvent ||
                                 TRACKER == kNextEvent + 100 || TRACKER == kDeltaIso ||
                                 ((TRACKER == kDecomposition || TRACKER == kResidualRatioNee) && GRID != kNanoVdb);
    // the refill loop's surface check has no closing surfaces (CLOSE_ISOSURFACES): persistent batches then
    if (schedule == kScheduleRefill && kRefillable && !features && !P.iso_close) {
        if constexpr (kRefillable) {
            int blocks = refill_blocks<TRACKER, INTERP, GRID, TF>(persistent_blocks);
            cudaMemsetAsync(P.work_counter, 0, sizeof(unsigned long long), stream);
            trace_refill_kernel<TRACKER, INTERP, GRID, TF><<<blocks, kTraceBlock, 0, stream>>>(P, total);
            count_launches(1);
            return cudaGetLastError();
        }
    }
    if (schedule == kScheduleRefill) schedule = kSchedulePersistent;
    if (schedule == kScheduleTiles) {
        uint64_t blocks = (total + kTraceBlock - 1) / kTraceBlock;
        trace_tiles_kernel<TRACKER, INTERP, GRID, TF><<<(unsigned)blocks, kTraceBlock, 0, stream>>>(P, features);
        count_launches(1);
    } else {
        if (persistent_blocks <= 0) {
            // one wave of resident blocks: SMs x blocks per SM from the occupancy calculator
            static int per_sm = 0;
            if (per_sm == 0) {
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_persistent_kernel<TRACKER, INTERP, GRID, TF>,
                                                              kTraceBlock, 0);
                if (per_sm <= 0) per_sm = 1;
            }
            int dev = 0, sms = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            persistent_blocks = per_sm * sms;
        }
        cudaMemsetAsync(P.work_counter, 0, sizeof(unsigned long long), stream);
        trace_persistent_kernel<TRACKER, INTERP, GRID, TF><<<persistent_blocks, kTraceBlock, 0, stream>>>(P, features,
                                                                                                           total);
        count_launches(1);
    }
    return cudaGetLastError();
}

template <int TRACKER, int GRID, bool TF>
static cudaError_t launch_interp_tf(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s) {
    switch (P.interp) {
        case kNearest: return launch_trace_t<TRACKER, kNearest, GRID, TF>(P, schedule, features, pb, s);
        case kStochastic: return launch_trace_t<TRACKER, kStochastic, GRID, TF>(P, schedule, features, pb, s);
        default: return launch_trace_t<TRACKER, kTrilinear, GRID, TF>(P, schedule, features, pb, s);
    }
}

// transfer-function variants exist for the trackers whose transfer-function appearance the reference
// defines (delta, next event and the spectral trackers); the others reject a table
template <int TRACKER, int GRID>
static cudaError_t launch_interp(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s) {
    constexpr int base = TRACKER >= 100 ? TRACKER - 100 : TRACKER;
    constexpr bool kTfTracker =
        base == kDelta || base == kNextEvent || base == kSpectralDelta || base == kSpectralNextEvent;
    if (P.tf) {
        if constexpr (kTfTracker) return launch_interp_tf<TRACKER, GRID, true>(P, schedule, features, pb, s);
        else return cudaErrorNotSupported;
    }
    return launch_interp_tf<TRACKER, GRID, false>(P, schedule, features, pb, s);
}

// One tracker family on one grid kind: interpolation and transfer-function variants behind it.
// Defined (explicitly specialised) in the vpt_trace_*.cu unit of the family.
template <int TRACKER, int GRID>
cudaError_t launch_tracker(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s);

#define VPT_DECLARE_TRACKER(T, G) \
    template <>                  \
    cudaError_t launch_tracker<T, G>(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s)
#define VPT_DEFINE_TRACKER(T, G) \
    VPT_DECLARE_TRACKER(T, G) { return launch_interp<T, G>(P, schedule, features, pb, s); }
// The density read through the grid's 3D texture object: no transfer-function variant (the host does
// not pick these kernels with a transfer function).
#define VPT_DEFINE_TRACKER_TEX(T)                                                \
    VPT_DECLARE_TRACKER(T, kDenseTex) {                                          \
        if (P.tf || !P.density_tex) return cudaErrorNotSupported;                \
        return launch_interp_tf<T, kDenseTex, false>(P, schedule, features, pb, s); \
    }

VPT_DECLARE_TRACKER(kDelta, kDense);
VPT_DECLARE_TRACKER(kDelta, kDenseTex);
VPT_DECLARE_TRACKER(kDelta, kNanoVdb);
VPT_DECLARE_TRACKER(kRatio, kDense);
VPT_DECLARE_TRACKER(kRatio, kDenseTex);
VPT_DECLARE_TRACKER(kRatio, kNanoVdb);
VPT_DECLARE_TRACKER(kDecomposition, kDense);
VPT_DECLARE_TRACKER(kDecomposition, kDenseTex);
VPT_DECLARE_TRACKER(kDecomposition, kNanoVdb);
VPT_DECLARE_TRACKER(kResidualRatio, kDense);
VPT_DECLARE_TRACKER(kResidualRatioNee, kDense);
VPT_DECLARE_TRACKER(kResidualRatioNee, kDenseTex);
VPT_DECLARE_TRACKER(kNextEvent, kDense);
VPT_DECLARE_TRACKER(kNextEvent, kDenseTex);
VPT_DECLARE_TRACKER(kNextEvent + 100, kDense);
VPT_DECLARE_TRACKER(kNextEvent + 100, kDenseTex);
VPT_DECLARE_TRACKER(kNextEvent, kNanoVdb);
VPT_DECLARE_TRACKER(kSpectralDelta, kDense);
VPT_DECLARE_TRACKER(kSpectralDelta, kNanoVdb);
VPT_DECLARE_TRACKER(kSpectralNextEvent, kDense);
VPT_DECLARE_TRACKER(kSpectralNextEvent + 100, kDense);
VPT_DECLARE_TRACKER(kSpectralNextEvent, kNanoVdb);
// delta tracking with isosurfaces: dense grids, trilinear lookups, no transfer function
cudaError_t launch_tracker_delta_iso(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s);
cudaError_t launch_tracker_spectral_delta_iso(const TraceParams& P, int schedule, int features, int pb,
                                              cudaStream_t s);
cudaError_t launch_tracker_nee_iso(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s);
cudaError_t launch_tracker_spectral_nee_iso(const TraceParams& P, int schedule, int features, int pb, cudaStream_t s);

}  // namespace vpt
