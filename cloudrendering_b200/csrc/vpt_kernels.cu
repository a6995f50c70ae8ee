// vpt_kernels.cu - CUDA kernels of the tracing path and their launchers.
//
//  * trace kernels: one camera path per thread; TRACKER x INTERP x FEATURES are template
//    parameters (the reference selects them with shader #defines, VolumetricPathTracingPass.cpp:
//    1558-1782).  Two schedules: a plain grid over 16x16 pixel tiles and a persistent grid whose
//    warps pull 32-path batches from a global counter (no block waits on its slowest warp).
//  * grid preparation: min/max reduction and normalisation (DensityField.cpp:136-154, 262-267),
//    seeded fBm scene generator, supervoxel and occupancy builders (SuperVoxelGrid.cpp,
//    ComputeOccupancyGrid.glsl), octahedral environment pyramid (OctahedralMapper.glsl).
//  * film readout: FP64 sums -> fp32 mean, channels x H x W.
#include <cuda_runtime.h>
#include <stdint.h>
#include "vpt_device.cuh"
#include "vpt_trackers.cuh"
#include "vpt_kernels.h"

namespace vpt {

// Number of kernels this library has launched (all launch sites below and in vpt_denoise.cu).
static unsigned long long g_launches = 0;
void count_launches(unsigned n) { __atomic_fetch_add(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }
unsigned long long launch_count() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

// Density access of the trackers: the dense texture or the sparse (NanoVDB) volume.
// TF: transfer-function variant (density = the table's alpha); compiled only where a table is in
// use, so that the ordinary lookup carries no check of its own
template <int INTERP, int GRID, bool TF = false>
struct Sampler {
    const TraceParams& P;
    F3 tf_rgb = {0.0f, 0.0f, 0.0f};  // transfer-function colour of the last lookup
    static constexpr bool kSparse = GRID == kNanoVdb;
    VPT_DEV float operator()(F3 pos, Rng& rng) {
        float v;
        if constexpr (GRID == kNanoVdb) v = sample_sparse<INTERP>(P, pos, rng);
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
    VPT_DEV F3 normal(F3 pos, Rng& rng) const {
        // getCloudFiniteDifference returns 0 for NanoVDB grids (VptUtils.glsl:726-729)
        if constexpr (GRID == kNanoVdb) return f3(0.0f, 0.0f, 0.0f);
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
    if (ray_box(P.box_min, P.box_max, x, w, tmin, tmax)) {
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
template <class S>
VPT_DEV void accumulate_features(const TraceParams& P, S& sample, Rng& rng, size_t pix, const FirstEvent& fe,
                                 F3 result, F3 x_camera, F3 w_camera) {
    float* f = P.feat + pix * kFeatStride;
    if (P.feat_background) {
        const F3 bg = fe.has ? sky_only(P, w_camera) : result;
        atomicAdd(f + kFeatBackground + 0, bg.x);
        atomicAdd(f + kFeatBackground + 1, bg.y);
        atomicAdd(f + kFeatBackground + 2, bg.z);
    }
    if (fe.has) {
        F3 n = sample.normal(fe.x, rng);
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
    if constexpr (TRACKER == kSpectralDelta) return track_delta_spectral(P, sample, rng, x, w, fe, pc);
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
    frame = (uint32_t)(p / per_frame);
    uint32_t q = (uint32_t)(p - (uint64_t)frame * per_frame);
    uint32_t tile = q >> 8, within = q & 255u;
    x = (int)((tile % tiles_x) * 16u + (within & 15u));
    y = (int)((tile / tiles_x) * 16u + (within >> 4));
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
    if (features) accumulate_features(P, sample, rng, pix, fe, L, x, w);
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
enum : int { kModePrimary = 0, kModeShadow = 1 };
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
    if (ray_box(P.box_min, P.box_max, x, w, tmin, tmax)) {
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
                         unsigned long long* counters, int* error_flags) {
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
    int scene = 0;
    uint32_t steps = 0;
    size_t pix = 0;
    uint32_t lookups = 0, paths = 0;
    bool guard_hit = false;

    while (true) {
        // ---- refill lanes without a path ----
        const bool need = !has && !exhausted;
        const unsigned m = __ballot_sync(FULL, need);
        if (m) {
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
                    iw = f3(1.0f, 1.0f, 1.0f);
                    iso_first = true;
                    iso_it = 0;
                    float tmin, tmax;
                    has = true;
                    if (ray_box(P.box_min, P.box_max, x, w, tmin, tmax)) {
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
            refill_finish<TRACKER>(P, pix, TRACKER == kNextEvent ? color : zero, has);
            continue;
        }
        const float t = free_path(rng, P.inv_extinction);
        bool escape = t > d;
        if (TRACKER == kNextEvent && mode == kModeShadow && light >= 0) {
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
        if (TRACKER == kNextEvent && mode == kModeShadow) {
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
            if (TRACKER == kNextEvent) L = ev ? color : color + sky_and_sun(P, w);
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
            if (TRACKER == kNextEvent) {
                L = P.emission ? color + sample.emission(x, rng) : (P.tf ? color + sample.tf_emission() : color);
            } else if (P.tf) {  // delta tracking (DeltaTracking.glsl:293-301)
                L = sample.tf_emission();
            }
            refill_finish<TRACKER>(P, pix, L, has);
            continue;
        }
        if (xi < density) {
            if (P.max_bounces > 0 && ++bounces > P.max_bounces) {
                refill_finish<TRACKER>(P, pix, TRACKER == kNextEvent ? color : zero, has);
                continue;
            }
            float tmin, tmax;
            if (TRACKER == kNextEvent) {
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
                if (ray_box(P.box_min, P.box_max, x, w, tmin, tmax)) {
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
            if (ray_box(P.box_min, P.box_max, x, w, tmin, tmax)) {
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
                                       P.counters, P.error_flags);
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
                                       error_flags);
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

cudaError_t launch_trace_batch(const BatchLaunch& b, cudaStream_t s) {
    return b.grid_kind == kNanoVdb ? batch_tracker<kNanoVdb>(b, s) : batch_tracker<kDense>(b, s);
}

uint64_t padded_paths(int width, int height, uint32_t frames) {
    uint64_t tiles = (uint64_t)((width + 15) / 16) * (uint64_t)((height + 15) / 16);
    return tiles * 256ull * frames;
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
    constexpr bool kRefillable = TRACKER == kDelta || TRACKER == kRatio || TRACKER == kNextEvent || TRACKER == kDeltaIso;
    if (schedule == kScheduleRefill && kRefillable && !features) {
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

cudaError_t launch_trace(const TraceParams& P, int tracker, int use_ess, int schedule, int features,
                         int persistent_blocks, cudaStream_t stream) {
    if (P.iso) {
        // isosurfaces: delta tracking on dense grids, trilinear lookups, no transfer function
        if (tracker != kDelta || P.grid_kind != kDense || P.tf) return cudaErrorNotSupported;
        return launch_trace_t<kDeltaIso, kTrilinear, kDense, false>(P, schedule, features, persistent_blocks, stream);
    }
    if (P.grid_kind == kNanoVdb) {
        // sparse grids: the trackers whose density access goes through sampleCloud, and the HDDA
        // decomposition tracker; residual ratio tracking and the occupancy grid are dense-only in the
        // reference (VolumetricPathTracingPass.cpp:1171-1186)
        switch (tracker) {
            case kDelta: return launch_interp<kDelta, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kRatio: return launch_interp<kRatio, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kDecomposition:
                return launch_interp<kDecomposition, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kNextEvent:
                if (use_ess) return cudaErrorNotSupported;
                return launch_interp<kNextEvent, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kSpectralDelta:
                return launch_interp<kSpectralDelta, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            case kSpectralNextEvent:
                if (use_ess) return cudaErrorNotSupported;
                return launch_interp<kSpectralNextEvent, kNanoVdb>(P, schedule, features, persistent_blocks, stream);
            default: return cudaErrorNotSupported;
        }
    }
    switch (tracker) {
        case kDelta: return launch_interp<kDelta, kDense>(P, schedule, features, persistent_blocks, stream);
        case kRatio: return launch_interp<kRatio, kDense>(P, schedule, features, persistent_blocks, stream);
        case kDecomposition: return launch_interp<kDecomposition, kDense>(P, schedule, features, persistent_blocks, stream);
        case kResidualRatio: return launch_interp<kResidualRatio, kDense>(P, schedule, features, persistent_blocks, stream);
        case kNextEvent:
            if (use_ess) return launch_interp<kNextEvent + 100, kDense>(P, schedule, features, persistent_blocks, stream);
            return launch_interp<kNextEvent, kDense>(P, schedule, features, persistent_blocks, stream);
        case kSpectralDelta: return launch_interp<kSpectralDelta, kDense>(P, schedule, features, persistent_blocks, stream);
        case kSpectralNextEvent:
            if (use_ess)
                return launch_interp<kSpectralNextEvent + 100, kDense>(P, schedule, features, persistent_blocks, stream);
            return launch_interp<kSpectralNextEvent, kDense>(P, schedule, features, persistent_blocks, stream);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------------------------
// Sparse volume queries (accessor checks against the reference's PNanoVDB).

__global__ void sparse_query_kernel(const __grid_constant__ SparseView v, const int* __restrict__ ijk, int count,
                                    float* __restrict__ values, uint32_t* __restrict__ dims,
                                    uint8_t* __restrict__ active) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int x = ijk[3 * i], y = ijk[3 * i + 1], z = ijk[3 * i + 2];
    values[i] = sparse_value(v, x, y, z);
    dims[i] = (uint32_t)sparse_dim(v, x, y, z);
    active[i] = sparse_is_active(v, x, y, z) ? 1 : 0;
}

cudaError_t launch_sparse_query(const SparseView& v, const int* ijk, int count, float* values, uint32_t* dims,
                                uint8_t* active, cudaStream_t s) {
    sparse_query_kernel<<<(count + 255) / 256, 256, 0, s>>>(v, ijk, count, values, dims, active);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Grid preparation.

__device__ __forceinline__ void atomic_min_float(float* addr, float v) {
    int* a = reinterpret_cast<int*>(addr);
    int old = *a;
    while (__int_as_float(old) > v) {
        int assumed = old;
        old = atomicCAS(a, assumed, __float_as_int(v));
        if (old == assumed) break;
    }
}
__device__ __forceinline__ void atomic_max_float(float* addr, float v) {
    int* a = reinterpret_cast<int*>(addr);
    int old = *a;
    while (__int_as_float(old) < v) {
        int assumed = old;
        old = atomicCAS(a, assumed, __float_as_int(v));
        if (old == assumed) break;
    }
}

// min/max over the raw grid (sgl::reduceFloatArrayMinMax semantics; order-independent, exact).
__global__ void minmax_kernel(const float* __restrict__ v, size_t n, float* out_minmax) {
    float lo = INFINITY, hi = -INFINITY;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float x = v[i];
        lo = fminf(lo, x);
        hi = fmaxf(hi, x);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __shared__ float slo[32], shi[32];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        slo[warp] = lo;
        shi[warp] = hi;
    }
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        lo = lane < nw ? slo[lane] : INFINITY;
        hi = lane < nw ? shi[lane] : -INFINITY;
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            atomic_min_float(out_minmax + 0, lo);
            atomic_max_float(out_minmax + 1, hi);
        }
    }
}

// (v - min) / (max - min), IEEE division as in DensityField::getDataFloatAtNorm.
__global__ void normalize_kernel(const float* __restrict__ in, float* __restrict__ out, size_t n, float vmin,
                                 float vmax) {
    const float range = vmax - vmin;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        out[i] = (in[i] - vmin) / range;
    }
}

// Improved Perlin noise (K. Perlin, "Improving Noise", SIGGRAPH 2002) with a seeded permutation;
// only +, -, *, floor, so the CPU oracle reproduces every value bit for bit.
struct PermTable {
    int p[512];
};

__device__ __forceinline__ float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
__device__ __forceinline__ float lerpf(float t, float a, float b) { return a + t * (b - a); }
__device__ __forceinline__ float grad(int h, float x, float y, float z) {
    h &= 15;
    float u = h < 8 ? x : y;
    float v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}

__device__ float perlin3(const int* __restrict__ p, float x, float y, float z) {
    float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
    x -= fx;
    y -= fy;
    z -= fz;
    float u = fade(x), v = fade(y), w = fade(z);
    int A = p[X] + Y, AA = p[A] + Z, AB = p[A + 1] + Z;
    int B = p[X + 1] + Y, BA = p[B] + Z, BB = p[B + 1] + Z;
    float r0 = lerpf(v, lerpf(u, grad(p[AA], x, y, z), grad(p[BA], x - 1.0f, y, z)),
                     lerpf(u, grad(p[AB], x, y - 1.0f, z), grad(p[BB], x - 1.0f, y - 1.0f, z)));
    float r1 = lerpf(v, lerpf(u, grad(p[AA + 1], x, y, z - 1.0f), grad(p[BA + 1], x - 1.0f, y, z - 1.0f)),
                     lerpf(u, grad(p[AB + 1], x, y - 1.0f, z - 1.0f), grad(p[BB + 1], x - 1.0f, y - 1.0f, z - 1.0f)));
    return lerpf(w, r0, r1);
}

__global__ void fbm_kernel(float* __restrict__ out, int nx, int ny, int nz, const __grid_constant__ PermTable perm,
                           FbmParams fp) {
    __shared__ int p[512];
    for (int i = threadIdx.x; i < 512; i += blockDim.x) p[i] = perm.p[i];
    __syncthreads();
    const size_t n = (size_t)nx * ny * nz;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int ix = (int)(i % (size_t)nx);
        int iy = (int)((i / (size_t)nx) % (size_t)ny);
        int iz = (int)(i / ((size_t)nx * ny));
        float px = ((float)ix + 0.5f) * fp.inv_max_dim;
        float py = ((float)iy + 0.5f) * fp.inv_max_dim;
        float pz = ((float)iz + 0.5f) * fp.inv_max_dim;
        float sum = 0.0f, amp = 1.0f, freq = fp.base_frequency, norm = 0.0f;
        for (int o = 0; o < fp.octaves; o++) {
            sum += amp * perlin3(p, px * freq, py * freq, pz * freq);
            norm += amp;
            amp *= fp.gain;
            freq *= fp.lacunarity;
        }
        float v = sum / norm;
        v = fminf(fmaxf(0.5f + fp.contrast * v, 0.0f), 1.0f);
        out[i] = v < fp.threshold ? 0.0f : v;
    }
}

// ---------------------------------------------------------------------------------------------
// Supervoxel grid: min / max / mean of the normalised density over each sv^3 block, with a one
// voxel halo unless the interpolation is NEAREST; voxels outside the grid count as 0 and a
// partial boundary supervoxel has min := 0 (SuperVoxelGrid.cpp:101-211, 316-396).  One thread
// per supervoxel accumulates the mean in the reference's z-y-x loop order, so the sum is
// bit-identical; min/max are order-independent.
__global__ void supervoxel_stats_kernel(const float* __restrict__ dens, int nx, int ny, int nz, int sv, int svx,
                                        int svy, int svz, int halo, float* __restrict__ out_min,
                                        float* __restrict__ out_max, float* __restrict__ out_avg,
                                        uint8_t* __restrict__ out_occ) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    int total = svx * svy * svz;
    if (idx >= total) return;
    int bx = idx % svx, by = (idx / svx) % svy, bz = idx / (svx * svy);
    float lo = 3.402823466e+38f, hi = -3.402823466e+38f, sum = 0.0f;
    int cnt = 0;
    int o0 = halo ? -1 : 0, o1 = halo ? sv : sv - 1;
    for (int oz = o0; oz <= o1; oz++) {
        int z = bz * sv + oz;
        for (int oy = o0; oy <= o1; oy++) {
            int y = by * sv + oy;
            for (int ox = o0; ox <= o1; ox++) {
                int x = bx * sv + ox;
                float v = 0.0f;
                if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) {
                    v = __ldg(dens + ((size_t)z * ny + y) * nx + x);
                }
                lo = fminf(lo, v);
                hi = fmaxf(hi, v);
                sum += v;
                cnt++;
            }
        }
    }
    float avg = sum / (float)cnt;
    if ((nx % sv != 0 && bx == svx - 1) || (ny % sv != 0 && by == svy - 1) || (nz % sv != 0 && bz == svz - 1)) {
        lo = 0.0f;
    }
    out_min[idx] = lo;
    out_max[idx] = hi;
    if (out_avg) out_avg[idx] = avg;
    if (out_occ) out_occ[idx] = hi < 1e-5f ? 0 : 1;
}

// Residual-ratio-tracking control and residual extinctions (SuperVoxelGrid.cpp:218-256):
// mu_r_bar = max(mu_max - mu_min, 0.1), mu_c = clamp(mu_min + mu_r_bar * gamma^(1/(D mu_r_bar) - 1),
// mu_min, mu_avg) with gamma = 2, D = sqrt(3) * sv.
__global__ void rrt_params_kernel(const float* __restrict__ mn, const float* __restrict__ mx,
                                  const float* __restrict__ avg, int total, float extinction, float D,
                                  float* __restrict__ out_pairs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    float mu_min = mn[i] * extinction, mu_max = mx[i] * extinction, mu_avg = avg[i] * extinction;
    float mu_r = fmaxf(mu_max - mu_min, 0.1f);
    float mu_c = mu_min + mu_r * m_pow(2.0f, (1.0f / (D * mu_r)) - 1.0f);
    mu_c = fminf(fmaxf(mu_c, mu_min), mu_avg);
    out_pairs[2 * i + 0] = mu_c;
    out_pairs[2 * i + 1] = mu_r;
}

__global__ void interleave_kernel(const float* __restrict__ a, const float* __restrict__ b, int total,
                                  float* __restrict__ out_pairs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    out_pairs[2 * i + 0] = a[i];
    out_pairs[2 * i + 1] = b[i];
}

// Occupancy grid for NEE empty-space skipping.  The reference shader's loop never executes
// (ComputeOccupancyGrid.glsl:108-109) so every block is marked occupied; `ref_compat` reproduces
// that.  Otherwise one warp per block votes whether any voxel of the block (plus a one-voxel halo
// for stochastic / trilinear lookups) exceeds `threshold`.
__global__ void occupancy_kernel(const float* __restrict__ dens, int nx, int ny, int nz, int bs, int gx, int gy,
                                 int gz, int halo, float threshold, int ref_compat, uint8_t* __restrict__ out) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int total = gx * gy * gz;
    if (warp >= total) return;
    if (ref_compat) {
        if (lane == 0) out[warp] = 1;
        return;
    }
    int bx = warp % gx, by = (warp / gx) % gy, bz = warp / (gx * gy);
    int ext = bs + 2 * halo;
    int n = ext * ext * ext;
    bool occ = false;
    for (int i = lane; i < n && !__any_sync(__activemask(), occ); i += 32) {
        int ox = i % ext - halo, oy = (i / ext) % ext - halo, oz = i / (ext * ext) - halo;
        int x = bx * bs + ox, y = by * bs + oy, z = bz * bs + oz;
        if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) {
            occ |= __ldg(dens + ((size_t)z * ny + y) * nx + x) > threshold;
        }
    }
    occ = __any_sync(0xffffffffu, occ);
    if (lane == 0) out[warp] = occ ? 1 : 0;
}

// ---------------------------------------------------------------------------------------------
// Octahedral max-luminance pyramid of the environment image (OctahedralMapper.glsl:65-85, then a
// 2x2 box reduction per level like vkCmdBlitImage mip generation).
__global__ void env_octahedral_level0_kernel(const __grid_constant__ TraceParams P, float* __restrict__ out, int res) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= res || y >= res) return;
    float best = -1.0f;
    for (int i = 0; i < 5; i++) {
        float sxo = 0.1f + 0.2f * (float)i;
        for (int j = 0; j < 5; j++) {
            float syo = 0.1f + 0.2f * (float)j;
            float u = ((float)x + sxo) / (float)res;
            float v = ((float)y + syo) / (float)res;
            F3 dir = octahedral_uv_to_world(u, v);
            float tu = m_atan2(dir.z, dir.x) / (2.0f * kPi) + 0.5f;
            float tv = -m_asin(dir.y) / kPi + 0.5f;
            F3 c = env_image_fetch(P, tu, tv);
            c = f3(fminf(c.x, 100000.0f), fminf(c.y, 100000.0f), fminf(c.z, 100000.0f));
            best = fmaxf(best, length3(c));
        }
    }
    out[(size_t)y * res + x] = best;
}

__global__ void env_downsample_kernel(const float* __restrict__ in, float* __restrict__ out, int res_out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= res_out || y >= res_out) return;
    int ri = res_out * 2;
    float a = in[(size_t)(2 * y) * ri + 2 * x], b = in[(size_t)(2 * y) * ri + 2 * x + 1];
    float c = in[(size_t)(2 * y + 1) * ri + 2 * x], d = in[(size_t)(2 * y + 1) * ri + 2 * x + 1];
    out[(size_t)y * res_out + x] = ((a + b) + (c + d)) * 0.25f;
}

// ---------------------------------------------------------------------------------------------
// Film readout: mean = sum / frames as channels x H x W (alpha = 1 for 4 channels).
__global__ void film_to_chw_kernel(const double* __restrict__ film, int width, int height, double inv_frames,
                                   int channels, float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = width * height;
    if (i >= n) return;
    for (int c = 0; c < 3; c++) out[(size_t)c * n + i] = (float)(film[(size_t)i * 3 + c] * inv_frames);
    if (channels == 4) out[(size_t)3 * n + i] = 1.0f;
}

__global__ void film_to_rgba_kernel(const double* __restrict__ film, int n, double inv_frames, float4* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4((float)(film[(size_t)i * 3 + 0] * inv_frames), (float)(film[(size_t)i * 3 + 1] * inv_frames),
                         (float)(film[(size_t)i * 3 + 2] * inv_frames), 1.0f);
}

__global__ void rgba_to_chw_kernel(const float4* __restrict__ in, int n, int channels, float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = in[i];
    out[i] = v.x;
    out[(size_t)n + i] = v.y;
    out[(size_t)2 * n + i] = v.z;
    if (channels == 4) out[(size_t)3 * n + i] = v.w;
}

// ---------------------------------------------------------------------------------------------
// Launchers (declared in vpt_kernels.h).

static unsigned grid_for(size_t n, int block, unsigned cap = 148u * 32u) {
    size_t g = (n + block - 1) / block;
    if (g > cap) g = cap;
    if (g == 0) g = 1;
    return (unsigned)g;
}

cudaError_t launch_minmax(const float* v, size_t n, float* out_minmax, cudaStream_t s) {
    float init[2] = {INFINITY, -INFINITY};
    cudaMemcpyAsync(out_minmax, init, sizeof(init), cudaMemcpyHostToDevice, s);
    minmax_kernel<<<grid_for(n, 256), 256, 0, s>>>(v, n, out_minmax);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_normalize(const float* in, float* out, size_t n, float vmin, float vmax, cudaStream_t s) {
    normalize_kernel<<<grid_for(n, 256), 256, 0, s>>>(in, out, n, vmin, vmax);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fbm(float* out, int nx, int ny, int nz, const int* perm512, const FbmParams& fp, cudaStream_t s) {
    PermTable t;
    for (int i = 0; i < 512; i++) t.p[i] = perm512[i];
    size_t n = (size_t)nx * ny * nz;
    fbm_kernel<<<grid_for(n, 256), 256, 0, s>>>(out, nx, ny, nz, t, fp);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_supervoxel_stats(const float* dens, int nx, int ny, int nz, int sv, int svx, int svy, int svz,
                                    int halo, float* mn, float* mx, float* avg, uint8_t* occ, cudaStream_t s) {
    int total = svx * svy * svz;
    supervoxel_stats_kernel<<<(total + 127) / 128, 128, 0, s>>>(dens, nx, ny, nz, sv, svx, svy, svz, halo, mn, mx,
                                                                avg, occ);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_rrt_params(const float* mn, const float* mx, const float* avg, int total, float extinction,
                              float D, float* out_pairs, cudaStream_t s) {
    rrt_params_kernel<<<(total + 255) / 256, 256, 0, s>>>(mn, mx, avg, total, extinction, D, out_pairs);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_interleave(const float* a, const float* b, int total, float* out_pairs, cudaStream_t s) {
    interleave_kernel<<<(total + 255) / 256, 256, 0, s>>>(a, b, total, out_pairs);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_occupancy(const float* dens, int nx, int ny, int nz, int bs, int gx, int gy, int gz, int halo,
                             float threshold, int ref_compat, uint8_t* out, cudaStream_t s) {
    int total = gx * gy * gz;
    size_t threads = (size_t)total * 32;
    occupancy_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(dens, nx, ny, nz, bs, gx, gy, gz, halo,
                                                                       threshold, ref_compat, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_env_pyramid(const TraceParams& P, float* pyramid, const uint64_t* level_offsets_host, int levels,
                               cudaStream_t s) {
    int res = 1 << levels;
    dim3 b(16, 16);
    env_octahedral_level0_kernel<<<dim3((res + 15) / 16, (res + 15) / 16), b, 0, s>>>(P, pyramid, res);
    count_launches((unsigned)levels);
    for (int l = 1; l < levels; l++) {
        int r = res >> l;
        env_downsample_kernel<<<dim3((r + 15) / 16, (r + 15) / 16), b, 0, s>>>(
            pyramid + level_offsets_host[l - 1], pyramid + level_offsets_host[l], r);
    }
    return cudaGetLastError();
}

cudaError_t launch_film_to_chw(const double* film, int width, int height, double inv_frames, int channels,
                               float* out, cudaStream_t s) {
    int n = width * height;
    film_to_chw_kernel<<<(n + 255) / 256, 256, 0, s>>>(film, width, height, inv_frames, channels, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_film_to_rgba(const double* film, int n, double inv_frames, float* out_rgba, cudaStream_t s) {
    film_to_rgba_kernel<<<(n + 255) / 256, 256, 0, s>>>(film, n, inv_frames, reinterpret_cast<float4*>(out_rgba));
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_rgba_to_chw(const float* rgba, int n, int channels, float* out, cudaStream_t s) {
    rgba_to_chw_kernel<<<(n + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float4*>(rgba), n, channels, out);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace vpt
