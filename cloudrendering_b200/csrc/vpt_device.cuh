// vpt_device.cuh - device-side building blocks of the tracer: RNG, camera rays, box clipping,
// Henyey-Greenstein sampling, sky/sun models and dense-grid density lookups.
//
// Arithmetic conventions (identical in the CPU oracle, so that paths can be compared one by one):
//  * the parity build (libvpt_b200_dr.so) is compiled with --fmad=false: a*b+c is two IEEE-rounded
//    operations, as in the oracle; the product build contracts them into FMAs (a last-ulp difference
//    per operation, which changes the random decisions of a small fraction of paths only);
//  * divisions and square roots are IEEE-rounded (-prec-div/-prec-sqrt default true);
//  * the reference's per-step ratios are written in closed form: with majorant == extinction.x,
//    Pa = (1 - albedo) * density and 1 - Pn = density (DeltaTracking.glsl:262-268);
//  * world -> voxel coordinates use one multiply by voxels-per-unit, (pos - boxMin) * (N / extent),
//    and the stochastic jitter is added in voxel units (VptUtils.glsl:585-591 does the same in
//    texture units).
#pragma once
#include <stdint.h>
#include <math.h>
#include "vpt_params.h"

namespace vpt {

#define VPT_DEV __device__ __forceinline__

constexpr float kPi = 3.14159265359f;        // VptUtils.glsl:27
constexpr float kTwoPi = 2.0f * 3.14159265359f;

// Transcendental functions of the tracer.  By default they are CUDA's single-precision functions,
// which can differ from a CPU C library by an ulp on some arguments.  With VPT_DOUBLE_ROUNDED_MATH
// (the library variant libvpt_b200_dr.so) each one is evaluated in double precision and rounded
// once to float.  The CPU oracle has the same mode: both sides then return the correctly rounded
// float except where the exact result lies within about one double ulp of a float rounding
// boundary (probability ~2^-29 per call), so paths of thousands of bounces can be compared one by
// one without an ulp difference flipping a later comparison.
#ifdef VPT_DOUBLE_ROUNDED_MATH
VPT_DEV float m_log(float x) { return (float)log((double)x); }
VPT_DEV float m_exp(float x) { return (float)exp((double)x); }
VPT_DEV float m_sin(float x) { return (float)sin((double)x); }
VPT_DEV float m_cos(float x) { return (float)cos((double)x); }
VPT_DEV float m_pow(float x, float y) { return (float)pow((double)x, (double)y); }
VPT_DEV float m_atan2(float y, float x) { return (float)atan2((double)y, (double)x); }
VPT_DEV float m_asin(float x) { return (float)asin((double)x); }
VPT_DEV float m_acos(float x) { return (float)acos((double)x); }
VPT_DEV float m_tan(float x) { return (float)tan((double)x); }
VPT_DEV float m_pow5(float x) { return (float)pow((double)x, 5.0); }
#elif defined(VPT_FAST_MATH)
// The product's tracer units (vpt_trace_*.cu): the special-function unit's approximations of log2,
// exp2, sin and cos (a few ulp; sin and cos to ~2^-21 absolute on the phase angles in [0, 2 pi)), the
// precision GLSL's log / exp / sin / cos / pow are allowed and get from a GPU driver.  Argument ranges
// here: log of (0, 1] (free paths), sin / cos of [0, 2 pi) (phase and sphere sampling), pow of
// non-negative bases.
VPT_DEV float m_log(float x) { return __logf(x); }
VPT_DEV float m_exp(float x) { return __expf(x); }
VPT_DEV float m_sin(float x) { return __sinf(x); }
VPT_DEV float m_cos(float x) { return __cosf(x); }
VPT_DEV float m_pow(float x, float y) { return __powf(x, y); }
VPT_DEV float m_atan2(float y, float x) { return atan2f(y, x); }
VPT_DEV float m_asin(float x) { return asinf(x); }
VPT_DEV float m_acos(float x) { return acosf(x); }
VPT_DEV float m_tan(float x) { return tanf(x); }  // near its poles (Disney's anisotropic sampling) __tanf is far off
// pow(x, 5.0) of the Fresnel term: its base 1 - cos can round to a tiny negative value, which the
// exp2(5 log2 x) form of __powf would turn into NaN
VPT_DEV float m_pow5(float x) { const float x2 = x * x; return x2 * x2 * x; }
#else
VPT_DEV float m_log(float x) { return logf(x); }
VPT_DEV float m_exp(float x) { return expf(x); }
VPT_DEV float m_sin(float x) { return sinf(x); }
VPT_DEV float m_cos(float x) { return cosf(x); }
VPT_DEV float m_pow(float x, float y) { return powf(x, y); }
VPT_DEV float m_atan2(float y, float x) { return atan2f(y, x); }
VPT_DEV float m_asin(float x) { return asinf(x); }
VPT_DEV float m_acos(float x) { return acosf(x); }
VPT_DEV float m_tan(float x) { return tanf(x); }
VPT_DEV float m_pow5(float x) { return powf(x, 5.0f); }
#endif

VPT_DEV F3 f3(float x, float y, float z) { F3 r; r.x = x; r.y = y; r.z = z; return r; }
VPT_DEV F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
VPT_DEV F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
VPT_DEV F3 operator-(F3 a) { return f3(-a.x, -a.y, -a.z); }
VPT_DEV F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
VPT_DEV F3 operator*(float s, F3 a) { return f3(s * a.x, s * a.y, s * a.z); }
VPT_DEV F3 operator*(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
VPT_DEV F3 operator/(F3 a, F3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
VPT_DEV float dot3(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
VPT_DEV F3 cross3(F3 a, F3 b) {
    return f3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
VPT_DEV float length3(F3 a) { return sqrtf(dot3(a, a)); }
VPT_DEV F3 normalize3(F3 a) {
    float l = length3(a);
    return f3(a.x / l, a.y / l, a.z / l);
}
VPT_DEV float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
VPT_DEV float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
VPT_DEV float smoothstepf(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

// ---------------------------------------------------------------------------------------------
// Hybrid Tausworthe generator: three Tausworthe steps and one LCG step combined by XOR
// (VptUtils.glsl:48-65).  Integer part is bit-exact; the float is float(u32) * 2^-32 rounded.
struct Rng {
    uint32_t x, y, z, w;
};

VPT_DEV uint32_t taus_step(uint32_t z, int s1, int s2, int s3, uint32_t m) {
    uint32_t b = ((z << s1) ^ z) >> s2;
    return ((z & m) << s3) ^ b;
}

VPT_DEV float rng_next(Rng& r) {
    r.x = taus_step(r.x, 13, 19, 12, 4294967294u);
    r.y = taus_step(r.y, 2, 25, 4, 4294967288u);
    r.z = taus_step(r.z, 3, 11, 17, 4294967280u);
    r.w = 1664525u * r.w + 1013904223u;
    return 2.3283064365387e-10f * __uint2float_rn(r.x ^ r.y ^ r.z ^ r.w);
}

VPT_DEV Rng rng_init(uint32_t seed) {
    Rng r;
    r.x = r.y = r.z = r.w = seed;
    uint32_t n = seed % 7u + 2u;
    for (uint32_t i = 0; i < n; i++) rng_next(r);
    return r;
}

// ---------------------------------------------------------------------------------------------
// Camera ray through NDC (x, y): near-plane point and direction to the far-plane point
// (createCameraRay, VptUtils.glsl:750-761).
VPT_DEV void mat4_mul_point(const float* m, float x, float y, float z, float w, float out[4]) {
#pragma unroll
    for (int r = 0; r < 4; r++) {
        out[r] = ((m[0 * 4 + r] * x + m[1 * 4 + r] * y) + m[2 * 4 + r] * z) + m[3 * 4 + r] * w;
    }
}

VPT_DEV void camera_ray(const TraceParams& P, float sx, float sy, F3& x, F3& w) {
    float p[4], t[4];
    mat4_mul_point(P.inv_view_proj, sx, sy, 0.0f, 1.0f, p);
    mat4_mul_point(P.inv_view_proj, sx, sy, 1.0f, 1.0f, t);
    F3 vp = f3(p[0] / p[3], p[1] / p[3], p[2] / p[3]);
    F3 vt = f3(t[0] / t[3], t[1] / t[3], t[2] / t[3]);
    x = vp;
    w = normalize3(vt - vp);
}

// ---------------------------------------------------------------------------------------------
// Lights of the light editor (VptUtils.glsl:394-453), sampled by next event tracking.

// (m * vec4(v, w)).xyz for a column-major mat4, summed column by column.
VPT_DEV F3 mat4_mul_xyz(const float* m, F3 v, float w) {
    return f3(((m[0] * v.x + m[4] * v.y) + m[8] * v.z) + m[12] * w,
              ((m[1] * v.x + m[5] * v.y) + m[9] * v.z) + m[13] * w,
              ((m[2] * v.x + m[6] * v.y) + m[10] * v.z) + m[14] * w);
}

VPT_DEV F3 light_position(const TraceParams& P, const LightParams& L) {
    if (L.space == kLightSpaceView || L.space == kLightSpaceViewOrientation) {
        const float hom = (L.type == kLightDirectional || L.space == kLightSpaceViewOrientation) ? 0.0f : 1.0f;
        return mat4_mul_xyz(P.inv_view, L.position, hom);
    }
    return L.position;
}

// getHeadlightDirection: picks a light uniformly when there are several (one random number),
// returns the unit direction to it and its distance.
VPT_DEV F3 light_direction(const TraceParams& P, F3 pos, Rng& rng, int& idx, float& prob_factor, float& dist) {
    if (P.num_lights > 1) {
        const uint32_t k = (uint32_t)(rng_next(rng) * (float)P.num_lights);
        idx = (int)min(k, (uint32_t)P.num_lights - 1u);
        prob_factor *= (float)P.num_lights;
    }
    const LightParams& L = P.lights[idx];
    const F3 lp = light_position(P, L);
    const F3 dir = (L.type == kLightPoint || L.type == kLightSpot) ? lp - pos : lp;
    dist = length3(dir);
    const float s = dist + 1e-5f;
    return f3(dir.x / s, dir.y / s, dir.z / s);
}

// sampleHeadlight: radiance of light `idx` seen from `pos` (distance falloff, spot cone).
VPT_DEV F3 light_radiance(const TraceParams& P, F3 pos, int idx) {
    const LightParams& L = P.lights[idx];
    const F3 lp = light_position(P, L);
    float f = L.intensity;
    if ((L.type == kLightPoint || L.type == kLightSpot) && L.use_distance != 0) {
        const F3 diff = lp - pos;
        f /= fmaxf(dot3(diff, diff), 1e-3f);
    }
    if (L.type == kLightSpot) {
        const float total = m_cos(L.spot_total_width);
        const float falloff = L.spot_total_width > L.spot_falloff_start ? m_cos(L.spot_falloff_start) : total;
        const F3 p = pos - lp;
        F3 z = normalize3(L.spot_direction);
        if (L.space == kLightSpaceView || L.space == kLightSpaceViewOrientation) z = mat4_mul_xyz(P.inv_view, z, 0.0f);
        const float cos_theta = dot3(z, p) / (length3(z) * length3(p));
        f *= smoothstepf(total, falloff, cos_theta);
    }
    return f3(f * L.color.x, f * L.color.y, f * L.color.z);
}

// Slab test with a 1e-6 clamp of near-zero direction components (rayBoxIntersect,
// VptUtils.glsl:763-801; the clip plane is not supported).
VPT_DEV bool ray_box(F3 bmin, F3 bmax, F3 p, F3 d, float& tmin, float& tmax) {
    d.x = fabsf(d.x) <= 0.000001f ? 0.000001f : d.x;
    d.y = fabsf(d.y) <= 0.000001f ? 0.000001f : d.y;
    d.z = fabsf(d.z) <= 0.000001f ? 0.000001f : d.z;
    F3 cmin = (bmin - p) / d;
    F3 cmax = (bmax - p) / d;
    tmin = fmaxf(fmaxf(fminf(cmin.x, cmax.x), fminf(cmin.y, cmax.y)), fminf(cmin.z, cmax.z));
    tmin = fmaxf(0.0f, tmin);
    tmax = fminf(fminf(fmaxf(cmin.x, cmax.x), fmaxf(cmin.y, cmax.y)), fmaxf(cmin.z, cmax.z));
    return !(tmax <= tmin || tmax <= 0.0f);
}

// rayBoxIntersect of the volume box (VptUtils.glsl:763-801): with the clip plane on (USE_CLIP_PLANE,
// :776-799) the interval is cut to the plane's positive side, using the direction as modified for the
// box test; a ray parallel to the plane, or meeting it behind its origin, is kept whole or dropped
// by the side its origin lies on.
VPT_DEV bool ray_box_p(const TraceParams& P, F3 p, F3 d, float& tmin, float& tmax) {
    if (!ray_box(P.box_min, P.box_max, p, d, tmin, tmax)) return false;
    if (!P.use_clip) return true;
    d.x = fabsf(d.x) <= 0.000001f ? 0.000001f : d.x;
    d.y = fabsf(d.y) <= 0.000001f ? 0.000001f : d.y;
    d.z = fabsf(d.z) <= 0.000001f ? 0.000001f : d.z;
    const float denom = dot3(P.clip_n, d);
    const float dp = dot3(P.clip_n, p) - P.clip_d;
    if (fabsf(denom) < 0.001f) return dp > 0.0f;
    const float t_clip = (P.clip_d - dot3(P.clip_n, p)) / denom;
    if (t_clip <= 0.0f) return dp > 0.0f;
    if (dp > 0.0f) tmax = fminf(t_clip, tmax);
    else tmin = fmaxf(t_clip, tmin);
    return !(tmax <= tmin || tmax <= 0.0f);
}

// rayBoxIntersectionNormal (VptUtils.glsl:803-856, CLOSE_ISOSURFACES): the normal of the box face a ray
// from p enters through, or -clip_n where the clip plane is the entry surface; n stays as it is when the
// ray misses the box, or when the ray runs parallel to the plane or meets it behind p on its negative side.
VPT_DEV void ray_box_normal(const TraceParams& P, F3 p, F3 d, F3& n) {
    d.x = fabsf(d.x) <= 1e-6f ? 1e-6f : d.x;
    d.y = fabsf(d.y) <= 1e-6f ? 1e-6f : d.y;
    d.z = fabsf(d.z) <= 1e-6f ? 1e-6f : d.z;
    const F3 cmin = (P.box_min - p) / d;
    const F3 cmax = (P.box_max - p) / d;
    const float mx = fminf(cmin.x, cmax.x), my = fminf(cmin.y, cmax.y), mz = fminf(cmin.z, cmax.z);
    const float tmin = fmaxf(0.0f, fmaxf(fmaxf(mx, my), mz));
    const float tmax = fminf(fminf(fmaxf(cmin.x, cmax.x), fmaxf(cmin.y, cmax.y)), fmaxf(cmin.z, cmax.z));
    if (tmax <= tmin || tmax <= 0.0f) return;
    auto sgn = [](float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); };
    F3 nb;
    if (mx > my && mx > mz) nb = f3(-sgn(d.x), 0.0f, 0.0f);
    else if (my > mz) nb = f3(0.0f, -sgn(d.y), 0.0f);
    else nb = f3(0.0f, 0.0f, -sgn(d.z));
    if (P.use_clip) {
        const float denom = dot3(P.clip_n, d);
        const float dp = dot3(P.clip_n, p) - P.clip_d;
        if (fabsf(denom) < 1e-3f) {
            if (dp > 0.0f) n = nb;
            return;
        }
        const float t_clip = (P.clip_d - dot3(P.clip_n, p)) / denom;
        if (t_clip <= 0.0f) {
            if (dp > 0.0f) n = nb;
            return;
        }
        if (dp <= 0.0f && t_clip >= tmin) {
            n = f3(-P.clip_n.x, -P.clip_n.y, -P.clip_n.z);
            return;
        }
    }
    n = nb;
}

// ---------------------------------------------------------------------------------------------
// Direction sampling (VptUtils.glsl:67-123).
VPT_DEV void orthonormal_basis(F3 d, F3& b, F3& t) {
    F3 other = fabsf(d.z) >= 0.9999f ? f3(1.0f, 0.0f, 0.0f) : f3(0.0f, 0.0f, 1.0f);
    b = normalize3(cross3(other, d));
    t = normalize3(cross3(d, b));
}

VPT_DEV F3 random_direction(Rng& rng, F3 d) {
    float r1 = rng_next(rng);
    float r2 = rng_next(rng) * 2.0f - 1.0f;
    float sq = r2 * r2;
    float a = kTwoPi * r1;
    float s = sqrtf(1.0f - sq);
    float x = m_cos(a) * s;
    float y = m_sin(a) * s;
    F3 t0, t1;
    orthonormal_basis(d, t0, t1);
    return (t0 * x + t1 * y) + d * r2;
}

VPT_DEV float hg_invert_cdf(float g, float xi) {
    float t = (1.0f - g * g) / (1.0f - g + 2.0f * g * xi);
    return (0.5f / g) * ((1.0f + g * g) - t * t);
}

// importanceSamplePhase without the pdf (only evaluatePhase's pdf feeds the estimators).
VPT_DEV F3 sample_phase(Rng& rng, float g, F3 d) {
    if (fabsf(g) < 0.001f) {
        return random_direction(rng, -d);
    }
    float phi = rng_next(rng) * 2.0f * kPi;
    float cos_t = hg_invert_cdf(g, rng_next(rng));
    float sin_t = sqrtf(fmaxf(0.0f, 1.0f - cos_t * cos_t));
    F3 t0, t1;
    orthonormal_basis(d, t0, t1);
    return (t0 * (sin_t * m_sin(phi)) + t1 * (sin_t * m_cos(phi))) + d * cos_t;
}

VPT_DEV float evaluate_phase(float g, F3 a, F3 b) {
    float c = dot3(normalize3(a), normalize3(b));
    return ((0.25f / kPi) * (1.0f - g * g)) / m_pow((1.0f + g * g) - 2.0f * g * c, 1.5f);
}

// ---------------------------------------------------------------------------------------------
// Sky and sun (VptUtils.glsl:288-389).
VPT_DEV float srgb_to_linear(float c) {
    return c <= 0.04045f ? c / 12.92f : m_pow((c + 0.055f) / 1.055f, 2.4f);
}

VPT_DEV float linear_to_srgb(float c) {
    return c <= 0.0031308f ? c * 12.92f : 1.055f * m_pow(c, 1.0f / 2.4f) - 0.055f;
}

VPT_DEV F3 sky_default(F3 dir, int linear_rgb) {
    const float cr[5] = {0.1f, 0.01f, 0.8f, 0.1f, 0.01f};
    const float cg[5] = {0.05f, 0.05f, 0.9f, 0.3f, 0.1f};
    const float cb[5] = {0.01f, 0.2f, 1.0f, 1.0f, 0.7f};
    const float dists[5] = {-1.0f, -0.1f, 0.0f, 0.4f, 1.0f};
    float r = cr[0], g = cg[0], b = cb[0];
#pragma unroll
    for (int i = 1; i < 5; i++) {
        float s = smoothstepf(dists[i - 1], dists[i], dir.y);
        r = mixf(r, cr[i], s);
        g = mixf(g, cg[i], s);
        b = mixf(b, cb[i], s);
    }
    if (linear_rgb) {
        r = srgb_to_linear(r);
        g = srgb_to_linear(g);
        b = srgb_to_linear(b);
    }
    return f3(r, g, b);
}

// Phong lobe with exponent 10 around the sun direction, normalised by (N+1)/(2*3.14159)
// (sampleLight, VptUtils.glsl:370-374).
VPT_DEV F3 sun_lobe(const TraceParams& P, F3 dir) {
    const float norm = 11.0f / (2.0f * 3.14159f);
    float p = m_pow(fmaxf(0.0f, dot3(dir, P.sun_dir)), 10.0f);
    return f3((P.sun_intensity.x * p) * norm, (P.sun_intensity.y * p) * norm, (P.sun_intensity.z * p) * norm);
}

// Bilinear fetch of the equirectangular image with REPEAT addressing.
VPT_DEV F3 env_image_fetch(const TraceParams& P, float u, float v) {
    float fx = u * (float)P.env_w - 0.5f;
    float fy = v * (float)P.env_h - 0.5f;
    float x0f = floorf(fx), y0f = floorf(fy);
    float ax = fx - x0f, ay = fy - y0f;
    int x0 = (int)x0f, y0 = (int)y0f;
    int w = P.env_w, h = P.env_h;
    int xa = ((x0 % w) + w) % w, xb = (((x0 + 1) % w) + w) % w;
    int ya = ((y0 % h) + h) % h, yb = (((y0 + 1) % h) + h) % h;
    const float4* img = reinterpret_cast<const float4*>(P.env_rgba);
    float4 c00 = __ldg(img + (size_t)ya * w + xa), c10 = __ldg(img + (size_t)ya * w + xb);
    float4 c01 = __ldg(img + (size_t)yb * w + xa), c11 = __ldg(img + (size_t)yb * w + xb);
    F3 r;
    r.x = mixf(mixf(c00.x, c10.x, ax), mixf(c01.x, c11.x, ax), ay);
    r.y = mixf(mixf(c00.y, c10.y, ax), mixf(c01.y, c11.y, ax), ay);
    r.z = mixf(mixf(c00.z, c10.z, ax), mixf(c01.z, c11.z, ax), ay);
    return r;
}

// parameters.envMapDirRot * v and its transpose (invEnvMapDirRot) * v, columns summed in order
VPT_DEV F3 env_rotate(const float* m, F3 v) {
    return f3((m[0] * v.x + m[3] * v.y) + m[6] * v.z, (m[1] * v.x + m[4] * v.y) + m[7] * v.z,
              (m[2] * v.x + m[5] * v.y) + m[8] * v.z);
}
VPT_DEV F3 env_rotate_inverse(const float* m, F3 v) {
    return f3((m[0] * v.x + m[1] * v.y) + m[2] * v.z, (m[3] * v.x + m[4] * v.y) + m[5] * v.z,
              (m[6] * v.x + m[7] * v.y) + m[8] * v.z);
}

// sampleSkybox for an environment image (VptUtils.glsl:303-328), with USE_ENV_MAP_ROTATION the
// direction rotated first.
VPT_DEV F3 sky_image(const TraceParams& P, F3 dir) {
    if (P.env_rot) dir = env_rotate(P.env_rot_m, dir);
    float u = m_atan2(dir.z, dir.x) / kTwoPi + 0.5f;
    float v = -m_asin(dir.y) / kPi + 0.5f;
    F3 c = env_image_fetch(P, u, v);
    c.x = fminf(c.x, 100000.0f);
    c.y = fminf(c.y, 100000.0f);
    c.z = fminf(c.z, 100000.0f);
    if (!P.env_image_linear && P.use_linear_rgb) {
        c = f3(srgb_to_linear(c.x), srgb_to_linear(c.y), srgb_to_linear(c.z));
    } else if (P.env_image_linear && !P.use_linear_rgb) {
        c = f3(linear_to_srgb(c.x), linear_to_srgb(c.y), linear_to_srgb(c.z));
    }
    return P.env_intensity * c;
}

// sampleSkybox(dir) + sampleLight(dir) for the configured environment.
VPT_DEV F3 sky_and_sun(const TraceParams& P, F3 dir) {
    switch (P.env_kind) {
        case kEnvDefault: return sky_default(dir, P.use_linear_rgb) + sun_lobe(P, dir);
        case kEnvBlack: return f3(0.0f, 0.0f, 0.0f);
        case kEnvSingleColor: return P.sun_intensity;
        case kEnvConstantSun: return P.sky_color + sun_lobe(P, dir);
        default: return sky_image(P, dir);
    }
}

// sampleSkybox(dir) only (background feature map).
VPT_DEV F3 sky_only(const TraceParams& P, F3 dir) {
    switch (P.env_kind) {
        case kEnvDefault: return sky_default(dir, P.use_linear_rgb);
        case kEnvBlack: return f3(0.0f, 0.0f, 0.0f);
        case kEnvSingleColor: return P.sun_intensity;
        case kEnvConstantSun: return P.sky_color;
        default: return sky_image(P, dir);
    }
}

// Octahedral map helpers (VptUtils.glsl:127-170, without the rotation; see importance_sample_env_image).
VPT_DEV float signf(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }

VPT_DEV F3 octahedral_uv_to_world(float u, float v) {
    u = u * 2.0f - 1.0f;
    v = v * 2.0f - 1.0f;
    float sx = signf(u), sy = signf(v);
    u = fabsf(u);
    v = fabsf(v);
    float r = 1.0f - fabsf(1.0f - u - v);
    float phi = 0.25f * kPi * ((v - u) / r + 1.0f);
    if (r == 0.0f) phi = 0.0f;
    float r2 = r * r;
    float s = sqrtf(2.0f - r2);
    float x = sx * m_cos(phi) * r * s;
    float y = sy * m_sin(phi) * r * s;
    float z = signf(1.0f - u - v) * (1.0f - r2);
    return f3(x, y, z);
}

VPT_DEV void world_to_octahedral_uv(F3 dir, float& u, float& v) {
    dir = normalize3(dir);
    float sx = signf(dir.x), sy = signf(dir.y), sz = signf(dir.z);
    dir = f3(fabsf(dir.x), fabsf(dir.y), fabsf(dir.z));
    float phi = m_atan2(dir.y, dir.x);
    float r = sqrtf(1.0f - dir.z);
    float vv = r * 2.0f / kPi * phi;
    float uu = r - vv;
    if (sz < 0.0f) {
        float t = uu;
        uu = 1.0f - vv;
        vv = 1.0f - t;
    }
    u = uu * sx * 0.5f + 0.5f;
    v = vv * sy * 0.5f + 0.5f;
}

VPT_DEV float pyr_fetch(const TraceParams& P, int level, int x, int y) {
    int res = P.env_base_res >> level;
    return __ldg(P.env_pyramid + P.env_level_offset[level] + (size_t)y * res + x) + 0.001f;
}

// Hierarchical sample of the octahedral max-luminance pyramid (importanceSampleSkybox,
// VptUtils.glsl:172-220).
VPT_DEV F3 importance_sample_env_image(const TraceParams& P, Rng& rng, float& pdf) {
    float rx = rng_next(rng);
    float ry = rng_next(rng);
    int px = 0, py = 0;
    pdf = 0.25f / kPi;
    for (int mip = P.env_levels - 1; mip >= 0; mip--) {
        px *= 2;
        py *= 2;
        pdf *= 4.0f;
        float ul = pyr_fetch(P, mip, px, py), ur = pyr_fetch(P, mip, px + 1, py);
        float dl = pyr_fetch(P, mip, px, py + 1), dr = pyr_fetch(P, mip, px + 1, py + 1);
        float l = ul + dl, r = ur + dr, total = l + r;
        float hs = l / total, vs;
        if (rx < hs) {
            rx = rx / hs;
            vs = ul / l;
            pdf *= hs;
        } else {
            px += 1;
            rx = (rx - hs) / (1.0f - hs);
            vs = ur / r;
            pdf *= (1.0f - hs);
        }
        if (ry < vs) {
            ry = ry / vs;
            pdf *= vs;
        } else {
            py += 1;
            ry = (ry - vs) / (1.0f - vs);
            pdf *= (1.0f - vs);
        }
    }
    float inv = 1.0f / (float)P.env_base_res;
    // octahedralUVToWorld with USE_ENV_MAP_ROTATION returns invEnvMapDirRot * direction
    // (VptUtils.glsl:142-146); the pyramid itself is built from unrotated directions
    const F3 dir = octahedral_uv_to_world(((float)px + rx) * inv, ((float)py + ry) * inv);
    return P.env_rot ? env_rotate_inverse(P.env_rot_m, dir) : dir;
}

// Light sample for NEE: environment image -> pyramid, builtin -> uniform sphere.
VPT_DEV F3 importance_sample_sky(const TraceParams& P, Rng& rng, float& pdf) {
    if (P.env_kind == kEnvImage) return importance_sample_env_image(P, rng, pdf);
    pdf = 1.0f / (4.0f * kPi);
    return random_direction(rng, f3(1.0f, 0.0f, 0.0f));
}

// ---------------------------------------------------------------------------------------------
// Dense density lookup with CLAMP_TO_BORDER semantics (sampleCloud/sampleCloudRaw,
// VptUtils.glsl:583-591, 674-683).  Values in `density` are already normalised.
VPT_DEV float dense_texel(const TraceParams& P, int ix, int iy, int iz) {
    if ((unsigned)ix >= (unsigned)P.nx || (unsigned)iy >= (unsigned)P.ny || (unsigned)iz >= (unsigned)P.nz) {
        return P.border_density;
    }
    return __ldg(P.density + ((size_t)iz * (size_t)P.ny + (size_t)iy) * (size_t)P.nx + (size_t)ix);
}

// Lookup at continuous voxel coordinates u (texel i covers [i, i+1)).
template <int INTERP>
VPT_DEV float sample_dense_vox(const TraceParams& P, float ux, float uy, float uz) {
    if (INTERP != kTrilinear) {
        return dense_texel(P, (int)floorf(ux), (int)floorf(uy), (int)floorf(uz));
    }
    ux = ux - 0.5f;
    uy = uy - 0.5f;
    uz = uz - 0.5f;
    float fx0 = floorf(ux), fy0 = floorf(uy), fz0 = floorf(uz);
    float ax = ux - fx0, ay = uy - fy0, az = uz - fz0;
    int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
    float f000 = dense_texel(P, x0, y0, z0), f100 = dense_texel(P, x0 + 1, y0, z0);
    float f010 = dense_texel(P, x0, y0 + 1, z0), f110 = dense_texel(P, x0 + 1, y0 + 1, z0);
    float f001 = dense_texel(P, x0, y0, z0 + 1), f101 = dense_texel(P, x0 + 1, y0, z0 + 1);
    float f011 = dense_texel(P, x0, y0 + 1, z0 + 1), f111 = dense_texel(P, x0 + 1, y0 + 1, z0 + 1);
    float f0 = mixf(mixf(f000, f100, ax), mixf(f010, f110, ax), ay);
    float f1 = mixf(mixf(f001, f101, ax), mixf(f011, f111, ax), ay);
    return mixf(f0, f1, az);
}

template <int INTERP>
VPT_DEV float sample_dense(const TraceParams& P, F3 pos, Rng& rng) {
    float ux = (pos.x - P.box_min.x) * P.vox_per_unit.x;
    float uy = (pos.y - P.box_min.y) * P.vox_per_unit.y;
    float uz = (pos.z - P.box_min.z) * P.vox_per_unit.z;
    if (INTERP == kStochastic) {
        float jx = rng_next(rng) - 0.5f;
        float jy = rng_next(rng) - 0.5f;
        float jz = rng_next(rng) - 0.5f;
        ux = ux + jx;
        uy = uy + jy;
        uz = uz + jz;
    }
    return sample_dense_vox<INTERP>(P, ux, uy, uz);
}

// The same lookups through the grid's 3D texture object (point filtering, unnormalised coordinates,
// border colour 0 = the border density when the grid's minimum is 0): the texel index is computed
// here as in dense_texel and fetched at its centre, so the value is the same texel, bit for bit; the
// texture unit does the bounds test and the address arithmetic and reads the array's 3D block layout.
VPT_DEV float tex_texel(const TraceParams& P, float fx, float fy, float fz) {
    return tex3D<float>((cudaTextureObject_t)P.density_tex, fx + 0.5f, fy + 0.5f, fz + 0.5f);
}

template <int INTERP>
VPT_DEV float sample_dense_tex(const TraceParams& P, F3 pos, Rng& rng) {
    float ux = (pos.x - P.box_min.x) * P.vox_per_unit.x;
    float uy = (pos.y - P.box_min.y) * P.vox_per_unit.y;
    float uz = (pos.z - P.box_min.z) * P.vox_per_unit.z;
    if (INTERP == kStochastic) {
        float jx = rng_next(rng) - 0.5f;
        float jy = rng_next(rng) - 0.5f;
        float jz = rng_next(rng) - 0.5f;
        ux = ux + jx;
        uy = uy + jy;
        uz = uz + jz;
    }
    if (INTERP != kTrilinear) return tex_texel(P, floorf(ux), floorf(uy), floorf(uz));
    ux = ux - 0.5f;
    uy = uy - 0.5f;
    uz = uz - 0.5f;
    const float fx0 = floorf(ux), fy0 = floorf(uy), fz0 = floorf(uz);
    const float ax = ux - fx0, ay = uy - fy0, az = uz - fz0;
    const float fx1 = fx0 + 1.0f, fy1 = fy0 + 1.0f, fz1 = fz0 + 1.0f;
    float f000 = tex_texel(P, fx0, fy0, fz0), f100 = tex_texel(P, fx1, fy0, fz0);
    float f010 = tex_texel(P, fx0, fy1, fz0), f110 = tex_texel(P, fx1, fy1, fz0);
    float f001 = tex_texel(P, fx0, fy0, fz1), f101 = tex_texel(P, fx1, fy0, fz1);
    float f011 = tex_texel(P, fx0, fy1, fz1), f111 = tex_texel(P, fx1, fy1, fz1);
    float f0 = mixf(mixf(f000, f100, ax), mixf(f010, f110, ax), ay);
    float f1 = mixf(mixf(f001, f101, ax), mixf(f011, f111, ax), ay);
    return mixf(f0, f1, az);
}

// Transfer function (sampleCloudDensityEmission, VptUtils.glsl:647-672; transferFunctionTexture, a
// one-row array texture): linear filtering along the normalised density with clamp to edge.
VPT_DEV void tf_lookup(const TraceParams& P, float v, F3& rgb, float& alpha) {
    const float u = v * (float)P.tf_size - 0.5f;
    const float fu = floorf(u);
    const float a = u - fu;
    int x0 = (int)fu, x1 = x0 + 1;
    x0 = x0 < 0 ? 0 : (x0 >= P.tf_size ? P.tf_size - 1 : x0);
    x1 = x1 < 0 ? 0 : (x1 >= P.tf_size ? P.tf_size - 1 : x1);
    const float* c0 = P.tf + 4 * x0;
    const float* c1 = P.tf + 4 * x1;
    rgb = f3(mixf(__ldg(c0), __ldg(c1), a), mixf(__ldg(c0 + 1), __ldg(c1 + 1), a), mixf(__ldg(c0 + 2), __ldg(c1 + 2), a));
    alpha = mixf(__ldg(c0 + 3), __ldg(c1 + 3), a);
}

// Emission (sampleEmission / sampleEmissionRaw, VptUtils.glsl:604-626): the emission grid at the
// point (its own world box, the density texture's filter and stochastic jitter, zero outside),
// t = clamp(value * cap, 0, 1), radiance (t^2, t^4, t^8) * strength.
VPT_DEV float emission_texel(const TraceParams& P, int ix, int iy, int iz) {
    if ((unsigned)ix >= (unsigned)P.enx || (unsigned)iy >= (unsigned)P.eny || (unsigned)iz >= (unsigned)P.enz)
        return 0.0f;
    return __ldg(P.emission + ((size_t)iz * (size_t)P.eny + (size_t)iy) * (size_t)P.enx + (size_t)ix);
}

template <int INTERP>
VPT_DEV F3 sample_emission(const TraceParams& P, F3 pos, Rng& rng) {
    float ux = (pos.x - P.emission_box_min.x) * P.emission_vox_per_unit.x;
    float uy = (pos.y - P.emission_box_min.y) * P.emission_vox_per_unit.y;
    float uz = (pos.z - P.emission_box_min.z) * P.emission_vox_per_unit.z;
    if (INTERP == kStochastic) {
        float jx = rng_next(rng) - 0.5f;
        float jy = rng_next(rng) - 0.5f;
        float jz = rng_next(rng) - 0.5f;
        ux = ux + jx;
        uy = uy + jy;
        uz = uz + jz;
    }
    float v;
    if (INTERP != kTrilinear) {
        v = emission_texel(P, (int)floorf(ux), (int)floorf(uy), (int)floorf(uz));
    } else {
        ux = ux - 0.5f;
        uy = uy - 0.5f;
        uz = uz - 0.5f;
        const float fx0 = floorf(ux), fy0 = floorf(uy), fz0 = floorf(uz);
        const float ax = ux - fx0, ay = uy - fy0, az = uz - fz0;
        const int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
        const float f0 = mixf(mixf(emission_texel(P, x0, y0, z0), emission_texel(P, x0 + 1, y0, z0), ax),
                              mixf(emission_texel(P, x0, y0 + 1, z0), emission_texel(P, x0 + 1, y0 + 1, z0), ax), ay);
        const float f1 =
            mixf(mixf(emission_texel(P, x0, y0, z0 + 1), emission_texel(P, x0 + 1, y0, z0 + 1), ax),
                 mixf(emission_texel(P, x0, y0 + 1, z0 + 1), emission_texel(P, x0 + 1, y0 + 1, z0 + 1), ax), ay);
        v = mixf(f0, f1, az);
    }
    const float t = fminf(fmaxf(v * P.emission_cap, 0.0f), 1.0f);
    const float r = t * t, g = r * r, b = g * g;
    return f3(r * P.emission_strength, g * P.emission_strength, b * P.emission_strength);
}

// Normal feature: central differences of the density one voxel apart, scaled by 100/dim and
// normalised when longer than 1e-5 (getCloudFiniteDifference, VptUtils.glsl:726-748).
template <int INTERP>
VPT_DEV F3 density_normal(const TraceParams& P, F3 pos, Rng& rng) {
    float ux = (pos.x - P.box_min.x) * P.vox_per_unit.x;
    float uy = (pos.y - P.box_min.y) * P.vox_per_unit.y;
    float uz = (pos.z - P.box_min.z) * P.vox_per_unit.z;
    if (INTERP == kStochastic) {
        float jx = rng_next(rng) - 0.5f;
        float jy = rng_next(rng) - 0.5f;
        float jz = rng_next(rng) - 0.5f;
        ux = ux + jx;
        uy = uy + jy;
        uz = uz + jz;
    }
    F3 d;
    d.x = sample_dense_vox<INTERP>(P, ux - 1.0f, uy, uz) - sample_dense_vox<INTERP>(P, ux + 1.0f, uy, uz);
    d.y = sample_dense_vox<INTERP>(P, ux, uy - 1.0f, uz) - sample_dense_vox<INTERP>(P, ux, uy + 1.0f, uz);
    d.z = sample_dense_vox<INTERP>(P, ux, uy, uz - 1.0f) - sample_dense_vox<INTERP>(P, ux, uy, uz + 1.0f);
    d = f3((d.x / (float)P.nx) * 100.0f, (d.y / (float)P.ny) * 100.0f, (d.z / (float)P.nz) * 100.0f);
    float l = length3(d);
    if (l > 1e-5f) d = f3(d.x / l, d.y / l, d.z / l);
    return d;
}

// ---------------------------------------------------------------------------------------------
// Isosurfaces of the density field or of its gradient magnitude (USE_ISOSURFACES with
// ISOSURFACE_TYPE_DENSITY / ISOSURFACE_TYPE_GRADIENT; dense grids).

// gradientImage (ISOSURFACE_TYPE_GRADIENT): the raw gradient magnitudes through a linear filter with
// border 0 (the density texture's sampler), at continuous voxel coordinates u.
VPT_DEV float grad_texel(const TraceParams& P, int ix, int iy, int iz) {
    if ((unsigned)ix >= (unsigned)P.nx || (unsigned)iy >= (unsigned)P.ny || (unsigned)iz >= (unsigned)P.nz) {
        return 0.0f;
    }
    return __ldg(P.iso_grad + ((size_t)iz * (size_t)P.ny + (size_t)iy) * (size_t)P.nx + (size_t)ix);
}

VPT_DEV float grad_filtered(const TraceParams& P, float ux, float uy, float uz) {
    ux = ux - 0.5f;
    uy = uy - 0.5f;
    uz = uz - 0.5f;
    const float fx0 = floorf(ux), fy0 = floorf(uy), fz0 = floorf(uz);
    const float ax = ux - fx0, ay = uy - fy0, az = uz - fz0;
    const int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
    const float f0 = mixf(mixf(grad_texel(P, x0, y0, z0), grad_texel(P, x0 + 1, y0, z0), ax),
                          mixf(grad_texel(P, x0, y0 + 1, z0), grad_texel(P, x0 + 1, y0 + 1, z0), ax), ay);
    const float f1 = mixf(mixf(grad_texel(P, x0, y0, z0 + 1), grad_texel(P, x0 + 1, y0, z0 + 1), ax),
                          mixf(grad_texel(P, x0, y0 + 1, z0 + 1), grad_texel(P, x0 + 1, y0 + 1, z0 + 1), ax), ay);
    return mixf(f0, f1, az);
}

// sampleCloudGradient (VptUtils.glsl:687-699): the filtered magnitude at a world position, the value
// gradient isosurfaces are found in (no random number drawn: lookups are trilinear with isosurfaces);
// the texture coordinate is formed as the shader forms it, (pos - boxMin) / (boxMax - boxMin)
VPT_DEV float iso_gradient_at(const TraceParams& P, F3 pos) {
    const F3 c = (pos - P.box_min) / (P.box_max - P.box_min);
    return grad_filtered(P, c.x * (float)P.nx, c.y * (float)P.ny, c.z * (float)P.nz);
}

// The iso image's linear filter at a normalised texture coordinate (sampleIsoImage, VptUtils.glsl:599):
// the density texture (its texels are normalised already) or, for gradient isosurfaces, gradientImage
// normalised with the density's min and range as the shader does.
VPT_DEV float iso_tex(const TraceParams& P, float cx, float cy, float cz) {
    if (P.iso_grad) {
        return (grad_filtered(P, cx * (float)P.nx, cy * (float)P.ny, cz * (float)P.nz) - P.iso_norm_min) /
               P.iso_norm_range;
    }
    return sample_dense_vox<kTrilinear>(P, cx * (float)P.nx, cy * (float)P.ny, cz * (float)P.nz);
}

// getNearestMultiple (VptUtils.glsl:896-906) with GLSL mod(n, x) = n - x * floor(n / x).
VPT_DEV float iso_nearest_multiple(float n, float x, bool smaller) {
    const float rest = n - x * floorf(n / x);
    if (smaller) return n - rest;
    if (rest == 0.0f) return n;
    return x + n - rest;
}

// trilinearInterpolationDensity (VptUtils.glsl:908-959): the eight lattice points k / (size - 1)
// around c looked up through the texture filter, blended with the fractions of c * (size - 1).
VPT_DEV float iso_trilinear(const TraceParams& P, float cx, float cy, float cz) {
    const float sx = (float)P.nx - 1.0f, sy = (float)P.ny - 1.0f, sz = (float)P.nz - 1.0f;
    const float dx = 1.0f / sx, dy = 1.0f / sy, dz = 1.0f / sz;
    const float x0 = iso_nearest_multiple(cx, dx, true), x1 = iso_nearest_multiple(cx, dx, false);
    const float y0 = iso_nearest_multiple(cy, dy, true), y1 = iso_nearest_multiple(cy, dy, false);
    const float z0 = iso_nearest_multiple(cz, dz, true), z1 = iso_nearest_multiple(cz, dz, false);
    const float d000 = iso_tex(P, x0, y0, z0), d100 = iso_tex(P, x1, y0, z0);
    const float d110 = iso_tex(P, x1, y1, z0), d010 = iso_tex(P, x0, y1, z0);
    const float d001 = iso_tex(P, x0, y0, z1), d101 = iso_tex(P, x1, y0, z1);
    const float d111 = iso_tex(P, x1, y1, z1), d011 = iso_tex(P, x0, y1, z1);
    const float px = cx * sx, py = cy * sy, pz = cz * sz;
    const float fx = px - floorf(px), fy = py - floorf(py), fz = pz - floorf(pz);
    const float t00 = mixf(d000, d100, fx), t10 = mixf(d010, d110, fx);
    const float t01 = mixf(d001, d101, fx), t11 = mixf(d011, d111, fx);
    return mixf(mixf(t00, t10, fy), mixf(t01, t11, fy), fz);
}

// Surface normal (computeGradient with DIFFERENCES_NEIGHBOR, VptUtils.glsl:965-984): central
// differences four lattice spacings apart, (0, 0, 1) when shorter than 1e-3.
VPT_DEV F3 iso_normal(const TraceParams& P, F3 pos) {
    const F3 c = (pos - P.box_min) / (P.box_max - P.box_min);
    const float hx = 4.0f * (1.0f / (float)(P.nx - 1)), hy = 4.0f * (1.0f / (float)(P.ny - 1)),
                hz = 4.0f * (1.0f / (float)(P.nz - 1));
    const F3 g = f3(0.5f * (iso_trilinear(P, c.x + hx, c.y, c.z) - iso_trilinear(P, c.x - hx, c.y, c.z)),
                    0.5f * (iso_trilinear(P, c.x, c.y + hy, c.z) - iso_trilinear(P, c.x, c.y - hy, c.z)),
                    0.5f * (iso_trilinear(P, c.x, c.y, c.z + hz) - iso_trilinear(P, c.x, c.y, c.z - hz)));
    const float l = length3(g);
    if (l < 1e-3f) return f3(0.0f, 0.0f, 1.0f);
    return f3(g.x / l, g.y / l, g.z / l);
}

// The shading frame at a surface hit: the normal turned against the ray, ComputeDefaultBasis's
// tangent and bitangent (RayTracingUtilities.glsl:20-28), and the direction back along the ray.
struct IsoFrame {
    F3 n, t, b, view;
};

// One BRDF sample at a surface hit (computeBrdf of the selected BRDF file): the new direction, the value
// the throughput is multiplied by, the lobe flags and the lobe's samplingPDF (read by MIS).
struct IsoBrdfSample {
    F3 dir, value;
    bool specular, clearcoat;
    float pdf;
};

// mat3(t, b, n) * (x, y, z), summed in the order of a GLSL matrix-vector product
VPT_DEV F3 iso_frame(F3 t, F3 b, F3 n, float x, float y, float z) {
    return f3((t.x * x + b.x * y) + n.x * z, (t.y * x + b.y * y) + n.y * z, (t.z * x + b.z * y) + n.z * z);
}

// CookTorrance.glsl computeBrdf: sampleBrdf picks the GGX lobe with probability
// (metallic + (1 - r)(1 + specular)) / (that + 1 - metallic), r = clamp(roughness, 0.05, 1), else its
// own cosine lobe (theta = asin(sqrt(u))); evaluateBrdf returns the diffuse colour (1 - F)(1 - metallic)
// plus F G v.h / (n.h v.n) for a GGX sample or F G D v.h sin(theta_h) / v.n for a diffuse one
// (F Schlick with f0 = mix(0.16 specular^2, colour, metallic), D GGX, G Smith-Schlick with k = r^2 / 2),
// and the throughput takes that value as it is.  sel, u are the hit's second and third random numbers.
VPT_DEV IsoBrdfSample iso_cook_torrance(const TraceParams& P, Rng& rng, const IsoFrame& fr, float sel, float u) {
    const F3 n = fr.n, t = fr.t, b = fr.b, view = fr.view;
    const float pi = 3.14159265358979323846f;  // M_PI as the shader's float
    const float v = rng_next(rng);
    const float metallic = P.brdf[kBrdfMetallic], specular = P.brdf[kBrdfSpecular];
    const float rough = fminf(fmaxf(P.brdf[kBrdfRoughness], 0.05f), 1.0f);
    const float specular_w = metallic + (1.0f - rough) * (1.0f + specular);
    const float diffuse_w = 1.0f - metallic;
    const float specular_p = specular_w * (1.0f / (specular_w + diffuse_w));
    const float alpha = rough * rough;
    const float alpha2 = alpha * alpha;
    const bool specular_hit = sel < specular_p;
    const float phi = (2.0f * pi) * v;
    F3 l;
    if (specular_hit) {  // sample_GGX
        const float theta = m_acos(sqrtf((1.0f - u) / (u * (alpha2 - 1.0f) + 1.0f)));
        const float st = m_sin(theta);
        const F3 h = iso_frame(t, b, n, st * m_cos(phi), st * m_sin(phi), m_cos(theta));
        const float vh = fabsf(dot3(view, h));
        const float s = 2.0f * (vh > 0.001f ? vh : 0.001f);  // avoidZero(v.h, 0.001)
        l = f3(s * h.x - view.x, s * h.y - view.y, s * h.z - view.z);
    } else {  // sample_Lambertian
        const float theta = m_asin(sqrtf(u));
        const float st = m_sin(theta);
        l = iso_frame(t, b, n, st * m_cos(phi), st * m_sin(phi), m_cos(theta));
    }
    const F3 h = normalize3(f3(l.x + view.x, l.y + view.y, l.z + view.z));
    const float ndoth = dot3(h, n), vdotn = dot3(view, n), ldotn = dot3(l, n), vdoth = dot3(view, h);
    const float f0s = 0.16f * (specular * specular);
    const float p5 = m_pow5(1.0f - vdoth);
    const float k = alpha / 2.0f;
    const float gl = ldotn < 0.001f ? 0.001f : ldotn, gv = vdotn < 0.001f ? 0.001f : vdotn;
    const float g = (gl / (gl * (1.0f - k) + k)) * (gv / (gv * (1.0f - k) + k));
    const float bq = (ndoth * ndoth) * (alpha2 - 1.0f) + 1.0f;
    const float d = ((1.0f / pi) * alpha2) / (bq * bq);
    const float sth = sqrtf(1.0f - fminf(ndoth * ndoth, 0.95f));
    const float cx[3] = {P.iso_color.x, P.iso_color.y, P.iso_color.z};
    float o[3];
    for (int i = 0; i < 3; ++i) {
        const float f0 = f0s * (1.0f - metallic) + cx[i] * metallic;
        const float f = f0 + (1.0f - f0) * p5;
        const float spec = specular_hit ? ((f * g) * vdoth) / (ndoth * vdotn)
                                        : ((((f * g) * d) * vdoth) * sth) / vdotn;
        o[i] = (cx[i] * (1.0f - f)) * (1.0f - metallic) + spec;
    }
    IsoBrdfSample r;
    r.dir = l;
    r.value = f3(o[0], o[1], o[2]);
    r.specular = specular_hit;
    r.clearcoat = false;
    r.pdf = specular_hit ? d : 1.0f / pi;  // samplingPDF
    return r;
}

// CookTorrance.glsl evaluateBrdfPdf at the light direction l: the diffuse-sample form of the value
// (F G D v.h sin(theta_h) / v.n) plus the diffuse colour / pi
VPT_DEV F3 cook_torrance_pdf_value(const TraceParams& P, const IsoFrame& fr, F3 l) {
    const float pi = 3.14159265358979323846f;
    const float metallic = P.brdf[kBrdfMetallic], specular = P.brdf[kBrdfSpecular];
    const float rough = fminf(fmaxf(P.brdf[kBrdfRoughness], 0.05f), 1.0f);
    const float alpha = rough * rough;
    const float alpha2 = alpha * alpha;
    const F3 view = fr.view, n = fr.n;
    const F3 h = normalize3(f3(l.x + view.x, l.y + view.y, l.z + view.z));
    const float ndoth = dot3(h, n), vdotn = dot3(view, n), ldotn = dot3(l, n), vdoth = dot3(view, h);
    const float f0s = 0.16f * (specular * specular);
    const float p5 = m_pow5(1.0f - vdoth);
    const float k = alpha / 2.0f;
    const float gl = ldotn < 0.001f ? 0.001f : ldotn, gv = vdotn < 0.001f ? 0.001f : vdotn;
    const float g = (gl / (gl * (1.0f - k) + k)) * (gv / (gv * (1.0f - k) + k));
    const float bq = (ndoth * ndoth) * (alpha2 - 1.0f) + 1.0f;
    const float d = ((1.0f / pi) * alpha2) / (bq * bq);
    const float sth = sqrtf(1.0f - fminf(ndoth * ndoth, 0.95f));
    const float cx[3] = {P.iso_color.x, P.iso_color.y, P.iso_color.z};
    float o[3];
    for (int i = 0; i < 3; ++i) {
        const float f0 = f0s * (1.0f - metallic) + cx[i] * metallic;
        const float f = f0 + (1.0f - f0) * p5;
        const float spec = ((((f * g) * d) * vdoth) * sth) / vdotn;
        o[i] = ((cx[i] * (1.0f - f)) * (1.0f - metallic)) * (1.0f / pi) + spec;
    }
    return f3(o[0], o[1], o[2]);
}

// Disney2012.glsl computeBrdf: sampleBrdf picks the anisotropic specular lobe (weight metallic +
// (1 + specular)(1 - roughness)), the diffuse lobe ((1 - metallic)(1 + roughness) + subsurface) or the
// clearcoat lobe (clamp(clearcoat, 0, 1)); evaluateBrdf returns diffuse + specular + clearcoat as the
// shader writes them (its cos-of-a-cosine Fresnel arguments and its D term included), and the throughput
// takes that value as it is.  sel, u are the hit's second and third random numbers.
VPT_DEV IsoBrdfSample iso_disney(const TraceParams& P, Rng& rng, const IsoFrame& fr, float sel, float u) {
    const F3 n = fr.n, t = fr.t, b = fr.b, view = fr.view;
    const float pi = 3.14159265358979323846f;  // M_PI
    const float pi_c = 3.14159265359f;         // PI (VptUtils.glsl:27), used by GTR1 and atan2
    const float* q = P.brdf;
    const float roughness = q[kBrdfRoughness], metallic = q[kBrdfMetallic];
    const float aspect = sqrtf(1.0f - q[kBrdfAnisotropic] * 0.9f);
    const float r2 = roughness * roughness;
    const float ax0 = r2 / aspect, ay0 = r2 * aspect;
    const float ax = 0.001f < ax0 ? ax0 : 0.001f, ay = 0.001f < ay0 ? ay0 : 0.001f;
    // sampleBrdf
    const float specular_w = metallic + (1.0f + q[kBrdfSpecular]) * (1.0f - roughness);
    const float diffuse_w = (1.0f - metallic) * (1.0f + roughness) + q[kBrdfSubsurface];
    const float clearcoat_w = fminf(fmaxf(q[kBrdfClearcoat], 0.0f), 1.0f);
    const float norm = 1.0f / ((specular_w + diffuse_w) + clearcoat_w);
    const float specular_p = specular_w * norm, diffuse_p = diffuse_w * norm;
    const float v0 = rng_next(rng);
    const int lobe = sel < specular_p ? 0 : (sel < specular_p + diffuse_p ? 1 : 2);  // specular, diffuse, clearcoat
    const bool specular_hit = lobe != 1, clearcoat_hit = lobe == 2;
    float th;
    F3 h, l;
    if (lobe == 0) {  // sample_specular_disney
        const float us = fminf(fmaxf(u, 0.05f), 0.95f), vs = fminf(fmaxf(v0, 0.05f), 0.95f);
        const float a = (2.0f * pi) * us;
        const float y = ay * m_tan(a);
        // the shader's own atan2 (Disney2012.glsl): atan(y, x) when |x| > |y|, else PI / 2 - atan(x, y)
        const float phi = fabsf(ax) > fabsf(y) ? m_atan2(y, ax) : pi_c / 2.0f - m_atan2(ax, y);
        const float cp = m_cos(phi), sp = m_sin(phi);
        th = m_acos(sqrtf((1.0f - vs) / (1.0f + ((cp * cp) / (ax * ax) + (sp * sp) / (ay * ay)) * vs)));
        const float sq = sqrtf(vs / (1.0f - vs));
        const float ca = ax * m_cos(a), sa = ay * m_sin(a);
        const F3 m = f3(ca * t.x + sa * b.x, ca * t.y + sa * b.y, ca * t.z + sa * b.z);
        h = normalize3(f3(sq * m.x + n.x, sq * m.y + n.y, sq * m.z + n.z));
    } else {
        const float phi = (2.0f * pi) * v0;
        float cth;
        if (!clearcoat_hit) {  // sample_diffuse_disney
            th = m_asin(sqrtf(u));
            cth = m_cos(th);
        } else {  // sample_clearcoat_disney with alpha = mix(0.1, 0.001, clearcoatGloss)
            const float g = q[kBrdfClearcoatGloss];
            const float alpha = 0.1f * (1.0f - g) + 0.001f * g;
            const float alpha2 = alpha * alpha;
            th = m_acos(sqrtf((1.0f - m_pow(alpha2, 1.0f - u)) / (1.0f - alpha2)));
            cth = m_cos(th);
        }
        const float st = m_sin(th);
        h = iso_frame(t, b, n, st * m_cos(phi), st * m_sin(phi), cth);
    }
    if (specular_hit) {
        const float vh = fabsf(dot3(view, h));
        const float s = 2.0f * (vh > 0.001f ? vh : 0.001f);  // avoidZero(v.h, 0.001)
        l = f3(s * h.x - view.x, s * h.y - view.y, s * h.z - view.z);
    } else {
        l = h;  // the diffuse lobe samples the direction itself
    }
    // evaluateBrdf
    const F3 hh = normalize3(f3(l.x + view.x, l.y + view.y, l.z + view.z));
    const float cos_h = dot3(hh, n), cos_d = dot3(l, hh), cos_v = dot3(view, n), cos_l = dot3(l, n);
    const float vdoth = dot3(view, hh);
    const float c[3] = {P.iso_color.x, P.iso_color.y, P.iso_color.z};
    const float lum = (0.3f * c[0] + 0.6f * c[1]) + 0.1f * c[2];
    const float cd = m_cos(cos_d);
    const float cd2 = cd * cd;  // pow(x, 2) of a positive x
    const float f_d90 = 0.5f + (2.0f * roughness) * cd2;
    const float pl = m_pow5(1.0f - m_cos(cos_l)), pv = m_pow5(1.0f - m_cos(cos_v));
    const float f_d = (1.0f + (f_d90 - 1.0f) * pl) * (1.0f + (f_d90 - 1.0f) * pv);
    const float fss90 = roughness * cd2;
    const float f_ss = (1.0f + (fss90 - 1.0f) * pl) * (1.0f + (fss90 - 1.0f) * pv);
    const float lv = cos_l + cos_v;
    const float f_dss = 1.25f * (f_ss * (1.0f / (lv < 0.001f ? 0.001f : lv) - 0.5f) + 0.5f);
    const float f_h = m_pow5(1.0f - cos_d);
    const float sub = q[kBrdfSubsurface];
    const float fd_mix = f_d * (1.0f - sub) + f_dss * sub;
    const float dx = dot3(t, hh) / ax, dy = dot3(b, hh) / ay;
    const float dd = dx * dx + dy * dy;
    const float d_spec = 1.0f / (((pi * ax) * ay) * (dd * dd) + cos_h * cos_h);
    const float glx = dot3(t, l) * ax, gly = dot3(b, l) * ay, gvx = dot3(t, view) * ax, gvy = dot3(b, view) * ay;
    float g_spec = 1.0f / (cos_v + sqrtf((glx * glx + gly * gly) + cos_v * cos_v));
    g_spec = g_spec * (1.0f / (cos_v + sqrtf((gvx * gvx + gvy * gvy) + cos_v * cos_v)));
    const float sin_th = m_sin(th);
    const float f_cc = 0.04f * (1.0f - f_h) + 1.0f * f_h;
    const float gloss = q[kBrdfClearcoatGloss];
    const float a_cc = 0.1f * (1.0f - gloss) + 0.001f * gloss;
    float d_cc;  // GTR1(cos_h, a_cc)
    if (a_cc >= 1.0f) {
        d_cc = 1.0f / pi_c;
    } else {
        const float a2 = a_cc * a_cc;
        d_cc = (a2 - 1.0f) / ((pi_c * m_log(a2)) * (1.0f + ((a2 - 1.0f) * cos_h) * cos_h));
    }
    const float bl = cos_l * cos_l, bv = cos_v * cos_v, ag = 0.25f * 0.25f;
    const float g_cc = (1.0f / ((cos_l < -0.99f ? -0.99f : cos_l) + sqrtf((ag + bl) - ag * bl))) *
                       (1.0f / ((cos_v < -0.99f ? -0.99f : cos_v) + sqrtf((ag + bv) - ag * bv)));
    const float cc = q[kBrdfClearcoat];
    const float clear = (specular_hit && clearcoat_hit)
                            ? (((((cc * f_cc) * g_cc) * cos_l) * vdoth) * sin_th) / cos_h
                            : ((((((cc * f_cc) * d_cc) * g_cc) * cos_l) * vdoth) * sin_th);
    const float st = q[kBrdfSpecularTint], sh = q[kBrdfSheenTint];
    const float spec_scale = q[kBrdfSpecular] * 0.08f;
    float o[3];
    for (int i = 0; i < 3; ++i) {
        const float tint = lum > 0.0f ? c[i] / lum : 1.0f;
        const float spec0 = (spec_scale * (1.0f * (1.0f - st) + tint * st)) * (1.0f - metallic) + c[i] * metallic;
        const float sheen_c = 1.0f * (1.0f - sh) + tint * sh;
        const float sheen = (f_h * q[kBrdfSheen]) * sheen_c;
        float diffuse = (c[i] * fd_mix + sheen) * (1.0f - metallic);
        if (specular_hit) diffuse = diffuse * (1.0f / pi);
        const float f_spec = spec0 * (1.0f - f_h) + 1.0f * f_h;
        const float spec = (specular_hit && !clearcoat_hit)
                               ? (((((f_spec * g_spec) * 4.0f) * cos_l) * vdoth) * sin_th) / cos_h
                               : ((((((f_spec * d_spec) * g_spec) * 4.0f) * cos_l) * vdoth) * sin_th);
        o[i] = (diffuse + spec) + clear;
    }
    IsoBrdfSample r;
    r.dir = l;
    r.value = f3(o[0], o[1], o[2]);
    r.specular = specular_hit;
    r.clearcoat = clearcoat_hit;
    r.pdf = specular_hit ? (clearcoat_hit ? d_cc : d_spec) : 1.0f / pi;  // samplingPDF
    return r;
}

// Disney2012.glsl evaluateBrdfPdf at the light direction l: the terms of evaluateBrdf in their
// non-specular-sample form, the diffuse term always divided by pi, sin(theta_h) from
// sqrt(1 - min(n.h^2, 0.95)), and 0.01 as the floor of the subsurface denominator
VPT_DEV F3 disney_pdf_value(const TraceParams& P, const IsoFrame& fr, F3 l) {
    const float pi = 3.14159265358979323846f, pi_c = 3.14159265359f;
    const float* q = P.brdf;
    const float roughness = q[kBrdfRoughness], metallic = q[kBrdfMetallic];
    const float aspect = sqrtf(1.0f - q[kBrdfAnisotropic] * 0.9f);
    const float r2 = roughness * roughness;
    const float ax0 = r2 / aspect, ay0 = r2 * aspect;
    const float ax = 0.001f < ax0 ? ax0 : 0.001f, ay = 0.001f < ay0 ? ay0 : 0.001f;
    const F3 view = fr.view, n = fr.n, t = fr.t, b = fr.b;
    const F3 hh = normalize3(f3(l.x + view.x, l.y + view.y, l.z + view.z));
    const float cos_h = dot3(hh, n), cos_d = dot3(l, hh), cos_v = dot3(view, n), cos_l = dot3(l, n);
    const float vdoth = dot3(view, hh);
    const float c[3] = {P.iso_color.x, P.iso_color.y, P.iso_color.z};
    const float lum = (0.3f * c[0] + 0.6f * c[1]) + 0.1f * c[2];
    const float cd = m_cos(cos_d);
    const float cd2 = cd * cd;
    const float f_d90 = 0.5f + (2.0f * roughness) * cd2;
    const float pl = m_pow5(1.0f - m_cos(cos_l)), pv = m_pow5(1.0f - m_cos(cos_v));
    const float f_d = (1.0f + (f_d90 - 1.0f) * pl) * (1.0f + (f_d90 - 1.0f) * pv);
    const float fss90 = roughness * cd2;
    const float f_ss = (1.0f + (fss90 - 1.0f) * pl) * (1.0f + (fss90 - 1.0f) * pv);
    const float lv = cos_l + cos_v;
    const float f_dss = 1.25f * (f_ss * (1.0f / (lv < 0.01f ? 0.01f : lv) - 0.5f) + 0.5f);
    const float f_h = m_pow5(1.0f - cos_d);
    const float sub = q[kBrdfSubsurface];
    const float fd_mix = f_d * (1.0f - sub) + f_dss * sub;
    const float dx = dot3(t, hh) / ax, dy = dot3(b, hh) / ay;
    const float dd = dx * dx + dy * dy;
    const float d_spec = 1.0f / (((pi * ax) * ay) * (dd * dd) + cos_h * cos_h);
    const float glx = dot3(t, l) * ax, gly = dot3(b, l) * ay, gvx = dot3(t, view) * ax, gvy = dot3(b, view) * ay;
    float g_spec = 1.0f / (cos_v + sqrtf((glx * glx + gly * gly) + cos_v * cos_v));
    g_spec = g_spec * (1.0f / (cos_v + sqrtf((gvx * gvx + gvy * gvy) + cos_v * cos_v)));
    const float sth = sqrtf(1.0f - fminf(cos_h * cos_h, 0.95f));
    const float f_cc = 0.04f * (1.0f - f_h) + 1.0f * f_h;
    const float gloss = q[kBrdfClearcoatGloss];
    const float a_cc = 0.1f * (1.0f - gloss) + 0.001f * gloss;
    float d_cc;
    if (a_cc >= 1.0f) {
        d_cc = 1.0f / pi_c;
    } else {
        const float a2 = a_cc * a_cc;
        d_cc = (a2 - 1.0f) / ((pi_c * m_log(a2)) * (1.0f + ((a2 - 1.0f) * cos_h) * cos_h));
    }
    const float bl = cos_l * cos_l, bv = cos_v * cos_v, ag = 0.25f * 0.25f;
    const float g_cc = (1.0f / ((cos_l < -0.99f ? -0.99f : cos_l) + sqrtf((ag + bl) - ag * bl))) *
                       (1.0f / ((cos_v < -0.99f ? -0.99f : cos_v) + sqrtf((ag + bv) - ag * bv)));
    const float clear = (((((q[kBrdfClearcoat] * f_cc) * d_cc) * g_cc) * cos_l) * vdoth) * sth;
    const float st = q[kBrdfSpecularTint], sh = q[kBrdfSheenTint];
    const float spec_scale = q[kBrdfSpecular] * 0.08f;
    float o[3];
    for (int i = 0; i < 3; ++i) {
        const float tint = lum > 0.0f ? c[i] / lum : 1.0f;
        const float spec0 = (spec_scale * (1.0f * (1.0f - st) + tint * st)) * (1.0f - metallic) + c[i] * metallic;
        const float sheen = (f_h * q[kBrdfSheen]) * (1.0f * (1.0f - sh) + tint * sh);
        const float diffuse = ((c[i] * fd_mix + sheen) * (1.0f - metallic)) * (1.0f / pi);
        const float f_spec = spec0 * (1.0f - f_h) + 1.0f * f_h;
        const float spec = ((((((f_spec * d_spec) * g_spec) * 4.0f) * cos_l) * vdoth) * sth);
        o[i] = (diffuse + spec) + clear;
    }
    return f3(o[0], o[1], o[2]);
}

// An opaque surface hit (getIsoSurfaceHit, VptUtils.glsl:1151-1334): one random number for the
// opacity test, the normal turned against the ray, the ComputeDefaultBasis frame
// (RayTracingUtilities.glsl:20-28), then the selected BRDF.  Lambertian: a cosine-weighted direction
// (Lambertian.glsl is included before UNIFORM_SAMPLING is defined, so the concentric-disk map of
// VptUtils.glsl:1078-1098 and a pdf factor equal to the cosine), value color * cos / cos.  This part
// ends at computeBrdf and returns the frame and the sample.
VPT_DEV IsoBrdfSample iso_sample(const TraceParams& P, Rng& rng, F3 p, F3 w, IsoFrame& fr, const F3* cam = nullptr) {
    (void)rng_next(rng);  // isoSurfaceOpacity (1) < random() never holds
    F3 n = iso_normal(P, p);
    if (cam) ray_box_normal(P, *cam, w, n);  // a closing surface (CLOSE_ISOSURFACES): the face entered
    else if (dot3(w, n) > 0.0f) n = -n;
    const float yz = -n.y * n.z;
    const F3 b = normalize3(fabsf(n.z) > 0.99999f ? f3(-n.x * n.y, 1.0f - n.y * n.y, yz)
                                                  : f3(-n.x * n.z, yz, 1.0f - n.z * n.z));
    const F3 t = cross3(b, n);
    fr.n = n;
    fr.t = t;
    fr.b = b;
    fr.view = normalize3(f3(-w.x, -w.y, -w.z));
    const float xi0 = rng_next(rng);
    const float xi1 = rng_next(rng);
    if (P.iso_brdf == kBrdfCookTorrance) return iso_cook_torrance(P, rng, fr, xi0, xi1);
    if (P.iso_brdf == kBrdfDisney) return iso_disney(P, rng, fr, xi0, xi1);
    IsoBrdfSample r;
    r.specular = false;
    r.clearcoat = false;
    r.pdf = 0.0f;
    if (P.iso_brdf != kBrdfLambertian) {
        // BlinnPhong.glsl / ConstantLighting.glsl: a uniformly sampled hemisphere direction
        // (sampleHemisphere, VptUtils.glsl:1071-1077: phi = 2 pi xi.y, z = xi.x) in the same frame
        const float pi = 3.14159265358979323846f;  // M_PI as the shader's float
        const float phi = (2.0f * pi) * xi1;
        const float rr = sqrtf(1.0f - xi0 * xi0);
        const float lx = m_cos(phi) * rr, ly = m_sin(phi) * rr;
        const F3 out = f3((t.x * lx + b.x * ly) + n.x * xi0, (t.y * lx + b.y * ly) + n.y * xi0,
                          (t.z * lx + b.z * ly) + n.z * xi0);
        F3 c = P.iso_color;  // ConstantLighting.glsl: the colour, whatever the direction
        if (P.iso_brdf == kBrdfBlinnPhong) {
            // BlinnPhong.glsl evaluateBrdf: 2 pi colour (n.h)^10 / norm, h = normalize(normalize(-w) + l),
            // norm = clamp((n + 2) / (4 pi 2^(-n/2)), (n + 2) / (8 pi), (n + 4) / (8 pi)) with n = 10
            const F3 h = normalize3(f3(fr.view.x + out.x, fr.view.y + out.y, fr.view.z + out.z));
            const float e = 10.0f;
            const float norm = fminf(fmaxf((e + 2.0f) / ((4.0f * pi) * 0.03125f), (e + 2.0f) / (8.0f * pi)),
                                     (e + 4.0f) / (8.0f * pi));
            const float s = m_pow(fmaxf(dot3(n, h), 0.0f), e) / norm;
            const float k = 2.0f * pi;
            c = f3((k * P.iso_color.x) * s, (k * P.iso_color.y) * s, (k * P.iso_color.z) * s);
        }
        r.dir = out;
        r.value = c;
        return r;
    }
    const float ox = 2.0f * xi0 - 1.0f, oy = 2.0f * xi1 - 1.0f;
    float dx = 0.0f, dy = 0.0f;
    if (!(ox == 0.0f && oy == 0.0f)) {
        float rad, th;
        if (fabsf(ox) > fabsf(oy)) {
            rad = ox;
            th = 0.785398185f * (oy / ox);  // pi / 4 in float
        } else {
            rad = oy;
            th = 1.57079637f - 0.785398185f * (ox / oy);  // pi / 2 - pi / 4 * ...
        }
        dx = rad * cosf(th);
        dy = rad * sinf(th);
    }
    const float hz = sqrtf(1.0f - dx * dx - dy * dy);
    const F3 out = f3((t.x * dx + b.x * dy) + n.x * hz, (t.y * dx + b.y * dy) + n.y * hz,
                      (t.z * dx + b.z * dy) + n.z * hz);
    const float cosv = dot3(out, n);
    r.dir = out;
    r.value = f3((P.iso_color.x * cosv) / cosv, (P.iso_color.y * cosv) / cosv, (P.iso_color.z * cosv) / cosv);
    return r;
}

// An opaque surface hit without next-event estimation: throughput *= the BRDF value, w = its direction.
VPT_DEV void iso_scatter(const TraceParams& P, Rng& rng, F3 p, F3& w, F3& weights) {
    IsoFrame fr;
    const IsoBrdfSample s = iso_sample(P, rng, p, w, fr);
    weights = f3(weights.x * s.value.x, weights.y * s.value.y, weights.z * s.value.z);
    w = s.dir;
}

// evaluateBrdfNee of the selected BRDF for the light direction l (USE_ISOSURFACE_NEE): the value the
// light sample is weighed with, and the sampling pdfs of the BRDF's own direction and of l that MIS
// reads (the specular BRDFs only).  Lambertian.glsl takes its non-uniform branch (UNIFORM_SAMPLING is
// defined after it is included): colour / pi * n.l.
VPT_DEV F3 iso_brdf_nee(const TraceParams& P, const IsoFrame& fr, const IsoBrdfSample& s, F3 l, float& pdf_out,
                        float& pdf_nee) {
    const float pi = 3.14159265358979323846f;
    const F3 c = P.iso_color;
    pdf_out = 0.0f;
    pdf_nee = 0.0f;
    if (P.iso_brdf == kBrdfLambertian) {
        const float th = dot3(fr.n, l);
        return f3((c.x / pi) * th, (c.y / pi) * th, (c.z / pi) * th);
    }
    if (P.iso_brdf == kBrdfAmbient) {
        const float k = 2.0f * pi;
        return f3(c.x / k, c.y / k, c.z / k);
    }
    if (P.iso_brdf == kBrdfBlinnPhong) {
        const float e = 10.0f;
        const float norm = fminf(fmaxf((e + 2.0f) / ((4.0f * pi) * 0.03125f), (e + 2.0f) / (8.0f * pi)),
                                 (e + 4.0f) / (8.0f * pi));
        const F3 h = normalize3(f3(fr.view.x + l.x, fr.view.y + l.y, fr.view.z + l.z));
        const float v = m_pow(fmaxf(dot3(fr.n, h), 0.0f), e) / norm;
        return f3(c.x * v, c.y * v, c.z * v);
    }
    const F3 h = normalize3(f3(s.dir.x + fr.view.x, s.dir.y + fr.view.y, s.dir.z + fr.view.z));
    const float cos_h = dot3(h, fr.n);
    const float sin_h = sqrtf(1.0f / (cos_h * cos_h));  // as the shaders write it
    const F3 hn = normalize3(f3(l.x + fr.view.x, l.y + fr.view.y, l.z + fr.view.z));
    const float cos_hn = dot3(hn, fr.n);
    const float sin_hn = sqrtf(1.0f - fminf(cos_hn * cos_hn, 0.95f));
    if (P.iso_brdf == kBrdfDisney && s.specular) {
        pdf_out = s.pdf * cos_h;
        pdf_nee = s.pdf * cos_hn;
    } else {
        pdf_out = (s.pdf * cos_h) * sin_h;
        pdf_nee = (s.pdf * cos_hn) * sin_hn;
    }
    const F3 v = P.iso_brdf == kBrdfDisney ? disney_pdf_value(P, fr, l) : cook_torrance_pdf_value(P, fr, l);
    const float nl = dot3(l, fr.n);
    return f3(v.x * nl, v.y * nl, v.z * nl);
}

}  // namespace vpt
