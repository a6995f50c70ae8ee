// vpt_oracle.cpp - CPU oracle (TEST INFRASTRUCTURE ONLY): a restatement of the reference's
// volumetric path-tracing shaders for checking the CUDA core and for the timed CPU baseline.
// Each function cites the reference file:line it follows (paths inside chrismile/CloudRendering).
// Build: oracle/build_oracle.py (g++ -O3 -fopenmp -ffp-contract=off).
#include "vpt_oracle.h"

#include <math.h>
#include <string.h>
#include <algorithm>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const float PI = 3.14159265359f;  // VptUtils.glsl:27
const float TWO_PI = 2.0f * 3.14159265359f;

// Transcendentals of the tracer: the C library's float functions, or (oracle_set_double_rounded_math)
// the double-precision functions rounded once to float, the mode of the CUDA core's
// libvpt_b200_dr.so.  In that mode both sides return the correctly rounded float except on
// arguments whose exact result lies within about one double ulp of a float rounding boundary.
bool g_dr_math = false;
inline float m_log(float x) { return g_dr_math ? (float)log((double)x) : logf(x); }
inline float m_exp(float x) { return g_dr_math ? (float)exp((double)x) : expf(x); }
inline float m_sin(float x) { return g_dr_math ? (float)sin((double)x) : sinf(x); }
inline float m_cos(float x) { return g_dr_math ? (float)cos((double)x) : cosf(x); }
inline float m_pow(float x, float y) { return g_dr_math ? (float)pow((double)x, (double)y) : powf(x, y); }
inline float m_atan2(float y, float x) { return g_dr_math ? (float)atan2((double)y, (double)x) : atan2f(y, x); }
inline float m_asin(float x) { return g_dr_math ? (float)asin((double)x) : asinf(x); }
inline float m_acos(float x) { return g_dr_math ? (float)acos((double)x) : acosf(x); }
inline float m_tan(float x) { return g_dr_math ? (float)tan((double)x) : tanf(x); }
inline float m_pow5(float x) { return g_dr_math ? (float)pow((double)x, 5.0) : powf(x, 5.0f); }

struct V3 {
    float x, y, z;
};
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 mul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 mulv(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 divv(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
inline float length(V3 a) { return sqrtf(dot(a, a)); }
inline V3 normalize(V3 a) {
    float l = length(a);
    return v3(a.x / l, a.y / l, a.z / l);
}
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline float clampf(float v, float lo, float hi) { return std::min(std::max(v, lo), hi); }
inline float smoothstepf(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
inline float signf(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }

// ---- RNG (VptUtils.glsl:48-65) ----
struct Rng {
    uint32_t x, y, z, w;
};
inline uint32_t taus(uint32_t z, int s1, int s2, int s3, uint32_t m) {
    uint32_t b = ((z << s1) ^ z) >> s2;
    return ((z & m) << s3) ^ b;
}
inline float rnd(Rng& r) {
    r.x = taus(r.x, 13, 19, 12, 4294967294u);
    r.y = taus(r.y, 2, 25, 4, 4294967288u);
    r.z = taus(r.z, 3, 11, 17, 4294967280u);
    r.w = 1664525u * r.w + 1013904223u;
    return 2.3283064365387e-10f * (float)(r.x ^ r.y ^ r.z ^ r.w);
}
inline Rng rng_init(uint32_t seed) {
    Rng r{seed, seed, seed, seed};
    for (uint32_t i = 0; i < seed % 7u + 2u; i++) rnd(r);
    return r;
}

// ---- camera ray (VptUtils.glsl:750-761) ----
void mat_point(const float* m, float x, float y, float z, float w, float o[4]) {
    for (int r = 0; r < 4; r++) o[r] = ((m[r] * x + m[4 + r] * y) + m[8 + r] * z) + m[12 + r] * w;
}
void camera_ray(const OracleScene& S, float sx, float sy, V3& x, V3& w) {
    float p[4], t[4];
    mat_point(S.inv_view_proj, sx, sy, 0.0f, 1.0f, p);
    mat_point(S.inv_view_proj, sx, sy, 1.0f, 1.0f, t);
    V3 vp = v3(p[0] / p[3], p[1] / p[3], p[2] / p[3]);
    V3 vt = v3(t[0] / t[3], t[1] / t[3], t[2] / t[3]);
    x = vp;
    w = normalize(sub(vt, vp));
}

// USE_CLIP_PLANE: the normalised plane normal and distance of the scene being rendered, or null
static const float* g_clip = nullptr;

// ---- rayBoxIntersect (VptUtils.glsl:763-801), with the clip plane's interval cut when it is on ----
bool ray_box(V3 bmin, V3 bmax, V3 p, V3 d, float& tmin, float& tmax) {
    d.x = fabsf(d.x) <= 0.000001f ? 0.000001f : d.x;
    d.y = fabsf(d.y) <= 0.000001f ? 0.000001f : d.y;
    d.z = fabsf(d.z) <= 0.000001f ? 0.000001f : d.z;
    V3 cmin = divv(sub(bmin, p), d), cmax = divv(sub(bmax, p), d);
    tmin = std::max(std::max(std::min(cmin.x, cmax.x), std::min(cmin.y, cmax.y)), std::min(cmin.z, cmax.z));
    tmin = std::max(0.0f, tmin);
    tmax = std::min(std::min(std::max(cmin.x, cmax.x), std::max(cmin.y, cmax.y)), std::max(cmin.z, cmax.z));
    if (tmax <= tmin || tmax <= 0.0f) return false;
    if (g_clip) {  // the part of the ray on the plane's positive side (the direction as modified above)
        const V3 n = v3(g_clip[0], g_clip[1], g_clip[2]);
        const float denom = dot(n, d);
        const float dp = dot(n, p) - g_clip[3];
        if (fabsf(denom) < 0.001f) return dp > 0.0f;
        const float t_clip = (g_clip[3] - dot(n, p)) / denom;
        if (t_clip <= 0.0f) return dp > 0.0f;
        if (dp > 0.0f) tmax = std::min(t_clip, tmax);
        else tmin = std::max(t_clip, tmin);
        if (tmax <= tmin || tmax <= 0.0f) return false;
    }
    return true;
}

// rayBoxIntersectionNormal (VptUtils.glsl:803-856, CLOSE_ISOSURFACES): the entered face's normal, or
// -clip normal where the clip plane is the entry surface; n unchanged in the cases the shader leaves it
void ray_box_normal(V3 bmin, V3 bmax, V3 p, V3 d, V3& n) {
    d.x = fabsf(d.x) <= 1e-6f ? 1e-6f : d.x;
    d.y = fabsf(d.y) <= 1e-6f ? 1e-6f : d.y;
    d.z = fabsf(d.z) <= 1e-6f ? 1e-6f : d.z;
    const V3 cmin = divv(sub(bmin, p), d), cmax = divv(sub(bmax, p), d);
    const float mx = std::min(cmin.x, cmax.x), my = std::min(cmin.y, cmax.y), mz = std::min(cmin.z, cmax.z);
    const float tmin = std::max(0.0f, std::max(std::max(mx, my), mz));
    const float tmax = std::min(std::min(std::max(cmin.x, cmax.x), std::max(cmin.y, cmax.y)), std::max(cmin.z, cmax.z));
    if (tmax <= tmin || tmax <= 0.0f) return;
    auto sgn = [](float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); };
    V3 nb;
    if (mx > my && mx > mz) nb = v3(-sgn(d.x), 0.0f, 0.0f);
    else if (my > mz) nb = v3(0.0f, -sgn(d.y), 0.0f);
    else nb = v3(0.0f, 0.0f, -sgn(d.z));
    if (g_clip) {
        const V3 cn = v3(g_clip[0], g_clip[1], g_clip[2]);
        const float denom = dot(cn, d);
        const float dp = dot(cn, p) - g_clip[3];
        if (fabsf(denom) < 1e-3f) {
            if (dp > 0.0f) n = nb;
            return;
        }
        const float t_clip = (g_clip[3] - dot(cn, p)) / denom;
        if (t_clip <= 0.0f) {
            if (dp > 0.0f) n = nb;
            return;
        }
        if (dp <= 0.0f && t_clip >= tmin) {
            n = v3(-cn.x, -cn.y, -cn.z);
            return;
        }
    }
    n = nb;
}

// ---- directions (VptUtils.glsl:67-123) ----
void basis(V3 d, V3& b, V3& t) {
    V3 other = fabsf(d.z) >= 0.9999f ? v3(1, 0, 0) : v3(0, 0, 1);
    b = normalize(cross(other, d));
    t = normalize(cross(d, b));
}
V3 random_direction(Rng& r, V3 d) {
    float r1 = rnd(r);
    float r2 = rnd(r) * 2.0f - 1.0f;
    float s = sqrtf(1.0f - r2 * r2);
    float a = TWO_PI * r1;
    float x = m_cos(a) * s, y = m_sin(a) * s;
    V3 t0, t1;
    basis(d, t0, t1);
    return add(add(mul(t0, x), mul(t1, y)), mul(d, r2));
}
V3 sample_phase(Rng& r, float g, V3 d) {
    if (fabsf(g) < 0.001f) return random_direction(r, neg(d));
    float phi = rnd(r) * 2.0f * PI;
    float xi = rnd(r);
    float t = (1.0f - g * g) / (1.0f - g + 2.0f * g * xi);
    float cos_t = (0.5f / g) * ((1.0f + g * g) - t * t);
    float sin_t = sqrtf(std::max(0.0f, 1.0f - cos_t * cos_t));
    V3 t0, t1;
    basis(d, t0, t1);
    return add(add(mul(t0, sin_t * m_sin(phi)), mul(t1, sin_t * m_cos(phi))), mul(d, cos_t));
}
float eval_phase(float g, V3 a, V3 b) {
    float c = dot(normalize(a), normalize(b));
    return ((0.25f / PI) * (1.0f - g * g)) / m_pow((1.0f + g * g) - 2.0f * g * c, 1.5f);
}

// ---- sky and sun (VptUtils.glsl:288-389, 125-267) ----
float srgb_to_lin(float c) { return c <= 0.04045f ? c / 12.92f : m_pow((c + 0.055f) / 1.055f, 2.4f); }
float lin_to_srgb(float c) { return c <= 0.0031308f ? c * 12.92f : 1.055f * m_pow(c, 1.0f / 2.4f) - 0.055f; }

V3 sky_default(V3 dir, int lin) {
    const float cr[5] = {0.1f, 0.01f, 0.8f, 0.1f, 0.01f};
    const float cg[5] = {0.05f, 0.05f, 0.9f, 0.3f, 0.1f};
    const float cb[5] = {0.01f, 0.2f, 1.0f, 1.0f, 0.7f};
    const float ds[5] = {-1.0f, -0.1f, 0.0f, 0.4f, 1.0f};
    float r = cr[0], g = cg[0], b = cb[0];
    for (int i = 1; i < 5; i++) {
        float s = smoothstepf(ds[i - 1], ds[i], dir.y);
        r = mixf(r, cr[i], s);
        g = mixf(g, cg[i], s);
        b = mixf(b, cb[i], s);
    }
    if (lin) return v3(srgb_to_lin(r), srgb_to_lin(g), srgb_to_lin(b));
    return v3(r, g, b);
}
V3 sun_lobe(const OracleScene& S, V3 dir) {
    const float norm = 11.0f / (2.0f * 3.14159f);
    float p = m_pow(std::max(0.0f, dot(dir, v3(S.sun_dir[0], S.sun_dir[1], S.sun_dir[2]))), 10.0f);
    return v3((S.sun_intensity[0] * p) * norm, (S.sun_intensity[1] * p) * norm, (S.sun_intensity[2] * p) * norm);
}
V3 env_fetch(const OracleScene& S, float u, float v) {
    float fx = u * (float)S.env_w - 0.5f, fy = v * (float)S.env_h - 0.5f;
    float x0f = floorf(fx), y0f = floorf(fy);
    float ax = fx - x0f, ay = fy - y0f;
    int x0 = (int)x0f, y0 = (int)y0f, w = S.env_w, h = S.env_h;
    int xa = ((x0 % w) + w) % w, xb = (((x0 + 1) % w) + w) % w;
    int ya = ((y0 % h) + h) % h, yb = (((y0 + 1) % h) + h) % h;
    const float* c00 = S.env_rgba + ((size_t)ya * w + xa) * 4;
    const float* c10 = S.env_rgba + ((size_t)ya * w + xb) * 4;
    const float* c01 = S.env_rgba + ((size_t)yb * w + xa) * 4;
    const float* c11 = S.env_rgba + ((size_t)yb * w + xb) * 4;
    float o[3];
    for (int c = 0; c < 3; c++) o[c] = mixf(mixf(c00[c], c10[c], ax), mixf(c01[c], c11[c], ax), ay);
    return v3(o[0], o[1], o[2]);
}
// USE_ENV_MAP_ROTATION (VptUtils.glsl:142-153, 303-306): parameters.envMapDirRot * v (column-major,
// columns summed in order) and the transpose invEnvMapDirRot * v
V3 env_rot(const OracleScene& S, V3 v) {
    const float* m = S.env_rot_m;
    return v3((m[0] * v.x + m[3] * v.y) + m[6] * v.z, (m[1] * v.x + m[4] * v.y) + m[7] * v.z,
              (m[2] * v.x + m[5] * v.y) + m[8] * v.z);
}
V3 env_rot_inv(const OracleScene& S, V3 v) {
    const float* m = S.env_rot_m;
    return v3((m[0] * v.x + m[1] * v.y) + m[2] * v.z, (m[3] * v.x + m[4] * v.y) + m[5] * v.z,
              (m[6] * v.x + m[7] * v.y) + m[8] * v.z);
}
V3 sky_image(const OracleScene& S, V3 dir) {
    if (S.env_rot) dir = env_rot(S, dir);
    float u = m_atan2(dir.z, dir.x) / TWO_PI + 0.5f;
    float v = -m_asin(dir.y) / PI + 0.5f;
    V3 c = env_fetch(S, u, v);
    c = v3(std::min(c.x, 100000.0f), std::min(c.y, 100000.0f), std::min(c.z, 100000.0f));
    if (!S.env_image_linear && S.use_linear_rgb) c = v3(srgb_to_lin(c.x), srgb_to_lin(c.y), srgb_to_lin(c.z));
    else if (S.env_image_linear && !S.use_linear_rgb) c = v3(lin_to_srgb(c.x), lin_to_srgb(c.y), lin_to_srgb(c.z));
    return mulv(v3(S.env_intensity[0], S.env_intensity[1], S.env_intensity[2]), c);
}
V3 sky_and_sun(const OracleScene& S, V3 dir) {
    switch (S.env_kind) {
        case 0: return add(sky_default(dir, S.use_linear_rgb), sun_lobe(S, dir));
        case 1: return v3(0, 0, 0);
        case 2: return v3(S.sun_intensity[0], S.sun_intensity[1], S.sun_intensity[2]);
        case 3: return add(v3(S.sky_color[0], S.sky_color[1], S.sky_color[2]), sun_lobe(S, dir));
        default: return sky_image(S, dir);
    }
}

V3 oct_to_world(float u, float v) {
    u = u * 2.0f - 1.0f;
    v = v * 2.0f - 1.0f;
    float sx = signf(u), sy = signf(v);
    u = fabsf(u);
    v = fabsf(v);
    float r = 1.0f - fabsf(1.0f - u - v);
    float phi = 0.25f * PI * ((v - u) / r + 1.0f);
    if (r == 0.0f) phi = 0.0f;
    float r2 = r * r, s = sqrtf(2.0f - r2);
    return v3(sx * m_cos(phi) * r * s, sy * m_sin(phi) * r * s, signf(1.0f - u - v) * (1.0f - r2));
}

struct Pyramid {
    std::vector<size_t> off;
};
float pyr(const OracleScene& S, const size_t* off, int level, int x, int y) {
    int res = (1 << S.env_levels) >> level;
    return S.env_pyramid[off[level] + (size_t)y * res + x] + 0.001f;
}
V3 sample_env_image(const OracleScene& S, const size_t* off, Rng& r, float& pdf) {
    float rx = rnd(r), ry = rnd(r);
    int px = 0, py = 0;
    pdf = 0.25f / PI;
    for (int mip = S.env_levels - 1; mip >= 0; mip--) {
        px *= 2;
        py *= 2;
        pdf *= 4.0f;
        float ul = pyr(S, off, mip, px, py), ur = pyr(S, off, mip, px + 1, py);
        float dl = pyr(S, off, mip, px, py + 1), dr = pyr(S, off, mip, px + 1, py + 1);
        float l = ul + dl, rr = ur + dr, total = l + rr;
        float hs = l / total, vs;
        if (rx < hs) {
            rx = rx / hs;
            vs = ul / l;
            pdf *= hs;
        } else {
            px += 1;
            rx = (rx - hs) / (1.0f - hs);
            vs = ur / rr;
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
    float inv = 1.0f / (float)(1 << S.env_levels);
    const V3 dir = oct_to_world(((float)px + rx) * inv, ((float)py + ry) * inv);
    return S.env_rot ? env_rot_inv(S, dir) : dir;
}

// ---- NanoVDB float grids: the read path of PNanoVDB.glsl restated ----
// Layout of a version-32 float grid (PNanoVDB.glsl:712-1171): map at 296 (mMatF, mInvMatF, mVecF),
// tree at 672 (root offset at +24), root: bbox at 0/12, tile count 24, background 28, 32-byte tiles
// from 64 (key, child, state, value); upper: value mask 32, child mask 4128, 8-byte table 8256;
// lower: masks 32 / 544, table 1088; leaf: bbox min 0, value mask 16, values 96.
template <class T>
T rdv(const uint8_t* b, size_t off) {
    T v;
    memcpy(&v, b + off, sizeof(T));
    return v;
}

struct Nano {
    const uint8_t* b = nullptr;
    size_t root = 0;
    uint32_t tiles = 0;
    float background = 0.0f;
    float mat[9], inv[9], vec[3];
    int rmin[3], rmax[3];
    bool fp16 = false;

    void init(const uint8_t* buf, bool half) {
        b = buf;
        fp16 = half;
        for (int i = 0; i < 9; i++) {
            mat[i] = rdv<float>(b, 296 + 4 * i);
            inv[i] = rdv<float>(b, 332 + 4 * i);
        }
        for (int i = 0; i < 3; i++) vec[i] = rdv<float>(b, 368 + 4 * i);
        root = 672 + rdv<uint64_t>(b, 672 + 24);
        for (int i = 0; i < 3; i++) {
            rmin[i] = rdv<int32_t>(b, root + 4 * i);
            rmax[i] = rdv<int32_t>(b, root + 12 + 4 * i);
        }
        tiles = rdv<uint32_t>(b, root + 24);
        background = rdv<float>(b, root + 28);
    }
    bool bit(size_t mask, uint32_t n) const { return (rdv<uint32_t>(b, mask + 4 * (n >> 5)) >> (n & 31u)) & 1u; }
    static uint64_t key(int x, int y, int z) {
        return (uint64_t)((uint32_t)z >> 12) | ((uint64_t)((uint32_t)y >> 12) << 21) |
               ((uint64_t)((uint32_t)x >> 12) << 42);
    }
    static uint32_t upper_off(int x, int y, int z) {
        return (((uint32_t)(x & 4095) >> 7) << 10) | (((uint32_t)(y & 4095) >> 7) << 5) | ((uint32_t)(z & 4095) >> 7);
    }
    static uint32_t lower_off(int x, int y, int z) {
        return (((uint32_t)(x & 127) >> 3) << 8) | (((uint32_t)(y & 127) >> 3) << 4) | ((uint32_t)(z & 127) >> 3);
    }
    static uint32_t leaf_off(int x, int y, int z) {
        return ((uint32_t)(x & 7) << 6) | ((uint32_t)(y & 7) << 3) | (uint32_t)(z & 7);
    }
    // pnanovdb_root_find_tile: linear search over the root tiles; 0 when absent
    size_t find_tile(int x, int y, int z) const {
        const uint64_t k = key(x, y, z);
        for (uint32_t t = 0; t < tiles; t++) {
            size_t tile = root + 64 + 32 * (size_t)t;
            if (rdv<uint64_t>(b, tile) == k) return tile;
        }
        return 0;
    }
    // Node holding (x, y, z): level 0 leaf, 1 lower tile, 2 upper tile, 3 root tile, 4 background.
    struct Where {
        int level;
        size_t tile, upper, lower, leaf;
        uint32_t un, ln;
    };
    Where where(int x, int y, int z) const {
        Where w{4, 0, 0, 0, 0, 0, 0};
        w.tile = find_tile(x, y, z);
        if (!w.tile) return w;
        int64_t child = rdv<int64_t>(b, w.tile + 8);
        if (child == 0) {
            w.level = 3;
            return w;
        }
        w.upper = root + (size_t)child;
        w.un = upper_off(x, y, z);
        if (!bit(w.upper + 4128, w.un)) {
            w.level = 2;
            return w;
        }
        w.lower = w.upper + (size_t)rdv<int64_t>(b, w.upper + 8256 + 8 * (size_t)w.un);
        w.ln = lower_off(x, y, z);
        if (!bit(w.lower + 544, w.ln)) {
            w.level = 1;
            return w;
        }
        w.leaf = w.lower + (size_t)rdv<int64_t>(b, w.lower + 1088 + 8 * (size_t)w.ln);
        w.level = 0;
        return w;
    }
    float leaf_value(size_t leaf, uint32_t off) const {
        float v = rdv<float>(b, leaf + 96 + 4 * (size_t)off);
        if (fp16) v = (float)(_Float16)v;
        return v;
    }
    float value(int x, int y, int z) const {
        Where w = where(x, y, z);
        switch (w.level) {
            case 0: return leaf_value(w.leaf, leaf_off(x, y, z));
            case 1: return rdv<float>(b, w.lower + 1088 + 8 * (size_t)w.ln);
            case 2: return rdv<float>(b, w.upper + 8256 + 8 * (size_t)w.un);
            case 3: return rdv<float>(b, w.tile + 20);
            default: return background;
        }
    }
    int dim(int x, int y, int z) const {
        static const int d[5] = {1, 8, 128, 4096, 4096};
        return d[where(x, y, z).level];
    }
    bool active(int x, int y, int z) const {
        Where w = where(x, y, z);
        switch (w.level) {
            case 0: return bit(w.leaf + 16, leaf_off(x, y, z));
            case 1: return bit(w.lower + 32, w.ln);
            case 2: return bit(w.upper + 32, w.un);
            case 3: return rdv<uint32_t>(b, w.tile + 16) != 0u;
            default: return false;
        }
    }
    // Cell classification of the sparse decomposition tracker at the leaf level
    // (DecompositionTracking.glsl:178-248); returns the level and writes the node box.
    int cell(int x, int y, int z, bool& is_active, V3& bmin, V3& bmax) const {
        Where w = where(x, y, z);
        is_active = false;
        auto box = [&](size_t node) {
            bmin = v3((float)rdv<int32_t>(b, node), (float)rdv<int32_t>(b, node + 4), (float)rdv<int32_t>(b, node + 8));
            bmax = v3((float)rdv<int32_t>(b, node + 12), (float)rdv<int32_t>(b, node + 16),
                      (float)rdv<int32_t>(b, node + 20));
        };
        switch (w.level) {
            case 0: {
                is_active = true;
                int bx = rdv<int32_t>(b, w.leaf), by = rdv<int32_t>(b, w.leaf + 4), bz = rdv<int32_t>(b, w.leaf + 8);
                bmin = v3((float)bx, (float)by, (float)bz);
                bmax = v3((float)(bx + 8), (float)(by + 8), (float)(bz + 8));
                break;
            }
            case 1: is_active = bit(w.lower + 32, w.ln); box(w.lower); break;
            case 2: is_active = bit(w.upper + 32, w.un); box(w.upper); break;
            case 3: is_active = rdv<uint32_t>(b, w.tile + 16) != 0u; box(root); break;
            default: break;
        }
        return w.level;
    }
    // pnanovdb_map_apply_inverse / _inverse_jacobi / _apply (PNanoVDB.glsl:1996-2040)
    V3 world_to_index(V3 p) const {
        float sx = p.x - vec[0], sy = p.y - vec[1], sz = p.z - vec[2];
        return v3((sx * inv[0] + sy * inv[1]) + sz * inv[2], (sx * inv[3] + sy * inv[4]) + sz * inv[5],
                  (sx * inv[6] + sy * inv[7]) + sz * inv[8]);
    }
    V3 world_to_index_dir(V3 d) const {
        return v3((d.x * inv[0] + d.y * inv[1]) + d.z * inv[2], (d.x * inv[3] + d.y * inv[4]) + d.z * inv[5],
                  (d.x * inv[6] + d.y * inv[7]) + d.z * inv[8]);
    }
    V3 index_to_world(V3 p) const {
        return v3(((p.x * mat[0] + p.y * mat[1]) + p.z * mat[2]) + vec[0],
                  ((p.x * mat[3] + p.y * mat[4]) + p.z * mat[5]) + vec[1],
                  ((p.x * mat[6] + p.y * mat[7]) + p.z * mat[8]) + vec[2]);
    }
};

// ---- hierarchical DDA (pnanovdb_hdda_*, PNanoVDB.glsl:2233-2452) ----
inline float pmin(float a, float b) { return a < b ? a : b; }
inline float pmax(float a, float b) { return a > b ? a : b; }

struct HddaState {
    int dim;
    float tmin, tmax;
    int voxel[3], step[3];
    float delta[3], next[3];
};

bool hdda_clip(V3 bmin, V3 bmax, V3 o, float& tmin, V3 d, float& tmax) {
    float ix = 1.0f / d.x, iy = 1.0f / d.y, iz = 1.0f / d.z;
    float t0x = (bmin.x - o.x) * ix, t0y = (bmin.y - o.y) * iy, t0z = (bmin.z - o.z) * iz;
    float t1x = (bmax.x - o.x) * ix, t1y = (bmax.y - o.y) * iy, t1z = (bmax.z - o.z) * iz;
    float tnear = pmax(pmin(t0x, t1x), pmax(pmin(t0y, t1y), pmin(t0z, t1z)));
    float tfar = pmin(pmax(t0x, t1x), pmin(pmax(t0y, t1y), pmax(t0z, t1z)));
    bool hit = tnear <= tfar;
    tmin = pmax(tmin, tnear);
    tmax = pmin(tmax, tfar);
    return hit;
}

void hdda_start(HddaState& h, V3 o, float tmin, V3 d, float tmax, int dim) {
    h.dim = dim;
    h.tmin = tmin;
    h.tmax = tmax;
    float pos[3] = {d.x * tmin + o.x, d.y * tmin + o.y, d.z * tmin + o.z};
    float dd[3] = {d.x, d.y, d.z};
    for (int a = 0; a < 3; a++) h.voxel[a] = (int)floorf(pos[a]) & ~(dim - 1);
    for (int a = 0; a < 3; a++) {
        float inv = 1.0f / dd[a];
        if (dd[a] == 0.0f) {
            h.next[a] = 1e38f;
            h.step[a] = 0;
            h.delta[a] = 0.0f;
        } else if (inv > 0.0f) {
            h.step[a] = 1;
            h.next[a] = h.tmin + ((float)(h.voxel[a] + dim) - pos[a]) * inv;
            h.delta[a] = inv;
        } else {
            h.step[a] = -1;
            h.next[a] = h.tmin + ((float)h.voxel[a] - pos[a]) * inv;
            h.delta[a] = -inv;
        }
    }
}

void hdda_set_dim(HddaState& h, V3 o, V3 d, int dim) {
    if (h.dim == dim) return;
    h.dim = dim;
    float pos[3] = {d.x * h.tmin + o.x, d.y * h.tmin + o.y, d.z * h.tmin + o.z};
    float inv[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    for (int a = 0; a < 3; a++) h.voxel[a] = (int)floorf(pos[a]) & ~(dim - 1);
    for (int a = 0; a < 3; a++) {
        if (h.step[a] != 0) {
            h.next[a] = h.tmin + ((float)h.voxel[a] - pos[a]) * inv[a];
            if (h.step[a] > 0) h.next[a] += (float)dim * inv[a];
        }
    }
}

bool hdda_advance(HddaState& h) {
    int a = (h.next[0] < h.next[1] && h.next[0] < h.next[2]) ? 0 : (h.next[1] < h.next[2] ? 1 : 2);
    if (h.next[a] <= h.tmin) h.next[a] += (h.tmin - 0.999999f * h.next[a]) + 1.0e-6f;
    h.tmin = h.next[a];
    h.next[a] += (float)h.dim * h.delta[a];
    h.voxel[a] += h.dim * h.step[a];
    return h.tmin <= h.tmax;
}

// ---- density lookup (VptUtils.glsl:583-591, 674-683; CLAMP_TO_BORDER) ----
struct Tracer {
    const OracleScene& S;
    std::vector<size_t> env_off;
    uint64_t lookups = 0;
    uint32_t steps = 0;

    Nano nano;

    explicit Tracer(const OracleScene& s) : S(s) {
        if (S.nanovdb) nano.init(S.nanovdb, S.sparse_fp16 != 0);
        if (S.env_kind == 4) {
            size_t o = 0;
            for (int l = 0; l < S.env_levels; l++) {
                env_off.push_back(o);
                size_t r = (size_t)1 << (S.env_levels - l);
                o += r * r;
            }
        }
    }
    V3 bmin() const { return v3(S.box_min[0], S.box_min[1], S.box_min[2]); }
    V3 bmax() const { return v3(S.box_max[0], S.box_max[1], S.box_max[2]); }

    float texel(int x, int y, int z) const {
        if (x < 0 || y < 0 || z < 0 || x >= S.nx || y >= S.ny || z >= S.nz) return S.border_density;
        return S.density[((size_t)z * S.ny + y) * S.nx + x];
    }
    float at_vox(float ux, float uy, float uz) const {
        if (S.interp != 2) return texel((int)floorf(ux), (int)floorf(uy), (int)floorf(uz));
        ux = ux - 0.5f;
        uy = uy - 0.5f;
        uz = uz - 0.5f;
        float fx = floorf(ux), fy = floorf(uy), fz = floorf(uz);
        float ax = ux - fx, ay = uy - fy, az = uz - fz;
        int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
        float f0 = mixf(mixf(texel(x0, y0, z0), texel(x0 + 1, y0, z0), ax),
                        mixf(texel(x0, y0 + 1, z0), texel(x0 + 1, y0 + 1, z0), ax), ay);
        float f1 = mixf(mixf(texel(x0, y0, z0 + 1), texel(x0 + 1, y0, z0 + 1), ax),
                        mixf(texel(x0, y0 + 1, z0 + 1), texel(x0 + 1, y0 + 1, z0 + 1), ax), ay);
        return mixf(f0, f1, az);
    }
    // sampleCloud (VptUtils.glsl:674-683) + sampleCloudRaw for NanoVDB (VptUtils.glsl:517-581)
    float sample_sparse(V3 pos, Rng& r) {
        V3 c;
        c.x = ((pos.x - S.box_min[0]) / (S.box_max[0] - S.box_min[0])) * (S.grid_max[0] - S.grid_min[0]) + S.grid_min[0];
        c.y = ((pos.y - S.box_min[1]) / (S.box_max[1] - S.box_min[1])) * (S.grid_max[1] - S.grid_min[1]) + S.grid_min[1];
        c.z = ((pos.z - S.box_min[2]) / (S.box_max[2] - S.box_min[2])) * (S.grid_max[2] - S.grid_min[2]) + S.grid_min[2];
        V3 p = nano.world_to_index(c);
        if (S.interp == 0) return nano.value((int)floorf(p.x), (int)floorf(p.y), (int)floorf(p.z));
        if (S.interp == 1) {
            float jx = rnd(r) - 0.5f, jy = rnd(r) - 0.5f, jz = rnd(r) - 0.5f;
            return nano.value((int)floorf(p.x + jx), (int)floorf(p.y + jy), (int)floorf(p.z + jz));
        }
        p = v3(p.x - 0.5f, p.y - 0.5f, p.z - 0.5f);
        int ix = (int)floorf(p.x), iy = (int)floorf(p.y), iz = (int)floorf(p.z);
        float fx = p.x - (float)ix, fy = p.y - (float)iy, fz = p.z - (float)iz;
        float f00 = mixf(nano.value(ix, iy, iz), nano.value(ix + 1, iy, iz), fx);
        float f10 = mixf(nano.value(ix, iy + 1, iz), nano.value(ix + 1, iy + 1, iz), fx);
        float f0 = mixf(f00, f10, fy);
        float f01 = mixf(nano.value(ix, iy, iz + 1), nano.value(ix + 1, iy, iz + 1), fx);
        float f11 = mixf(nano.value(ix, iy + 1, iz + 1), nano.value(ix + 1, iy + 1, iz + 1), fx);
        float f1 = mixf(f01, f11, fy);
        return mixf(f0, f1, fz);
    }
    // sampleCloud with USE_TRANSFER_FUNCTION (VptUtils.glsl:647-672): the table (a one-row texture,
    // linear filtering, clamp to edge) at the normalised density; its rgb kept for the absorption
    V3 tf_rgb = v3(0, 0, 0);
    float tf_apply(float v) {
        if (!S.tf) return v;
        const float u = v * (float)S.tf_size - 0.5f;
        const float fu = floorf(u);
        const float a = u - fu;
        int x0 = (int)fu, x1 = x0 + 1;
        x0 = x0 < 0 ? 0 : (x0 >= S.tf_size ? S.tf_size - 1 : x0);
        x1 = x1 < 0 ? 0 : (x1 >= S.tf_size ? S.tf_size - 1 : x1);
        const float* c0 = S.tf + 4 * x0;
        const float* c1 = S.tf + 4 * x1;
        tf_rgb = v3(mixf(c0[0], c1[0], a), mixf(c0[1], c1[1], a), mixf(c0[2], c1[2], a));
        return mixf(c0[3], c1[3], a);
    }
    V3 tf_emission() const { return mul(tf_rgb, S.emission_strength); }
    float sample(V3 pos, Rng& r) { return tf_apply(sample_raw(pos, r)); }
    float sample_raw(V3 pos, Rng& r) {
        lookups++;
        if (S.nanovdb) return sample_sparse(pos, r);
        float ux = (pos.x - S.box_min[0]) * S.vox_per_unit[0];
        float uy = (pos.y - S.box_min[1]) * S.vox_per_unit[1];
        float uz = (pos.z - S.box_min[2]) * S.vox_per_unit[2];
        if (S.interp == 1) {
            float jx = rnd(r) - 0.5f, jy = rnd(r) - 0.5f, jz = rnd(r) - 0.5f;
            ux = ux + jx;
            uy = uy + jy;
            uz = uz + jz;
        }
        return at_vox(ux, uy, uz);
    }
    float free_path(Rng& r) const { return -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) * (1.0f / S.extinction); }
    // sampleEmission (VptUtils.glsl:604-626): the emission grid at pos (the density texture's filter
    // and stochastic jitter, zero outside its box), t = clamp(value * cap, 0, 1) -> (t^2, t^4, t^8) * strength
    float emission_texel(int x, int y, int z) const {
        if (x < 0 || y < 0 || z < 0 || x >= S.enx || y >= S.eny || z >= S.enz) return 0.0f;
        return S.emission[((size_t)z * S.eny + y) * S.enx + x];
    }
    V3 emission(V3 pos, Rng& r) const {
        float ux = (pos.x - S.emission_box_min[0]) * S.emission_vox_per_unit[0];
        float uy = (pos.y - S.emission_box_min[1]) * S.emission_vox_per_unit[1];
        float uz = (pos.z - S.emission_box_min[2]) * S.emission_vox_per_unit[2];
        if (S.interp == 1) {
            float jx = rnd(r) - 0.5f, jy = rnd(r) - 0.5f, jz = rnd(r) - 0.5f;
            ux = ux + jx;
            uy = uy + jy;
            uz = uz + jz;
        }
        float v;
        if (S.interp != 2) {
            v = emission_texel((int)floorf(ux), (int)floorf(uy), (int)floorf(uz));
        } else {
            ux = ux - 0.5f;
            uy = uy - 0.5f;
            uz = uz - 0.5f;
            float fx = floorf(ux), fy = floorf(uy), fz = floorf(uz);
            float ax = ux - fx, ay = uy - fy, az = uz - fz;
            int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
            float f0 = mixf(mixf(emission_texel(x0, y0, z0), emission_texel(x0 + 1, y0, z0), ax),
                            mixf(emission_texel(x0, y0 + 1, z0), emission_texel(x0 + 1, y0 + 1, z0), ax), ay);
            float f1 = mixf(mixf(emission_texel(x0, y0, z0 + 1), emission_texel(x0 + 1, y0, z0 + 1), ax),
                            mixf(emission_texel(x0, y0 + 1, z0 + 1), emission_texel(x0 + 1, y0 + 1, z0 + 1), ax), ay);
            v = mixf(f0, f1, az);
        }
        const float t = std::min(std::max(v * S.emission_cap, 0.0f), 1.0f);
        const float rr = t * t, gg = rr * rr, bb = gg * gg;
        return v3(rr * S.emission_strength, gg * S.emission_strength, bb * S.emission_strength);
    }
    bool guard() { return ++steps > (1u << 24); }
    V3 sky(V3 d) const { return sky_and_sun(S, d); }

    // deltaTracking (DeltaTracking.glsl:168-344)
    V3 delta(V3 x, V3 w, Rng& r, bool& ev) {
        float tmin, tmax;
        const float absorb = 1.0f - S.albedo;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            int bounces = 0;
            while (true) {
                if (guard()) return v3(0, 0, 0);
                float t = free_path(r);
                if (t > d) break;
                V3 xn = add(x, mul(w, t));
                float dens = sample(xn, r);
                x = xn;
                float xi = rnd(r);
                if (xi < absorb * dens) {
                    ev = true;
                    // USE_TRANSFER_FUNCTION (DeltaTracking.glsl:293-301)
                    return S.tf ? tf_emission() : v3(0, 0, 0);
                }
                if (xi < dens) {
                    if (S.max_bounces > 0 && ++bounces > S.max_bounces) return v3(0, 0, 0);
                    w = sample_phase(r, S.g, w);
                    ev = true;
                    if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
                        x = add(x, mul(w, tmin));
                        d = tmax - tmin;
                    }
                } else {
                    d -= t;
                }
            }
        }
        return sky(w);
    }

    // ---- isosurfaces (USE_ISOSURFACES, ISOSURFACE_TYPE_DENSITY, SURFACE_BRDF_LAMBERTIAN) ----
    // the isosurface field at a texture coordinate: the density texture's linear filter there
    // (sampleIsoImage, VptUtils.glsl:599; the texel values are normalised already)
    float iso_tex(V3 c) const {
        if (S.iso_grad) {  // gradientImage normalised with the density's range (sampleIsoImage)
            return (grad_vox(c.x * (float)S.nx, c.y * (float)S.ny, c.z * (float)S.nz) - S.iso_norm_min) /
                   S.iso_norm_range;
        }
        return at_vox(c.x * (float)S.nx, c.y * (float)S.ny, c.z * (float)S.nz);
    }
    // gradientImage (ISOSURFACE_TYPE_GRADIENT): raw magnitudes, linear filter, border 0
    float grad_texel(int x, int y, int z) const {
        if (x < 0 || y < 0 || z < 0 || x >= S.nx || y >= S.ny || z >= S.nz) return 0.0f;
        return S.iso_grad[((size_t)z * S.ny + y) * S.nx + x];
    }
    float grad_vox(float ux, float uy, float uz) const {
        ux = ux - 0.5f;
        uy = uy - 0.5f;
        uz = uz - 0.5f;
        const float fx = floorf(ux), fy = floorf(uy), fz = floorf(uz);
        const float ax = ux - fx, ay = uy - fy, az = uz - fz;
        const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
        const float f0 = mixf(mixf(grad_texel(x0, y0, z0), grad_texel(x0 + 1, y0, z0), ax),
                              mixf(grad_texel(x0, y0 + 1, z0), grad_texel(x0 + 1, y0 + 1, z0), ax), ay);
        const float f1 = mixf(mixf(grad_texel(x0, y0, z0 + 1), grad_texel(x0 + 1, y0, z0 + 1), ax),
                              mixf(grad_texel(x0, y0 + 1, z0 + 1), grad_texel(x0 + 1, y0 + 1, z0 + 1), ax), ay);
        return mixf(f0, f1, az);
    }
    // sampleCloudIso: the density, or the filtered gradient magnitude (sampleCloudGradient,
    // VptUtils.glsl:687-699) for gradient isosurfaces
    float iso_value_at(V3 pos, Rng& r) {
        if (S.iso_grad) {  // the shader's texture coordinate (pos - boxMin) / (boxMax - boxMin)
            const V3 c = divv(sub(pos, bmin()), sub(bmax(), bmin()));
            return grad_vox(c.x * (float)S.nx, c.y * (float)S.ny, c.z * (float)S.nz);
        }
        return sample(pos, r);
    }
    // getNearestMultiple (VptUtils.glsl:896-906) with GLSL mod(n, x) = n - x * floor(n / x)
    static float nearest_multiple(float n, float x, bool smaller) {
        const float rest = n - x * floorf(n / x);
        if (smaller) return n - rest;
        if (rest == 0.0f) return n;
        return x + n - rest;
    }
    // trilinearInterpolationDensity (VptUtils.glsl:908-959): the eight lattice points k / (size - 1)
    // around c looked up through the texture filter, blended with the fractions of c * (size - 1)
    float iso_trilinear(V3 c) const {
        const float dx = 1.0f / ((float)S.nx - 1.0f), dy = 1.0f / ((float)S.ny - 1.0f),
                    dz = 1.0f / ((float)S.nz - 1.0f);
        const float x0 = nearest_multiple(c.x, dx, true), x1 = nearest_multiple(c.x, dx, false);
        const float y0 = nearest_multiple(c.y, dy, true), y1 = nearest_multiple(c.y, dy, false);
        const float z0 = nearest_multiple(c.z, dz, true), z1 = nearest_multiple(c.z, dz, false);
        const float d000 = iso_tex(v3(x0, y0, z0)), d100 = iso_tex(v3(x1, y0, z0));
        const float d110 = iso_tex(v3(x1, y1, z0)), d010 = iso_tex(v3(x0, y1, z0));
        const float d001 = iso_tex(v3(x0, y0, z1)), d101 = iso_tex(v3(x1, y0, z1));
        const float d111 = iso_tex(v3(x1, y1, z1)), d011 = iso_tex(v3(x0, y1, z1));
        const float px = c.x * ((float)S.nx - 1.0f), py = c.y * ((float)S.ny - 1.0f), pz = c.z * ((float)S.nz - 1.0f);
        const float fx = px - floorf(px), fy = py - floorf(py), fz = pz - floorf(pz);
        const float t00 = mixf(d000, d100, fx), t10 = mixf(d010, d110, fx);
        const float t01 = mixf(d001, d101, fx), t11 = mixf(d011, d111, fx);
        return mixf(mixf(t00, t10, fy), mixf(t01, t11, fy), fz);
    }
    // computeGradient with DIFFERENCES_NEIGHBOR (VptUtils.glsl:965-984): central differences four
    // voxel spacings (1 / (size - 1)) apart, (0, 0, 1) when shorter than 1e-3
    V3 iso_normal(V3 pos) const {
        const V3 c = divv(sub(pos, bmin()), sub(bmax(), bmin()));
        const float hx = 4.0f * (1.0f / (float)(S.nx - 1)), hy = 4.0f * (1.0f / (float)(S.ny - 1)),
                    hz = 4.0f * (1.0f / (float)(S.nz - 1));
        const V3 g = v3(0.5f * (iso_trilinear(v3(c.x + hx, c.y, c.z)) - iso_trilinear(v3(c.x - hx, c.y, c.z))),
                        0.5f * (iso_trilinear(v3(c.x, c.y + hy, c.z)) - iso_trilinear(v3(c.x, c.y - hy, c.z))),
                        0.5f * (iso_trilinear(v3(c.x, c.y, c.z + hz)) - iso_trilinear(v3(c.x, c.y, c.z - hz))));
        const float l = length(g);
        if (l < 1e-3f) return v3(0.0f, 0.0f, 1.0f);
        return v3(g.x / l, g.y / l, g.z / l);
    }
    // refineIsoSurfaceHit (VptUtils.glsl:1045-1058): 8 bisection steps
    void iso_refine(V3& cur, V3 last, float step_sign, Rng& r) {
        for (int i = 0; i < 8; i++) {
            const V3 mid = v3((cur.x + last.x) * 0.5f, (cur.y + last.y) * 0.5f, (cur.z + last.z) * 0.5f);
            const float v = iso_value_at(mid, r);
            if ((v - S.iso_value) * step_sign >= 0.0f) cur = mid;
            else last = mid;
        }
    }
    // getIsoSurfaceHit (VptUtils.glsl:1151-1334) for an opaque Lambertian surface: one random number
    // for the opacity test, normal facing the ray, a direction in the ComputeDefaultBasis frame
    // (RayTracingUtilities.glsl:20-28), throughput *= color * cos / pdf factor.  Lambertian.glsl is
    // included (VptUtils.glsl:1121) before UNIFORM_SAMPLING is defined (:1144), so it samples the
    // cosine-weighted hemisphere through the concentric disk map (VptUtils.glsl:1078-1098) and its
    // pdf factor is the cosine itself
    // CookTorrance.glsl computeBrdf = sampleBrdf + evaluateBrdf (no division by the lobe probability):
    // sel picks sample_GGX (theta = acos(sqrt((1 - u) / (u (a^2 - 1) + 1))), reflected about the half
    // vector) over sample_Lambertian (theta = asin(sqrt(u))); the value is the diffuse colour
    // (1 - F)(1 - metallic) plus F G v.h / (n.h v.n) (GGX sample) or F G D v.h sin(theta_h) / v.n
    V3 frame(V3 t, V3 b, V3 n, float x, float y, float z) const {
        return v3((t.x * x + b.x * y) + n.x * z, (t.y * x + b.y * y) + n.y * z, (t.z * x + b.z * y) + n.z * z);
    }
    struct Frame {
        V3 n, t, b, view;
    };
    struct BrdfS {  // one computeBrdf sample: direction, value, lobe flags, samplingPDF
        V3 dir, value;
        bool spec, cc;
        float pdf;
    };
    BrdfS cook_torrance(const Frame& fr, float sel, float u, Rng& r) {
        const V3 n = fr.n, t = fr.t, b = fr.b, view = fr.view;
        const float pi = 3.14159265358979323846f;
        const float v = rnd(r);
        const float metallic = S.brdf[1], specular = S.brdf[2];
        const float rough = std::min(std::max(S.brdf[4], 0.05f), 1.0f);
        const float specular_w = metallic + (1.0f - rough) * (1.0f + specular);
        const float diffuse_w = 1.0f - metallic;
        const float specular_p = specular_w * (1.0f / (specular_w + diffuse_w));
        const float alpha = rough * rough, alpha2 = alpha * alpha;
        const bool specular_hit = sel < specular_p;
        const float phi = (2.0f * pi) * v;
        V3 l;
        if (specular_hit) {
            const float theta = m_acos(sqrtf((1.0f - u) / (u * (alpha2 - 1.0f) + 1.0f)));
            const float st = m_sin(theta);
            const V3 h = frame(t, b, n, st * m_cos(phi), st * m_sin(phi), m_cos(theta));
            const float vh = fabsf(dot(view, h));
            const float s = 2.0f * (vh > 0.001f ? vh : 0.001f);
            l = v3(s * h.x - view.x, s * h.y - view.y, s * h.z - view.z);
        } else {
            const float theta = m_asin(sqrtf(u));
            const float st = m_sin(theta);
            l = frame(t, b, n, st * m_cos(phi), st * m_sin(phi), m_cos(theta));
        }
        const V3 h = normalize(add(l, view));
        const float ndoth = dot(h, n), vdotn = dot(view, n), ldotn = dot(l, n), vdoth = dot(view, h);
        const float f0s = 0.16f * (specular * specular);
        const float p5 = m_pow5(1.0f - vdoth);
        const float k = alpha / 2.0f;
        const float gl = ldotn < 0.001f ? 0.001f : ldotn, gv = vdotn < 0.001f ? 0.001f : vdotn;
        const float g = (gl / (gl * (1.0f - k) + k)) * (gv / (gv * (1.0f - k) + k));
        const float bq = (ndoth * ndoth) * (alpha2 - 1.0f) + 1.0f;
        const float d = ((1.0f / pi) * alpha2) / (bq * bq);
        const float sth = sqrtf(1.0f - std::min(ndoth * ndoth, 0.95f));
        float o[3];
        for (int i = 0; i < 3; ++i) {
            const float c = S.iso_color[i];
            const float f0 = f0s * (1.0f - metallic) + c * metallic;
            const float f = f0 + (1.0f - f0) * p5;
            const float spec = specular_hit ? ((f * g) * vdoth) / (ndoth * vdotn)
                                            : ((((f * g) * d) * vdoth) * sth) / vdotn;
            o[i] = (c * (1.0f - f)) * (1.0f - metallic) + spec;
        }
        return BrdfS{l, v3(o[0], o[1], o[2]), specular_hit, false, specular_hit ? d : 1.0f / pi};
    }
    // CookTorrance.glsl evaluateBrdfPdf at l: the diffuse-sample specular term plus the diffuse colour / pi
    V3 cook_torrance_pdf_value(const Frame& fr, V3 l) const {
        const float pi = 3.14159265358979323846f;
        const float metallic = S.brdf[1], specular = S.brdf[2];
        const float rough = std::min(std::max(S.brdf[4], 0.05f), 1.0f);
        const float alpha = rough * rough, alpha2 = alpha * alpha;
        const V3 view = fr.view, n = fr.n;
        const V3 h = normalize(add(l, view));
        const float ndoth = dot(h, n), vdotn = dot(view, n), ldotn = dot(l, n), vdoth = dot(view, h);
        const float f0s = 0.16f * (specular * specular);
        const float p5 = m_pow5(1.0f - vdoth);
        const float k = alpha / 2.0f;
        const float gl = ldotn < 0.001f ? 0.001f : ldotn, gv = vdotn < 0.001f ? 0.001f : vdotn;
        const float g = (gl / (gl * (1.0f - k) + k)) * (gv / (gv * (1.0f - k) + k));
        const float bq = (ndoth * ndoth) * (alpha2 - 1.0f) + 1.0f;
        const float d = ((1.0f / pi) * alpha2) / (bq * bq);
        const float sth = sqrtf(1.0f - std::min(ndoth * ndoth, 0.95f));
        float o[3];
        for (int i = 0; i < 3; ++i) {
            const float c = S.iso_color[i];
            const float f0 = f0s * (1.0f - metallic) + c * metallic;
            const float f = f0 + (1.0f - f0) * p5;
            o[i] = ((c * (1.0f - f)) * (1.0f - metallic)) * (1.0f / pi) + ((((f * g) * d) * vdoth) * sth) / vdotn;
        }
        return v3(o[0], o[1], o[2]);
    }
    // Disney2012.glsl computeBrdf = sampleBrdf + evaluateBrdf, its terms as the shader writes them:
    // lobes specular (metallic + (1 + specular)(1 - roughness)), diffuse ((1 - metallic)(1 + roughness)
    // + subsurface) and clearcoat (clamp(clearcoat, 0, 1)); the value is diffuse + specular + clearcoat
    BrdfS disney(const Frame& fr, float sel, float u, Rng& r) {
        const V3 n = fr.n, t = fr.t, b = fr.b, view = fr.view;
        const float pi = 3.14159265358979323846f, pi_c = 3.14159265359f;
        const float* q = S.brdf;
        const float roughness = q[4], metallic = q[1];
        const float aspect = sqrtf(1.0f - q[5] * 0.9f);
        const float r2 = roughness * roughness;
        const float ax0 = r2 / aspect, ay0 = r2 * aspect;
        const float ax = 0.001f < ax0 ? ax0 : 0.001f, ay = 0.001f < ay0 ? ay0 : 0.001f;
        const float specular_w = metallic + (1.0f + q[2]) * (1.0f - roughness);
        const float diffuse_w = (1.0f - metallic) * (1.0f + roughness) + q[0];
        const float clearcoat_w = std::min(std::max(q[8], 0.0f), 1.0f);
        const float norm = 1.0f / ((specular_w + diffuse_w) + clearcoat_w);
        const float specular_p = specular_w * norm, diffuse_p = diffuse_w * norm;
        const float v0 = rnd(r);
        const int lobe = sel < specular_p ? 0 : (sel < specular_p + diffuse_p ? 1 : 2);
        const bool specular_hit = lobe != 1, clearcoat_hit = lobe == 2;
        float th;
        V3 h, l;
        if (lobe == 0) {  // sample_specular_disney
            const float us = std::min(std::max(u, 0.05f), 0.95f), vs = std::min(std::max(v0, 0.05f), 0.95f);
            const float a = (2.0f * pi) * us;
            const float y = ay * m_tan(a);
            const float phi = fabsf(ax) > fabsf(y) ? m_atan2(y, ax) : pi_c / 2.0f - m_atan2(ax, y);
            const float cp = m_cos(phi), sp = m_sin(phi);
            th = m_acos(sqrtf((1.0f - vs) / (1.0f + ((cp * cp) / (ax * ax) + (sp * sp) / (ay * ay)) * vs)));
            const float sq = sqrtf(vs / (1.0f - vs));
            const float ca = ax * m_cos(a), sa = ay * m_sin(a);
            const V3 m = v3(ca * t.x + sa * b.x, ca * t.y + sa * b.y, ca * t.z + sa * b.z);
            h = normalize(v3(sq * m.x + n.x, sq * m.y + n.y, sq * m.z + n.z));
        } else {
            const float phi = (2.0f * pi) * v0;
            if (!clearcoat_hit) {
                th = m_asin(sqrtf(u));
            } else {
                const float g = q[9];
                const float alpha = 0.1f * (1.0f - g) + 0.001f * g;
                const float alpha2 = alpha * alpha;
                th = m_acos(sqrtf((1.0f - m_pow(alpha2, 1.0f - u)) / (1.0f - alpha2)));
            }
            const float st = m_sin(th);
            h = frame(t, b, n, st * m_cos(phi), st * m_sin(phi), m_cos(th));
        }
        if (specular_hit) {
            const float vh = fabsf(dot(view, h));
            const float s = 2.0f * (vh > 0.001f ? vh : 0.001f);
            l = v3(s * h.x - view.x, s * h.y - view.y, s * h.z - view.z);
        } else {
            l = h;
        }
        const V3 hh = normalize(add(l, view));
        const float cos_h = dot(hh, n), cos_d = dot(l, hh), cos_v = dot(view, n), cos_l = dot(l, n);
        const float vdoth = dot(view, hh);
        const float* c = S.iso_color;
        const float lum = (0.3f * c[0] + 0.6f * c[1]) + 0.1f * c[2];
        const float cd = m_cos(cos_d);
        const float cd2 = cd * cd;
        const float f_d90 = 0.5f + (2.0f * roughness) * cd2;
        const float pl = m_pow5(1.0f - m_cos(cos_l)), pv = m_pow5(1.0f - m_cos(cos_v));
        const float f_d = (1.0f + (f_d90 - 1.0f) * pl) * (1.0f + (f_d90 - 1.0f) * pv);
        const float fss90 = roughness * cd2;
        const float f_ss = (1.0f + (fss90 - 1.0f) * pl) * (1.0f + (fss90 - 1.0f) * pv);
        const float lv = cos_l + cos_v;
        const float f_dss = 1.25f * (f_ss * (1.0f / (lv < 0.001f ? 0.001f : lv) - 0.5f) + 0.5f);
        const float f_h = m_pow5(1.0f - cos_d);
        const float fd_mix = f_d * (1.0f - q[0]) + f_dss * q[0];
        const float dx = dot(t, hh) / ax, dy = dot(b, hh) / ay;
        const float dd = dx * dx + dy * dy;
        const float d_spec = 1.0f / (((pi * ax) * ay) * (dd * dd) + cos_h * cos_h);
        const float glx = dot(t, l) * ax, gly = dot(b, l) * ay, gvx = dot(t, view) * ax, gvy = dot(b, view) * ay;
        float g_spec = 1.0f / (cos_v + sqrtf((glx * glx + gly * gly) + cos_v * cos_v));
        g_spec = g_spec * (1.0f / (cos_v + sqrtf((gvx * gvx + gvy * gvy) + cos_v * cos_v)));
        const float sin_th = m_sin(th);
        const float f_cc = 0.04f * (1.0f - f_h) + 1.0f * f_h;
        const float a_cc = 0.1f * (1.0f - q[9]) + 0.001f * q[9];
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
        const float cc = q[8];
        const float clear = (specular_hit && clearcoat_hit)
                                ? (((((cc * f_cc) * g_cc) * cos_l) * vdoth) * sin_th) / cos_h
                                : ((((((cc * f_cc) * d_cc) * g_cc) * cos_l) * vdoth) * sin_th);
        const float st = q[3], sh = q[7];
        const float spec_scale = q[2] * 0.08f;
        float o[3];
        for (int i = 0; i < 3; ++i) {
            const float tint = lum > 0.0f ? c[i] / lum : 1.0f;
            const float spec0 = (spec_scale * (1.0f * (1.0f - st) + tint * st)) * (1.0f - metallic) + c[i] * metallic;
            const float sheen = (f_h * q[6]) * (1.0f * (1.0f - sh) + tint * sh);
            float diffuse = (c[i] * fd_mix + sheen) * (1.0f - metallic);
            if (specular_hit) diffuse = diffuse * (1.0f / pi);
            const float f_spec = spec0 * (1.0f - f_h) + 1.0f * f_h;
            const float spec = (specular_hit && !clearcoat_hit)
                                   ? (((((f_spec * g_spec) * 4.0f) * cos_l) * vdoth) * sin_th) / cos_h
                                   : ((((((f_spec * d_spec) * g_spec) * 4.0f) * cos_l) * vdoth) * sin_th);
            o[i] = (diffuse + spec) + clear;
        }
        return BrdfS{l, v3(o[0], o[1], o[2]), specular_hit, clearcoat_hit,
                     specular_hit ? (clearcoat_hit ? d_cc : d_spec) : 1.0f / pi};
    }
    // Disney2012.glsl evaluateBrdfPdf at l: the non-specular-sample terms, diffuse / pi, sin(theta_h) =
    // sqrt(1 - min(n.h^2, 0.95)), 0.01 as the floor of the subsurface denominator
    V3 disney_pdf_value(const Frame& fr, V3 l) const {
        const float pi = 3.14159265358979323846f, pi_c = 3.14159265359f;
        const float* q = S.brdf;
        const float roughness = q[4], metallic = q[1];
        const float aspect = sqrtf(1.0f - q[5] * 0.9f);
        const float r2 = roughness * roughness;
        const float ax0 = r2 / aspect, ay0 = r2 * aspect;
        const float ax = 0.001f < ax0 ? ax0 : 0.001f, ay = 0.001f < ay0 ? ay0 : 0.001f;
        const V3 view = fr.view, n = fr.n, t = fr.t, b = fr.b;
        const V3 hh = normalize(add(l, view));
        const float cos_h = dot(hh, n), cos_d = dot(l, hh), cos_v = dot(view, n), cos_l = dot(l, n);
        const float vdoth = dot(view, hh);
        const float* c = S.iso_color;
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
        const float fd_mix = f_d * (1.0f - q[0]) + f_dss * q[0];
        const float dx = dot(t, hh) / ax, dy = dot(b, hh) / ay;
        const float dd = dx * dx + dy * dy;
        const float d_spec = 1.0f / (((pi * ax) * ay) * (dd * dd) + cos_h * cos_h);
        const float glx = dot(t, l) * ax, gly = dot(b, l) * ay, gvx = dot(t, view) * ax, gvy = dot(b, view) * ay;
        float g_spec = 1.0f / (cos_v + sqrtf((glx * glx + gly * gly) + cos_v * cos_v));
        g_spec = g_spec * (1.0f / (cos_v + sqrtf((gvx * gvx + gvy * gvy) + cos_v * cos_v)));
        const float sth = sqrtf(1.0f - std::min(cos_h * cos_h, 0.95f));
        const float f_cc = 0.04f * (1.0f - f_h) + 1.0f * f_h;
        const float a_cc = 0.1f * (1.0f - q[9]) + 0.001f * q[9];
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
        const float clear = (((((q[8] * f_cc) * d_cc) * g_cc) * cos_l) * vdoth) * sth;
        const float st = q[3], sh = q[7];
        const float spec_scale = q[2] * 0.08f;
        float o[3];
        for (int i = 0; i < 3; ++i) {
            const float tint = lum > 0.0f ? c[i] / lum : 1.0f;
            const float spec0 = (spec_scale * (1.0f * (1.0f - st) + tint * st)) * (1.0f - metallic) + c[i] * metallic;
            const float sheen = (f_h * q[6]) * (1.0f * (1.0f - sh) + tint * sh);
            const float diffuse = ((c[i] * fd_mix + sheen) * (1.0f - metallic)) * (1.0f / pi);
            const float f_spec = spec0 * (1.0f - f_h) + 1.0f * f_h;
            const float spec = ((((((f_spec * d_spec) * g_spec) * 4.0f) * cos_l) * vdoth) * sth);
            o[i] = (diffuse + spec) + clear;
        }
        return v3(o[0], o[1], o[2]);
    }
    // getIsoSurfaceHit (VptUtils.glsl:1151-1334) up to computeBrdf: one random number for the opacity
    // test, the normal turned against the ray, the ComputeDefaultBasis frame (RayTracingUtilities.glsl:
    // 20-28), the selected BRDF's sample.  Lambertian.glsl is included (VptUtils.glsl:1121) before
    // UNIFORM_SAMPLING is defined (:1144), so it samples the cosine-weighted hemisphere through the
    // concentric disk map (VptUtils.glsl:1078-1098) and its pdf factor is the cosine itself
    BrdfS iso_sample(V3 p, V3 w, Frame& fr, Rng& r, const V3* cam = nullptr) {
        (void)rnd(r);  // isoSurfaceOpacity (1) < random() never holds
        V3 n = iso_normal(p);
        if (cam) ray_box_normal(bmin(), bmax(), *cam, w, n);  // a closing surface (CLOSE_ISOSURFACES)
        else if (dot(w, n) > 0.0f) n = neg(n);
        const float yz = -n.y * n.z;
        const V3 b = normalize(fabsf(n.z) > 0.99999f ? v3(-n.x * n.y, 1.0f - n.y * n.y, yz)
                                                     : v3(-n.x * n.z, yz, 1.0f - n.z * n.z));
        const V3 t = cross(b, n);
        fr = Frame{n, t, b, normalize(neg(w))};
        const float xi0 = rnd(r), xi1 = rnd(r);
        if (S.iso_brdf == 3) return cook_torrance(fr, xi0, xi1, r);
        if (S.iso_brdf == 4) return disney(fr, xi0, xi1, r);
        if (S.iso_brdf != 0) {
            // BlinnPhong.glsl / ConstantLighting.glsl: sampleHemisphere (VptUtils.glsl:1071-1077), uniform
            const float pi = 3.14159265358979323846f;
            const float phi = (2.0f * pi) * xi1;
            const float rr = sqrtf(1.0f - xi0 * xi0);
            const float lx = m_cos(phi) * rr, ly = m_sin(phi) * rr;
            const V3 out = v3((t.x * lx + b.x * ly) + n.x * xi0, (t.y * lx + b.y * ly) + n.y * xi0,
                              (t.z * lx + b.z * ly) + n.z * xi0);
            V3 c = v3(S.iso_color[0], S.iso_color[1], S.iso_color[2]);
            if (S.iso_brdf == 1) {  // BlinnPhong.glsl evaluateBrdf
                const V3 h = normalize(add(fr.view, out));
                const float e = 10.0f;
                const float norm = std::min(std::max((e + 2.0f) / ((4.0f * pi) * 0.03125f), (e + 2.0f) / (8.0f * pi)),
                                            (e + 4.0f) / (8.0f * pi));
                const float s = m_pow(std::max(dot(n, h), 0.0f), e) / norm;
                const float k = 2.0f * pi;
                c = v3((k * S.iso_color[0]) * s, (k * S.iso_color[1]) * s, (k * S.iso_color[2]) * s);
            }
            return BrdfS{out, c, false, false, 0.0f};
        }
        const float ox = 2.0f * xi0 - 1.0f, oy = 2.0f * xi1 - 1.0f;
        float dx = 0.0f, dy = 0.0f;
        if (!(ox == 0.0f && oy == 0.0f)) {
            float rad, th;
            if (fabsf(ox) > fabsf(oy)) {
                rad = ox;
                th = 0.785398185f * (oy / ox);  // M_PI / 4 in float
            } else {
                rad = oy;
                th = 1.57079637f - 0.785398185f * (ox / oy);  // M_PI / 2 - M_PI / 4 * ...
            }
            dx = rad * cosf(th);
            dy = rad * sinf(th);
        }
        const float hz = sqrtf(1.0f - dx * dx - dy * dy);
        const V3 out = v3((t.x * dx + b.x * dy) + n.x * hz, (t.y * dx + b.y * dy) + n.y * hz,
                          (t.z * dx + b.z * dy) + n.z * hz);
        const float cosv = dot(out, n);
        return BrdfS{out,
                     v3((S.iso_color[0] * cosv) / cosv, (S.iso_color[1] * cosv) / cosv,
                        (S.iso_color[2] * cosv) / cosv),
                     false, false, 0.0f};
    }
    void iso_scatter(V3 p, V3& w, V3& weights, Rng& r) {
        Frame fr;
        const BrdfS bs = iso_sample(p, w, fr, r);
        weights = v3(weights.x * bs.value.x, weights.y * bs.value.y, weights.z * bs.value.z);
        w = bs.dir;
    }
    // evaluateBrdfNee of each BRDF file (USE_ISOSURFACE_NEE) for the light direction l, with the
    // sampling pdfs MIS reads (Cook-Torrance, Disney)
    V3 brdf_nee(const Frame& fr, const BrdfS& bs, V3 l, float& pdf_out, float& pdf_nee) const {
        const float pi = 3.14159265358979323846f;
        const float* c = S.iso_color;
        pdf_out = 0.0f;
        pdf_nee = 0.0f;
        if (S.iso_brdf == 0) {  // Lambertian.glsl, non-uniform branch: colour / pi * n.l
            const float th = dot(fr.n, l);
            return v3((c[0] / pi) * th, (c[1] / pi) * th, (c[2] / pi) * th);
        }
        if (S.iso_brdf == 2) {  // ConstantLighting.glsl: colour / (2 pi)
            const float k = 2.0f * pi;
            return v3(c[0] / k, c[1] / k, c[2] / k);
        }
        if (S.iso_brdf == 1) {  // BlinnPhong.glsl: colour (n.h)^10 / norm
            const float e = 10.0f;
            const float norm = std::min(std::max((e + 2.0f) / ((4.0f * pi) * 0.03125f), (e + 2.0f) / (8.0f * pi)),
                                        (e + 4.0f) / (8.0f * pi));
            const V3 h = normalize(add(fr.view, l));
            const float v = m_pow(std::max(dot(fr.n, h), 0.0f), e) / norm;
            return v3(c[0] * v, c[1] * v, c[2] * v);
        }
        const V3 h = normalize(add(bs.dir, fr.view));
        const float cos_h = dot(h, fr.n);
        const float sin_h = sqrtf(1.0f / (cos_h * cos_h));
        const V3 hn = normalize(add(l, fr.view));
        const float cos_hn = dot(hn, fr.n);
        const float sin_hn = sqrtf(1.0f - std::min(cos_hn * cos_hn, 0.95f));
        if (S.iso_brdf == 4 && bs.spec) {
            pdf_out = bs.pdf * cos_h;
            pdf_nee = bs.pdf * cos_hn;
        } else {
            pdf_out = (bs.pdf * cos_h) * sin_h;
            pdf_nee = (bs.pdf * cos_hn) * sin_hn;
        }
        const V3 v = S.iso_brdf == 4 ? disney_pdf_value(fr, l) : cook_torrance_pdf_value(fr, l);
        const float nl = dot(l, fr.n);
        return v3(v.x * nl, v.y * nl, v.z * nl);
    }
    // calculateTransmittance with USE_TRANSMITTANCE_DELTA_TRACKING (defined by the isosurface block of
    // NeeTransmittance.glsl): 0 at the first real collision, else 1; the bisected crossings on the way
    // change nothing without ISOSURFACE_USE_TF and are not looked for
    float transmittance_delta(V3 x, V3 w, Rng& r) {
        float tmin, tmax;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            while (true) {
                if (guard()) return 0.0f;
                float t = free_path(r);
                if (t > d) break;
                V3 xn = add(x, mul(w, t));
                float dens = sample(xn, r);
                x = xn;
                if (rnd(r) > 1.0f - dens) return 0.0f;
                d -= t;
            }
        }
        return 1.0f;
    }
    // getIsoSurfaceHit's next-event estimate (USE_ISOSURFACE_NEE, VptUtils.glsl:1213-1325, no lights)
    void surface_nee(V3 x, const Frame& fr, const BrdfS& bs, V3 thr, V3& color, Rng& r) {
        float pdf_l;
        const V3 l = importance_sky(r, pdf_l);
        if (!(dot(fr.n, l) > 0.0f)) return;
        float pdf_out, pdf_nee;
        const V3 rdf = brdf_nee(fr, bs, l, pdf_out, pdf_nee);
        const bool mis = (S.iso_brdf == 3 || S.iso_brdf == 4) && bs.spec;
        if (mis) {
            const float pdf_l_out = 1.0f / (4.0f * 3.14159265359f);
            const float w_nee = pdf_l / (pdf_l + pdf_nee);
            const float w_out = pdf_out / (pdf_l_out + pdf_out);
            const float tr = transmittance_delta(add(x, mul(l, 1e-4f)), l, r);
            const V3 sk = sky(l);
            color = add(color, v3(((((thr.x * rdf.x) * w_nee) / pdf_l) * tr) * sk.x,
                                  ((((thr.y * rdf.y) * w_nee) / pdf_l) * tr) * sk.y,
                                  ((((thr.z * rdf.z) * w_nee) / pdf_l) * tr) * sk.z));
            const float tr2 = transmittance_delta(add(x, mul(bs.dir, 1e-4f)), bs.dir, r);
            const V3 sk2 = sky(bs.dir);
            color = add(color, v3((((thr.x * w_out) * bs.value.x) * tr2) * sk2.x,
                                  (((thr.y * w_out) * bs.value.y) * tr2) * sk2.y,
                                  (((thr.z * w_out) * bs.value.z) * tr2) * sk2.z));
        } else {
            const float tr = transmittance_delta(add(x, mul(l, 1e-4f)), l, r);
            const V3 sk = sky(l);
            color = add(color, v3((((thr.x * rdf.x) / pdf_l) * tr) * sk.x, (((thr.y * rdf.y) / pdf_l) * tr) * sk.y,
                                  (((thr.z * rdf.z) / pdf_l) * tr) * sk.z));
        }
    }
    // deltaTracking with USE_ISOSURFACES (DeltaTracking.glsl:168-344 with CheckIsosurfaceHit.glsl):
    // every free-flight segment [x, x_new] is checked at iso_subdivisions points for a sign change of
    // density - iso_value against the first point after the last surface event; a crossing is
    // bisected, the surface reflects, the path restarts from the box boundary; escapes carry the
    // surface throughput; 1000 loop iterations end the path with zero
    // CheckIsosurfaceHit.glsl for one free-flight segment [x, xn]: iso_subdivisions check points for a
    // sign change of sampleCloudIso - iso_value against the first point after the last surface event;
    // a crossing is bisected, the surface scatters, the path moves 1e-4 off it and restarts from the
    // box boundary.  Returns true on a surface event.
    // CLOSE_ISOSURFACES: `outside` is true until the path's first check point, where outside the volume
    // counts as sign(-iso_value) and a hit takes the face entered from the camera position `cam`
    bool iso_check(V3& x, V3 xn, V3& w, float& d, float& tmax, V3& weights, float& last_sign, bool& first_point,
                   Rng& r, bool& ev, V3* nee_color = nullptr, bool* outside = nullptr, V3 cam = V3{0, 0, 0}) {
        const int nsub = S.iso_subdivisions;
        for (int sub = 0; sub < nsub; sub++) {
            const float a0 = (float)sub / (float)nsub, a1 = (float)(sub + 1) / (float)nsub;
            const V3 x0 = add(mul(x, 1.0f - a0), mul(xn, a0));
            V3 x1 = add(mul(x, 1.0f - a1), mul(xn, a1));
            const float cur_sign = signf(iso_value_at(x1, r) - S.iso_value);
            const bool from_outside = outside && *outside;
            if (from_outside) {
                first_point = false;
                last_sign = signf(-S.iso_value);
            } else if (first_point) {
                first_point = false;
                last_sign = cur_sign;
            }
            if (last_sign != cur_sign) {
                iso_refine(x1, x0, cur_sign, r);
                x = x1;
                Frame fr;
                const BrdfS bs = iso_sample(x, w, fr, r, from_outside ? &cam : nullptr);
                if (nee_color) surface_nee(x, fr, bs, weights, *nee_color, r);  // USE_ISOSURFACE_NEE
                weights = v3(weights.x * bs.value.x, weights.y * bs.value.y, weights.z * bs.value.z);
                w = bs.dir;
                x = add(x, mul(w, 1e-4f));
                first_point = true;
                if (outside) *outside = false;
                ev = true;
                float tmin;
                if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
                    x = add(x, mul(w, tmin));
                    d = tmax - tmin;
                }
                return true;
            }
            if (outside) *outside = false;
        }
        return false;
    }
    V3 delta_iso(V3 x, V3 w, Rng& r, bool& ev) {
        const V3 cam = x;  // cameraPosition (Clouds.glsl:99)
        bool outside = S.use_iso && S.iso_close;
        float tmin, tmax;
        const float absorb = 1.0f - S.albedo;
        V3 weights = v3(1, 1, 1);
        float last_sign = 0.0f;
        bool first_point = true;
        int it = 0;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            int bounces = 0;
            while (true) {
                if (++it == 1000) return v3(0, 0, 0);
                if (guard()) return v3(0, 0, 0);
                float t = free_path(r);
                if (t > d) break;
                V3 xn = add(x, mul(w, t));
                float dens = sample(xn, r);
                if (iso_check(x, xn, w, d, tmax, weights, last_sign, first_point, r, ev, nullptr, S.iso_close ? &outside : nullptr, cam)) {
                    if (weights.x < 1e-3f && weights.y < 1e-3f && weights.z < 1e-3f) return v3(0, 0, 0);
                    continue;
                }
                x = xn;
                float xi = rnd(r);
                if (xi < absorb * dens) {
                    ev = true;
                    return v3(0, 0, 0);
                }
                if (xi < dens) {
                    if (S.max_bounces > 0 && ++bounces > S.max_bounces) return v3(0, 0, 0);
                    w = sample_phase(r, S.g, w);
                    ev = true;
                    if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
                        x = add(x, mul(w, tmin));
                        d = tmax - tmin;
                    }
                } else {
                    d -= t;
                }
            }
        }
        return mulv(weights, sky(w));
    }

    // ratioTracking (RatioTracking.glsl:26-95)
    V3 ratio(V3 x, V3 w, Rng& r, bool& ev) {
        float trans = 1.0f, tmin, tmax;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            int bounces = 0;
            while (true) {
                if (guard()) return v3(0, 0, 0);
                float t = free_path(r);
                if (t > d) break;
                x = add(x, mul(w, t));
                float dens = sample(x, r);
                float xi = rnd(r);
                if (xi < dens) {
                    if (S.max_bounces > 0 && ++bounces > S.max_bounces) return v3(0, 0, 0);
                    float pa = (1.0f - S.albedo) * dens, ps = S.albedo * dens;
                    trans *= 1.0f - pa / (pa + ps);
                    w = sample_phase(r, S.g, w);
                    ev = true;
                    if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
                        x = add(x, mul(w, tmin));
                        d = tmax - tmin;
                    }
                } else {
                    d -= t;
                }
            }
        }
        V3 l = sky(w);
        return v3(l.x * trans, l.y * trans, l.z * trans);
    }

    // calculateTransmittance (NeeTransmittance.glsl:5-119), ratio tracking T *= P_n
    float transmittance(V3 x, V3 w, Rng& r) {
        float trans = 1.0f, tmin, tmax;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            while (true) {
                if (guard()) return 0.0f;
                float t = free_path(r);
                if (t > d) break;
                V3 xn = add(x, mul(w, t));
                float dens = sample(xn, r);
                x = xn;
                trans *= 1.0f - dens;
                d -= t;
            }
        }
        return trans;
    }

    void sv_step(V3 smin, V3 smax, V3 x, V3 w, int& ix, int& iy, int& iz) const {
        V3 c = mul(add(smin, smax), 0.5f);
        V3 mov = sub(add(x, mul(w, 0.00001f)), c);
        float sx = signf(mov.x), sy = signf(mov.y), sz = signf(mov.z);
        mov = v3(mov.x * sx, mov.y * sy, mov.z * sz);
        ix += (mov.x >= mov.y && mov.x >= mov.z ? 1 : 0) * (int)sx;
        iy += (mov.y >= mov.x && mov.y >= mov.z ? 1 : 0) * (int)sy;
        iz += (mov.z >= mov.x && mov.z >= mov.y ? 1 : 0) * (int)sz;
    }
    V3 grid_f() const { return v3((float)S.nx, (float)S.ny, (float)S.nz); }
    V3 svs_f() const { return v3((float)S.sv_size, (float)S.sv_size, (float)S.sv_size); }
    V3 svw() const { return v3(S.sv_world[0], S.sv_world[1], S.sv_world[2]); }

    // calculateTransmittance with USE_OCCUPANCY_GRID (NeeTransmittance.glsl:121-259)
    float transmittance_ess(V3 x, V3 w, Rng& r) {
        float trans = 1.0f;
        V3 eps = v3(1e-6f, 1e-6f, 1e-6f);
        float tminv, tmaxv;
        if (!ray_box(add(bmin(), eps), sub(bmax(), eps), x, w, tminv, tmaxv)) return trans;
        V3 delta = sub(bmax(), bmin());
        x = add(x, mul(w, tminv));
        V3 sp = divv(mulv(divv(sub(x, bmin()), delta), grid_f()), svs_f());
        int ix = (int)floorf(sp.x), iy = (int)floorf(sp.y), iz = (int)floorf(sp.z);
        int cx = ix, cy = iy, cz = iz;
        bool empty = false;
        while (ix >= 0 && iy >= 0 && iz >= 0 && ix < S.svx && iy < S.svy && iz < S.svz) {
            if (guard()) return 0.0f;
            V3 smin = add(bmin(), mulv(v3((float)ix, (float)iy, (float)iz), svw()));
            V3 smax = add(smin, svw());
            float ts0 = 0.0f, ts1 = 0.0f;
            ray_box(smin, smax, x, w, ts0, ts1);
            float dmax = ts1 - ts0;
            x = add(x, mul(w, ts0));
            if (cx != ix || cy != iy || cz != iz) {
                empty = S.occupancy[((size_t)iz * S.svy + iy) * S.svx + ix] == 0;
                cx = ix;
                cy = iy;
                cz = iz;
            }
            if (empty) {
                x = add(x, mul(w, dmax));
            } else {
                // t counts from the supervoxel entry x0 (the reference steps from the moving x,
                // NeeTransmittance.glsl:173-228, which overshoots; ess_ref_compat keeps that)
                const V3 x0 = x;
                float t = 0.0f;
                while (true) {
                    if (guard()) return 0.0f;
                    t -= m_log(std::max(0.0000000001f, 1.0f - rnd(r))) * (1.0f / S.extinction);
                    if (t >= dmax) {
                        x = add(S.ess_ref_compat ? x : x0, mul(w, dmax));
                        break;
                    }
                    V3 xn = add(S.ess_ref_compat ? x : x0, mul(w, t));
                    float dens = sample(xn, r);
                    x = xn;
                    trans *= 1.0f - dens;
                }
            }
            sv_step(smin, smax, x, w, ix, iy, iz);
        }
        return trans;
    }

    V3 importance_sky(Rng& r, float& pdf) {
        if (S.env_kind == 4) return sample_env_image(S, env_off.data(), r, pdf);
        pdf = 1.0f / (4.0f * PI);
        return random_direction(r, v3(1, 0, 0));
    }

    // nextEventTracking (NextEventTracking.glsl:224-393)
    // ---- lights (VptUtils.glsl:394-453) ----
    const float* light(int i) const { return S.lights + 16 * i; }
    V3 inv_view_xyz(V3 v, float wv) const {
        const float* m = S.inv_view;
        return v3(((m[0] * v.x + m[4] * v.y) + m[8] * v.z) + m[12] * wv,
                  ((m[1] * v.x + m[5] * v.y) + m[9] * v.z) + m[13] * wv,
                  ((m[2] * v.x + m[6] * v.y) + m[10] * v.z) + m[14] * wv);
    }
    V3 light_pos(int i) const {
        const float* L = light(i);
        int type = (int)L[0], space = (int)L[1];
        V3 p = v3(L[8], L[9], L[10]);
        if (space == 1 || space == 2) p = inv_view_xyz(p, (type == 2 || space == 2) ? 0.0f : 1.0f);
        return p;
    }
    // getHeadlightDirection
    V3 light_dir(V3 pos, Rng& r, int& idx, float& factor, float& dist) const {
        if (S.num_lights > 1) {
            uint32_t k = (uint32_t)(rnd(r) * (float)S.num_lights);
            idx = (int)std::min(k, (uint32_t)S.num_lights - 1u);
            factor *= (float)S.num_lights;
        }
        int type = (int)light(idx)[0];
        V3 lp = light_pos(idx);
        V3 dir = (type == 0 || type == 1) ? sub(lp, pos) : lp;
        dist = length(dir);
        float s = dist + 1e-5f;
        return v3(dir.x / s, dir.y / s, dir.z / s);
    }
    // sampleHeadlight
    V3 light_rad(V3 pos, int idx) const {
        const float* L = light(idx);
        int type = (int)L[0], space = (int)L[1];
        V3 lp = light_pos(idx);
        float f = L[7];
        if ((type == 0 || type == 1) && L[11] != 0.0f) {
            V3 diff = sub(lp, pos);
            f /= std::max(dot(diff, diff), 1e-3f);
        }
        if (type == 1) {
            float total = m_cos(L[2]);
            float falloff = L[2] > L[3] ? m_cos(L[3]) : total;
            V3 p = sub(pos, lp);
            V3 z = normalize(v3(L[12], L[13], L[14]));
            if (space == 1 || space == 2) z = inv_view_xyz(z, 0.0f);
            float ct = dot(z, p) / (length(z) * length(p));
            f *= smoothstepf(total, falloff, ct);
        }
        return v3(f * L[4], f * L[5], f * L[6]);
    }
    // calculateTransmittanceDistance (NeeTransmittance.glsl:264-381), ratio tracking
    float transmittance_distance(V3 x, V3 w, float max_dist, Rng& r) {
        float trans = 1.0f, tmin, tmax, cur = 0.0f;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            cur += tmin;
            float d = tmax - tmin;
            while (true) {
                if (guard()) return 0.0f;
                float t = free_path(r);
                cur += t;
                if (t > d || cur > max_dist) break;
                V3 xn = add(x, mul(w, t));
                float dens = sample(xn, r);
                x = xn;
                trans *= 1.0f - dens;
                d -= t;
            }
        }
        return trans;
    }

    // nextEventTracking with USE_ISOSURFACES and USE_ISOSURFACE_NEE (NextEventTracking.glsl:224-393; no
    // lights): the 1000-iteration cap, the segment check with next-event estimation at surface hits,
    // delta-tracked shadow rays, volume light samples scaled by the surface throughput, the sky at the
    // end only for a path without any event
    V3 nee_iso(V3 x, V3 w, Rng& r, bool& ev) {
        const V3 cam = x;  // cameraPosition (Clouds.glsl:99)
        bool outside = S.use_iso && S.iso_close;
        V3 color = v3(0, 0, 0), weights = v3(1, 1, 1);
        float last_sign = 0.0f;
        bool first_point = true;
        int it = 0;
        float tmin, tmax;
        const float absorb = 1.0f - S.albedo;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            int bounces = 0;
            while (true) {
                if (++it == 1000) return v3(0, 0, 0);
                if (guard()) return color;
                float t = free_path(r);
                if (t > d) break;
                V3 xn = add(x, mul(w, t));
                float dens = sample(xn, r);
                if (iso_check(x, xn, w, d, tmax, weights, last_sign, first_point, r, ev, &color, S.iso_close ? &outside : nullptr, cam)) {
                    if (weights.x < 1e-3f && weights.y < 1e-3f && weights.z < 1e-3f) return v3(0, 0, 0);
                    continue;
                }
                x = xn;
                float xi = rnd(r);
                if (xi < absorb * dens) {
                    ev = true;
                    if (S.emission) {
                        const V3 e = emission(x, r);
                        return add(color, v3(weights.x * e.x, weights.y * e.y, weights.z * e.z));
                    }
                    return color;
                }
                if (xi < dens) {
                    if (S.max_bounces > 0 && ++bounces > S.max_bounces) return color;
                    V3 nw = sample_phase(r, S.g, w);
                    ev = true;
                    float pdf_l;
                    V3 dl = importance_sky(r, pdf_l);
                    float pdf_p = eval_phase(S.g, w, dl);
                    w = nw;
                    float tr = transmittance_delta(x, dl, r);
                    float f = (pdf_p / pdf_l) * tr;
                    V3 l = sky(dl);
                    color = add(color, v3((f * l.x) * weights.x, (f * l.y) * weights.y, (f * l.z) * weights.z));
                    if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
                        x = add(x, mul(w, tmin));
                        d = tmax - tmin;
                    }
                } else {
                    d -= t;
                }
            }
        }
        if (!ev) color = add(color, sky(w));
        return color;
    }
    V3 nee(V3 x, V3 w, Rng& r, bool& ev) {
        V3 color = v3(0, 0, 0);
        float tmin, tmax;
        const float absorb = 1.0f - S.albedo;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            int bounces = 0;
            while (true) {
                if (guard()) return color;
                float t = free_path(r);
                if (t > d) break;
                V3 xn = add(x, mul(w, t));
                float dens = sample(xn, r);
                x = xn;
                float xi = rnd(r);
                if (xi < absorb * dens) {
                    ev = true;
                    // USE_EMISSION (NextEventTracking.glsl:296-301); else USE_TRANSFER_FUNCTION (:303-310)
                    return S.emission ? add(color, emission(x, r)) : (S.tf ? add(color, tf_emission()) : color);
                }
                if (xi < dens) {
                    if (S.max_bounces > 0 && ++bounces > S.max_bounces) return color;
                    V3 nw = sample_phase(r, S.g, w);
                    ev = true;
                    // NextEventTracking.glsl:335-369: lights or sky, 1/2 each (lights only when the
                    // environment is black)
                    bool to_light = false;
                    float factor = 1.0f, ldist = 0.0f, pdf_l = 0.0f;
                    int lidx = 0;
                    if (S.num_lights > 0) {
                        to_light = S.env_is_black ? true : (rnd(r) > 0.5f);
                        factor = S.env_is_black ? 1.0f : 2.0f;
                    }
                    V3 dl = to_light ? light_dir(x, r, lidx, factor, ldist) : importance_sky(r, pdf_l);
                    float pdf_p = eval_phase(S.g, w, dl);
                    w = nw;
                    if (S.num_lights > 0) {
                        float common = factor * pdf_p;
                        if (to_light) {
                            float tr = transmittance_distance(x, dl, ldist, r);
                            float f = common * tr;
                            V3 l = light_rad(x, lidx);
                            color = add(color, v3(f * l.x, f * l.y, f * l.z));
                        } else {
                            float tr = S.use_ess ? transmittance_ess(x, dl, r) : transmittance(x, dl, r);
                            float f = (common / pdf_l) * tr;
                            V3 l = sky(dl);
                            color = add(color, v3(f * l.x, f * l.y, f * l.z));
                        }
                    } else {
                        float tr = S.use_ess ? transmittance_ess(x, dl, r) : transmittance(x, dl, r);
                        float f = (pdf_p / pdf_l) * tr;
                        V3 l = sky(dl);
                        color = add(color, v3(f * l.x, f * l.y, f * l.z));
                    }
                    if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
                        x = add(x, mul(w, tmin));
                        d = tmax - tmin;
                    }
                } else {
                    d -= t;
                }
            }
        }
        if (!ev) color = add(color, sky(w));
        return color;
    }

    // ---- spectral tracking (Kutz et al. 2017) ----
    V3 ext3() const {
        if (S.ext_rgb[0] == 0.0f && S.ext_rgb[1] == 0.0f && S.ext_rgb[2] == 0.0f)
            return v3(S.extinction, S.extinction, S.extinction);
        return v3(S.ext_rgb[0], S.ext_rgb[1], S.ext_rgb[2]);
    }
    V3 alb3() const {
        if (S.ext_rgb[0] == 0.0f && S.ext_rgb[1] == 0.0f && S.ext_rgb[2] == 0.0f)
            return v3(S.albedo, S.albedo, S.albedo);
        return v3(S.albedo_rgb[0], S.albedo_rgb[1], S.albedo_rgb[2]);
    }
    static float maxc(V3 v) { return std::max(v.x, std::max(v.y, v.z)); }
    static float avgc(V3 v) { return ((v.x + v.y) + v.z) / 3.0f; }
    static V3 cmin(V3 v, float c) { return v3(std::min(v.x, c), std::min(v.y, c), std::min(v.z, c)); }
    static V3 cmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
    // the collision probabilities of one real-or-null collision (DeltaTracking.glsl:90-110)
    void sdt_step(float dens, V3 weights, float maj, V3& sa, V3& ss, V3& sn, float& pa, float& ps, float& pn) const {
        const V3 ext = ext3();
        V3 alb = alb3();
        if (S.tf && S.tf_albedo_strength > 0.0f) {  // mix(scatteringAlbedo, TF rgb, strength), DeltaTracking.glsl:76-81
            const float s = S.tf_albedo_strength;
            alb = v3(alb.x * (1.0f - s) + tf_rgb.x * s, alb.y * (1.0f - s) + tf_rgb.y * s,
                     alb.z * (1.0f - s) + tf_rgb.z * s);
        }
        const V3 aa = v3(1.0f - alb.x, 1.0f - alb.y, 1.0f - alb.z);
        sa = v3((aa.x * ext.x) * dens, (aa.y * ext.y) * dens, (aa.z * ext.z) * dens);
        ss = v3((alb.x * ext.x) * dens, (alb.y * ext.y) * dens, (alb.z * ext.z) * dens);
        sn = v3(maj - ext.x * dens, maj - ext.y * dens, maj - ext.z * dens);
        if (S.sdt_prob == 0) {
            pa = maxc(sa);
            ps = maxc(ss);
            pn = maxc(sn);
        } else if (S.sdt_prob == 1) {
            pa = avgc(sa);
            ps = avgc(ss);
            pn = avgc(sn);
        } else {
            pa = avgc(cmul(sa, weights));
            ps = avgc(cmul(ss, weights));
            pn = avgc(cmul(sn, weights));
        }
        const float c = (pa + ps) + pn;
        pa /= c;
        ps /= c;
        pn /= c;
    }
    static V3 reweight(V3 weights, V3 sigma, float maj, float p) {
        const float den = maj * p;
        return v3(weights.x * (sigma.x / den), weights.y * (sigma.y / den), weights.z * (sigma.z / den));
    }

    // deltaTrackingSpectral (DeltaTracking.glsl:33-163)
    // with isosurfaces (USE_ISOSURFACES, DeltaTracking.glsl:37-63 and the CheckIsosurfaceHit.glsl include):
    // the 1000-iteration cap, the segment check and the surface throughput in the spectral weights
    V3 spectral_delta(V3 x, V3 w, Rng& r, bool& ev) {
        const V3 cam = x;  // cameraPosition (Clouds.glsl:99)
        bool outside = S.use_iso && S.iso_close;
        const float maj = maxc(ext3());
        V3 weights = v3(1, 1, 1);
        float last_sign = 0.0f;
        bool first_point = true;
        int it = 0;
        float tmin, tmax;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            int bounces = 0;
            while (true) {
                if (S.use_iso && ++it == 1000) return v3(0, 0, 0);
                if (guard()) return v3(0, 0, 0);
                float t = -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) * (1.0f / maj);
                if (t > d) break;
                V3 xn = add(x, mul(w, t));
                float dens = sample(xn, r);
                if (S.use_iso && iso_check(x, xn, w, d, tmax, weights, last_sign, first_point, r, ev, nullptr, S.iso_close ? &outside : nullptr, cam)) {
                    if (weights.x < 1e-3f && weights.y < 1e-3f && weights.z < 1e-3f) return v3(0, 0, 0);
                    continue;
                }
                x = xn;
                V3 sa, ss, sn;
                float pa, ps, pn;
                sdt_step(dens, weights, maj, sa, ss, sn, pa, ps, pn);
                float xi = rnd(r);
                if (xi < pa) {
                    ev = true;
                    if (S.tf) {  // USE_TRANSFER_FUNCTION (DeltaTracking.glsl:125-127)
                        const V3 le = tf_emission();
                        const float den = maj * pa;
                        return v3(weights.x * sa.x / den * le.x, weights.y * sa.y / den * le.y,
                                  weights.z * sa.z / den * le.z);
                    }
                    return v3(0, 0, 0);
                }
                if (xi < pa + ps) {
                    if (S.max_bounces > 0 && ++bounces > S.max_bounces) return v3(0, 0, 0);
                    w = sample_phase(r, S.g, w);
                    ev = true;
                    if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
                        x = add(x, mul(w, tmin));
                        d = tmax - tmin;
                    }
                    weights = reweight(weights, ss, maj, ps);
                } else {
                    d -= t;
                    weights = reweight(weights, sn, maj, pn);
                }
                if (S.sdt_prob == 2) weights = cmin(weights, 100.0f);
            }
        }
        return cmul(cmin(weights, 100000.0f), sky(w));
    }

    // nextEventTrackingSpectral (NextEventTracking.glsl:31-220)
    V3 spectral_nee(V3 x, V3 w, Rng& r, bool& ev) {
        const V3 cam = x;  // cameraPosition (Clouds.glsl:99)
        bool outside = S.use_iso && S.iso_close;
        const float maj = maxc(ext3());
        V3 weights = v3(1, 1, 1), color = v3(0, 0, 0);
        float last_sign = 0.0f;
        bool first_point = true;
        int it = 0;
        float tmin, tmax;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            int bounces = 0;
            while (true) {
                if (S.use_iso && ++it == 1000) return v3(0, 0, 0);
                if (guard()) return color;
                float t = -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) * (1.0f / maj);
                if (t > d) break;
                V3 xn = add(x, mul(w, t));
                // with a transfer function the reference looks up the previous point x
                // (NextEventTracking.glsl:74, sampleCloudDensityEmission(x))
                float dens = sample(S.tf ? x : xn, r);
                // isosurfaces (CheckIsosurfaceHit.glsl with USE_ISOSURFACE_NEE)
                if (S.use_iso && iso_check(x, xn, w, d, tmax, weights, last_sign, first_point, r, ev, &color, S.iso_close ? &outside : nullptr, cam)) {
                    if (weights.x < 1e-3f && weights.y < 1e-3f && weights.z < 1e-3f) return v3(0, 0, 0);
                    continue;
                }
                x = xn;
                V3 sa, ss, sn;
                float pa, ps, pn;
                sdt_step(dens, weights, maj, sa, ss, sn, pa, ps, pn);
                float xi = rnd(r);
                if (xi < pa) {
                    ev = true;
                    // USE_EMISSION (NextEventTracking.glsl:125-131); else USE_TRANSFER_FUNCTION (:133-139)
                    if (S.use_iso && S.emission) {  // the surface throughput applies (NextEventTracking.glsl:118-124)
                        const V3 e = emission(x, r);
                        return add(color, v3(weights.x * e.x, weights.y * e.y, weights.z * e.z));
                    }
                    return S.emission ? add(color, emission(x, r)) : (S.tf ? tf_emission() : color);
                }
                if (xi < pa + ps) {
                    if (S.max_bounces > 0 && ++bounces > S.max_bounces) return color;
                    V3 nw = sample_phase(r, S.g, w);
                    ev = true;
                    bool to_light = false;
                    float factor = 1.0f, ldist = 0.0f, pdf_l = 0.0f;
                    int lidx = 0;
                    if (S.num_lights > 0) {
                        to_light = S.env_is_black ? true : (rnd(r) > 0.5f);
                        factor = S.env_is_black ? 1.0f : 2.0f;
                    }
                    V3 dl = to_light ? light_dir(x, r, lidx, factor, ldist) : importance_sky(r, pdf_l);
                    float pdf_p = eval_phase(S.g, w, dl);
                    w = nw;
                    weights = reweight(weights, ss, maj, ps);
                    const V3 wc = cmin(weights, 100000.0f);
                    if (S.num_lights > 0) {
                        const float cf = factor * pdf_p;
                        const V3 common = v3(cf * wc.x, cf * wc.y, cf * wc.z);
                        if (to_light) {
                            float tr = transmittance_distance(x, dl, ldist, r);
                            V3 l = light_rad(x, lidx);
                            color = add(color, v3((common.x * tr) * l.x, (common.y * tr) * l.y, (common.z * tr) * l.z));
                        } else {
                            float tr = S.use_ess ? transmittance_ess(x, dl, r) : transmittance(x, dl, r);
                            V3 l = sky(dl);
                            color = add(color, v3(((common.x / pdf_l) * tr) * l.x, ((common.y / pdf_l) * tr) * l.y,
                                                  ((common.z / pdf_l) * tr) * l.z));
                        }
                    } else {
                        // with isosurfaces every shadow ray is delta tracked (USE_TRANSMITTANCE_DELTA_TRACKING)
                        float tr = S.use_iso ? transmittance_delta(x, dl, r)
                                             : (S.use_ess ? transmittance_ess(x, dl, r) : transmittance(x, dl, r));
                        float f = (pdf_p / pdf_l) * tr;
                        V3 l = sky(dl);
                        color = add(color, v3((f * wc.x) * l.x, (f * wc.y) * l.y, (f * wc.z) * l.z));
                    }
                    if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
                        x = add(x, mul(w, tmin));
                        d = tmax - tmin;
                    }
                } else {
                    d -= t;
                    weights = reweight(weights, sn, maj, pn);
                }
                if (S.sdt_prob == 2) weights = cmin(weights, 100.0f);
            }
        }
        if (!ev) {
            const V3 wc = cmin(weights, 100000.0f);
            const V3 l = sky(w);
            color = add(color, v3((1.0f * wc.x) * l.x, (1.0f * wc.y) * l.y, (1.0f * wc.z) * l.z));
        }
        return color;
    }

    // analogDecompositionTracking over a NanoVDB grid with the HDDA
    // (DecompositionTracking.glsl:130-360)
    V3 decomposition_sparse(V3 x, V3 w, Rng& r) {
        V3 origin = nano.world_to_index(x);
        V3 dir = nano.world_to_index_dir(w);
        float scale = 1.0f / length(dir);
        dir = mul(dir, scale);
        float tmin = 0.0f, tmax = 1e10f;
        V3 rlo = v3((float)nano.rmin[0], (float)nano.rmin[1], (float)nano.rmin[2]);
        V3 rhi = v3((float)(nano.rmax[0] + 1), (float)(nano.rmax[1] + 1), (float)(nano.rmax[2] + 1));
        bool hit = hdda_clip(rlo, rhi, origin, tmin, dir, tmax);
        if (hit && tmax < 1e20f) {
            const float majorant = S.extinction;
            const float absorb = 1.0f - S.albedo;
            const int lowest = S.sparse_lowest_level;
            int bounces = 0;
            HddaState h;
            hdda_start(h, origin, tmin - 1e-4f, dir, tmax + 1e-4f, lowest);
            for (int iteration = 0;; iteration++) {
                if (guard()) return v3(0, 0, 0);
                if (iteration > 0) {
                    if (!hdda_advance(h)) break;
                    int d = std::max(nano.dim(h.voxel[0], h.voxel[1], h.voxel[2]), lowest);
                    hdda_set_dim(h, origin, dir, d);
                }
                bool active = false;
                V3 nmin = v3(0, 0, 0), nmax = v3(0, 0, 0);
                if (lowest == 8) {
                    nano.cell(h.voxel[0], h.voxel[1], h.voxel[2], active, nmin, nmax);
                } else {
                    active = nano.active(h.voxel[0], h.voxel[1], h.voxel[2]);
                    nmin = v3((float)h.voxel[0], (float)h.voxel[1], (float)h.voxel[2]);
                    nmax = v3((float)(h.voxel[0] + 1), (float)(h.voxel[1] + 1), (float)(h.voxel[2] + 1));
                }
                if (!active) continue;
                float tn0 = 0.0f, tn1 = 1e10f;
                bool hits_node = hdda_clip(nmin, nmax, origin, tn0, dir, tn1);
                x = nano.index_to_world(add(origin, mul(dir, tn0)));
                if (!hits_node) continue;
                float d_max = scale * (std::min(std::min(h.next[0], h.next[1]), h.next[2]) - h.tmin);
                const float mu_c = 0.0000000001f;
                const float mu_r = std::max(0.0000000001f, majorant * 1.0f - mu_c);
                bool changed = false;
                float t_c = -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) / mu_c;
                float t_r = 0.0f;
                while (true) {
                    if (guard()) return v3(0, 0, 0);
                    t_r -= m_log(std::max(0.0000000001f, 1.0f - rnd(r))) / mu_r;
                    if (t_c >= d_max && t_r >= d_max) {
                        x = add(x, mul(w, d_max));
                        break;
                    }
                    V3 xs = add(x, mul(w, std::min(t_c, t_r)));
                    bool collision;
                    if (t_c <= t_r) {
                        collision = true;
                    } else {
                        float dens = sample(xs, r);
                        collision = rnd(r) * mu_r < S.extinction * dens - mu_c;
                    }
                    if (collision) {
                        x = xs;
                        if (rnd(r) < absorb) return v3(0, 0, 0);
                        if (S.max_bounces > 0 && ++bounces > S.max_bounces) return v3(0, 0, 0);
                        w = sample_phase(r, S.g, w);
                        t_r = 0.0f;
                        t_c = -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) / mu_c;
                        origin = nano.world_to_index(x);
                        dir = normalize(nano.world_to_index_dir(w));
                        float tl0 = 0.0f, tl1 = 1e10f;
                        ray_box(nmin, nmax, origin, dir, tl0, tl1);
                        hdda_clip(nmin, nmax, origin, tl0, dir, tl1);
                        d_max = scale * (tl1 - tl0);
                        changed = true;
                    }
                }
                if (changed) {
                    tmin = 0.0f;
                    tmax = 1e10f;
                    hdda_clip(rlo, rhi, origin, tmin, dir, tmax);
                    hdda_start(h, origin, tmin + d_max / scale + 1e-4f, dir, tmax + 1e-4f, lowest);
                }
            }
        }
        return sky(w);
    }

    // analogDecompositionTracking, dense (DecompositionTracking.glsl:35-123)
    V3 decomposition(V3 x, V3 w, Rng& r) {
        V3 eps = v3(1e-6f, 1e-6f, 1e-6f);
        float tminv, tmaxv;
        if (ray_box(add(bmin(), eps), sub(bmax(), eps), x, w, tminv, tmaxv)) {
            const float maj = S.extinction, absorb = 1.0f - S.albedo;
            V3 delta = sub(bmax(), bmin());
            x = add(x, mul(w, tminv));
            V3 sp = divv(mulv(divv(sub(x, bmin()), delta), grid_f()), svs_f());
            int ix = (int)floorf(sp.x), iy = (int)floorf(sp.y), iz = (int)floorf(sp.z);
            int cx = -1, cy = -1, cz = -1;
            float mn = 0.0f, mx = 0.0f;
            int bounces = 0;
            while (ix >= 0 && iy >= 0 && iz >= 0 && ix < S.svx && iy < S.svy && iz < S.svz) {
                if (guard()) return v3(0, 0, 0);
                V3 smin = add(bmin(), mulv(v3((float)ix, (float)iy, (float)iz), svw()));
                V3 smax = add(smin, svw());
                float ts0 = 0.0f, ts1 = 0.0f;
                ray_box(smin, smax, x, w, ts0, ts1);
                float dmax = ts1 - ts0;
                x = add(x, mul(w, ts0));
                if (cx != ix || cy != iy || cz != iz) {
                    size_t k = ((size_t)iz * S.svy + iy) * S.svx + ix;
                    mn = S.sv_data[2 * k];
                    mx = S.sv_data[2 * k + 1];
                    cx = ix;
                    cy = iy;
                    cz = iz;
                }
                if (mx < 1e-5f) {
                    x = add(x, mul(w, dmax));
                } else {
                    float mu_c = std::max(0.0000000001f, maj * mn);
                    float mu_r = std::max(0.0000000001f, maj * mx - mu_c);
                    float t_c = -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) / mu_c;
                    float t_r = 0.0f;
                    while (true) {
                        if (guard()) return v3(0, 0, 0);
                        t_r -= m_log(std::max(0.0000000001f, 1.0f - rnd(r))) / mu_r;
                        if (t_c >= dmax && t_r >= dmax) {
                            x = add(x, mul(w, dmax));
                            break;
                        }
                        V3 xs = add(x, mul(w, std::min(t_c, t_r)));
                        bool coll;
                        if (t_c <= t_r) {
                            coll = true;
                        } else {
                            float dens = sample(xs, r);
                            coll = rnd(r) * mu_r < S.extinction * dens - mu_c;
                        }
                        if (coll) {
                            x = xs;
                            if (rnd(r) < absorb) return v3(0, 0, 0);
                            if (S.max_bounces > 0 && ++bounces > S.max_bounces) return v3(0, 0, 0);
                            w = sample_phase(r, S.g, w);
                            t_r = 0.0f;
                            t_c = -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) / mu_c;
                            ray_box(smin, smax, x, w, ts0, ts1);
                            dmax = ts1 - ts0;
                        }
                    }
                }
                sv_step(smin, smax, x, w, ix, iy, iz);
            }
        }
        return sky(w);
    }

    // residualRatioTrackingEstimator (ResidualRatioTracking.glsl:34-76)
    float rrt_est(V3 x, V3 w, float d0, float d1, float T, float& wsum, float& res_t, float& res_d, float mu_c,
                  float mu_r, Rng& r) {
        float tc = m_exp(-mu_c * (d1 - d0));
        float tr = 1.0f;
        float dt = d0;
        while (true) {
            if (guard()) break;
            float t = -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) / mu_r;
            x = add(x, mul(w, t));
            dt += t;
            if (dt >= d1) break;
            float dens = sample(x, r);
            float mu = S.extinction * dens;
            tr *= 1.0f - (mu - mu_c) / mu_r;
            float tcl = m_exp(-mu_c * (dt - d0));
            float tl = (T * tr) * tcl;
            wsum += tl;
            float xi = rnd(r);
            if (xi < tl / wsum) {
                res_t = tl;
                res_d = dt;
            }
        }
        return tc * tr;
    }

    // residualRatioTracking (ResidualRatioTracking.glsl:78-223)
    V3 rrt(V3 x, V3 w, Rng& r) {
        float wsum = 0.0f, res_t = 0.0f, res_d = 0.0f, T = 1.0f;
        V3 acc = v3(0, 0, 0);
        V3 eps = v3(1e-6f, 1e-6f, 1e-6f);
        V3 n = grid_f(), sv = svs_f(), delta = sub(bmax(), bmin());
        V3 old_x = x;
        int iteration = 0;
        while (true) {
            float tminv, tmaxv;
            if (!ray_box(add(bmin(), eps), sub(bmax(), eps), x, w, tminv, tmaxv)) break;
            x = add(x, mul(w, tminv));
            old_x = x;
            float dtot = tmaxv - tminv;
            V3 sp = divv(mulv(divv(sub(x, bmin()), delta), n), sv);
            V3 ep = divv(mulv(divv(sub(add(x, mul(w, dtot)), bmin()), delta), n), sv);
            float spv[3] = {sp.x, sp.y, sp.z}, epv[3] = {ep.x, ep.y, ep.z};
            int step[3], idx[3];
            float tdel[3], tmx[3];
            for (int a = 0; a < 3; a++) {
                float diff = epv[a] - spv[a];
                step[a] = (int)signf(diff);
                tdel[a] = step[a] != 0 ? std::min((float)step[a] / diff, 1e7f) : 1e7f;
                float fr = spv[a] - floorf(spv[a]);
                tmx[a] = step[a] > 0 ? tdel[a] * (1.0f - fr) : tdel[a] * fr;
                idx[a] = (int)floorf(spv[a]);
            }
            if (step[0] == 0 && step[1] == 0 && step[2] == 0) break;
            while (idx[0] >= 0 && idx[1] >= 0 && idx[2] >= 0 && idx[0] < S.svx && idx[1] < S.svy && idx[2] < S.svz) {
                if (guard()) return acc;
                size_t k = ((size_t)idx[2] * S.svy + idx[1]) * S.svx + idx[0];
                float mu_c = S.sv_data[2 * k], mu_r = S.sv_data[2 * k + 1];
                V3 vmin = v3((float)(idx[0] * S.sv_size), (float)(idx[1] * S.sv_size), (float)(idx[2] * S.sv_size));
                V3 vmax = v3((float)(idx[0] * S.sv_size + S.sv_size), (float)(idx[1] * S.sv_size + S.sv_size),
                             (float)(idx[2] * S.sv_size + S.sv_size));
                vmin = add(mulv(divv(vmin, n), delta), bmin());
                vmax = add(mulv(divv(vmax, n), delta), bmin());
                float tv0 = 0.0f, tv1 = 0.0f;
                ray_box(vmin, vmax, old_x, w, tv0, tv1);
                x = add(old_x, mul(w, tv0));
                T *= rrt_est(x, w, tv0, tv1, T, wsum, res_t, res_d, mu_c, mu_r, r);
                if (tmx[0] < tmx[1]) {
                    if (tmx[0] < tmx[2]) {
                        idx[0] += step[0];
                        tmx[0] += tdel[0];
                    } else {
                        idx[2] += step[2];
                        tmx[2] += tdel[2];
                    }
                } else {
                    if (tmx[1] < tmx[2]) {
                        idx[1] += step[1];
                        tmx[1] += tdel[1];
                    } else {
                        idx[2] += step[2];
                        tmx[2] += tdel[2];
                    }
                }
            }
            float xi = rnd(r);
            if (xi > wsum || iteration >= 10) break;
            V3 l = sky(w);
            acc = add(acc, v3(l.x * T, l.y * T, l.z * T));
            iteration++;
            T = res_t;
            x = add(old_x, mul(w, res_d));
            w = sample_phase(r, S.g, w);
            wsum = 0.0f;
            res_t = 0.0f;
            res_d = 0.0f;
        }
        V3 l = sky(w);
        return add(acc, v3(l.x * T, l.y * T, l.z * T));
    }

    // ---- unbiased residual ratio tracking (no reference counterpart; the CUDA core's
    // track_residual_ratio_nee): next-event estimation with residual ratio tracking (Novak et al.
    // 2014) for the shadow rays over the supervoxel (mu_c, mu_r_bar) of SuperVoxelGrid.cpp:218-265, and
    // delta tracking with each supervoxel's majorant (extinction * largest density incl. a one-voxel
    // halo) for the free paths; empty supervoxels are crossed without random numbers.  sv_local: 4
    // floats per supervoxel (mu_c, mu_r_bar, 1 / max, 1 / majorant).
    struct Walk {
        int idx[3], step[3];
        float next[3], delta[3];
    };
    void walk_begin(V3 x, V3 w, Walk& s) const {
        const float xv[3] = {x.x, x.y, x.z}, wv[3] = {w.x, w.y, w.z};
        const int n[3] = {S.svx, S.svy, S.svz};
        for (int a = 0; a < 3; a++) {
            int i = (int)floorf((xv[a] - S.box_min[a]) * S.sv_inv_world[a]);
            i = std::min(std::max(i, 0), n[a] - 1);
            s.idx[a] = i;
            if (wv[a] > 0.0f) {
                s.step[a] = 1;
                s.next[a] = ((S.box_min[a] + (float)(i + 1) * S.sv_world[a]) - xv[a]) / wv[a];
                s.delta[a] = S.sv_world[a] / wv[a];
            } else if (wv[a] < 0.0f) {
                s.step[a] = -1;
                s.next[a] = ((S.box_min[a] + (float)i * S.sv_world[a]) - xv[a]) / wv[a];
                s.delta[a] = -S.sv_world[a] / wv[a];
            } else {
                s.step[a] = 0;
                s.next[a] = INFINITY;
                s.delta[a] = INFINITY;
            }
        }
    }
    static int walk_axis(const Walk& s) {
        return s.next[0] < s.next[1] ? (s.next[0] < s.next[2] ? 0 : 2) : (s.next[1] < s.next[2] ? 1 : 2);
    }
    bool walk_advance(Walk& s, int a) const {
        s.idx[a] += s.step[a];
        s.next[a] += s.delta[a];
        const int n = a == 0 ? S.svx : (a == 1 ? S.svy : S.svz);
        return s.idx[a] >= 0 && s.idx[a] < n;
    }
    const float* walk_cell(const Walk& s) const {
        return S.sv_local + 4 * (((size_t)s.idx[2] * S.svy + s.idx[1]) * S.svx + s.idx[0]);
    }
    float transmittance_residual_ratio(V3 x, V3 w, float max_dist, Rng& r) {
        float tmin, tmax;
        if (!ray_box(bmin(), bmax(), x, w, tmin, tmax)) return 1.0f;
        const float d = std::min(tmax, max_dist) - tmin;
        if (!(d > 0.0f)) return 1.0f;
        x = add(x, mul(w, tmin));
        Walk s;
        walk_begin(x, w, s);
        float T = 1.0f, t0 = 0.0f;
        while (true) {
            if (guard()) return 0.0f;
            const int a = walk_axis(s);
            const float t1 = std::min(s.next[a], d);
            const float* c = walk_cell(s);
            if (c[3] > 0.0f && t1 > t0) {
                T *= m_exp(-c[0] * (t1 - t0));
                const float inv_mu_r = 1.0f / c[1];
                float t = t0;
                while (true) {
                    if (guard()) return 0.0f;
                    t += -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) * inv_mu_r;
                    if (t >= t1) break;
                    const float dens = sample(add(x, mul(w, t)), r);
                    T *= 1.0f - (S.extinction * dens - c[0]) * inv_mu_r;
                }
            }
            if (t1 >= d) break;
            t0 = std::max(t0, t1);
            if (!walk_advance(s, a)) break;
        }
        return T;
    }
    V3 residual_ratio_nee(V3 x, V3 w, Rng& r, bool& ev) {
        V3 color = v3(0, 0, 0);
        float tmin, tmax;
        const float absorb = 1.0f - S.albedo;
        if (ray_box(bmin(), bmax(), x, w, tmin, tmax)) {
            x = add(x, mul(w, tmin));
            float d = tmax - tmin;
            int bounces = 0;
            while (true) {
                Walk s;
                walk_begin(x, w, s);
                float t0 = 0.0f, t = 0.0f;
                bool collided = false;
                while (true) {
                    if (guard()) return color;
                    const int a = walk_axis(s);
                    const float t1 = std::min(s.next[a], d);
                    const float* c = walk_cell(s);
                    if (c[3] > 0.0f && t1 > t0) {
                        t = t0;
                        while (true) {
                            if (guard()) return color;
                            t += -m_log(std::max(0.0000000001f, 1.0f - rnd(r))) * c[3];
                            if (t >= t1) break;
                            const float dens = sample(add(x, mul(w, t)), r);
                            const float ratio = dens * c[2];
                            const float xi = rnd(r);
                            if (xi < absorb * ratio) {
                                ev = true;
                                return S.emission ? add(color, emission(add(x, mul(w, t)), r)) : color;
                            }
                            if (xi < ratio) {
                                collided = true;
                                break;
                            }
                        }
                        if (collided) break;
                    }
                    if (t1 >= d) break;
                    t0 = std::max(t0, t1);
                    if (!walk_advance(s, a)) break;
                }
                if (!collided) break;
                x = add(x, mul(w, t));
                if (S.max_bounces > 0 && ++bounces > S.max_bounces) return color;
                V3 nw = sample_phase(r, S.g, w);
                ev = true;
                bool to_light = false;
                float factor = 1.0f, ldist = 0.0f, pdf_l = 0.0f;
                int lidx = 0;
                if (S.num_lights > 0) {
                    to_light = S.env_is_black ? true : (rnd(r) > 0.5f);
                    factor = S.env_is_black ? 1.0f : 2.0f;
                }
                V3 dl = to_light ? light_dir(x, r, lidx, factor, ldist) : importance_sky(r, pdf_l);
                float pdf_p = eval_phase(S.g, w, dl);
                w = nw;
                if (to_light) {
                    float tr = transmittance_residual_ratio(x, dl, ldist, r);
                    float f = (factor * pdf_p) * tr;
                    V3 l = light_rad(x, lidx);
                    color = add(color, v3(f * l.x, f * l.y, f * l.z));
                } else {
                    float tr = transmittance_residual_ratio(x, dl, INFINITY, r);
                    float f = ((factor * pdf_p) / pdf_l) * tr;
                    V3 l = sky(dl);
                    color = add(color, v3(f * l.x, f * l.y, f * l.z));
                }
                if (!ray_box(bmin(), bmax(), x, w, tmin, tmax)) break;
                x = add(x, mul(w, tmin));
                d = tmax - tmin;
            }
        }
        if (!ev) color = add(color, sky(w));
        return color;
    }

    // pathTraceSample (Clouds.glsl:73-141): seed, jittered camera ray, tracker
    V3 path(int px, int py, uint32_t frame) {
        steps = 0;
        uint32_t W = (uint32_t)S.width, H = (uint32_t)S.height;
        uint32_t seed = (S.frame_count + frame) * W * H + (uint32_t)px + (uint32_t)py * W;
        seed += S.seed_offset;
        Rng r = rng_init(seed);
        float rx = rnd(r), ry = rnd(r);
        float sx = (2.0f * ((float)px + rx)) / (float)S.width - 1.0f;
        float sy = (2.0f * ((float)py + ry)) / (float)S.height - 1.0f;
        V3 x, w;
        camera_ray(S, sx, sy, x, w);
        bool ev = false;
        switch (S.mode) {
            case 0: return S.use_iso ? delta_iso(x, w, r, ev) : delta(x, w, r, ev);
            case 1: return spectral_delta(x, w, r, ev);
            case 6: return spectral_nee(x, w, r, ev);
            case 2: return ratio(x, w, r, ev);
            case 3: return S.nanovdb ? decomposition_sparse(x, w, r) : decomposition(x, w, r);
            case 4: return rrt(x, w, r);
            case 9: return residual_ratio_nee(x, w, r, ev);
            default: return S.use_iso ? nee_iso(x, w, r, ev) : nee(x, w, r, ev);
        }
    }
};

int threads_or_default(int t) {
#ifdef _OPENMP
    return t > 0 ? t : omp_get_max_threads();
#else
    (void)t;
    return 1;
#endif
}

}  // namespace

extern "C" {

// inputs a tracker dereferences: the scene is rejected (status 2) rather than read through null
static bool scene_inputs_ok(const OracleScene* s) {
    if (!s || (!s->density && !s->nanovdb)) return false;
    const bool nee = s->mode == 5 || s->mode == 6;
    if (nee && s->use_ess && !s->occupancy) return false;
    if ((s->mode == 3 && !s->nanovdb) || s->mode == 4) {
        if (!s->sv_data) return false;
    }
    if (s->mode == 9 && (!s->sv_local || s->nanovdb)) return false;
    if (s->env_kind == 4 && (!s->env_rgba || !s->env_pyramid)) return false;
    return true;
}

int oracle_render_rows(const OracleScene* s, int row0, int row1, double* film, uint64_t* lookups, int threads) {
    if (!scene_inputs_ok(s)) return 2;
    g_clip = s->use_clip ? s->clip : nullptr;
    const OracleScene& S = *s;
    uint64_t total_lookups = 0;
    int nt = threads_or_default(threads);
    const int rows = row1 - row0;
#pragma omp parallel num_threads(nt) reduction(+ : total_lookups)
    {
        Tracer T(S);
#pragma omp for schedule(dynamic, 1)
        for (int yy = 0; yy < rows; yy++) {
            int y = row0 + yy;
            for (int x = 0; x < S.width; x++) {
                double acc[3] = {0, 0, 0};
                for (uint32_t f = 0; f < S.num_frames; f++) {
                    V3 L = T.path(x, y, f);
                    acc[0] += L.x;
                    acc[1] += L.y;
                    acc[2] += L.z;
                }
                size_t p = (size_t)y * S.width + x;
                film[p * 3 + 0] += acc[0];
                film[p * 3 + 1] += acc[1];
                film[p * 3 + 2] += acc[2];
            }
        }
        total_lookups += T.lookups;
    }
    if (lookups) *lookups += total_lookups;
    return 0;
}

int oracle_render(const OracleScene* s, double* film, double* film_sq, uint64_t* lookups, int threads) {
    if (!scene_inputs_ok(s)) return 2;
    g_clip = s->use_clip ? s->clip : nullptr;
    const OracleScene& S = *s;
    uint64_t total_lookups = 0;
    int nt = threads_or_default(threads);
#pragma omp parallel num_threads(nt) reduction(+ : total_lookups)
    {
        Tracer T(S);
#pragma omp for schedule(dynamic, 1)
        for (int y = 0; y < S.height; y++) {
            for (int x = 0; x < S.width; x++) {
                double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
                for (uint32_t f = 0; f < S.num_frames; f++) {
                    V3 L = T.path(x, y, f);
                    acc[0] += L.x;
                    acc[1] += L.y;
                    acc[2] += L.z;
                    acc2[0] += (double)L.x * L.x;
                    acc2[1] += (double)L.y * L.y;
                    acc2[2] += (double)L.z * L.z;
                }
                size_t p = (size_t)y * S.width + x;
                for (int c = 0; c < 3; c++) {
                    film[p * 3 + c] += acc[c];
                    if (film_sq) film_sq[p * 3 + c] += acc2[c];
                }
            }
        }
        total_lookups += T.lookups;
    }
    if (lookups) *lookups += total_lookups;
    return 0;
}

int oracle_trace_paths(const OracleScene* s, const int* xs, const int* ys, const uint32_t* frames, int n,
                       float* out_rgb, int threads) {
    if (!scene_inputs_ok(s)) return 2;
    g_clip = s->use_clip ? s->clip : nullptr;
    int nt = threads_or_default(threads);
#pragma omp parallel num_threads(nt)
    {
        Tracer T(*s);
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < n; i++) {
            V3 L = T.path(xs[i], ys[i], frames[i]);
            out_rgb[3 * i + 0] = L.x;
            out_rgb[3 * i + 1] = L.y;
            out_rgb[3 * i + 2] = L.z;
        }
    }
    return 0;
}

// ---- scene generation: improved Perlin noise (Perlin 2002), seeded permutation ----
static uint32_t pcg(uint32_t& st) {
    st = st * 747796405u + 2891336453u;
    uint32_t word = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
    return (word >> 22u) ^ word;
}
static float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
static float lerpf(float t, float a, float b) { return a + t * (b - a); }
static float grad(int h, float x, float y, float z) {
    h &= 15;
    float u = h < 8 ? x : y;
    float v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
static float perlin(const int* p, float x, float y, float z) {
    float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
    x -= fx;
    y -= fy;
    z -= fz;
    float u = fade(x), v = fade(y), w = fade(z);
    int A = p[X] + Y, AA = p[A] + Z, AB = p[A + 1] + Z, B = p[X + 1] + Y, BA = p[B] + Z, BB = p[B + 1] + Z;
    float r0 = lerpf(v, lerpf(u, grad(p[AA], x, y, z), grad(p[BA], x - 1.0f, y, z)),
                     lerpf(u, grad(p[AB], x, y - 1.0f, z), grad(p[BB], x - 1.0f, y - 1.0f, z)));
    float r1 = lerpf(v, lerpf(u, grad(p[AA + 1], x, y, z - 1.0f), grad(p[BA + 1], x - 1.0f, y, z - 1.0f)),
                     lerpf(u, grad(p[AB + 1], x, y - 1.0f, z - 1.0f), grad(p[BB + 1], x - 1.0f, y - 1.0f, z - 1.0f)));
    return lerpf(w, r0, r1);
}

void oracle_fbm(float* out, int nx, int ny, int nz, uint32_t seed, int octaves, float lacunarity, float gain,
                float base_frequency, float threshold, float contrast) {
    int perm[256], p[512];
    for (int i = 0; i < 256; i++) perm[i] = i;
    uint32_t st = seed;
    for (int i = 255; i > 0; i--) {
        uint32_t j = pcg(st) % (uint32_t)(i + 1);
        std::swap(perm[i], perm[j]);
    }
    for (int i = 0; i < 512; i++) p[i] = perm[i & 255];
    const float inv = 1.0f / (float)std::max(nx, std::max(ny, nz));
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                float px = ((float)x + 0.5f) * inv, py = ((float)y + 0.5f) * inv, pz = ((float)z + 0.5f) * inv;
                float sum = 0.0f, amp = 1.0f, freq = base_frequency, norm = 0.0f;
                for (int o = 0; o < octaves; o++) {
                    sum += amp * perlin(p, px * freq, py * freq, pz * freq);
                    norm += amp;
                    amp *= gain;
                    freq *= lacunarity;
                }
                float v = sum / norm;
                v = std::min(std::max(0.5f + contrast * v, 0.0f), 1.0f);
                out[((size_t)z * ny + y) * nx + x] = v < threshold ? 0.0f : v;
            }
}

void oracle_minmax(const float* v, uint64_t n, float* out_min, float* out_max) {
    float lo = INFINITY, hi = -INFINITY;
    for (uint64_t i = 0; i < n; i++) {
        lo = std::min(lo, v[i]);
        hi = std::max(hi, v[i]);
    }
    if (lo == hi) lo = 0.0f;  // DensityField.cpp:146-150
    *out_min = lo;
    *out_max = hi;
}

void oracle_normalize(const float* in, float* out, uint64_t n, float vmin, float vmax) {
    const float range = vmax - vmin;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) out[i] = (in[i] - vmin) / range;
}

// CloudData::computeGridBounds (CloudData.cpp:63-78) with voxel size 1
void oracle_grid_bounds(int nx, int ny, int nz, float e, float* bmin, float* bmax) {
    float sx = (float)nx, sy = (float)ny, sz = (float)nz;
    float ms = std::max(sx, std::max(sy, sz));
    bmax[0] = sx * e / ms;
    bmax[1] = sy * e / ms;
    bmax[2] = sz * e / ms;
    for (int i = 0; i < 3; i++) bmin[i] = -bmax[i];
}

// SuperVoxelGridResidualRatioTracking::computeSuperVoxels / SuperVoxelGridDecompositionTracking
// (SuperVoxelGrid.cpp:101-211, 316-396)
void oracle_supervoxel_stats(const float* dens, int nx, int ny, int nz, int sv, int halo, float* out_min,
                             float* out_max, float* out_avg, uint8_t* out_occ) {
    int gx = (nx + sv - 1) / sv, gy = (ny + sv - 1) / sv, gz = (nz + sv - 1) / sv;
    int total = gx * gy * gz;
#pragma omp parallel for schedule(static)
    for (int idx = 0; idx < total; idx++) {
        int bx = idx % gx, by = (idx / gx) % gy, bz = idx / (gx * gy);
        float lo = 3.402823466e+38f, hi = -3.402823466e+38f, sum = 0.0f;
        int cnt = 0;
        int o0 = halo ? -1 : 0, o1 = halo ? sv : sv - 1;
        for (int oz = o0; oz <= o1; oz++)
            for (int oy = o0; oy <= o1; oy++)
                for (int ox = o0; ox <= o1; ox++) {
                    int x = bx * sv + ox, y = by * sv + oy, z = bz * sv + oz;
                    float v = 0.0f;
                    if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) v = dens[((size_t)z * ny + y) * nx + x];
                    lo = std::min(lo, v);
                    hi = std::max(hi, v);
                    sum += v;
                    cnt++;
                }
        float avg = sum / (float)cnt;
        if ((nx % sv != 0 && bx == gx - 1) || (ny % sv != 0 && by == gy - 1) || (nz % sv != 0 && bz == gz - 1)) lo = 0.0f;
        out_min[idx] = lo;
        out_max[idx] = hi;
        if (out_avg) out_avg[idx] = avg;
        if (out_occ) out_occ[idx] = hi < 1e-5f ? 0 : 1;
    }
}

// SuperVoxelGridResidualRatioTracking::recomputeSuperVoxels (SuperVoxelGrid.cpp:218-256)
void oracle_rrt_params(const float* mn, const float* mx, const float* avg, int total, float extinction, int sv,
                       float* out_pairs) {
    const float gamma = 2.0f;
    const float D = sqrtf(3.0f) * (float)sv;
    for (int i = 0; i < total; i++) {
        float mu_min = mn[i] * extinction, mu_max = mx[i] * extinction, mu_avg = avg[i] * extinction;
        float mu_r = std::max(mu_max - mu_min, 0.1f);
        float mu_c = mu_min + mu_r * m_pow(gamma, (1.0f / (D * mu_r)) - 1.0f);
        mu_c = std::min(std::max(mu_c, mu_min), mu_avg);
        out_pairs[2 * i] = mu_c;
        out_pairs[2 * i + 1] = mu_r;
    }
}

// Supervoxel grid of the unbiased residual ratio tracker (the CUDA core's rrt_local_kernel): the
// (mu_c, mu_r_bar) of oracle_rrt_params, then 1 / max and 1 / (extinction * max) (0 when empty).
void oracle_rrt_local(const float* mn, const float* mx, const float* avg, int total, float extinction, int sv,
                      float* out4) {
    const float D = sqrtf(3.0f) * (float)sv;
    for (int i = 0; i < total; i++) {
        const float dmax = mx[i];
        float mu_min = mn[i] * extinction, mu_max = dmax * extinction, mu_avg = avg[i] * extinction;
        float mu_r = std::max(mu_max - mu_min, 0.1f);
        float mu_c = mu_min + mu_r * m_pow(2.0f, (1.0f / (D * mu_r)) - 1.0f);
        mu_c = std::min(std::max(mu_c, mu_min), mu_avg);
        const bool empty = !(dmax > 0.0f) || !(mu_max > 0.0f);
        out4[4 * i + 0] = mu_c;
        out4[4 * i + 1] = mu_r;
        out4[4 * i + 2] = empty ? 0.0f : 1.0f / dmax;
        out4[4 * i + 3] = empty ? 0.0f : 1.0f / mu_max;
    }
}

// Occupancy of bs^3 blocks: any voxel (plus halo) above `threshold` (intent of
// ComputeOccupancyGrid.glsl:91-143).
void oracle_occupancy(const float* dens, int nx, int ny, int nz, int bs, int halo, float threshold, uint8_t* out) {
    int gx = (nx + bs - 1) / bs, gy = (ny + bs - 1) / bs, gz = (nz + bs - 1) / bs;
    for (int bz = 0; bz < gz; bz++)
        for (int by = 0; by < gy; by++)
            for (int bx = 0; bx < gx; bx++) {
                bool occ = false;
                for (int z = bz * bs - halo; z < bz * bs + bs + halo && !occ; z++)
                    for (int y = by * bs - halo; y < by * bs + bs + halo && !occ; y++)
                        for (int x = bx * bs - halo; x < bx * bs + bs + halo && !occ; x++)
                            if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz &&
                                dens[((size_t)z * ny + y) * nx + x] > threshold)
                                occ = true;
                out[((size_t)bz * gy + by) * gx + bx] = occ ? 1 : 0;
            }
}

// OctahedralMapper.glsl:65-85 + 2x2 mip reduction
void oracle_env_pyramid(const float* rgba, int w, int h, int levels, float* pyramid) {
    OracleScene S;
    memset(&S, 0, sizeof(S));
    S.env_rgba = rgba;
    S.env_w = w;
    S.env_h = h;
    int res = 1 << levels;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < res; y++)
        for (int x = 0; x < res; x++) {
            float best = -1.0f;
            for (int i = 0; i < 5; i++) {
                float sxo = 0.1f + 0.2f * (float)i;
                for (int j = 0; j < 5; j++) {
                    float syo = 0.1f + 0.2f * (float)j;
                    V3 dir = oct_to_world(((float)x + sxo) / (float)res, ((float)y + syo) / (float)res);
                    float tu = m_atan2(dir.z, dir.x) / (2.0f * PI) + 0.5f;
                    float tv = -m_asin(dir.y) / PI + 0.5f;
                    V3 c = env_fetch(S, tu, tv);
                    c = v3(std::min(c.x, 100000.0f), std::min(c.y, 100000.0f), std::min(c.z, 100000.0f));
                    best = std::max(best, length(c));
                }
            }
            pyramid[(size_t)y * res + x] = best;
        }
    size_t off_in = 0, off_out = (size_t)res * res;
    for (int l = 1; l < levels; l++) {
        int r = res >> l, ri = r * 2;
        for (int y = 0; y < r; y++)
            for (int x = 0; x < r; x++) {
                const float* in = pyramid + off_in;
                float a = in[(size_t)(2 * y) * ri + 2 * x], b = in[(size_t)(2 * y) * ri + 2 * x + 1];
                float c = in[(size_t)(2 * y + 1) * ri + 2 * x], d = in[(size_t)(2 * y + 1) * ri + 2 * x + 1];
                pyramid[off_out + (size_t)y * r + x] = ((a + b) + (c + d)) * 0.25f;
            }
        off_in = off_out;
        off_out += (size_t)r * r;
    }
}

// EAWDenoise.glsl:216-314 (compute path) / 92-158 (fragment path colour weight)
// ---- SVGF (Data/Shaders/Denoiser/SVGF/SVGF.glsl; compute_weight svgf_common.glsl:29-41) ----
// One frame of the filter on prepared maps (all w*h, rgba = 4 floats): the reprojection pass
// (SVGF.glsl:210-267 with is_reprj_valid :80-94, try_2x2_tap :96-147, try_3x3_bilat :149-193), the
// moments filter (:286-347), `iterations` a-trous passes (:401-495; iteration 0 refreshes the colour
// history) and the history update (moments, normal, depth of this frame).  Two choices where the
// shader's result is not defined: the moments filter reads the pre-filter values of its neighbours
// (the shader filters temp_accum in place while neighbours read it), and filter_variance clamps its
// 3x3 reads to the image (the shader's texelFetch may leave it).
static float svgf_weight_o(float cd, float od, float phi_d, const float* cn, const float* on, float cc, float oc,
                           float phi_c) {
    float wn = powf(std::max(0.0f, (cn[0] * on[0] + cn[1] * on[1]) + cn[2] * on[2]), 128.0f);
    float wz = (phi_d == 0.0f) ? 0.0f : fabsf(cd - od) / phi_d;
    float wc = fabsf(cc - oc) * 2.0f / phi_c;
    return expf(0.0f - std::max(wc, 0.0f) - std::max(wz, 0.0f)) * wn;
}

void oracle_svgf_frame(const float* noisy, const float* normal, const float* depth, const float* fwidth,
                       const float* motion, float* color_hist, float* moments_hist, float* normal_hist,
                       float* depth_hist, int w, int h, float zt, float nt, int iterations, float* out) {
    const size_t n = (size_t)w * h;
    std::vector<float> moments(n * 4), temp(n * 4), filt(n * 4), a(n * 4), b(n * 4);
    auto valid = [&](int x, int y, float z, float zp, const float* nn, const float* np) {
        if (x < 1 || y < 1 || x > w - 1 || y > h - 1) return false;
        if (fabsf(zp - z) > zt) return false;
        float dx = np[0] - nn[0], dy = np[1] - nn[1], dz = np[2] - nn[2];
        return !(sqrtf((dx * dx + dy * dy) + dz * dz) > nt);
    };
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const size_t i = (size_t)y * w + x;
            const float mvx = motion[2 * i], mvy = motion[2 * i + 1];
            int pxp = (int)(0.5f + ((float)x - mvx)), pyp = (int)(0.5f + ((float)y - mvy));
            float pm0 = 0.0f, pm1 = 0.0f, hist_len = 0.0f;
            bool ok = !(pxp < 0 || pyp < 0 || pxp >= w || pyp >= h);
            if (ok) {
                const float* r = moments_hist + ((size_t)pyp * w + pxp) * 4;
                pm0 = r[0];
                pm1 = r[1];
                hist_len = r[2];
            }
            const float* col = noisy + i * 4;
            float last[3] = {color_hist[i * 4], color_hist[i * 4 + 1], color_hist[i * 4 + 2]};
            if (ok) {
                float fx = 0.01f + ((float)x - mvx), fy = 0.01f + ((float)y - mvy);
                int ix = (int)fx, iy = (int)fy;
                const float d = depth[i];
                const float* nn = normal + i * 4;
                const int ox[4] = {0, 0, 1, 1}, oy[4] = {0, 1, 0, 1};
                bool vs[4], found = false;
                for (int k = 0; k < 4; k++) {
                    int qx = ix + ox[k], qy = iy + oy[k];
                    bool inside = qx >= 0 && qy >= 0 && qx < w && qy < h;
                    vs[k] = inside && valid(qx, qy, d, depth_hist[(size_t)qy * w + qx], nn,
                                            normal_hist + ((size_t)qy * w + qx) * 4);
                    found = found || vs[k];
                }
                if (found) {
                    float ax = fx - floorf(fx), ay = fy - floorf(fy);
                    const float wk[4] = {(1 - ax) * (1 - ay), ax * (1 - ay), (1 - ax) * ay, ax * ay};
                    float cb[3] = {0, 0, 0}, mb[2] = {0, 0}, sw = 0.0f;
                    for (int k = 0; k < 4; k++) {
                        if (!vs[k]) continue;
                        const size_t q = (size_t)(iy + oy[k]) * w + (ix + ox[k]);
                        mb[0] += wk[k] * moments_hist[q * 4];
                        mb[1] += wk[k] * moments_hist[q * 4 + 1];
                        for (int c = 0; c < 3; c++) cb[c] += wk[k] * color_hist[q * 4 + c];
                        sw += wk[k];
                    }
                    found = sw >= 0.001f;
                    if (found) {
                        for (int c = 0; c < 3; c++) last[c] = cb[c] / sw;
                        pm0 = mb[0] / sw;
                        pm1 = mb[1] / sw;
                    }
                }
                if (!found) {
                    float nv = 0.0f, fc[3] = {0, 0, 0}, fm[2] = {0, 0};
                    for (int yy = -1; yy <= 1; yy++)
                        for (int xx = -1; xx <= 1; xx++) {
                            int qx = ix + xx, qy = iy + yy;
                            if (qx < 1 || qy < 1 || qx >= w || qy >= h) continue;
                            const size_t q = (size_t)qy * w + qx;
                            if (valid(qx, qy, d, depth_hist[q], nn, normal_hist + q * 4)) {
                                for (int c = 0; c < 3; c++) fc[c] += color_hist[q * 4 + c];
                                fm[0] += moments_hist[q * 4];
                                fm[1] += moments_hist[q * 4 + 1];
                                nv += 1.0f;
                            }
                        }
                    if (nv > 0.0f) {
                        for (int c = 0; c < 3; c++) last[c] = fc[c] / nv;
                        pm0 = fm[0] / nv;
                        pm1 = fm[1] / nv;
                        found = true;
                    }
                }
                ok = found;
            }
            hist_len = std::min(ok ? hist_len + 1.0f : 1.0f, 32.0f);
            const float a_c = ok ? std::max(0.01f, 1.0f / hist_len) : 1.0f;
            const float a_m = ok ? std::max(0.2f, 1.0f / hist_len) : 1.0f;
            float m1 = col[0], m2 = m1 * m1;
            m1 = pm0 * (1.0f - a_m) + m1 * a_m;
            m2 = pm1 * (1.0f - a_m) + m2 * a_m;
            const float var = std::max(0.0f, m2 - m1 * m1);
            moments[i * 4] = m1;
            moments[i * 4 + 1] = m2;
            moments[i * 4 + 2] = hist_len;
            moments[i * 4 + 3] = 0.0f;
            for (int c = 0; c < 3; c++) temp[i * 4 + c] = last[c] * (1.0f - a_c) + col[c] * a_c;
            temp[i * 4 + 3] = var;
        }
    // moments filter
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const size_t i = (size_t)y * w + x;
            const float hl = moments[i * 4 + 2];
            if (hl >= 4.0f) {
                for (int c = 0; c < 4; c++) filt[i * 4 + c] = temp[i * 4 + c];
                continue;
            }
            const float cd = depth[i], cfw = fwidth[i];
            const float* cn = normal + i * 4;
            float sw = 0.0f, sc[3] = {0, 0, 0}, sm[2] = {0, 0};
            for (int yy = -3; yy <= 3; yy++)
                for (int xx = -3; xx <= 3; xx++) {
                    int qx = x + xx, qy = y + yy;
                    if (qx < 0 || qy < 0 || qx >= w || qy >= h) continue;
                    const size_t q = (size_t)qy * w + qx;
                    float wt = svgf_weight_o(cd, depth[q], fabsf(cfw) + 0.0001f, cn, normal + q * 4, temp[i * 4],
                                             temp[q * 4], 10.0f);
                    sw += wt;
                    for (int c = 0; c < 3; c++) sc[c] += wt * temp[q * 4 + c];
                    sm[0] += wt * moments[q * 4];
                    sm[1] += wt * moments[q * 4 + 1];
                }
            sw = std::max(sw, 1e-6f);
            for (int c = 0; c < 3; c++) filt[i * 4 + c] = sc[c] / sw;
            const float m0 = sm[0] / sw, m1v = sm[1] / sw;
            float var = m1v - m0 * m0;
            var *= 4.0f / hl;
            filt[i * 4 + 3] = var;
        }
    // a-trous
    const float* src = filt.data();
    if (iterations < 1) std::copy(filt.begin(), filt.end(), color_hist);
    const float kv2[2][2] = {{1.0f / 4.0f, 1.0f / 8.0f}, {1.0f / 8.0f, 1.0f / 16.0f}};
    const float kvals[3] = {1.0f, 2.0f / 3.0f, 1.0f / 6.0f};
    for (int it = 0; it < iterations; it++) {
        float* dst = (it & 1) ? b.data() : a.data();
        const int step = 1 << it;
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                const size_t i = (size_t)y * w + x;
                const float* cc = src + i * 4;
                float fv = 0.0f;
                for (int yy = -1; yy <= 1; yy++)
                    for (int xx = -1; xx <= 1; xx++) {
                        int qx = std::min(std::max(x + xx, 0), w - 1), qy = std::min(std::max(y + yy, 0), h - 1);
                        fv += src[((size_t)qy * w + qx) * 4 + 3] * kv2[abs(xx)][abs(yy)];
                    }
                const float* cn = normal + i * 4;
                const float cz = depth[i], cfw = fwidth[i];
                const float phi_c = sqrtf(std::max(0.0f, 1e-10f + fv));
                float accw = kvals[0] * kvals[0];
                float sum[4] = {cc[0] * accw, cc[1] * accw, cc[2] * accw, cc[3] * accw};
                for (int yy = -2; yy <= 2; yy++)
                    for (int xx = -2; xx <= 2; xx++) {
                        int qx = x + xx * step, qy = y + yy * step;
                        bool inside = qx >= 0 && qy >= 0 && qx < w && qy < h;
                        if (!inside || (xx == 0 && yy == 0)) continue;
                        const float kval = kvals[abs(xx)] * kvals[abs(yy)];
                        const size_t q = (size_t)qy * w + qx;
                        const float len = sqrtf((float)(xx * xx + yy * yy));
                        const float wt = svgf_weight_o(cz, depth[q], fabsf(cfw * len * (float)step) + 0.0001f, cn,
                                                       normal + q * 4, cc[0], src[q * 4], phi_c) *
                                         kval;
                        for (int c = 0; c < 3; c++) sum[c] += wt * src[q * 4 + c];
                        sum[3] += wt * wt * src[q * 4 + 3];
                        accw += wt;
                    }
                for (int c = 0; c < 3; c++) dst[i * 4 + c] = sum[c] / accw;
                dst[i * 4 + 3] = sum[3] / (accw * accw);
                if (it == 0)
                    for (int c = 0; c < 4; c++) color_hist[i * 4 + c] = dst[i * 4 + c];
            }
        src = dst;
    }
    for (size_t i = 0; i < n; i++) {
        for (int c = 0; c < 4; c++) {
            moments_hist[i * 4 + c] = moments[i * 4 + c];
            normal_hist[i * 4 + c] = normal[i * 4 + c];
            out[i * 4 + c] = src[i * 4 + c];
        }
        depth_hist[i] = depth[i];
    }
}

void oracle_eaw(const float* color, const float* pos, const float* nrm, int w, int h, int iterations, float phi_c,
                float phi_p, float phi_n, int quirk, float* out) {
    std::vector<float> a(color, color + (size_t)w * h * 4), b((size_t)w * h * 4);
    float kern[25];
    for (int i = 0; i < 25; i++) {
        int x = i % 5 - 2, y = i / 5 - 2;
        kern[i] = expf(-float(x * x + y * y) / 2.0f);
    }
    auto ld = [&](const float* img, int x, int y, int c) {
        x = std::min(std::max(x, 0), w - 1);
        y = std::min(std::max(y, 0), h - 1);
        return img[((size_t)y * w + x) * 4 + c];
    };
    int step = 1;
    for (int it = 0; it < iterations; it++) {
        const float* src = a.data();
#pragma omp parallel for schedule(static)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                float cc[4], cp[4] = {0, 0, 0, 0}, cn[4] = {0, 0, 0, 0};
                for (int c = 0; c < 4; c++) {
                    cc[c] = ld(src, x, y, c);
                    if (pos) cp[c] = ld(pos, x, y, c);
                    if (nrm) cn[c] = ld(nrm, x, y, c);
                }
                float sum[4] = {0, 0, 0, 0}, acc = 0.0f;
                const float qwc = std::min(expf(-1.0f / phi_c), 1.0f);
                for (int i = 0; i < 25; i++) {
                    int sx = x + (i % 5 - 2) * step, sy = y + (i / 5 - 2) * step;
                    float oc[4];
                    for (int c = 0; c < 4; c++) oc[c] = ld(src, sx, sy, c);
                    float weight = 1.0f;
                    float d[4];
                    for (int c = 0; c < 4; c++) d[c] = cc[c] - oc[c];
                    float dist = ((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) + d[3] * d[3];
                    weight *= quirk ? qwc : std::min(expf(-dist / phi_c), 1.0f);
                    if (pos) {
                        for (int c = 0; c < 4; c++) d[c] = cp[c] - ld(pos, sx, sy, c);
                        dist = ((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) + d[3] * d[3];
                        weight *= std::min(expf(-dist / phi_p), 1.0f);
                    }
                    if (nrm) {
                        for (int c = 0; c < 4; c++) d[c] = cn[c] - ld(nrm, sx, sy, c);
                        dist = ((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) + d[3] * d[3];
                        weight *= std::min(expf(-dist / phi_n), 1.0f);
                    }
                    float wk = weight * kern[i];
                    for (int c = 0; c < 4; c++) sum[c] += oc[c] * wk;
                    acc += wk;
                }
                for (int c = 0; c < 4; c++) b[((size_t)y * w + x) * 4 + c] = sum[c] / acc;
            }
        std::swap(a, b);
        step *= 2;
    }
    memcpy(out, a.data(), a.size() * sizeof(float));
}

void oracle_set_double_rounded_math(int on) { g_dr_math = on != 0; }

// ---- kernel-predicting denoiser (modules/kpn_module/src/Kernel.cu) ----

// torch::softmax(x, 1): exp(x - max) / sum over the channel dimension, per pixel
void oracle_softmax_channels(const float* in, int n, int k, int h, int w, float* out) {
    const size_t plane = (size_t)h * w;
    for (int b = 0; b < n; b++)
        for (size_t i = 0; i < plane; i++) {
            const float* x = in + (size_t)b * k * plane + i;
            float* y = out + (size_t)b * k * plane + i;
            float m = -INFINITY;
            for (int t = 0; t < k; t++) m = std::max(m, x[(size_t)t * plane]);
            float s = 0.0f;
            for (int t = 0; t < k; t++) {
                y[(size_t)t * plane] = expf(x[(size_t)t * plane] - m);
                s += y[(size_t)t * plane];
            }
            for (int t = 0; t < k; t++) y[(size_t)t * plane] = y[(size_t)t * plane] / s;
        }
}

// perPixelKernelForwardKernel (Kernel.cu:38-81): output size min(image, weights), taps outside it skipped
void oracle_kpn_apply(const float* image, const float* weights, int n, int c, int h, int w, int wh, int ww, int k,
                      float* out) {
    const int ho = std::min(h, wh), wo = std::min(w, ww);
    const int K = k * k;
    for (int b = 0; b < n; b++)
        for (int y = 0; y < ho; y++)
            for (int x = 0; x < wo; x++) {
                float acc[4] = {0, 0, 0, 0};
                int t = 0;
                for (int dy = -k / 2; dy <= k / 2; dy++) {
                    int ky = y + dy;
                    for (int dx = -k / 2; dx <= k / 2; dx++, t++) {
                        int kx = x + dx;
                        if (kx >= 0 && kx < wo && ky >= 0 && ky < ho) {
                            float wt = weights[(size_t)b * ww * wh * K + (size_t)t * ww * wh + (size_t)y * ww + x];
                            for (int ch = 0; ch < c; ch++)
                                acc[ch] += wt * image[(size_t)b * w * h * c + (size_t)ch * w * h + (size_t)ky * w + kx];
                        }
                    }
                }
                for (int ch = 0; ch < c; ch++) out[(size_t)b * wo * ho * c + (size_t)ch * wo * ho + (size_t)y * wo + x] = acc[ch];
            }
}

// getInvIterBaseKernel (Kernel.cu:138-186); pixels whose low-resolution texel is out of range stay 0
void oracle_kpn_inv_iter_base(const float* x_hi, const float* pred_lo, const float* x_lo, const float* prev,
                              const float* fused, int n, int c, int h, int w, int lh, int lw, int wh, int ww, int k,
                              int use_prev, float* out) {
    const int ho = std::min(h, wh), wo = std::min(w, ww);
    const int K = k * k;
    const size_t plane = (size_t)wh * ww;
    for (size_t i = 0; i < (size_t)n * c * ho * wo; i++) out[i] = 0.0f;
    for (int b = 0; b < n; b++)
        for (int y = 0; y < ho; y++)
            for (int x = 0; x < wo; x++) {
                int lx = x / 2, ly = y / 2;
                if (lx >= lw || ly >= lh) continue;
                for (int ch = 0; ch < c; ch++) {
                    const float* wb = fused + (size_t)b * (K + 3) * plane + (size_t)y * ww + x;
                    float lf_w = 1.0f / (1.0f + expf(-wb[(size_t)K * plane]));
                    float hf_w = 1.0f / (1.0f + expf(-wb[(size_t)(K + 1) * plane]));
                    float pv_w = 1.0f / (1.0f + expf(-wb[(size_t)(K + 2) * plane]));
                    float xh = x_hi[((size_t)b * c + ch) * h * w + (size_t)y * w + x];
                    float xl = x_lo[((size_t)b * c + ch) * lh * lw + (size_t)ly * lw + lx];
                    float pl = pred_lo[((size_t)b * c + ch) * lh * lw + (size_t)ly * lw + lx];
                    float lf = lf_w * pl + (1.0f - lf_w) * xl;
                    if (use_prev) {
                        float pr = prev[((size_t)b * c + ch) * h * w + (size_t)y * w + x];
                        lf = lf * (1.0 - pv_w) + pr * pv_w;  // double literal, as in the reference
                    }
                    out[((size_t)b * c + ch) * ho * wo + (size_t)y * wo + x] = hf_w * (xh - xl + lf) + (1.0f - hf_w) * lf;
                }
            }
}

// torch::avg_pool2d(x, 2, 2)
void oracle_avg_pool2(const float* in, int nc, int h, int w, float* out) {
    const int ho = h / 2, wo = w / 2;
    for (int i = 0; i < nc; i++)
        for (int y = 0; y < ho; y++)
            for (int x = 0; x < wo; x++) {
                const float* b = in + ((size_t)i * h + 2 * y) * w + 2 * x;
                out[((size_t)i * ho + y) * wo + x] = (((b[0] + b[1]) + b[w]) + b[w + 1]) / 4.0f;
            }
}

// torch::grid_sampler_2d(prev, uv * 2 - 1, bilinear, zeros, align_corners = false)
void oracle_grid_sample(const float* prev, const float* uv, int n, int c, int ph, int pw, int h, int w, float* out) {
    const size_t plane = (size_t)h * w;
    for (int b = 0; b < n; b++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                float gx = uv[((size_t)b * 2 + 0) * plane + (size_t)y * w + x] * 2.0f - 1.0f;
                float gy = uv[((size_t)b * 2 + 1) * plane + (size_t)y * w + x] * 2.0f - 1.0f;
                float ix = ((gx + 1.0f) * (float)pw - 1.0f) / 2.0f;
                float iy = ((gy + 1.0f) * (float)ph - 1.0f) / 2.0f;
                float x0 = floorf(ix), y0 = floorf(iy), x1 = x0 + 1.0f, y1 = y0 + 1.0f;
                float nw = (x1 - ix) * (y1 - iy), ne = (ix - x0) * (y1 - iy);
                float sw = (x1 - ix) * (iy - y0), se = (ix - x0) * (iy - y0);
                int xi0 = (int)x0, yi0 = (int)y0, xi1 = xi0 + 1, yi1 = yi0 + 1;
                auto in = [&](int xx, int yy) { return xx >= 0 && xx < pw && yy >= 0 && yy < ph; };
                for (int ch = 0; ch < c; ch++) {
                    const float* src = prev + ((size_t)b * c + ch) * ph * pw;
                    float v = 0.0f;
                    if (in(xi0, yi0)) v += src[(size_t)yi0 * pw + xi0] * nw;
                    if (in(xi1, yi0)) v += src[(size_t)yi0 * pw + xi1] * ne;
                    if (in(xi0, yi1)) v += src[(size_t)yi1 * pw + xi0] * sw;
                    if (in(xi1, yi1)) v += src[(size_t)yi1 * pw + xi1] * se;
                    out[((size_t)b * c + ch) * plane + (size_t)y * w + x] = v;
                }
            }
}

void oracle_nanovdb_query(const uint8_t* buf, int n, const int32_t* ijk, float* value, uint32_t* dim,
                          uint8_t* active) {
    Nano g;
    g.init(buf, false);
    for (int i = 0; i < n; i++) {
        int x = ijk[3 * i], y = ijk[3 * i + 1], z = ijk[3 * i + 2];
        value[i] = g.value(x, y, z);
        dim[i] = (uint32_t)g.dim(x, y, z);
        active[i] = g.active(x, y, z) ? 1 : 0;
    }
}

int oracle_nanovdb_hdda_walk(const uint8_t* buf, const float world_origin[3], const float world_dir[3],
                             int lowest_level, int max_visits, int32_t* out_voxel, int32_t* out_dim,
                             uint8_t* out_active, int32_t* out_level, float* out_box, float* out_t) {
    Nano g;
    g.init(buf, false);
    V3 origin = g.world_to_index(v3(world_origin[0], world_origin[1], world_origin[2]));
    V3 dir = g.world_to_index_dir(v3(world_dir[0], world_dir[1], world_dir[2]));
    float scale = 1.0f / length(dir);
    dir = mul(dir, scale);
    float tmin = 0.0f, tmax = 1e10f;
    V3 rlo = v3((float)g.rmin[0], (float)g.rmin[1], (float)g.rmin[2]);
    V3 rhi = v3((float)(g.rmax[0] + 1), (float)(g.rmax[1] + 1), (float)(g.rmax[2] + 1));
    if (!(hdda_clip(rlo, rhi, origin, tmin, dir, tmax) && tmax < 1e20f)) return -1;
    HddaState h;
    hdda_start(h, origin, tmin - 1e-4f, dir, tmax + 1e-4f, lowest_level);
    int visits = 0;
    for (int iteration = 0; visits < max_visits; iteration++) {
        if (iteration > 0) {
            if (!hdda_advance(h)) break;
            hdda_set_dim(h, origin, dir, std::max(g.dim(h.voxel[0], h.voxel[1], h.voxel[2]), lowest_level));
        }
        bool active = false;
        int level = -1;
        V3 nmin = v3(0, 0, 0), nmax = v3(0, 0, 0);
        if (lowest_level == 8) {
            level = g.cell(h.voxel[0], h.voxel[1], h.voxel[2], active, nmin, nmax);
        } else {
            active = g.active(h.voxel[0], h.voxel[1], h.voxel[2]);
            nmin = v3((float)h.voxel[0], (float)h.voxel[1], (float)h.voxel[2]);
            nmax = v3((float)(h.voxel[0] + 1), (float)(h.voxel[1] + 1), (float)(h.voxel[2] + 1));
        }
        for (int a = 0; a < 3; a++) out_voxel[3 * visits + a] = h.voxel[a];
        out_dim[visits] = h.dim;
        out_active[visits] = active ? 1 : 0;
        out_level[visits] = level;
        float tn0 = 0.0f, tn1 = 1e10f;
        float* bx = out_box + 6 * visits;
        if (active) {
            bx[0] = nmin.x; bx[1] = nmin.y; bx[2] = nmin.z;
            bx[3] = nmax.x; bx[4] = nmax.y; bx[5] = nmax.z;
            hdda_clip(nmin, nmax, origin, tn0, dir, tn1);
        } else {
            for (int k = 0; k < 6; k++) bx[k] = 0.0f;
        }
        out_t[3 * visits] = h.tmin;
        out_t[3 * visits + 1] = pmin(pmin(h.next[0], h.next[1]), h.next[2]);
        out_t[3 * visits + 2] = tn0;
        visits++;
    }
    return visits;
}

void oracle_rng_stream(uint32_t seed, int n, float* out, uint32_t* st4) {
    Rng r = rng_init(seed);
    for (int i = 0; i < n; i++) out[i] = rnd(r);
    if (st4) {
        st4[0] = r.x;
        st4[1] = r.y;
        st4[2] = r.z;
        st4[3] = r.w;
    }
}

}  // extern "C"
