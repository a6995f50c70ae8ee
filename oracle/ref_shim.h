// ref_shim.h - GLSL-to-C++ shim for compiling the reference's tracer shaders on the CPU
// (TEST INFRASTRUCTURE ONLY).  Provides the GLSL types, built-ins, samplers and images the shaders
// use, so that oracle/ref_build.py can compile Data/Shaders/VPT/*.glsl from the reference tree
// unmodified (apart from a mechanical rewrite of parameter qualifiers and float literals).
//
// Texture semantics follow the Vulkan specification: NEAREST picks texel floor(u * size),
// LINEAR blends the four/eight texels around u * size - 0.5 in fp32; CLAMP_TO_BORDER returns 0,
// REPEAT wraps.  Arithmetic is fp32 like the shaders (literals are rewritten to float).
#pragma once
#include <stdint.h>
#include <math.h>
#include <vector>

namespace glslref {

typedef uint32_t uint;

struct vec2;
struct vec3;
struct vec4;
struct ivec2;
struct ivec3;
struct uvec2;
struct uvec3;
struct uvec4;

template <int A, int B>
struct Sw2 {
    float v[4];
    operator vec2() const;
    Sw2& operator=(const vec2& o);
};
template <int A, int B, int C>
struct Sw3 {
    float v[4];
    operator vec3() const;
    Sw3& operator=(const vec3& o);
    Sw3& operator/=(float s);
};

struct vec2 {
    union {
        struct { float x, y; };
        struct { float r, g; };
    };
    vec2() : x(0), y(0) {}
    explicit vec2(float s) : x(s), y(s) {}
    vec2(float a, float b) : x(a), y(b) {}
    vec2(const ivec2& o);
    vec2(const uvec2& o);
    float& operator[](int i) { return (&x)[i]; }
    float operator[](int i) const { return (&x)[i]; }
};

struct vec3 {
    union {
        struct { float x, y, z; };
        struct { float r, g, b; };
        Sw2<0, 1> xy;
        Sw2<0, 1> rg;
    };
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    vec3(const vec2& a, float c) : x(a.x), y(a.y), z(c) {}
    vec3(const ivec3& o);
    vec3(const vec3& o) : x(o.x), y(o.y), z(o.z) {}
    vec3& operator=(const vec3& o) {
        x = o.x;
        y = o.y;
        z = o.z;
        return *this;
    }
    float& operator[](int i) { return (&x)[i]; }
    float operator[](int i) const { return (&x)[i]; }
};

struct vec4 {
    union {
        struct { float x, y, z, w; };
        struct { float r, g, b, a; };
        Sw3<0, 1, 2> xyz;
        Sw3<0, 1, 2> rgb;
        Sw2<0, 1> xy;
        Sw2<0, 1> rg;
    };
    vec4() : x(0), y(0), z(0), w(0) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    vec4(const vec3& v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    vec4(const vec2& v, float c, float d) : x(v.x), y(v.y), z(c), w(d) {}
    vec4(const vec4& o) : x(o.x), y(o.y), z(o.z), w(o.w) {}
    vec4& operator=(const vec4& o) {
        x = o.x;
        y = o.y;
        z = o.z;
        w = o.w;
        return *this;
    }
};

template <int A, int B>
Sw2<A, B>::operator vec2() const { return vec2(v[A], v[B]); }
template <int A, int B>
Sw2<A, B>& Sw2<A, B>::operator=(const vec2& o) {
    v[A] = o.x;
    v[B] = o.y;
    return *this;
}
template <int A, int B, int C>
Sw3<A, B, C>::operator vec3() const { return vec3(v[A], v[B], v[C]); }
template <int A, int B, int C>
Sw3<A, B, C>& Sw3<A, B, C>::operator=(const vec3& o) {
    v[A] = o.x;
    v[B] = o.y;
    v[C] = o.z;
    return *this;
}
template <int A, int B, int C>
Sw3<A, B, C>& Sw3<A, B, C>::operator/=(float s) {
    v[A] /= s;
    v[B] /= s;
    v[C] /= s;
    return *this;
}

struct ivec2 {
    int x, y;
    ivec2() : x(0), y(0) {}
    explicit ivec2(int s) : x(s), y(s) {}
    ivec2(int a, int b) : x(a), y(b) {}
    explicit ivec2(const vec2& v) : x((int)v.x), y((int)v.y) {}
    explicit ivec2(const uvec2& v);
};
struct ivec3 {
    int x, y, z;
    ivec3() : x(0), y(0), z(0) {}
    explicit ivec3(int s) : x(s), y(s), z(s) {}
    ivec3(int a, int b, int c) : x(a), y(b), z(c) {}
    explicit ivec3(const vec3& v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
    explicit ivec3(const uvec3& v);
    int& operator[](int i) { return (&x)[i]; }
};
struct uvec2 {
    uint x, y;
    uvec2() : x(0), y(0) {}
    uvec2(uint a, uint b) : x(a), y(b) {}
};
struct USw2 {
    uint v[3];
    operator uvec2() const { return uvec2(v[0], v[1]); }
};
struct uvec3 {
    union {
        struct { uint x, y, z; };
        USw2 xy;
    };
    uvec3() : x(0), y(0), z(0) {}
    uvec3(uint a, uint b, uint c) : x(a), y(b), z(c) {}
};
struct uvec4 {
    uint x, y, z, w;
    uvec4() : x(0), y(0), z(0), w(0) {}
    explicit uvec4(uint s) : x(s), y(s), z(s), w(s) {}
    uvec4(uint a, uint b, uint c, uint d) : x(a), y(b), z(c), w(d) {}
};
struct bvec3 {
    bool x, y, z;
};

inline vec2::vec2(const ivec2& o) : x((float)o.x), y((float)o.y) {}
inline vec2::vec2(const uvec2& o) : x((float)o.x), y((float)o.y) {}
inline vec3::vec3(const ivec3& o) : x((float)o.x), y((float)o.y), z((float)o.z) {}
inline ivec2::ivec2(const uvec2& v) : x((int)v.x), y((int)v.y) {}
inline ivec3::ivec3(const uvec3& v) : x((int)v.x), y((int)v.y), z((int)v.z) {}

// ---- operators ----
#define SHIM_V2(op)                                                                                   \
    inline vec2 operator op(const vec2& a, const vec2& b) { return vec2(a.x op b.x, a.y op b.y); }   \
    inline vec2 operator op(const vec2& a, float s) { return vec2(a.x op s, a.y op s); }            \
    inline vec2 operator op(float s, const vec2& a) { return vec2(s op a.x, s op a.y); }            \
    inline vec2 operator op(const vec2& a, const ivec2& b) { return a op vec2(b); }                  \
    inline vec2 operator op(const uvec2& a, const vec2& b) { return vec2(a) op b; }
SHIM_V2(+) SHIM_V2(-) SHIM_V2(*) SHIM_V2(/)
#undef SHIM_V2
#define SHIM_V3(op)                                                                                              \
    inline vec3 operator op(const vec3& a, const vec3& b) { return vec3(a.x op b.x, a.y op b.y, a.z op b.z); }  \
    inline vec3 operator op(const vec3& a, float s) { return vec3(a.x op s, a.y op s, a.z op s); }             \
    inline vec3 operator op(float s, const vec3& a) { return vec3(s op a.x, s op a.y, s op a.z); }             \
    inline vec3 operator op(const vec3& a, const ivec3& b) { return a op vec3(b); }                             \
    inline vec3 operator op(const ivec3& a, const vec3& b) { return vec3(a) op b; }
SHIM_V3(+) SHIM_V3(-) SHIM_V3(*) SHIM_V3(/)
#undef SHIM_V3
#define SHIM_V4(op)                                                                                         \
    inline vec4 operator op(const vec4& a, const vec4& b) {                                                \
        return vec4(a.x op b.x, a.y op b.y, a.z op b.z, a.w op b.w);                                       \
    }                                                                                                      \
    inline vec4 operator op(const vec4& a, float s) { return vec4(a.x op s, a.y op s, a.z op s, a.w op s); } \
    inline vec4 operator op(float s, const vec4& a) { return vec4(s op a.x, s op a.y, s op a.z, s op a.w); }
SHIM_V4(+) SHIM_V4(-) SHIM_V4(*) SHIM_V4(/)
#undef SHIM_V4
#define SHIM_I3(op)                                                                                              \
    inline ivec3 operator op(const ivec3& a, const ivec3& b) { return ivec3(a.x op b.x, a.y op b.y, a.z op b.z); } \
    inline ivec3 operator op(const ivec3& a, int s) { return ivec3(a.x op s, a.y op s, a.z op s); }
SHIM_I3(+) SHIM_I3(-) SHIM_I3(*) SHIM_I3(/)
#undef SHIM_I3
inline ivec2 operator+(const ivec2& a, const ivec2& b) { return ivec2(a.x + b.x, a.y + b.y); }
inline ivec2 operator*(const ivec2& a, int s) { return ivec2(a.x * s, a.y * s); }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec2 operator-(const vec2& a) { return vec2(-a.x, -a.y); }
inline vec2 operator+(const USw2& a, const vec2& b) { return vec2(uvec2(a)) + b; }
inline vec3& operator+=(vec3& a, const vec3& b) { return a = a + b; }
inline vec3& operator-=(vec3& a, const vec3& b) { return a = a - b; }
inline vec3& operator*=(vec3& a, const vec3& b) { return a = a * b; }
inline vec3& operator*=(vec3& a, float s) { return a = a * s; }
inline vec3& operator/=(vec3& a, float s) { return a = a / s; }
inline vec3& operator/=(vec3& a, const vec3& b) { return a = a / b; }
inline vec2& operator+=(vec2& a, const vec2& b) { return a = a + b; }
inline vec2& operator*=(vec2& a, const vec2& b) { return a = a * b; }
inline vec2& operator*=(vec2& a, float s) { return a = a * s; }
inline vec2& operator/=(vec2& a, float s) { return a = a / s; }
inline vec4& operator+=(vec4& a, const vec4& b) { return a = a + b; }
inline vec4& operator/=(vec4& a, float s) { return a = a / s; }
inline ivec3& operator+=(ivec3& a, const ivec3& b) { return a = a + b; }
inline ivec2& operator*=(ivec2& a, int s) { return a = a * s; }
inline ivec2& operator+=(ivec2& a, const ivec2& b) { return a = a + b; }
inline bool operator==(const ivec3& a, const ivec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool operator!=(const ivec3& a, const ivec3& b) { return !(a == b); }

// ---- matrices (column-major like GLSL) ----
struct mat3 {
    vec3 c[3];
    mat3() {}
    mat3(const vec3& c0, const vec3& c1, const vec3& c2) {
        c[0] = c0;
        c[1] = c1;
        c[2] = c2;
    }
};
struct mat4 {
    vec4 c[4];
    mat4() {}
};
inline vec3 operator*(const mat3& m, const vec3& v) {
    return vec3(m.c[0].x * v.x + m.c[1].x * v.y + m.c[2].x * v.z, m.c[0].y * v.x + m.c[1].y * v.y + m.c[2].y * v.z,
                m.c[0].z * v.x + m.c[1].z * v.y + m.c[2].z * v.z);
}
inline vec4 operator*(const mat4& m, const vec4& v) {
    vec4 r;
    r.x = ((m.c[0].x * v.x + m.c[1].x * v.y) + m.c[2].x * v.z) + m.c[3].x * v.w;
    r.y = ((m.c[0].y * v.x + m.c[1].y * v.y) + m.c[2].y * v.z) + m.c[3].y * v.w;
    r.z = ((m.c[0].z * v.x + m.c[1].z * v.y) + m.c[2].z * v.z) + m.c[3].z * v.w;
    r.w = ((m.c[0].w * v.x + m.c[1].w * v.y) + m.c[2].w * v.z) + m.c[3].w * v.w;
    return r;
}

// ---- built-in functions ----
inline float abs(float v) { return fabsf(v); }
inline int abs(int v) { return v < 0 ? -v : v; }
inline vec3 abs(const vec3& v) { return vec3(fabsf(v.x), fabsf(v.y), fabsf(v.z)); }
inline vec2 abs(const vec2& v) { return vec2(fabsf(v.x), fabsf(v.y)); }
inline float sign(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }
inline vec2 sign(const vec2& v) { return vec2(sign(v.x), sign(v.y)); }
inline vec3 sign(const vec3& v) { return vec3(sign(v.x), sign(v.y), sign(v.z)); }
inline float floor(float v) { return floorf(v); }
inline vec3 floor(const vec3& v) { return vec3(floorf(v.x), floorf(v.y), floorf(v.z)); }
inline vec3 ceil(const vec3& v) { return vec3(ceilf(v.x), ceilf(v.y), ceilf(v.z)); }
inline float fract(float v) { return v - floorf(v); }
// GLSL mod: x - y * floor(x / y)
inline float mod(float x, float y) { return x - y * floorf(x / y); }
inline float min(float a, float b) { return b < a ? b : a; }
inline float max(float a, float b) { return a < b ? b : a; }
inline int min(int a, int b) { return b < a ? b : a; }
inline int max(int a, int b) { return a < b ? b : a; }
inline uint min(uint a, uint b) { return b < a ? b : a; }
inline float max(int a, float b) { return max((float)a, b); }
inline float max(float a, int b) { return max(a, (float)b); }
inline float min(int a, float b) { return min((float)a, b); }
inline float min(float a, int b) { return min(a, (float)b); }
inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 max(const vec3& a, float b) { return vec3(max(a.x, b), max(a.y, b), max(a.z, b)); }
inline float clamp(float v, float lo, float hi) { return min(max(v, lo), hi); }
inline ivec3 clamp(const ivec3& v, const ivec3& lo, const ivec3& hi) {
    return ivec3(min(max(v.x, lo.x), hi.x), min(max(v.y, lo.y), hi.y), min(max(v.z, lo.z), hi.z));
}
inline float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline vec2 mix(const vec2& a, const vec2& b, float t) { return a * (1.0f - t) + b * t; }
inline vec3 mix(const vec3& a, const vec3& b, float t) { return a * (1.0f - t) + b * t; }
inline vec4 mix(const vec4& a, const vec4& b, float t) { return a * (1.0f - t) + b * t; }
inline vec3 mix(const vec3& a, const vec3& b, const vec3& t) { return a * (vec3(1.0f) - t) + b * t; }
inline vec3 mix(const vec3& a, const vec3& b, const bvec3& s) {
    return vec3(s.x ? b.x : a.x, s.y ? b.y : a.y, s.z ? b.z : a.z);
}
inline float smoothstep(float e0, float e1, float x) {
    float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
inline float exp(float v) { return expf(v); }
inline float log(float v) { return logf(v); }
inline float pow(float a, float b) { return powf(a, b); }
inline vec3 pow(const vec3& a, const vec3& b) { return vec3(powf(a.x, b.x), powf(a.y, b.y), powf(a.z, b.z)); }
inline float sqrt(float v) { return sqrtf(v); }
inline float cos(float v) { return cosf(v); }
inline float sin(float v) { return sinf(v); }
inline float atan(float y, float x) { return atan2f(y, x); }
inline float asin(float v) { return asinf(v); }
inline float dot(const vec3& a, const vec3& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }
inline float dot(const vec4& a, const vec4& b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }
inline float length(const vec3& v) { return sqrtf(dot(v, v)); }
inline float length(const vec2& v) { return sqrtf(dot(v, v)); }
inline float distance(const vec3& a, const vec3& b) { return length(a - b); }
inline vec3 normalize(const vec3& v) {
    float l = length(v);
    return vec3(v.x / l, v.y / l, v.z / l);
}
inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
inline bvec3 lessThanEqual(const vec3& a, const vec3& b) { return bvec3{a.x <= b.x, a.y <= b.y, a.z <= b.z}; }
inline bvec3 greaterThanEqual(const ivec3& a, const ivec3& b) { return bvec3{a.x >= b.x, a.y >= b.y, a.z >= b.z}; }
inline bvec3 lessThan(const ivec3& a, const ivec3& b) { return bvec3{a.x < b.x, a.y < b.y, a.z < b.z}; }
inline bool all(const bvec3& b) { return b.x && b.y && b.z; }
inline bool any(const bvec3& b) { return b.x || b.y || b.z; }

// ---- samplers and images ----
enum Filter { FILTER_NEAREST = 0, FILTER_LINEAR = 1 };
enum Address { ADDRESS_CLAMP_TO_BORDER = 0, ADDRESS_REPEAT = 1, ADDRESS_CLAMP_TO_EDGE = 2 };

struct sampler3D {
    const float* data = nullptr;  // `channels` floats per texel, x fastest
    int w = 0, h = 0, d = 0, channels = 1;
    int filter = FILTER_NEAREST;
    vec4 texel(int x, int y, int z) const {
        if (x < 0 || y < 0 || z < 0 || x >= w || y >= h || z >= d) return vec4(0.0f);  // transparent black
        const float* p = data + (((size_t)z * h + y) * w + x) * channels;
        return vec4(p[0], channels > 1 ? p[1] : 0.0f, channels > 2 ? p[2] : 0.0f, channels > 3 ? p[3] : 1.0f);
    }
};
typedef sampler3D usampler3D;

struct sampler2D {
    std::vector<const float*> levels;  // mip chain, level 0 first
    int w = 0, h = 0, channels = 4;
    int filter = FILTER_LINEAR;
    int address = ADDRESS_REPEAT;
    vec4 texel(int x, int y, int lvl = 0) const {
        int lw = w >> lvl, lh = h >> lvl;
        if (address == ADDRESS_REPEAT) {
            x = ((x % lw) + lw) % lw;
            y = ((y % lh) + lh) % lh;
        } else {
            x = x < 0 ? 0 : (x >= lw ? lw - 1 : x);
            y = y < 0 ? 0 : (y >= lh ? lh - 1 : y);
        }
        const float* p = levels[lvl] + ((size_t)y * lw + x) * channels;
        return vec4(p[0], channels > 1 ? p[1] : 0.0f, channels > 2 ? p[2] : 0.0f, channels > 3 ? p[3] : 1.0f);
    }
};

inline vec4 texture(const sampler3D& s, const vec3& c) {
    float u = c.x * (float)s.w, v = c.y * (float)s.h, q = c.z * (float)s.d;
    if (s.filter == FILTER_NEAREST) return s.texel((int)floorf(u), (int)floorf(v), (int)floorf(q));
    u -= 0.5f;
    v -= 0.5f;
    q -= 0.5f;
    float fu = floorf(u), fv = floorf(v), fq = floorf(q);
    float a = u - fu, b = v - fv, cc = q - fq;
    int x = (int)fu, y = (int)fv, z = (int)fq;
    vec4 r0 = mix(mix(s.texel(x, y, z), s.texel(x + 1, y, z), a), mix(s.texel(x, y + 1, z), s.texel(x + 1, y + 1, z), a), b);
    vec4 r1 = mix(mix(s.texel(x, y, z + 1), s.texel(x + 1, y, z + 1), a),
                  mix(s.texel(x, y + 1, z + 1), s.texel(x + 1, y + 1, z + 1), a), b);
    return mix(r0, r1, cc);
}
// textureOffset: the lookup moved by whole texels
inline vec4 textureOffset(const sampler3D& s, const vec3& c, const ivec3& o) {
    return texture(s, vec3(c.x + float(o.x) / float(s.w), c.y + float(o.y) / float(s.h), c.z + float(o.z) / float(s.d)));
}
inline vec4 texture(const sampler2D& s, const vec2& c) {
    float u = c.x * (float)s.w - 0.5f, v = c.y * (float)s.h - 0.5f;
    float fu = floorf(u), fv = floorf(v);
    float a = u - fu, b = v - fv;
    int x = (int)fu, y = (int)fv;
    return mix(mix(s.texel(x, y), s.texel(x + 1, y), a), mix(s.texel(x, y + 1), s.texel(x + 1, y + 1), a), b);
}
// sampler1DArray (the transfer-function texture): RGBA fp32 rows, one per layer; linear filtering
// along u with clamp to edge; coordinate (u, layer)
struct sampler1DArray {
    const float* data = nullptr;
    int w = 0, layers = 1;
    vec4 texel(int x, int layer) const {
        x = x < 0 ? 0 : (x >= w ? w - 1 : x);
        const float* q = data + ((size_t)layer * w + x) * 4;
        return vec4(q[0], q[1], q[2], q[3]);
    }
};
inline vec4 texture(const sampler1DArray& s, const vec2& c) {
    int layer = (int)floorf(c.y + 0.5f);
    layer = layer < 0 ? 0 : (layer >= s.layers ? s.layers - 1 : layer);
    float u = c.x * (float)s.w - 0.5f;
    float fu = floorf(u);
    float a = u - fu;
    int x = (int)fu;
    return mix(s.texel(x, layer), s.texel(x + 1, layer), a);
}
inline vec4 texelFetch(const sampler3D& s, const ivec3& p, int) { return s.texel(p.x, p.y, p.z); }
inline vec4 texelFetch(const sampler2D& s, const ivec2& p, int lvl) { return s.texel(p.x, p.y, lvl); }
inline ivec3 textureSize(const sampler3D& s, int) { return ivec3(s.w, s.h, s.d); }
inline int textureQueryLevels(const sampler2D& s) { return (int)s.levels.size(); }

struct image2D {
    float* data = nullptr;  // RGBA fp32
    int w = 0, h = 0;
};
inline ivec2 imageSize(const image2D& im) { return ivec2(im.w, im.h); }
inline vec4 imageLoad(const image2D& im, const ivec2& p) {
    const float* q = im.data + ((size_t)p.y * im.w + p.x) * 4;
    return vec4(q[0], q[1], q[2], q[3]);
}
inline void imageStore(image2D& im, const ivec2& p, const vec4& v) {
    float* q = im.data + ((size_t)p.y * im.w + p.x) * 4;
    q[0] = v.x;
    q[1] = v.y;
    q[2] = v.z;
    q[3] = v.w;
}
struct uimage3D {
    const uint8_t* data = nullptr;
    int w = 0, h = 0, d = 0;
};
inline uvec4 imageLoad(const uimage3D& im, const ivec3& p) {
    return uvec4(im.data[((size_t)p.z * im.h + p.y) * im.w + p.x], 0, 0, 1);
}

// ---- the Parameters UBO (Data/Shaders/VPT/VptHeader.glsl:45-112) and FrameInfo (114-119) ----
struct Parameters {
    mat4 inverseViewProjMatrix, previousViewProjMatrix, inverseTransposedViewMatrix, inverseViewMatrix, viewMatrix;
    vec3 boxMin;
    float voxelValueMin;
    vec3 boxMax;
    float voxelValueMax;
    vec3 gridMin;
    float minGradientVal;
    vec3 gridMax;
    float maxGradientVal;
    vec3 emissionBoxMin, emissionBoxMax;
    vec3 extinction;
    float tfScatteringAlbedoStrength;
    vec3 scatteringAlbedo;
    float phaseG;
    vec3 sunDirection, sunIntensity, environmentMapIntensityFactor;
    mat3 envMapDirRot, invEnvMapDirRot;
    float emissionCap, emissionStrength;
    int numFeatureMapSamplesPerFrame;
    int useLinearRGB;
    ivec3 superVoxelSize, superVoxelGridSize, gridResolution;
    uint isEnvMapBlack;
    vec3 voxelTexelSize;
    float farDistance;
    // isosurfaces (VptHeader.glsl:88-93)
    vec3 isoSurfaceColor;
    float isoValue;
    float isoStepWidth;
    float maxAoDist;
    int numAoSamples;
    // clip plane (VptHeader.glsl:95-98)
    int useClipPlane;
    vec3 clipPlaneNormal;
    float clipPlaneDistance;
    // surface BRDF parameters (VptHeader.glsl:100-111)
    float subsurface, metallic, specular, specularTint, roughness, anisotropic, sheen, sheenTint;
    vec3 camForward;
    float clearcoat, clearcoatGloss;
};
struct FrameInfo {
    uint frameCount, globalFrameNumber;
};
// the LightsBuffer UBO (VptHeader.glsl:226-251)
const uint LIGHT_TYPE_POINT = 0u;
const uint LIGHT_TYPE_SPOT = 1u;
const uint LIGHT_TYPE_DIRECTIONAL = 2u;
const uint LIGHT_SPACE_WORLD = 0u;
const uint LIGHT_SPACE_VIEW = 1u;
const uint LIGHT_SPACE_VIEW_ORIENTATION = 2u;
struct Light {
    uint lightType;
    uint lightSpace;
    float spotTotalWidth;
    float spotFalloffStart;
    vec3 color;
    float intensity;
    vec3 position;
    uint useDistance;
    vec3 spotDirection;
    float padding;
};

}  // namespace glslref
