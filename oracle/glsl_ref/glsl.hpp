// Minimal GLSL-compute environment in C++ so the reference's own compute
// shaders (fluxfx/shaders/*.glsl) can be compiled and run on the CPU as a
// checker. TEST INFRASTRUCTURE ONLY: nothing in the product links this.
//
// Semantics follow the GLSL 4.x specification for the subset the hot-path
// shaders use: float/int vectors with component-wise arithmetic, swizzles .xy
// and .r/.a, texelFetch/textureSize on 3D samplers, imageStore,
// mix(x, y, a) = x*(1-a) + y*a, clamp = min(max(x, lo), hi), truncating
// float->int conversion. Compile with -fsingle-precision-constant so decimal
// literals are float as in GLSL, and -ffp-contract=off so a*b+c is not fused.
#pragma once
#include <cmath>
#include <cstdint>

namespace glsl {

// Plain aggregate: it also lives inside vec3's union as the .xy swizzle.
struct vec2 {
    float x, y;
};

struct ivec3;
struct vec4;

struct vec3 {
    union {
        struct { float x, y, z; };
        struct { vec2 xy; float z_; };
        float v[3];
    };
    vec3() = default;
    constexpr vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit constexpr vec3(float a) : x(a), y(a), z(a) {}
    inline explicit vec3(const ivec3& i);
    float& operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
};

struct ivec3 {
    union {
        struct { int x, y, z; };
        int v[3];
    };
    ivec3() = default;
    constexpr ivec3(int a, int b, int c) : x(a), y(b), z(c) {}
    explicit constexpr ivec3(int a) : x(a), y(a), z(a) {}
    explicit ivec3(const vec3& f) : x((int)f.x), y((int)f.y), z((int)f.z) {}
    int& operator[](int i) { return v[i]; }
    int operator[](int i) const { return v[i]; }
};
inline vec3::vec3(const ivec3& i) : x((float)i.x), y((float)i.y), z((float)i.z) {}

struct vec4 {
    union {
        struct { float x, y, z, w; };
        struct { float r, g, b, a; };
        float v[4];
    };
    vec4() = default;
    constexpr vec4(float a0, float a1, float a2, float a3) : x(a0), y(a1), z(a2), w(a3) {}
    explicit constexpr vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(const vec3& p, float s) : x(p.x), y(p.y), z(p.z), w(s) {}
    float& operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
    vec3 xyz() const { return vec3(x, y, z); }   // the build recipe rewrites `.xyz` reads to `.xyz()`
};

struct bvec3 { bool x, y, z; };

// ---- arithmetic ------------------------------------------------------------
#define GLSL_V3_OP(OP)                                                                                    \
    inline vec3 operator OP(const vec3& a, const vec3& b) { return vec3(a.x OP b.x, a.y OP b.y, a.z OP b.z); } \
    inline vec3 operator OP(const vec3& a, float s) { return vec3(a.x OP s, a.y OP s, a.z OP s); }          \
    inline vec3 operator OP(float s, const vec3& a) { return vec3(s OP a.x, s OP a.y, s OP a.z); }          \
    inline ivec3 operator OP(const ivec3& a, const ivec3& b) { return ivec3(a.x OP b.x, a.y OP b.y, a.z OP b.z); } \
    inline ivec3 operator OP(const ivec3& a, int s) { return ivec3(a.x OP s, a.y OP s, a.z OP s); }       \
    inline ivec3 operator OP(int s, const ivec3& a) { return ivec3(s OP a.x, s OP a.y, s OP a.z); }
GLSL_V3_OP(+)
GLSL_V3_OP(-)
GLSL_V3_OP(*)
GLSL_V3_OP(/)
#undef GLSL_V3_OP
inline vec2 operator-(const vec2& a, const vec2& b) { return vec2{a.x - b.x, a.y - b.y}; }
inline vec2 operator*(float s, const vec2& a) { return vec2{s * a.x, s * a.y}; }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec3& operator+=(vec3& a, const vec3& b) { a = a + b; return a; }
inline ivec3& operator+=(ivec3& a, const ivec3& b) { a = a + b; return a; }

// ---- scalar built-ins (float overloads keep single precision) --------------
inline float exp(float x) { return std::exp(x); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float floor(float x) { return std::floor(x); }
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float min(float a, float b) { return b < a ? b : a; }
inline float max(float a, float b) { return a < b ? b : a; }
inline int min(int a, int b) { return b < a ? b : a; }
inline int max(int a, int b) { return a < b ? b : a; }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline int clamp(int x, int lo, int hi) { return min(max(x, lo), hi); }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline float fract(float x) { return x - std::floor(x); }
inline float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline bool isnan(float x) { return std::isnan(x); }
inline bool isinf(float x) { return std::isinf(x); }

// ---- vector built-ins -------------------------------------------------------
inline vec3 floor(const vec3& a) { return vec3(floor(a.x), floor(a.y), floor(a.z)); }
inline vec3 fract(const vec3& a) { return vec3(fract(a.x), fract(a.y), fract(a.z)); }
inline vec3 abs(const vec3& a) { return vec3(abs(a.x), abs(a.y), abs(a.z)); }
inline vec3 sign(const vec3& a) { return vec3(sign(a.x), sign(a.y), sign(a.z)); }
inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline ivec3 min(const ivec3& a, const ivec3& b) { return ivec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline ivec3 max(const ivec3& a, const ivec3& b) { return ivec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 clamp(const vec3& x, const vec3& lo, const vec3& hi) { return min(max(x, lo), hi); }
inline vec3 clamp(const vec3& x, float lo, float hi) { return clamp(x, vec3(lo), vec3(hi)); }
inline ivec3 clamp(const ivec3& x, const ivec3& lo, const ivec3& hi) { return min(max(x, lo), hi); }
inline vec3 mix(const vec3& x, const vec3& y, const vec3& a) {
    return vec3(mix(x.x, y.x, a.x), mix(x.y, y.y, a.y), mix(x.z, y.z, a.z));
}
inline vec3 mix(const vec3& x, const vec3& y, float a) { return mix(x, y, vec3(a)); }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(const vec4& a, const vec4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float length(const vec3& a) { return sqrt(dot(a, a)); }
inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float distance(const vec3& a, const vec3& b) { return length(a - b); }

inline bvec3 lessThan(const vec3& a, const vec3& b) { return {a.x < b.x, a.y < b.y, a.z < b.z}; }
inline bvec3 greaterThan(const vec3& a, const vec3& b) { return {a.x > b.x, a.y > b.y, a.z > b.z}; }
inline bvec3 lessThanEqual(const vec3& a, const vec3& b) { return {a.x <= b.x, a.y <= b.y, a.z <= b.z}; }
inline bvec3 lessThan(const ivec3& a, const ivec3& b) { return {a.x < b.x, a.y < b.y, a.z < b.z}; }
inline bvec3 greaterThanEqual(const ivec3& a, const ivec3& b) { return {a.x >= b.x, a.y >= b.y, a.z >= b.z}; }
inline bool any(const bvec3& b) { return b.x || b.y || b.z; }
inline bool all(const bvec3& b) { return b.x && b.y && b.z; }

// ---- resources -------------------------------------------------------------
struct sampler3D {
    const float* data = nullptr;
    int sx = 0, sy = 0, sz = 0, channels = 1;
};
struct image3D {
    float* data = nullptr;
    int sx = 0, sy = 0, sz = 0, channels = 1;
};

extern thread_local long long g_out_of_range;

inline ivec3 textureSize(const sampler3D& s, int) { return ivec3(s.sx, s.sy, s.sz); }
inline vec4 texelFetch(const sampler3D& s, const ivec3& p, int) {
    if (!s.data || p.x < 0 || p.y < 0 || p.z < 0 || p.x >= s.sx || p.y >= s.sy || p.z >= s.sz) {
        ++g_out_of_range;
        return vec4(0.0f);
    }
    const float* t = s.data + (size_t)s.channels * ((size_t)p.x + (size_t)s.sx * ((size_t)p.y + (size_t)s.sy * p.z));
    if (s.channels == 4) return vec4(t[0], t[1], t[2], t[3]);
    return vec4(t[0], 0.0f, 0.0f, 1.0f);
}
inline void imageStore(image3D& img, const ivec3& p, const vec4& v) {
    if (p.x < 0 || p.y < 0 || p.z < 0 || p.x >= img.sx || p.y >= img.sy || p.z >= img.sz) {
        ++g_out_of_range;
        return;
    }
    float* t = img.data + (size_t)img.channels * ((size_t)p.x + (size_t)img.sx * ((size_t)p.y + (size_t)img.sy * p.z));
    for (int c = 0; c < img.channels; ++c) t[c] = v.v[c];
}

struct InvocationID {
    ivec3 xyz;
};
extern thread_local InvocationID gl_GlobalInvocationID;

}  // namespace glsl
