// Oracle (test infrastructure only): small float vector / matrix library with
// the semantics of the Metal Shading Language types the reference device
// library is written in (raymond/device/**).  Matrices are column-major as in
// Metal: m.c[i] is column i, M*v sums columns, v*M dots v with each column.
// Literals are float, because Metal evaluates `0.08 * x` in float.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>

namespace orc {

struct float2 {
    float x = 0, y = 0;
    float2() = default;
    constexpr float2(float a, float b) : x(a), y(b) {}
    explicit constexpr float2(float a) : x(a), y(a) {}
    float &operator[](int i) { return (&x)[i]; }
    float operator[](int i) const { return (&x)[i]; }
};
struct float3 {
    float x = 0, y = 0, z = 0;
    float3() = default;
    constexpr float3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit constexpr float3(float a) : x(a), y(a), z(a) {}
    constexpr float3(float2 v, float c) : x(v.x), y(v.y), z(c) {}
    float &operator[](int i) { return (&x)[i]; }
    float operator[](int i) const { return (&x)[i]; }
    float2 xy() const { return {x, y}; }
    float2 yz() const { return {y, z}; }
};
struct float4 {
    float x = 0, y = 0, z = 0, w = 0;
    float4() = default;
    constexpr float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    explicit constexpr float4(float a) : x(a), y(a), z(a), w(a) {}
    constexpr float4(float3 v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    constexpr float4(float2 v, float c, float d) : x(v.x), y(v.y), z(c), w(d) {}
    float &operator[](int i) { return (&x)[i]; }
    float operator[](int i) const { return (&x)[i]; }
    float3 xyz() const { return {x, y, z}; }
    float2 xy() const { return {x, y}; }
};

#define ORC_V2OP(op)                                                                   \
    inline float2 operator op(float2 a, float2 b) { return {a.x op b.x, a.y op b.y}; } \
    inline float2 operator op(float2 a, float s) { return {a.x op s, a.y op s}; }      \
    inline float2 operator op(float s, float2 a) { return {s op a.x, s op a.y}; }
#define ORC_V3OP(op)                                                                                  \
    inline float3 operator op(float3 a, float3 b) { return {a.x op b.x, a.y op b.y, a.z op b.z}; }   \
    inline float3 operator op(float3 a, float s) { return {a.x op s, a.y op s, a.z op s}; }          \
    inline float3 operator op(float s, float3 a) { return {s op a.x, s op a.y, s op a.z}; }
#define ORC_V4OP(op)                                                                                            \
    inline float4 operator op(float4 a, float4 b) { return {a.x op b.x, a.y op b.y, a.z op b.z, a.w op b.w}; } \
    inline float4 operator op(float4 a, float s) { return {a.x op s, a.y op s, a.z op s, a.w op s}; }          \
    inline float4 operator op(float s, float4 a) { return {s op a.x, s op a.y, s op a.z, s op a.w}; }
ORC_V2OP(+) ORC_V2OP(-) ORC_V2OP(*) ORC_V2OP(/)
ORC_V3OP(+) ORC_V3OP(-) ORC_V3OP(*) ORC_V3OP(/)
ORC_V4OP(+) ORC_V4OP(-) ORC_V4OP(*) ORC_V4OP(/)
#undef ORC_V2OP
#undef ORC_V3OP
#undef ORC_V4OP

inline float3 operator-(float3 a) { return {-a.x, -a.y, -a.z}; }
inline float2 operator-(float2 a) { return {-a.x, -a.y}; }
inline float4 operator-(float4 a) { return {-a.x, -a.y, -a.z, -a.w}; }
inline float3 &operator+=(float3 &a, float3 b) { return a = a + b; }
inline float3 &operator*=(float3 &a, float3 b) { return a = a * b; }
inline float3 &operator*=(float3 &a, float s) { return a = a * s; }
inline float3 &operator/=(float3 &a, float s) { return a = a / s; }
inline float3 &operator/=(float3 &a, float3 b) { return a = a / b; }
inline float2 &operator*=(float2 &a, float s) { return a = a * s; }

inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float3 cross(float3 a, float3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length_squared(float3 v) { return dot(v, v); }
inline float length(float3 v) { return std::sqrt(dot(v, v)); }
inline float length(float2 v) { return std::sqrt(dot(v, v)); }
inline float3 normalize(float3 v) { return v / std::sqrt(dot(v, v)); }

inline float saturate(float v) { return std::min(std::max(v, 0.0f), 1.0f); }
inline float3 saturate(float3 v) { return {saturate(v.x), saturate(v.y), saturate(v.z)}; }
inline float4 saturate(float4 v) { return {saturate(v.x), saturate(v.y), saturate(v.z), saturate(v.w)}; }
inline float clampf(float v, float lo, float hi) { return std::min(std::max(v, lo), hi); }
inline float3 vmin(float3 a, float3 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
inline float3 vmax(float3 a, float3 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
inline float4 vmin(float4 a, float4 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z), std::min(a.w, b.w)}; }
inline float4 vmax(float4 a, float4 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z), std::max(a.w, b.w)}; }
inline float3 vabs(float3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline float3 vfloor(float3 a) { return {std::floor(a.x), std::floor(a.y), std::floor(a.z)}; }
// Metal mix(): x + (y - x) * a
inline float mixf(float x, float y, float a) { return x + (y - x) * a; }
// Metal sign(): +-1, or 0 for zero / NaN
inline float signf(float x) { return x > 0 ? 1.0f : (x < 0 ? -1.0f : 0.0f); }
inline float smoothstep(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
inline float3 reflect(float3 i, float3 n) { return i - 2.0f * dot(n, i) * n; }
inline float3 refract(float3 i, float3 n, float eta) {
    float ndi = dot(n, i);
    float k = 1.0f - eta * eta * (1.0f - ndi * ndi);
    if (k < 0.0f) return float3(0.0f);
    return eta * i - (eta * ndi + std::sqrt(k)) * n;
}
inline bool isfinite3(float3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
inline bool any_nonzero(float3 v) { return v.x != 0 || v.y != 0 || v.z != 0; }
inline bool all_zero(float3 v) { return v.x == 0 && v.y == 0 && v.z == 0; }

constexpr float M_PI_F = 3.14159265358979323846f;
constexpr float M_1_PI_F = 0.318309886183790671538f;
constexpr float INF = INFINITY;

// column-major 3x3 (Metal float3x3)
struct float3x3 {
    float3 c[3];
    float3 &operator[](int i) { return c[i]; }
    const float3 &operator[](int i) const { return c[i]; }
};
inline float3 operator*(const float3x3 &m, float3 v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z; }
inline float3 operator*(float3 v, const float3x3 &m) { return {dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2])}; }
inline float3x3 transpose(const float3x3 &m) {
    float3x3 t;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t.c[i][j] = m.c[j][i];
    return t;
}
// column-major 4x4 (Metal float4x4)
struct float4x4 {
    float4 c[4];
};
inline float4 operator*(const float4x4 &m, float4 v) {
    return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z + m.c[3] * v.w;
}
// Metal float3x4: three float4 columns; `float4 * float3x4` dots with each column.
struct float3x4 {
    float4 c[3];
};
inline float3 operator*(float4 v, const float3x4 &m) { return {dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2])}; }

inline uint32_t float_as_uint(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float uint_as_float(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

}  // namespace orc
