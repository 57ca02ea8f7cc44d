// Vector / matrix helpers with the semantics of the Metal types the
// reference device library is written in: column-major matrices,
// M*v sums columns, v*M dots v with each column; lerp(a, b, v) = (1-v)a + vb
// (raymond/device/utils/math.hpp:29-30), mix(x, y, a) = x + (y - x)a (Metal).
// Compiled by nvcc for the static kernels and by NVRTC for the shading module,
// so it includes no system headers.
#pragma once

#ifndef RMD_HD
#define RMD_HD __device__ __forceinline__
#endif

#ifdef __CUDACC_RTC__
typedef unsigned int uint32_t;
typedef int int32_t;
typedef unsigned short uint16_t;
typedef unsigned char uint8_t;
typedef unsigned long long uint64_t;
typedef long long int64_t;
#else
#include <cstdint>
#endif

namespace rmd {

constexpr float M_PI_F = 3.14159265358979323846f;
constexpr float M_1_PI_F = 0.318309886183790671538f;

RMD_HD float inf_f() { return __int_as_float(0x7f800000); }
RMD_HD bool is_inf(float x) { return (__float_as_uint(x) & 0x7fffffffu) == 0x7f800000u; }
RMD_HD bool is_finite(float x) { return (__float_as_uint(x) & 0x7f800000u) != 0x7f800000u; }

RMD_HD float2 f2(float a, float b) { return make_float2(a, b); }
RMD_HD float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
RMD_HD float3 f3(float a) { return make_float3(a, a, a); }
RMD_HD float3 f3(float2 v, float c) { return make_float3(v.x, v.y, c); }
RMD_HD float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
RMD_HD float4 f4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
RMD_HD float4 f4(float a) { return make_float4(a, a, a, a); }
RMD_HD float4 f4(float3 v, float d) { return make_float4(v.x, v.y, v.z, d); }
RMD_HD float4 f4(float2 v, float c, float d) { return make_float4(v.x, v.y, c, d); }
RMD_HD float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }

#define RMD_V2OP(op)                                                                          \
    RMD_HD float2 operator op(float2 a, float2 b) { return make_float2(a.x op b.x, a.y op b.y); } \
    RMD_HD float2 operator op(float2 a, float s) { return make_float2(a.x op s, a.y op s); }      \
    RMD_HD float2 operator op(float s, float2 a) { return make_float2(s op a.x, s op a.y); }
#define RMD_V3OP(op)                                                                                         \
    RMD_HD float3 operator op(float3 a, float3 b) { return make_float3(a.x op b.x, a.y op b.y, a.z op b.z); } \
    RMD_HD float3 operator op(float3 a, float s) { return make_float3(a.x op s, a.y op s, a.z op s); }        \
    RMD_HD float3 operator op(float s, float3 a) { return make_float3(s op a.x, s op a.y, s op a.z); }
#define RMD_V4OP(op)                                                                                                   \
    RMD_HD float4 operator op(float4 a, float4 b) { return make_float4(a.x op b.x, a.y op b.y, a.z op b.z, a.w op b.w); } \
    RMD_HD float4 operator op(float4 a, float s) { return make_float4(a.x op s, a.y op s, a.z op s, a.w op s); }          \
    RMD_HD float4 operator op(float s, float4 a) { return make_float4(s op a.x, s op a.y, s op a.z, s op a.w); }
RMD_V2OP(+) RMD_V2OP(-) RMD_V2OP(*) RMD_V2OP(/)
RMD_V3OP(+) RMD_V3OP(-) RMD_V3OP(*) RMD_V3OP(/)
RMD_V4OP(+) RMD_V4OP(-) RMD_V4OP(*) RMD_V4OP(/)
#undef RMD_V2OP
#undef RMD_V3OP
#undef RMD_V4OP

RMD_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
RMD_HD float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
RMD_HD float3 &operator+=(float3 &a, float3 b) { return a = a + b; }
RMD_HD float3 &operator*=(float3 &a, float3 b) { return a = a * b; }
RMD_HD float3 &operator*=(float3 &a, float s) { return a = a * s; }
RMD_HD float3 &operator/=(float3 &a, float s) { return a = a / s; }

RMD_HD float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
RMD_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RMD_HD float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
RMD_HD float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
RMD_HD float length_squared(float3 v) { return dot(v, v); }
RMD_HD float length(float3 v) { return sqrtf(dot(v, v)); }
RMD_HD float3 normalize(float3 v) { return v / sqrtf(dot(v, v)); }

RMD_HD float saturate(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }
RMD_HD float3 saturate(float3 v) { return make_float3(saturate(v.x), saturate(v.y), saturate(v.z)); }
RMD_HD float4 saturate(float4 v) { return make_float4(saturate(v.x), saturate(v.y), saturate(v.z), saturate(v.w)); }
RMD_HD float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
RMD_HD float3 vmin(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
RMD_HD float3 vmax(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
RMD_HD float4 vmin(float4 a, float4 b) { return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w)); }
RMD_HD float4 vmax(float4 a, float4 b) { return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w)); }
RMD_HD float mixf(float x, float y, float a) { return x + (y - x) * a; }
RMD_HD float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
RMD_HD float smoothstep(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
RMD_HD float3 reflect(float3 i, float3 n) { return i - 2.0f * dot(n, i) * n; }
RMD_HD float3 refract(float3 i, float3 n, float eta) {
    float ndi = dot(n, i);
    float k = 1.0f - eta * eta * (1.0f - ndi * ndi);
    if (k < 0.0f) return f3(0.0f);
    return eta * i - (eta * ndi + sqrtf(k)) * n;
}
RMD_HD bool isfinite3(float3 v) { return is_finite(v.x) && is_finite(v.y) && is_finite(v.z); }
RMD_HD bool any_nonzero(float3 v) { return v.x != 0.0f || v.y != 0.0f || v.z != 0.0f; }
RMD_HD bool all_zero(float3 v) { return v.x == 0.0f && v.y == 0.0f && v.z == 0.0f; }
RMD_HD float comp(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// math.hpp:16-41
RMD_HD float safe_sqrtf(float f) { return sqrtf(fmaxf(f, 0.0f)); }
RMD_HD float sqr(float f) { return f * f; }
RMD_HD float safe_sqrt(float v) { return v <= 0.0f ? 0.0f : sqrtf(v); }
RMD_HD float lerp(float a, float b, float v) { return (1.0f - v) * a + v * b; }
RMD_HD float3 lerp(float3 a, float3 b, float v) { return (1.0f - v) * a + v * b; }
RMD_HD float4 lerp(float4 a, float4 b, float v) { return (1.0f - v) * a + v * b; }
RMD_HD float square(float v) { return v * v; }
RMD_HD float mean(float3 v) { return (v.x + v.y + v.z) / 3.0f; }

// Metal matrices, column-major
struct float3x3 {
    float3 c[3];
};
RMD_HD float3 operator*(const float3x3 &m, float3 v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z; }
RMD_HD float3 operator*(float3 v, const float3x3 &m) { return make_float3(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2])); }
struct float4x4 {
    float4 c[4];
};
RMD_HD float4 operator*(const float4x4 &m, float4 v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z + m.c[3] * v.w; }
struct float3x4 {  // three float4 columns; float4 * float3x4 dots with each
    float4 c[3];
};
RMD_HD float3 operator*(float4 v, const float3x4 &m) { return make_float3(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2])); }

// math.hpp:4-14 ("Building an Orthonormal Basis, Revisited", Duff et al. 2017)
RMD_HD float3x3 buildOrthonormalBasis(float3 n) {
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    float3x3 frame;
    frame.c[0] = make_float3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    frame.c[1] = make_float3(b, sign + n.y * n.y * a, -n.y);
    frame.c[2] = n;
    return frame;
}
// world -> local of the frame (v * M) and local -> world (v * transpose(M) = M * v)
RMD_HD float3 toLocal(const float3x3 &f, float3 v) { return v * f; }
RMD_HD float3 toWorld(const float3x3 &f, float3 v) { return f * v; }

// math.hpp:73-119 (Cycles ensure_valid_reflection)
RMD_HD float3 ensure_valid_reflection(float3 Ng, float3 I, float3 N) {
    float3 R = 2.0f * dot(N, I) * N - I;
    float threshold = fminf(0.9f * dot(Ng, I), 0.01f);
    if (dot(Ng, R) >= threshold) return N;
    float NdotNg = dot(N, Ng);
    float3 X = normalize(N - NdotNg * Ng);
    float Ix = dot(I, X), Iz = dot(I, Ng);
    float Ix2 = sqr(Ix), Iz2 = sqr(Iz);
    float a = Ix2 + Iz2;
    float b = safe_sqrtf(Ix2 * (a - sqr(threshold)));
    float c = Iz * threshold + a;
    float fac = 0.5f / a;
    float N1_z2 = fac * (b + c), N2_z2 = fac * (-b + c);
    bool valid1 = (N1_z2 > 1e-5f) && (N1_z2 <= (1.0f + 1e-5f));
    bool valid2 = (N2_z2 > 1e-5f) && (N2_z2 <= (1.0f + 1e-5f));
    float2 N_new;
    if (valid1 && valid2) {
        float2 N1 = make_float2(safe_sqrtf(1.0f - N1_z2), safe_sqrtf(N1_z2));
        float2 N2 = make_float2(safe_sqrtf(1.0f - N2_z2), safe_sqrtf(N2_z2));
        float R1 = 2.0f * (N1.x * Ix + N1.y * Iz) * N1.y - Iz;
        float R2 = 2.0f * (N2.x * Ix + N2.y * Iz) * N2.y - Iz;
        valid1 = (R1 >= 1e-5f);
        valid2 = (R2 >= 1e-5f);
        if (valid1 && valid2) N_new = (R1 < R2) ? N1 : N2;
        else N_new = (R1 > R2) ? N1 : N2;
    } else if (valid1 || valid2) {
        float Nz2 = valid1 ? N1_z2 : N2_z2;
        N_new = make_float2(safe_sqrtf(1.0f - Nz2), safe_sqrtf(Nz2));
    } else {
        return Ng;
    }
    return N_new.x * X + N_new.y * Ng;
}

namespace warp {
// warp.hpp:12-59
RMD_HD float3 uniformSquareToSphere(float2 uv) {
    float z = 1.0f - 2.0f * uv.y;
    float r = safe_sqrt(1.0f - z * z);
    float s, c;
    sincosf(2.0f * M_PI_F * uv.x, &s, &c);
    return make_float3(r * c, r * s, z);
}
RMD_HD float2 uniformSphereToSquare(float3 v) {
    float y = (1.0f - v.z) / 2.0f;
    float x = atan2f(v.y, v.x) / (2.0f * M_PI_F);
    return make_float2(x < 0.0f ? x + 1.0f : x, y);
}
RMD_HD float uniformSquareToSpherePdf() { return 1.0f / (4.0f * M_PI_F); }
// warp.hpp:5-10: longitude from atan2(x, y) shifted by a quarter turn, latitude from z
RMD_HD float2 equirectSphereToSquare(float3 v) {
    return make_float2((atan2f(v.x, v.y) + M_PI_F / 2.0f) / (2.0f * M_PI_F), acosf(v.z / length(v)) / M_PI_F);
}
RMD_HD float2 uniformSquareToDisk(float2 uv) {
    float s, c;
    sincosf(2.0f * M_PI_F * uv.x, &s, &c);
    float r = sqrtf(uv.y);
    return make_float2(r * c, r * s);
}
RMD_HD float3 uniformSquareToCosineWeightedHemisphere(float2 rnd) {
    float cosTheta = sqrtf(rnd.x);
    float sinTheta = sqrtf(1.0f - square(cosTheta));
    float s, c;
    sincosf(2.0f * M_PI_F * rnd.y, &s, &c);
    return make_float3(sinTheta * c, sinTheta * s, cosTheta);
}
RMD_HD float2 uniformSquareToTriangleBarycentric(float2 rnd) {
    float x = sqrtf(rnd.x);
    return make_float2(1.0f - x, x * rnd.y);
}
}  // namespace warp

}  // namespace rmd
