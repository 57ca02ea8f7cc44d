// Blender Perlin / fractal noise as the reference carries it in
// raymond/device/utils/noise.hpp (lookup3 hash :57-103, Perlin 1-4D :170-352,
// fractal :416-441).
#pragma once
#include "rt_math.cuh"

namespace rmd {
namespace noise {

RMD_HD uint32_t rot(uint32_t x, int k) { return __funnelshift_l(x, x, k); }

RMD_HD void final3(uint32_t &a, uint32_t &b, uint32_t &c) {
    c ^= b; c -= rot(b, 14);
    a ^= c; a -= rot(c, 11);
    b ^= a; b -= rot(a, 25);
    c ^= b; c -= rot(b, 16);
    a ^= c; a -= rot(c, 4);
    b ^= a; b -= rot(a, 14);
    c ^= b; c -= rot(b, 24);
}
RMD_HD void mix3(uint32_t &a, uint32_t &b, uint32_t &c) {
    a -= c; a ^= rot(c, 4);  c += b;
    b -= a; b ^= rot(a, 6);  a += c;
    c -= b; c ^= rot(b, 8);  b += a;
    a -= c; a ^= rot(c, 16); c += b;
    b -= a; b ^= rot(a, 19); a += c;
    c -= b; c ^= rot(b, 4);  b += a;
}
RMD_HD uint32_t hash_uint(uint32_t kx) {
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + (1u << 2) + 13u;
    a += kx;
    final3(a, b, c);
    return c;
}
RMD_HD uint32_t hash_uint2(uint32_t kx, uint32_t ky) {
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + (2u << 2) + 13u;
    b += ky;
    a += kx;
    final3(a, b, c);
    return c;
}
RMD_HD uint32_t hash_uint3(uint32_t kx, uint32_t ky, uint32_t kz) {
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + (3u << 2) + 13u;
    c += kz;
    b += ky;
    a += kx;
    final3(a, b, c);
    return c;
}
RMD_HD uint32_t hash_uint4(uint32_t kx, uint32_t ky, uint32_t kz, uint32_t kw) {
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + (4u << 2) + 13u;
    a += kx;
    b += ky;
    c += kz;
    mix3(a, b, c);
    a += kw;
    final3(a, b, c);
    return c;
}
RMD_HD float hash_uint_to_float(uint32_t kx) { return (float)hash_uint(kx) / 4294967296.0f; }
RMD_HD float hash_uint2_to_float(uint32_t kx, uint32_t ky) { return (float)hash_uint2(kx, ky) / 4294967296.0f; }
RMD_HD float hash_float_to_float(float k) { return hash_uint_to_float(__float_as_uint(k)); }
RMD_HD float hash_float2_to_float(float2 k) { return hash_uint2_to_float(__float_as_uint(k.x), __float_as_uint(k.y)); }

RMD_HD int quick_floor_to_int(float x) { return (int)x - ((x < 0.0f) ? 1 : 0); }
RMD_HD float floorfrac(float x, int *i) {
    *i = quick_floor_to_int(x);
    return x - (float)*i;
}
RMD_HD float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
RMD_HD float negate_if(float val, int condition) { return condition ? -val : val; }
RMD_HD float grad1(int hash, float x) {
    int h = hash & 15;
    float g = (float)(1 + (h & 7));
    return negate_if(g, h & 8) * x;
}
RMD_HD float grad2(int hash, float x, float y) {
    int h = hash & 7;
    float u = h < 4 ? x : y;
    float v = 2.0f * (h < 4 ? y : x);
    return negate_if(u, h & 1) + negate_if(v, h & 2);
}
RMD_HD float grad3(int hash, float x, float y, float z) {
    int h = hash & 15;
    float u = h < 8 ? x : y;
    float vt = ((h == 12) || (h == 14)) ? x : z;
    float v = h < 4 ? y : vt;
    return negate_if(u, h & 1) + negate_if(v, h & 2);
}
RMD_HD float grad4(int hash, float x, float y, float z, float w) {
    int h = hash & 31;
    float u = h < 24 ? x : y;
    float v = h < 16 ? y : z;
    float s = h < 8 ? z : w;
    return negate_if(u, h & 1) + negate_if(v, h & 2) + negate_if(s, h & 4);
}
RMD_HD float bi_mix(float v0, float v1, float v2, float v3, float x, float y) {
    float x1 = 1.0f - x;
    return (1.0f - y) * (v0 * x1 + v1 * x) + y * (v2 * x1 + v3 * x);
}
RMD_HD float tri_mix(float v0, float v1, float v2, float v3, float v4, float v5, float v6, float v7, float x, float y,
                     float z) {
    float x1 = 1.0f - x;
    float y1 = 1.0f - y;
    float z1 = 1.0f - z;
    return z1 * (y1 * (v0 * x1 + v1 * x) + y * (v2 * x1 + v3 * x)) + z * (y1 * (v4 * x1 + v5 * x) + y * (v6 * x1 + v7 * x));
}
RMD_HD float perlin_1d(float x) {
    int X;
    float fx = floorfrac(x, &X);
    float u = fade(fx);
    return mixf(grad1((int)hash_uint((uint32_t)X), fx), grad1((int)hash_uint((uint32_t)(X + 1)), fx - 1.0f), u);
}
RMD_HD float perlin_2d(float x, float y) {
    int X, Y;
    float fx = floorfrac(x, &X);
    float fy = floorfrac(y, &Y);
    float u = fade(fx), v = fade(fy);
    return bi_mix(grad2((int)hash_uint2(X, Y), fx, fy), grad2((int)hash_uint2(X + 1, Y), fx - 1.0f, fy),
                  grad2((int)hash_uint2(X, Y + 1), fx, fy - 1.0f),
                  grad2((int)hash_uint2(X + 1, Y + 1), fx - 1.0f, fy - 1.0f), u, v);
}
RMD_HD float perlin_3d(float x, float y, float z) {
    int X, Y, Z;
    float fx = floorfrac(x, &X);
    float fy = floorfrac(y, &Y);
    float fz = floorfrac(z, &Z);
    float u = fade(fx), v = fade(fy), w = fade(fz);
    return tri_mix(grad3((int)hash_uint3(X, Y, Z), fx, fy, fz),
                   grad3((int)hash_uint3(X + 1, Y, Z), fx - 1.0f, fy, fz),
                   grad3((int)hash_uint3(X, Y + 1, Z), fx, fy - 1.0f, fz),
                   grad3((int)hash_uint3(X + 1, Y + 1, Z), fx - 1.0f, fy - 1.0f, fz),
                   grad3((int)hash_uint3(X, Y, Z + 1), fx, fy, fz - 1.0f),
                   grad3((int)hash_uint3(X + 1, Y, Z + 1), fx - 1.0f, fy, fz - 1.0f),
                   grad3((int)hash_uint3(X, Y + 1, Z + 1), fx, fy - 1.0f, fz - 1.0f),
                   grad3((int)hash_uint3(X + 1, Y + 1, Z + 1), fx - 1.0f, fy - 1.0f, fz - 1.0f), u, v, w);
}
RMD_HD float perlin_4d(float x, float y, float z, float w) {
    int X, Y, Z, W;
    float fx = floorfrac(x, &X);
    float fy = floorfrac(y, &Y);
    float fz = floorfrac(z, &Z);
    float fw = floorfrac(w, &W);
    float u = fade(fx), v = fade(fy), t = fade(fz), s = fade(fw);
    float g[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1, dw = (i >> 3) & 1;
        g[i] = grad4((int)hash_uint4(X + dx, Y + dy, Z + dz, W + dw), fx - (float)dx, fy - (float)dy, fz - (float)dz,
                     fw - (float)dw);
    }
    return mixf(tri_mix(g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], u, v, t),
                tri_mix(g[8], g[9], g[10], g[11], g[12], g[13], g[14], g[15], u, v, t), s);
}
// noise.hpp:356-364
RMD_HD bool isfinite_safe(float f) {
    uint32_t x = __float_as_uint(f);
    return (f == f) && (x == 0 || x == (1u << 31) || (f != 2.0f * f)) && !((x << 1) > 0xff000000u);
}
RMD_HD float ensure_finite(float v) { return isfinite_safe(v) ? v : 0.0f; }
RMD_HD float snoise(float p) { return 0.2500f * ensure_finite(perlin_1d(p)); }
RMD_HD float snoise(float2 p) { return 0.6616f * ensure_finite(perlin_2d(p.x, p.y)); }
RMD_HD float snoise(float3 p) { return 0.9820f * ensure_finite(perlin_3d(p.x, p.y, p.z)); }
RMD_HD float snoise(float4 p) { return 0.8344f * ensure_finite(perlin_4d(p.x, p.y, p.z, p.w)); }
template <typename T>
RMD_HD float noise(T p) { return 0.5f * snoise(p) + 0.5f; }

// noise.hpp:416-441
template <typename T>
RMD_HD float fractal_noise(T p, float octaves, float roughness) {
    float fscale = 1.0f;
    float amp = 1.0f;
    float maxamp = 0.0f;
    float sum = 0.0f;
    octaves = clampf(octaves, 0.0f, 15.0f);
    int n = (int)octaves;
    for (int i = 0; i <= n; i++) {
        float t = noise(fscale * p);
        sum += t * amp;
        maxamp += amp;
        amp *= clampf(roughness, 0.0f, 1.0f);
        fscale *= 2.0f;
    }
    float rmd_ = octaves - floorf(octaves);
    if (rmd_ != 0.0f) {
        float t = noise(fscale * p);
        float sum2 = sum + t * amp;
        sum /= maxamp;
        sum2 /= maxamp + amp;
        return (1.0f - rmd_) * sum + rmd_ * sum2;
    }
    return sum / maxamp;
}

}  // namespace noise
}  // namespace rmd
