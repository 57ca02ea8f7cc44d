// Oracle (test infrastructure only): node structs of raymond/device/nodes/nodes.hpp
// and the JIT rules of raymond/host/scene/MaterialBuilder.swift, interpreted.
#include "nodes.h"

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cstdio>
#include <functional>
#include <map>
#include <set>

#include "noise.h"
#include "sky.h"

namespace orc {

// ------------------------------------------------------------ helpers
static inline float luminance(float3 c) { return dot(float3(0.2126f, 0.7152f, 0.0722f), c); }  // color.hpp:3-6

// color.hpp:9-41
static float3 rgb2hsv(float3 rgb) {
    const float cmax = std::max(rgb.x, std::max(rgb.y, rgb.z));
    const float cmin = std::min(rgb.x, std::min(rgb.y, rgb.z));
    const float cdelta = cmax - cmin;
    float h = 0, s = 0, v = cmax;
    if (cmax != 0) s = cdelta / cmax;
    if (s != 0) {
        const float3 c = (float3(cmax) - rgb) / cdelta;
        if (rgb.x == cmax) h = 0 + c.z - c.y;
        else if (rgb.y == cmax) h = 2 + c.x - c.z;
        else h = 4 + c.y - c.x;
        h /= 6;
        if (h < 0) h += 1;
    }
    return float3(h, s, v);
}
// color.hpp:43-72
static float3 hsv2rgb(float3 hsv) {
    float h = hsv.x;
    const float s = hsv.y, v = hsv.z;
    if (s == 0) return float3(v, v, v);
    if (h == 1) h = 0;
    h *= 6;
    const float i = std::floor(h);
    const float f = h - i;
    const float p = v * (1 - s);
    const float q = v * (1 - (s * f));
    const float t = v * (1 - (s * (1 - f)));
    switch ((int)i) {
        case 0: return float3(v, t, p);
        case 1: return float3(q, v, p);
        case 2: return float3(p, v, t);
        case 3: return float3(p, q, v);
        case 4: return float3(t, p, v);
        default: return float3(v, p, q);
    }
}
static inline float safe_divide(float a, float b, float fb) { return b == 0 ? fb : a / b; }  // math.hpp:130-132

// ------------------------------------------------------------ node structs (nodes.hpp)
struct FieldList {
    std::vector<FieldDesc> v;
    void add(const char *n, Kind k, size_t off) { v.push_back({n, k, off}); }
};
#define FLD(T, name, kind) fl.add(#name, kind, offsetof(T, name))

struct TextureCoordinate {  // nodes.hpp:223-237
    float3 generated, uv, object, normal, reflection;
    void compute(const SceneData &, ShadingContext &sh) {
        uv = sh.uv;
        generated = sh.generated;
        object = sh.object;
        normal = sh.normal;
        reflection = sh.normal;
    }
    static void describe(FieldList &fl) {
        using T = TextureCoordinate;
        FLD(T, generated, K_F3); FLD(T, uv, K_F3); FLD(T, object, K_F3); FLD(T, normal, K_F3); FLD(T, reflection, K_F3);
    }
};
struct UVMapCoordinate {  // nodes.hpp:239-245
    float3 uv;
    void compute(const SceneData &, ShadingContext &sh) { uv = sh.uv; }
    static void describe(FieldList &fl) { using T = UVMapCoordinate; FLD(T, uv, K_F3); }
};
struct NewGeometry {  // nodes.hpp:201-221
    float3 normal, trueNormal, tangent, position, parametric, incoming, randomPerIsland;
    float backfacing;
    void compute(const SceneData &, ShadingContext &sh) {
        normal = sh.normal;
        trueNormal = sh.trueNormal;
        tangent = sh.tu;
        position = sh.position;
        parametric = sh.uv;
        incoming = sh.wo;
        randomPerIsland = float3(0.0f);
        backfacing = dot(sh.wo, sh.normal) < 0 ? 1.0f : 0.0f;
    }
    static void describe(FieldList &fl) {
        using T = NewGeometry;
        FLD(T, normal, K_F3); FLD(T, trueNormal, K_F3); FLD(T, tangent, K_F3); FLD(T, position, K_F3);
        FLD(T, parametric, K_F3); FLD(T, incoming, K_F3); FLD(T, randomPerIsland, K_F3); FLD(T, backfacing, K_F1);
    }
};
struct LightPath {  // nodes.hpp:15-43 (bools exposed as 0/1 floats)
    float isCameraRay, isReflectionRay, isTransmissionRay, isShadowRay, isDiffuseRay, isGlossyRay, isSingularRay,
        rayLength;
    void compute(const SceneData &, ShadingContext &sh) {
        uint8_t f = sh.rayFlags;
        isCameraRay = (f & RayFlagsCamera) ? 1.f : 0.f;
        isReflectionRay = (f & RayFlagsReflection) ? 1.f : 0.f;
        isTransmissionRay = (f & RayFlagsTransmission) ? 1.f : 0.f;
        isShadowRay = (f & RayFlagsShadow) ? 1.f : 0.f;
        isDiffuseRay = (f & RayFlagsDiffuse) ? 1.f : 0.f;
        isGlossyRay = (f & RayFlagsGlossy) ? 1.f : 0.f;
        isSingularRay = (f & RayFlagsSingular) ? 1.f : 0.f;
        rayLength = sh.distance;
        if (isSingularRay != 0) isGlossyRay = 1.f;
    }
    static void describe(FieldList &fl) {
        using T = LightPath;
        FLD(T, isCameraRay, K_F1); FLD(T, isReflectionRay, K_F1); FLD(T, isTransmissionRay, K_F1);
        FLD(T, isShadowRay, K_F1); FLD(T, isDiffuseRay, K_F1); FLD(T, isGlossyRay, K_F1);
        FLD(T, isSingularRay, K_F1); FLD(T, rayLength, K_F1);
    }
};
struct TexChecker {  // nodes.hpp:247-264
    float scale;
    float4 color1, color2;
    float3 vector;
    float fac;
    float4 color;
    void compute(const SceneData &, ShadingContext &) {
        float3 p = (vector * scale + 0.000001f) * 0.999999f;
        int ix = (int)std::floor(p.x), iy = (int)std::floor(p.y), iz = (int)std::floor(p.z);
        const bool which = ((ix ^ iy ^ iz) & 1) != 0;
        color = which ? color1 : color2;
        fac = which ? 1.f : 0.f;
    }
    static void describe(FieldList &fl) {
        using T = TexChecker;
        FLD(T, scale, K_F1); FLD(T, color1, K_F4); FLD(T, color2, K_F4); FLD(T, vector, K_F3);
        FLD(T, fac, K_F1); FLD(T, color, K_F4);
    }
};
struct TexNoise {  // nodes.hpp:872-1011
    int dimension = 2;  // template parameter kTexNoise::Dimension (0..3 = 1D..4D)
    float detail, distortion, roughness, scale, w;
    float3 vector;
    float fac;
    float4 color;

    static float random_float_offset(float seed) { return 100.0f + noise::hash_float_to_float(seed) * 100.0f; }
    static float off2(float seed, float k) { return 100.0f + noise::hash_float2_to_float(float2(seed, k)) * 100.0f; }

    void noiseTexture1(float p) {
        if (distortion != 0) p += noise::snoise(p + random_float_offset(0)) * distortion;
        color = float4(noise::fractal_noise(p, detail, roughness),
                       noise::fractal_noise(p + random_float_offset(1), detail, roughness),
                       noise::fractal_noise(p + random_float_offset(2), detail, roughness), 1);
        fac = color.x;
    }
    void noiseTexture2(float2 p) {
        if (distortion != 0)
            p = p + distortion * float2(noise::snoise(p + float2(off2(0, 0), off2(0, 1))),
                                        noise::snoise(p + float2(off2(1, 0), off2(1, 1))));
        color = float4(noise::fractal_noise(p, detail, roughness),
                       noise::fractal_noise(p + float2(off2(2, 0), off2(2, 1)), detail, roughness),
                       noise::fractal_noise(p + float2(off2(3, 0), off2(3, 1)), detail, roughness), 1);
        fac = color.x;
    }
    static float3 off3(float s) { return float3(off2(s, 0), off2(s, 1), off2(s, 2)); }
    void noiseTexture3(float3 p) {
        if (distortion != 0)
            p += distortion *
                 float3(noise::snoise(p + off3(0)), noise::snoise(p + off3(1)), noise::snoise(p + off3(2)));
        color = float4(noise::fractal_noise(p, detail, roughness),
                       noise::fractal_noise(p + off3(3), detail, roughness),
                       noise::fractal_noise(p + off3(4), detail, roughness), 1);
        fac = color.x;
    }
    static float4 off4(float s) { return float4(off2(s, 0), off2(s, 1), off2(s, 2), off2(s, 3)); }
    void noiseTexture4(float4 p) {
        if (distortion != 0)
            p = p + distortion * float4(noise::snoise(p + off4(0)), noise::snoise(p + off4(1)),
                                        noise::snoise(p + off4(2)), noise::snoise(p + off4(3)));
        color = float4(noise::fractal_noise(p, detail, roughness),
                       noise::fractal_noise(p + off4(4), detail, roughness),
                       noise::fractal_noise(p + off4(5), detail, roughness), 1);
        fac = color.x;
    }
    void compute(const SceneData &, ShadingContext &) {
        float3 p = this->vector * scale;
        float ww = this->w * scale;
        switch (dimension) {
            case 0: noiseTexture1(ww); break;
            case 1: noiseTexture2(p.xy()); break;
            case 2: noiseTexture3(p); break;
            default: noiseTexture4(float4(p, ww)); break;
        }
    }
    static void describe(FieldList &fl) {
        using T = TexNoise;
        FLD(T, detail, K_F1); FLD(T, distortion, K_F1); FLD(T, roughness, K_F1); FLD(T, scale, K_F1);
        FLD(T, w, K_F1); FLD(T, vector, K_F3); FLD(T, fac, K_F1); FLD(T, color, K_F4);
    }
};
struct ColorRamp {  // nodes.hpp:1013-1046 (linear interpolation only, MaterialBuilder.swift:467-475)
    float fac;
    float4 color;
    int numElements = 0;
    float positions[32];
    float4 colors[32];
    void compute(const SceneData &, ShadingContext &) {
        if (fac < positions[0]) {
            color = colors[0];
            return;
        }
        if (fac > positions[numElements - 1]) {
            color = colors[numElements - 1];
            return;
        }
        for (int i = 1; i < numElements; ++i) {
            if (positions[i] >= fac) {
                float v = (fac - positions[i - 1]) / (positions[i] - positions[i - 1]);
                color = (1 - v) * colors[i - 1] + v * colors[i];
                return;
            }
        }
    }
    static void describe(FieldList &fl) { using T = ColorRamp; FLD(T, fac, K_F1); FLD(T, color, K_F4); }
};
struct ColorMix {  // nodes.hpp:1304-1385
    int blendType = 0;  // kColorMix::BlendType
    bool clampResult = false;
    float4 color1, color2;
    float fac;
    float4 color;
    void compute(const SceneData &, ShadingContext &) {
        switch (blendType) {
            case 0: color = lerp(color1, color2, fac); break;  // MIX
            case 1: color = color1 + fac * color2; break;      // ADD
            case 2: color = color1 * lerp(float4(1.0f), color2, fac); break;  // MULTIPLY
            case 3: color = float4(1.0f) - (float4(1.0f) - fac * color1) * (float4(1.0f) - color1); break;  // SCREEN
            case 4: {  // OVERLAY
                color = color1;
                for (int d = 0; d < 3; d++) {
                    if (color[d] < 0.5f) color[d] *= 1 - fac + 2 * fac * color2[d];
                    else color[d] = 1 - (1 - fac + 2 * fac * (1 - color2[d])) * (1 - color[d]);
                }
                break;
            }
            case 5: color = color1 - fac * color2; break;  // SUB
            case 6: {                                      // COLOR
                color = color1;
                float3 hsv2 = rgb2hsv(color2.xyz());
                if (hsv2.y == 0) {
                    color = color1;
                } else {
                    float3 hsv = rgb2hsv(color1.xyz());
                    hsv.x = hsv2.x;
                    hsv.y = hsv2.y;
                    color = lerp(color1, float4(hsv2rgb(hsv), color2.w), fac);
                }
                break;
            }
            case 7: color = lerp(color1, vmax(color1, color2), fac); break;  // LIGHTEN
            case 8: color = lerp(color1, vmin(color1, color2), fac); break;  // DARKEN
            case 9: {                                                         // VALUE
                float3 hsv = rgb2hsv(color1.xyz());
                hsv.z = rgb2hsv(color2.xyz()).z;
                color = lerp(color1, float4(hsv2rgb(hsv), color2.w), fac);
                break;
            }
        }
        if (clampResult) color = saturate(color);
    }
    static void describe(FieldList &fl) {
        using T = ColorMix;
        FLD(T, color1, K_F4); FLD(T, color2, K_F4); FLD(T, fac, K_F1); FLD(T, color, K_F4);
    }
};
struct Mix {  // nodes.hpp:1933-1974
    bool clampFactor = false, clampResult = false;
    int factorMode = 0;  // UNIFORM / NON_UNIFORM
    float4 a_Color, b_Color, result_Color;
    float a_Float, b_Float, result_Float;
    float3 a_Vector, b_Vector, result_Vector;
    float factor_Float;
    float3 factor_Vector;
    void compute(const SceneData &, ShadingContext &) {
        if (clampFactor) {
            factor_Float = saturate(factor_Float);
            factor_Vector = saturate(factor_Vector);
        }
        if (factorMode == 0) result_Vector = lerp(a_Vector, b_Vector, factor_Float);
        else result_Vector = a_Vector + (b_Vector - a_Vector) * factor_Vector;
        result_Float = lerp(a_Float, b_Float, factor_Float);
        result_Color = lerp(a_Color, b_Color, factor_Float);
        if (clampResult) result_Color = saturate(result_Color);
    }
    static void describe(FieldList &fl) {
        using T = Mix;
        FLD(T, a_Color, K_F4); FLD(T, b_Color, K_F4); FLD(T, result_Color, K_F4);
        FLD(T, a_Float, K_F1); FLD(T, b_Float, K_F1); FLD(T, result_Float, K_F1);
        FLD(T, a_Vector, K_F3); FLD(T, b_Vector, K_F3); FLD(T, result_Vector, K_F3);
        FLD(T, factor_Float, K_F1); FLD(T, factor_Vector, K_F3);
    }
};
struct MathNode {  // nodes.hpp:1128-1193 ("Math")
    int operation = 0;
    bool clamp = false;
    float value, value_001, value_002;
    void compute(const SceneData &, ShadingContext &) {
        switch (operation) {
            case 0: value = value + value_001; break;
            case 1: value = value - value_001; break;
            case 2: value = value * value_001; break;
            case 3: value = safe_divide(value, value_001, 0); break;
            case 4: value = value * value_001 + value_002; break;
            case 5: value = std::pow(value, value_001); break;
            case 6: value = std::min(value, value_001); break;
            case 7: value = std::max(value, value_001); break;
            case 8: value = std::tan(value); break;
            case 9: value = value < value_001 ? 1.f : 0.f; break;
            case 10: value = value > value_001 ? 1.f : 0.f; break;
            case 11: value = std::fmod(value, value_001); break;
        }
        if (clamp) value = saturate(value);
    }
    static void describe(FieldList &fl) {
        using T = MathNode;
        FLD(T, value, K_F1); FLD(T, value_001, K_F1); FLD(T, value_002, K_F1);
    }
};
struct VectorMath {  // nodes.hpp:151-199
    int operation = 0;
    float scale, value;
    float3 vector, vector_001, vector_002;
    void compute(const SceneData &, ShadingContext &) {
        switch (operation) {
            case 0: vector = vector + vector_001; break;
            case 1: vector = vector - vector_001; break;
            case 2: vector = vector * vector_001; break;
            case 3: vector = vector * vector_001 + vector_002; break;
            case 4: vector = normalize(vector); break;
            case 5: vector = vector * scale; break;
            case 6: vector = vmin(vector, vector_001); break;
            case 7: value = length(vector); break;
            case 8: vector = float3(dot(vector, vector_001)); break;
        }
    }
    static void describe(FieldList &fl) {
        using T = VectorMath;
        FLD(T, scale, K_F1); FLD(T, value, K_F1); FLD(T, vector, K_F3); FLD(T, vector_001, K_F3);
        FLD(T, vector_002, K_F3);
    }
};
struct SeparateVector {  // nodes.hpp:266-275
    float3 vector;
    float x, y, z;
    void compute(const SceneData &, ShadingContext &) { x = vector.x; y = vector.y; z = vector.z; }
    static void describe(FieldList &fl) {
        using T = SeparateVector;
        FLD(T, vector, K_F3); FLD(T, x, K_F1); FLD(T, y, K_F1); FLD(T, z, K_F1);
    }
};
struct CombineVector {  // nodes.hpp:277-284
    float x, y, z;
    float3 vector;
    void compute(const SceneData &, ShadingContext &) { vector = float3(x, y, z); }
    static void describe(FieldList &fl) {
        using T = CombineVector;
        FLD(T, x, K_F1); FLD(T, y, K_F1); FLD(T, z, K_F1); FLD(T, vector, K_F3);
    }
};
struct MapRange {  // nodes.hpp:314-344
    bool clamp = false;
    float fromMin, fromMax, toMin, toMax, steps, value, result;
    float3 vector, steps_Float3, from_Min_Float3, from_Max_Float3, to_Min_Float3, to_Max_Float3;
    void compute(const SceneData &, ShadingContext &) {
        float v = (value - fromMin) / (fromMax - fromMin);
        if (clamp) v = saturate(v);
        result = lerp(toMin, toMax, v);
    }
    static void describe(FieldList &fl) {
        using T = MapRange;
        FLD(T, fromMin, K_F1); FLD(T, fromMax, K_F1); FLD(T, toMin, K_F1); FLD(T, toMax, K_F1);
        FLD(T, steps, K_F1); FLD(T, value, K_F1); FLD(T, result, K_F1); FLD(T, vector, K_F3);
        FLD(T, steps_Float3, K_F3); FLD(T, from_Min_Float3, K_F3); FLD(T, from_Max_Float3, K_F3);
        FLD(T, to_Min_Float3, K_F3); FLD(T, to_Max_Float3, K_F3);
    }
};
struct Value {  // nodes.hpp:1716-1719
    float value;
    void compute(const SceneData &, ShadingContext &) {}
    static void describe(FieldList &fl) { using T = Value; FLD(T, value, K_F1); }
};
struct RGB {  // nodes.hpp:1721-1724
    float4 color;
    void compute(const SceneData &, ShadingContext &) {}
    static void describe(FieldList &fl) { using T = RGB; FLD(T, color, K_F4); }
};
struct RGBToBW {  // nodes.hpp:1726-1734
    float4 color;
    float val;
    void compute(const SceneData &, ShadingContext &) { val = luminance(color.xyz()); }
    static void describe(FieldList &fl) { using T = RGBToBW; FLD(T, color, K_F4); FLD(T, val, K_F1); }
};
struct ColorInvert {  // nodes.hpp:1387-1394
    float4 color;
    float fac;
    void compute(const SceneData &, ShadingContext &) {
        float3 c = color.xyz() - fac * (2 * color.xyz() - float3(1.0f));
        color = float4(c, color.w);
    }
    static void describe(FieldList &fl) { using T = ColorInvert; FLD(T, color, K_F4); FLD(T, fac, K_F1); }
};
// Metal's linear sampler with address::repeat over normalized coordinates
// (nodes.hpp:517): texel centres at (i + 1/2) / size, bilinear, wrapped.
static int wrapTexel(float i, int n) {
    const float m = i - std::floor(i / (float)n) * (float)n;
    const int k = (int)m;
    return k < 0 ? 0 : (k >= n ? n - 1 : k);
}
static float4 sampleLinearRepeat(const Texture &t, float2 uv) {
    const float x = uv.x * (float)t.width - 0.5f, y = uv.y * (float)t.height - 0.5f;
    const float x0f = std::floor(x), y0f = std::floor(y);
    const float ax = x - x0f, ay = y - y0f;
    const int x0 = wrapTexel(x0f, t.width), y0 = wrapTexel(y0f, t.height);
    const int x1 = x0 + 1 == t.width ? 0 : x0 + 1, y1 = y0 + 1 == t.height ? 0 : y0 + 1;
    const float4 *r0 = t.texels.data() + (size_t)y0 * t.width, *r1 = t.texels.data() + (size_t)y1 * t.width;
    return lerp(lerp(r0[x0], r0[x1], ax), lerp(r1[x0], r1[x1], ax), ay);
}
struct TexImage {  // nodes.hpp:486-564 (image and environment textures)
    float3 vector;
    float4 color;
    float alpha;
    int slot = 0, projection = 0, colorSpace = 1;  // projection: FLAT, BOX, EQUIRECTANGULAR, MIRROR_BALL
    bool singleChannel = true;
    static float srgbToLinear(float c) {
        if (c < 0.04045f) return c < 0 ? 0.0f : c * (1.0f / 12.92f);
        return std::pow((c + 0.055f) * (1.0f / 1.055f), 2.4f);
    }
    void compute(const SceneData &d, ShadingContext &) {
        float2 p(0, 0);
        if (projection == 0) p = float2(vector.x, 1 - vector.y);
        else if (projection == 2)  // warp.hpp:5-10
            p = float2((std::atan2(vector.x, vector.y) + (float)M_PI / 2) / (2 * (float)M_PI),
                       std::acos(vector.z / length(vector)) / (float)M_PI);
        color = sampleLinearRepeat(d.textures[slot], p);
        alpha = color.w;
        if (singleChannel) color = float4(color.x, color.x, color.x, 1);
        if (colorSpace == 1) {
            color = float4(srgbToLinear(color.x), srgbToLinear(color.y), srgbToLinear(color.z), color.w);
        } else if (colorSpace == 4) {  // color.hpp:74-78
            const float3 c = color.xyz();
            color = float4(3.240479f * c.x + -1.537150f * c.y + -0.498535f * c.z,
                           -0.969256f * c.x + 1.875991f * c.y + 0.041556f * c.z,
                           0.055648f * c.x + -0.204043f * c.y + 1.057311f * c.z, color.w);
        }
    }
    static void describe(FieldList &fl) {
        using T = TexImage;
        FLD(T, vector, K_F3); FLD(T, color, K_F4); FLD(T, alpha, K_F1);
    }
};
struct TexNishita {  // nodes.hpp:774-870 (sky_radiance_nishita, TexNishita)
    float scale = 1;
    float3 vector;
    float4 color;
    float data[10] = {};
    int slot = 0;
    void compute(const SceneData &d, ShadingContext &sh) {
        const float3 dir = sh.wo * float3(1, -1, -1);
        const float elev = data[6], rot = data[7], diameter = data[8], intensity = data[9];
        float3 xyz(0, 0, 0);
        const float theta = std::acos(dir.z), phi = std::atan2(dir.x, dir.y);
        const float pi = (float)M_PI, halfPi = (float)M_PI / 2;
        if (dir.z >= 0.0f) {
            const float3 sun = oracle_sky::direction(elev, rot + halfPi);
            const float angle = 2.f * std::atan2(length(dir - sun), length(dir + sun));
            const float half = diameter / 2.0f;
            const float dirElev = halfPi - theta;
            if (angle < half && diameter > 0) {
                const float3 bottom(data[0], data[1], data[2]), top(data[3], data[4], data[5]);
                if (elev - half > 0.0f) {
                    if (elev + half > 0.0f) {
                        const float y = ((dirElev - elev) / diameter) + 0.5f;
                        xyz = (bottom + (top - bottom) * y) * intensity;
                    }
                } else if (elev + half > 0.0f) {
                    const float y = dirElev / (elev + half);
                    xyz = (bottom + (top - bottom) * y) * intensity;
                }
                const float f = angle / half;
                xyz = xyz * (1.0f - 0.6f * (1.0f - std::sqrt(1.0f - f * f)));
            } else {
                float x = (phi + pi + rot) / (2 * pi);
                const float y = std::sqrt(dirElev / halfPi);
                if (x > 1.0f) x = x - 1.0f;
                xyz = sampleLinearRepeat(d.textures[slot], float2(x, y)).xyz();
            }
        } else if (dir.z >= -0.4f) {
            const float mul = std::pow(1.0f + dir.z * 2.5f, 3.0f);
            float x = (phi + pi + rot) / (2 * pi);
            if (x > 1.0f) x = x - 1.0f;
            xyz = sampleLinearRepeat(d.textures[slot], float2(x, 1e-3f)).xyz() * mul;
        }
        const float3 rgb(3.240479f * xyz.x + -1.537150f * xyz.y + -0.498535f * xyz.z,  // color.hpp:74-78
                         -0.969256f * xyz.x + 1.875991f * xyz.y + 0.041556f * xyz.z,
                         0.055648f * xyz.x + -0.204043f * xyz.y + 1.057311f * xyz.z);
        color = float4(scale * rgb.x, scale * rgb.y, scale * rgb.z, 1);
    }
    static void describe(FieldList &fl) {
        using T = TexNishita;
        FLD(T, vector, K_F3); FLD(T, color, K_F4);
    }
};
struct Mapping {  // nodes.hpp:346-364 with euler2mat of math.hpp:46-68 (one Type: MAPPING)
    float3 scale, rotation, location, vector;
    void compute(const SceneData &, ShadingContext &) {
        const float sx = std::sin(rotation.x), cx = std::cos(rotation.x);
        const float sy = std::sin(rotation.y), cy = std::cos(rotation.y);
        const float sz = std::sin(rotation.z), cz = std::cos(rotation.z);
        float3x3 m;
        m.c[0] = float3(cy * cz, cy * sz, -sy);
        m.c[1] = float3(sy * sx * cz - cx * sz, sy * sx * sz + cx * cz, cy * sx);
        m.c[2] = float3(sy * cx * cz + sx * sz, sy * cx * sz - sx * cz, cy * cx);
        vector = m * (vector * scale) + location;
    }
    static void describe(FieldList &fl) {
        using T = Mapping;
        FLD(T, scale, K_F3); FLD(T, rotation, K_F3); FLD(T, location, K_F3); FLD(T, vector, K_F3);
    }
};
struct NormalMap {  // nodes.hpp:1060-1097
    float4 color;
    float strength;
    float3 normal;
    int space = 0;  // 0 tangent, 1 world
    void compute(const SceneData &, ShadingContext &sh) {
        const float s = std::max(strength, 0.0f);
        float3 n = normalize(2 * color.xyz() - float3(1.0f));
        n = normalize(s * n + (1 - s) * float3(0, 0, 1));
        if (space == 0) {
            float3x3 onb;
            onb.c[0] = sh.tu;
            onb.c[1] = sh.tv;
            onb.c[2] = sh.normal;
            n = onb * n;
        }
        normal = n;
    }
    static void describe(FieldList &fl) {
        using T = NormalMap;
        FLD(T, color, K_F4); FLD(T, strength, K_F1); FLD(T, normal, K_F3);
    }
};
struct HueSaturation {  // nodes.hpp:1261-1277
    float4 color;
    float fac, hue, saturation, value;
    void compute(const SceneData &, ShadingContext &) {
        float3 hsv = rgb2hsv(color.xyz());
        hsv.x = std::fmod(hsv.x + hue + 0.5f, 1.0f);
        hsv.y = saturate(hsv.y * saturation);
        hsv.z *= value;
        float3 r = hsv2rgb(hsv);
        r = float3(std::max(r.x, 0.0f), std::max(r.y, 0.0f), std::max(r.z, 0.0f));
        color = float4(lerp(color.xyz(), r, fac), color.w);
    }
    static void describe(FieldList &fl) {
        using T = HueSaturation;
        FLD(T, color, K_F4); FLD(T, fac, K_F1); FLD(T, hue, K_F1); FLD(T, saturation, K_F1); FLD(T, value, K_F1);
    }
};
struct BrightnessContrast {  // nodes.hpp:1279-1290
    float bright, contrast;
    float4 color;
    void compute(const SceneData &, ShadingContext &) {
        const float a = 1 + contrast, b = bright - contrast / 2;
        for (int d = 0; d < 4; d++) color[d] = std::max(a * color[d] + b, 0.0f);
    }
    static void describe(FieldList &fl) {
        using T = BrightnessContrast;
        FLD(T, bright, K_F1); FLD(T, contrast, K_F1); FLD(T, color, K_F4);
    }
};
// Cycles' blackbody fit (the coefficient table of nodes.hpp:1421-1449)
static const float kBlackbodyR[7][3] = {
    {1.61919106e+03f, -2.05010916e-03f, 5.02995757e+00f}, {2.48845471e+03f, -1.11330907e-03f, 3.22621544e+00f},
    {3.34143193e+03f, -4.86551192e-04f, 1.76486769e+00f}, {4.09461742e+03f, -1.27446582e-04f, 7.25731635e-01f},
    {4.67028036e+03f, 2.91258199e-05f, 1.26703442e-01f},  {4.59509185e+03f, 2.87495649e-05f, 1.50345020e-01f},
    {3.78717450e+03f, 9.35907826e-06f, 3.99075871e-01f}};
static const float kBlackbodyG[7][3] = {
    {-4.88999748e+02f, 6.04330754e-04f, -7.55807526e-02f}, {-7.55994277e+02f, 3.16730098e-04f, 4.78306139e-01f},
    {-1.02363977e+03f, 1.20223470e-04f, 9.36662319e-01f},  {-1.26571316e+03f, 4.87340896e-06f, 1.27054498e+00f},
    {-1.42529332e+03f, -4.01150431e-05f, 1.43972784e+00f}, {-1.17554822e+03f, -2.16378048e-05f, 1.30408023e+00f},
    {-5.00799571e+02f, -4.59832026e-06f, 1.09098763e+00f}};
static const float kBlackbodyB[7][4] = {
    {5.96945309e-11f, -4.85742887e-08f, -9.70622247e-05f, -4.07936148e-03f},
    {2.40430366e-11f, 5.55021075e-08f, -1.98503712e-04f, 2.89312858e-02f},
    {-1.40949732e-11f, 1.89878968e-07f, -3.56632824e-04f, 9.10767778e-02f},
    {-3.61460868e-11f, 2.84822009e-07f, -4.93211319e-04f, 1.56723440e-01f},
    {-1.97075738e-11f, 1.75359352e-07f, -2.50542825e-04f, -2.22783266e-02f},
    {-1.61997957e-13f, -1.64216008e-08f, 3.86216271e-04f, -7.38077418e-01f},
    {6.72650283e-13f, -2.73078809e-08f, 4.24098264e-04f, -7.52335691e-01f}};
struct Blackbody {  // nodes.hpp:1451-1495
    float temperature;
    float4 color;
    void compute(const SceneData &, ShadingContext &) {
        const float t = temperature;
        float3 c;
        if (t >= 12000.0f) {
            c = float3(0.8262954810464208f, 0.9945080501520986f, 1.566307710274283f);
        } else if (t < 800.0f) {
            c = float3(5.413294490189271f, -0.20319390035873933f, -0.0822535242887164f);
        } else {
            const int i = t >= 6365.0f ? 6 : t >= 3315.0f ? 5 : t >= 1902.0f ? 4 : t >= 1449.0f ? 3
                        : t >= 1167.0f ? 2 : t >= 965.0f ? 1 : 0;
            const float *r = kBlackbodyR[i], *g = kBlackbodyG[i], *b = kBlackbodyB[i];
            const float inv = 1.0f / t;
            c = float3(r[0] * inv + r[1] * t + r[2], g[0] * inv + g[1] * t + g[2], ((b[0] * t + b[1]) * t + b[2]) * t + b[3]);
        }
        color = float4(c / luminance(c), 1.0f);
    }
    static void describe(FieldList &fl) { using T = Blackbody; FLD(T, temperature, K_F1); FLD(T, color, K_F4); }
};
struct Gamma {  // nodes.hpp:1292-1302
    float4 color;
    float gamma;
    void compute(const SceneData &, ShadingContext &) {
        if (gamma == 0) {
            color.x = color.y = color.z = 1;
        } else {
            for (int d = 0; d < 3; d++)
                if (color[d] > 0) color[d] = std::pow(color[d], gamma);
        }
    }
    static void describe(FieldList &fl) { using T = Gamma; FLD(T, color, K_F4); FLD(T, gamma, K_F1); }
};
struct Fresnel {  // nodes.hpp:1112-1126
    float ior;
    float3 normal;
    float fac;
    void compute(const SceneData &, ShadingContext &sh) {
        float cosI = dot(sh.wo, normal);
        bool backfacing = cosI < 0;
        float eta = std::max(ior, 1e-5f);
        eta = backfacing ? 1 / eta : eta;
        fac = fresnelDielectricCos(cosI, eta);
    }
    static void describe(FieldList &fl) {
        using T = Fresnel;
        FLD(T, ior, K_F1); FLD(T, normal, K_F3); FLD(T, fac, K_F1);
    }
};
struct LayerWeight {  // nodes.hpp:1689-1714
    float blend;
    float3 normal;
    float fresnel, facing;
    void compute(const SceneData &, ShadingContext &sh) {
        const bool backfacing = dot(sh.wo, normal) < 0;
        const float cosI = dot(sh.wo, normal);
        float eta = std::max(1 - blend, 1e-5f);
        eta = backfacing ? eta : 1 / eta;
        fresnel = fresnelDielectricCos(cosI, eta);
        facing = std::fabs(cosI);
        if (blend != 0.5f) {
            float b = clampf(blend, 0.0f, 1.0f - 1e-5f);
            b = (b < 0.5f) ? 2 * b : 0.5f / (1 - b);
            facing = std::pow(facing, b);
        }
        facing = 1 - facing;
    }
    static void describe(FieldList &fl) {
        using T = LayerWeight;
        FLD(T, blend, K_F1); FLD(T, normal, K_F3); FLD(T, fresnel, K_F1); FLD(T, facing, K_F1);
    }
};
struct Emission {  // nodes.hpp:1396-1407
    float4 color;
    float strength, weight;
    UberShader emission;
    void compute(const SceneData &, ShadingContext &) {
        emission.lobeProbabilities[0] = 1;
        emission.emission = color.xyz() * strength;
    }
    static void describe(FieldList &fl) {
        using T = Emission;
        FLD(T, color, K_F4); FLD(T, strength, K_F1); FLD(T, weight, K_F1); FLD(T, emission, K_SHADER);
    }
};
struct Background {  // nodes.hpp:1409-1419
    float4 color;
    float strength, weight;
    UberShader background;
    void compute(const SceneData &, ShadingContext &) { background.emission = color.xyz() * strength; }
    static void describe(FieldList &fl) {
        using T = Background;
        FLD(T, color, K_F4); FLD(T, strength, K_F1); FLD(T, weight, K_F1); FLD(T, background, K_SHADER);
    }
};
struct BsdfPrincipled {  // nodes.hpp:1581-1687
    float weight;
    float4 emission;
    float sheenTint, emissionStrength, transmission;
    float3 clearcoatNormal;
    float alpha, specularTint;
    float3 tangent;
    float roughness, subsurfaceIor, anisotropic, sheen;
    float3 subsurfaceRadius, normal;
    float subsurfaceAnisotropy;
    float4 baseColor;
    float transmissionRoughness, metallic, specular, clearcoatRoughness;
    float4 subsurfaceColor;
    float subsurface, ior, anisotropicRotation, clearcoat;
    UberShader bsdf;

    void compute(const SceneData &, ShadingContext &) {
        clearcoatRoughness = std::max(clearcoatRoughness, 1e-4f);
        roughness = std::max(roughness, 1e-4f);
        const float diffuseWeight = (1 - saturate(transmission)) * (1 - saturate(metallic));
        const float transmissionWeight = saturate(transmission) * (1 - saturate(metallic));
        const float specularWeight = 1 - transmissionWeight;
        const float lum = luminance(baseColor.xyz());
        const float3 tintColor = lum > 0.f ? baseColor.xyz() * (1 / lum) : float3(1.0f);
        const float3 sheenColor = lerp(float3(1.0f), tintColor, sheenTint);
        const float3 specularColor = lerp(float3(1.0f), tintColor, specularTint);
        const float3 Cspec0 = lerp(specular * 0.08f * specularColor, baseColor.xyz(), metallic);
        const float aspect = std::sqrt(1 - 0.9f * anisotropic);
        const float r2 = square(roughness);

        bsdf.diffuse = Diffuse{diffuseWeight * baseColor.xyz(), diffuseWeight * sheen * sheenColor, roughness, false};
        bsdf.specular = Specular{r2 / aspect, r2 * aspect, Cspec0, (2 / (1 - std::sqrt(0.08f * specular))) - 1,
                                 specularWeight};
        bsdf.transmission = Transmission{r2,
                                         square(1 - (1 - roughness) * (1 - transmissionRoughness)),
                                         baseColor.xyz(),
                                         lerp(float3(1.0f), baseColor.xyz(), specularTint),
                                         ior,
                                         transmissionWeight,
                                         false};
        bsdf.clearcoat = Clearcoat{square(clearcoatRoughness), clearcoat};
        bsdf.lobeProbabilities[0] = diffuseWeight;
        bsdf.lobeProbabilities[1] = specularWeight;
        bsdf.lobeProbabilities[2] = transmissionWeight;
        bsdf.lobeProbabilities[3] = clearcoat * 0.25f;
        float weightsSum = 0;
        for (int i = 0; i < 4; i++) weightsSum += bsdf.lobeProbabilities[i];
        for (int i = 0; i < 4; i++) bsdf.lobeProbabilities[i] /= weightsSum;
        bsdf.alpha = alpha;
        bsdf.normal = normal;
        bsdf.emission = alpha * emission.xyz() * emissionStrength;
    }
    static void describe(FieldList &fl) {
        using T = BsdfPrincipled;
        FLD(T, weight, K_F1); FLD(T, emission, K_F4); FLD(T, sheenTint, K_F1); FLD(T, emissionStrength, K_F1);
        FLD(T, transmission, K_F1); FLD(T, clearcoatNormal, K_F3); FLD(T, alpha, K_F1); FLD(T, specularTint, K_F1);
        FLD(T, tangent, K_F3); FLD(T, roughness, K_F1); FLD(T, subsurfaceIor, K_F1); FLD(T, anisotropic, K_F1);
        FLD(T, sheen, K_F1); FLD(T, subsurfaceRadius, K_F3); FLD(T, normal, K_F3);
        FLD(T, subsurfaceAnisotropy, K_F1); FLD(T, baseColor, K_F4); FLD(T, transmissionRoughness, K_F1);
        FLD(T, metallic, K_F1); FLD(T, specular, K_F1); FLD(T, clearcoatRoughness, K_F1);
        FLD(T, subsurfaceColor, K_F4); FLD(T, subsurface, K_F1); FLD(T, ior, K_F1);
        FLD(T, anisotropicRotation, K_F1); FLD(T, clearcoat, K_F1); FLD(T, bsdf, K_SHADER);
    }
};
struct BsdfDiffuse {  // nodes.hpp:1809-1827
    float4 color;
    float3 normal;
    float roughness, weight;
    UberShader bsdf;
    void compute(const SceneData &, ShadingContext &) {
        bsdf.diffuse = Diffuse{color.xyz(), float3(0.0f), roughness, false};
        bsdf.normal = normal;
        bsdf.lobeProbabilities[0] = 1;
    }
    static void describe(FieldList &fl) {
        using T = BsdfDiffuse;
        FLD(T, color, K_F4); FLD(T, normal, K_F3); FLD(T, roughness, K_F1); FLD(T, weight, K_F1);
        FLD(T, bsdf, K_SHADER);
    }
};
struct BsdfGlossy {  // nodes.hpp:1534-1567
    float4 color;
    float3 normal;
    float roughness, weight;
    UberShader bsdf;
    void compute(const SceneData &, ShadingContext &) {
        const float alpha = square(std::max(roughness, 1e-4f));
        bsdf.specular = Specular{alpha, alpha, color.xyz(), 1.45f, 1};
        bsdf.lobeProbabilities[1] = 1;
        bsdf.normal = normal;
    }
    static void describe(FieldList &fl) {
        using T = BsdfGlossy;
        FLD(T, color, K_F4); FLD(T, normal, K_F3); FLD(T, roughness, K_F1); FLD(T, weight, K_F1);
        FLD(T, bsdf, K_SHADER);
    }
};
struct BsdfGlass {  // nodes.hpp:1497-1532
    float4 color;
    float ior;
    float3 normal;
    float roughness, weight;
    UberShader bsdf;
    void compute(const SceneData &, ShadingContext &) {
        const float alpha = square(std::max(roughness, 1e-4f));
        bsdf.transmission = Transmission{alpha, alpha, color.xyz(), color.xyz(), ior, 1, false};
        bsdf.lobeProbabilities[2] = 1;
        bsdf.normal = normal;
    }
    static void describe(FieldList &fl) {
        using T = BsdfGlass;
        FLD(T, color, K_F4); FLD(T, ior, K_F1); FLD(T, normal, K_F3); FLD(T, roughness, K_F1);
        FLD(T, weight, K_F1); FLD(T, bsdf, K_SHADER);
    }
};
struct BsdfTransparent {  // nodes.hpp:1797-1807
    float4 color;
    float weight;
    UberShader bsdf;
    void compute(const SceneData &, ShadingContext &) {
        bsdf.alpha = 0;
        bsdf.alphaWeight = color.xyz();
    }
    static void describe(FieldList &fl) {
        using T = BsdfTransparent;
        FLD(T, color, K_F4); FLD(T, weight, K_F1); FLD(T, bsdf, K_SHADER);
    }
};
struct AddShader {  // nodes.hpp:1895-1911
    UberShader shader, shader_001;
    void compute(const SceneData &, ShadingContext &sh) {
        const float3 em = shader_001.emission + shader.emission;
        if (sh.rnd.x < 0.5f) {
            sh.rnd.x /= 0.5f;
            shader = shader_001;
        } else {
            sh.rnd.x = 2 * (sh.rnd.x - 0.5f);
        }
        shader.emission = em;
        shader.weight *= 2;
    }
    static void describe(FieldList &fl) {
        using T = AddShader;
        FLD(T, shader, K_SHADER); FLD(T, shader_001, K_SHADER);
    }
};
struct MixShader {  // nodes.hpp:1916-1931
    float fac;
    UberShader shader, shader_001;
    void compute(const SceneData &, ShadingContext &sh) {
        const float3 em = fac * shader_001.emission + (1 - fac) * shader.emission;
        if (sh.rnd.x < fac) {
            sh.rnd.x /= fac;
            shader = shader_001;
        } else {
            sh.rnd.x = (sh.rnd.x - fac) / (1 - fac);
        }
        shader.emission = em;
    }
    static void describe(FieldList &fl) {
        using T = MixShader;
        FLD(T, fac, K_F1); FLD(T, shader, K_SHADER); FLD(T, shader_001, K_SHADER);
    }
};
struct OutputMaterial {  // nodes.hpp:1976-1986
    float3 displacement;
    float thickness;
    UberShader surface, volume;
    void compute(const SceneData &, ShadingContext &sh) { sh.material = surface; }
    static void describe(FieldList &fl) {
        using T = OutputMaterial;
        FLD(T, displacement, K_F3); FLD(T, thickness, K_F1); FLD(T, surface, K_SHADER); FLD(T, volume, K_SHADER);
    }
};
struct OutputWorld {  // nodes.hpp:1988-1995
    float thickness;
    UberShader surface;
    void compute(const SceneData &, ShadingContext &sh) { sh.material = surface; }
    static void describe(FieldList &fl) {
        using T = OutputWorld;
        FLD(T, thickness, K_F1); FLD(T, surface, K_SHADER);
    }
};
struct OutputLight {  // nodes.hpp:1997-2005
    UberShader surface;
    void compute(const SceneData &, ShadingContext &sh) {
        sh.material.alpha = 0;
        sh.material.emission = surface.emission;
    }
    static void describe(FieldList &fl) { using T = OutputLight; FLD(T, surface, K_SHADER); }
};

template <class T>
struct Box final : NodeImpl {
    T v{};
    void compute(const SceneData &ctx, ShadingContext &sh) override { v.compute(ctx, sh); }
    std::unique_ptr<NodeImpl> clone() const override { return std::make_unique<Box<T>>(*this); }
    void copy_from(const NodeImpl &o) override { v = static_cast<const Box<T> &>(o).v; }
    void *base() override { return &v; }
    const std::vector<FieldDesc> &fields() const override {
        static std::vector<FieldDesc> f = [] {
            FieldList fl;
            T::describe(fl);
            return fl.v;
        }();
        return f;
    }
};

// ------------------------------------------------------------ identifiers
std::string makeIdentifier(const std::string &name) {
    size_t a = 0, b = name.size();
    while (a < b && name[a] == ' ') a++;
    while (b > a && name[b - 1] == ' ') b--;
    std::string trimmed = name.substr(a, b - a);
    if (trimmed.empty()) return "";
    // Foundation `capitalized`: first letter of every word upper, the rest lower;
    // words start after any character that is not a letter or digit.
    std::string cap;
    bool wordStart = true;
    for (char c : trimmed) {
        if (std::isalpha((unsigned char)c)) {
            cap += wordStart ? (char)std::toupper((unsigned char)c) : (char)std::tolower((unsigned char)c);
            wordStart = false;
        } else {
            cap += c;
            wordStart = !std::isdigit((unsigned char)c);
        }
    }
    std::string nospace;
    for (char c : cap)
        if (c != ' ') nospace += c;
    std::string out;
    out += (char)std::tolower((unsigned char)trimmed[0]);
    out += nospace.substr(1);
    for (auto &c : out)
        if (!(std::isalnum((unsigned char)c) || c == '_')) c = '_';
    return out;
}

// ------------------------------------------------------------ program build
static const rmd_node_param *findParam(const rmd_node &n, const char *key) {
    for (int i = 0; i < n.num_params; i++)
        if (n.params[i].key && std::string(n.params[i].key) == key) return &n.params[i];
    return nullptr;
}
static std::string paramString(const rmd_node &n, const char *key, const char *fb) {
    auto p = findParam(n, key);
    return (p && p->string_value) ? std::string(p->string_value) : std::string(fb);
}
static bool paramBool(const rmd_node &n, const char *key, bool fb) {
    auto p = findParam(n, key);
    return p ? p->number_value != 0 : fb;
}
static float paramNumber(const rmd_node &n, const char *key, float fb) {
    auto p = findParam(n, key);
    return (p && (p->kind == RMD_PARAM_NUMBER || p->kind == RMD_PARAM_BOOL)) ? (float)p->number_value : fb;
}

SkyParams skyParams(const rmd_node &n) {
    const float deg = (float)M_PI / 180.0f;
    SkyParams p;
    std::string type = paramString(n, "sky_type", "NISHITA");
    p.elevation = paramNumber(n, "sun_elevation", 15.0f * deg);
    p.rotation = paramNumber(n, "sun_rotation", 0.0f);
    p.disc = paramBool(n, "sun_disc", true);
    p.size = paramNumber(n, "sun_size", 0.545f * deg);
    p.intensity = paramNumber(n, "sun_intensity", 1.0f);
    p.altitude = paramNumber(n, "altitude", 0.0f);
    p.air = paramNumber(n, "air_density", 1.0f);
    p.dust = paramNumber(n, "dust_density", 1.0f);
    p.ozone = paramNumber(n, "ozone_density", 1.0f);
    p.scale = 1.0f;
    if (type == "HOSEK_WILKIE") {  // MaterialBuilder.swift:333-348
        float d[3] = {0, 0, 1};
        auto q = findParam(n, "sun_direction");
        if (q && q->num_numbers >= 3)
            for (int i = 0; i < 3; i++) d[i] = q->numbers[i];
        p.rotation = std::atan2(d[0], d[1]);
        p.elevation = std::max(std::asin(d[2]), 5 * deg);
        p.disc = false;
        p.air = 2;
        p.dust = 0.5f;
        p.ozone = 1;
        p.scale = 0.08f;
        type = "NISHITA";
    }
    if (type != "NISHITA") throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "TexSky: unsupported sky type " + type};
    return p;
}

std::string skyTextureKey(const SkyParams &p) {
    char buf[200];
    std::snprintf(buf, sizeof(buf), "sky %a %a %a %a %a", (double)p.elevation, (double)p.altitude, (double)p.air,
                  (double)p.dust, (double)p.ozone);
    return buf;
}

static int enumIndex(const std::string &v, std::initializer_list<const char *> names, int fb = -1) {
    // MaterialBuilder.swift:147-149: value with non-word characters replaced by '_', uppercased
    std::string e;
    for (char c : v) e += std::isalnum((unsigned char)c) || c == '_' ? (char)std::toupper((unsigned char)c) : '_';
    int i = 0;
    for (auto n : names) {
        if (e == n) return i;
        i++;
    }
    return fb;
}

// MaterialBuilder.swift:327-661 (the kernels this oracle implements)
static std::unique_ptr<NodeImpl> makeKernel(const rmd_node &n, const std::vector<std::string> &texNames,
                                            const std::vector<int> &texChannels) {
    std::string t = n.type ? n.type : "";
    auto unsupported = [&]() -> std::unique_ptr<NodeImpl> {
        throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "unsupported node type '" + t + "'"};
    };
    if (t == "TEX_COORD") return std::make_unique<Box<TextureCoordinate>>();
    if (t == "UVMAP") return std::make_unique<Box<UVMapCoordinate>>();
    if (t == "NEW_GEOMETRY") return std::make_unique<Box<NewGeometry>>();
    if (t == "LIGHT_PATH") return std::make_unique<Box<LightPath>>();
    if (t == "TEX_CHECKER") return std::make_unique<Box<TexChecker>>();
    if (t == "TEX_NOISE") {
        auto b = std::make_unique<Box<TexNoise>>();
        int d = enumIndex(paramString(n, "noise_dimensions", "3D"), {"1D", "2D", "3D", "4D"});
        if (d < 0) return unsupported();
        b->v.dimension = d;
        return b;
    }
    if (t == "VALTORGB") {
        auto b = std::make_unique<Box<ColorRamp>>();
        auto p = findParam(n, "elements");
        if (!p || p->num_numbers < 5 || p->num_numbers % 5 != 0 || p->num_numbers / 5 > 32)
            throw CodegenError{RMD_ERROR_INVALID_ARGUMENT, "ColorRamp needs 1..32 elements"};
        b->v.numElements = p->num_numbers / 5;
        for (int i = 0; i < b->v.numElements; i++) {
            b->v.positions[i] = p->numbers[5 * i];
            b->v.colors[i] = float4(p->numbers[5 * i + 1], p->numbers[5 * i + 2], p->numbers[5 * i + 3],
                                    p->numbers[5 * i + 4]);
        }
        return b;
    }
    if (t == "MIX_RGB") {
        auto b = std::make_unique<Box<ColorMix>>();
        int bt = enumIndex(paramString(n, "blend_type", "MIX"),
                           {"MIX", "ADD", "MULTIPLY", "SCREEN", "OVERLAY", "SUB", "COLOR", "LIGHTEN", "DARKEN",
                            "VALUE"});  // kColorMix names, nodes.hpp:1304-1317
        if (bt < 0) return unsupported();
        b->v.blendType = bt;
        b->v.clampResult = paramBool(n, "use_clamp", false);
        return b;
    }
    if (t == "MIX") {
        auto b = std::make_unique<Box<Mix>>();
        b->v.clampFactor = paramBool(n, "clamp_factor", true);
        b->v.clampResult = paramBool(n, "clamp_result", false);
        int fm = enumIndex(paramString(n, "factor_mode", "UNIFORM"), {"UNIFORM", "NON_UNIFORM"});
        if (fm < 0) return unsupported();
        b->v.factorMode = fm;
        return b;
    }
    if (t == "MATH") {
        auto b = std::make_unique<Box<MathNode>>();
        int op = enumIndex(paramString(n, "operation", "ADD"),
                           {"ADD", "SUBTRACT", "MULTIPLY", "DIVIDE", "MULTIPLY_ADD", "POWER", "MINIMUM", "MAXIMUM",
                            "TANGENT", "LESS_THAN", "GREATER_THAN", "MODULO"});
        if (op < 0) return unsupported();
        b->v.operation = op;
        b->v.clamp = paramBool(n, "use_clamp", false);
        return b;
    }
    if (t == "VECT_MATH") {
        auto b = std::make_unique<Box<VectorMath>>();
        int op = enumIndex(paramString(n, "operation", "ADD"),
                           {"ADD", "SUBTRACT", "MULTIPLY", "MULTIPLY_ADD", "NORMALIZE", "SCALE", "MINIMUM", "LENGTH",
                            "DOT_PRODUCT"});
        if (op < 0) return unsupported();
        b->v.operation = op;
        return b;
    }
    if (t == "SEPXYZ") return std::make_unique<Box<SeparateVector>>();
    if (t == "COMBXYZ") return std::make_unique<Box<CombineVector>>();
    if (t == "MAP_RANGE") {
        auto b = std::make_unique<Box<MapRange>>();
        b->v.clamp = paramBool(n, "clamp", true);
        return b;
    }
    if (t == "VALUE") {
        auto b = std::make_unique<Box<Value>>();
        auto p = findParam(n, "value");
        b->v.value = p ? (float)p->number_value : 0.0f;  // MaterialBuilder.swift:565-567
        return b;
    }
    if (t == "RGB") {
        auto b = std::make_unique<Box<RGB>>();
        auto p = findParam(n, "value");
        if (p && p->num_numbers >= 4)
            b->v.color = float4(p->numbers[0], p->numbers[1], p->numbers[2], p->numbers[3]);  // :568-575
        return b;
    }
    if (t == "RGBTOBW") return std::make_unique<Box<RGBToBW>>();
    if (t == "INVERT") return std::make_unique<Box<ColorInvert>>();
    if (t == "GAMMA") return std::make_unique<Box<Gamma>>();
    if (t == "MAPPING") {
        if (enumIndex(paramString(n, "type", "MAPPING"), {"MAPPING"}) < 0) return unsupported();
        return std::make_unique<Box<Mapping>>();
    }
    if (t == "NORMAL_MAP") {
        auto b = std::make_unique<Box<NormalMap>>();
        b->v.space = enumIndex(paramString(n, "space", "TANGENT"), {"TANGENT", "WORLD"});
        if (b->v.space < 0) return unsupported();
        return b;
    }
    if (t == "TEX_IMAGE" || t == "TEX_ENVIRONMENT") {  // MaterialBuilder.swift:387-433
        auto b = std::make_unique<Box<TexImage>>();
        const std::string file = paramString(n, "filepath", "");
        int slot = (int)texNames.size();
        for (size_t i = 0; i < texNames.size(); i++)
            if (texNames[i] == file) {
                slot = (int)i;
                break;
            }
        b->v.slot = slot;
        b->v.singleChannel = slot >= (int)texChannels.size() || texChannels[slot] == 1;
        if (enumIndex(paramString(n, "interpolation", "Linear"), {"LINEAR"}) < 0) return unsupported();
        b->v.projection = enumIndex(paramString(n, "projection", t == "TEX_IMAGE" ? "FLAT" : "EQUIRECTANGULAR"),
                                    {"FLAT", "BOX", "EQUIRECTANGULAR", "MIRROR_BALL"});
        b->v.colorSpace = enumIndex(paramString(n, "colorspace", "sRGB"),
                                    {"LINEAR", "SRGB", "NON_COLOR", "RAW", "XYZ", "FILMIC_LOG"});
        if (b->v.projection < 0 || b->v.colorSpace < 0) return unsupported();
        return b;
    }
    if (t == "TEX_SKY") {  // MaterialBuilder.swift:329-388
        const SkyParams p = skyParams(n);
        auto b = std::make_unique<Box<TexNishita>>();
        const std::string key = skyTextureKey(p);
        b->v.slot = (int)texNames.size();
        for (size_t i = 0; i < texNames.size(); i++)
            if (texNames[i] == key) b->v.slot = (int)i;
        oracle_sky::skyData(p.elevation, p.rotation, p.disc, p.size, p.intensity, p.altitude, p.air, p.dust,
                            b->v.data);
        b->v.scale = p.scale;
        return b;
    }
    if (t == "HUE_SAT") return std::make_unique<Box<HueSaturation>>();
    if (t == "BRIGHTCONTRAST") return std::make_unique<Box<BrightnessContrast>>();
    if (t == "BLACKBODY") return std::make_unique<Box<Blackbody>>();
    if (t == "FRESNEL") return std::make_unique<Box<Fresnel>>();
    if (t == "LAYER_WEIGHT") return std::make_unique<Box<LayerWeight>>();
    if (t == "EMISSION") return std::make_unique<Box<Emission>>();
    if (t == "BACKGROUND") return std::make_unique<Box<Background>>();
    if (t == "BSDF_PRINCIPLED") return std::make_unique<Box<BsdfPrincipled>>();
    if (t == "BSDF_DIFFUSE") return std::make_unique<Box<BsdfDiffuse>>();
    if (t == "BSDF_GLOSSY") return std::make_unique<Box<BsdfGlossy>>();
    if (t == "BSDF_GLASS") return std::make_unique<Box<BsdfGlass>>();
    if (t == "BSDF_TRANSPARENT") return std::make_unique<Box<BsdfTransparent>>();
    if (t == "ADD_SHADER") return std::make_unique<Box<AddShader>>();
    if (t == "MIX_SHADER") return std::make_unique<Box<MixShader>>();
    if (t == "OUTPUT_MATERIAL") return std::make_unique<Box<OutputMaterial>>();
    if (t == "OUTPUT_WORLD") return std::make_unique<Box<OutputWorld>>();
    if (t == "OUTPUT_LIGHT") return std::make_unique<Box<OutputLight>>();
    return unsupported();
}

static bool isOutput(const char *t) {
    std::string s = t ? t : "";
    return s == "OUTPUT_MATERIAL" || s == "OUTPUT_LIGHT" || s == "OUTPUT_WORLD";
}

// The coercion helpers of nodes.hpp:2007-2031 applied to a value of kind `k`.
static Kind coercedKind(const std::string &type) {
    if (type == "VALUE") return K_F1;
    if (type == "RGBA") return K_F4;
    if (type == "VECTOR") return K_F3;
    if (type == "SHADER") return K_SHADER;
    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "unsupported socket type '" + type + "'"};
}

// `field = TYPE(x)` compiles when the coerced type is the field's, or a scalar
// widened to a vector (Metal's implicit scalar-to-vector conversion).
static void checkAssignable(const std::string &type, Kind fieldKind, const std::string &field) {
    const Kind k = coercedKind(type);
    if (k == fieldKind) return;
    if (k == K_F1 && (fieldKind == K_F3 || fieldKind == K_F4)) return;
    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "cannot assign " + type + " to field '" + field + "'"};
}

static void coerce(const std::string &type, Kind k, const void *src, Kind dstKind, void *dst) {
    float f[4] = {0, 0, 0, 0};
    const UberShader *sh = nullptr;
    if (k == K_SHADER) sh = static_cast<const UberShader *>(src);
    else std::memcpy(f, src, sizeof(float) * (int)k);
    if (type == "VECTOR") {
        float3 r;
        switch (k) {
            case K_F1: r = float3(f[0]); break;
            case K_F2: r = float3(f[0], f[1], 0); break;
            case K_F3: r = float3(f[0], f[1], f[2]); break;
            case K_F4: r = float3(f[0], f[1], f[2]); break;
            case K_SHADER: r = float3(0.0f); break;
        }
        std::memcpy(dst, &r, sizeof(r));
    } else if (type == "RGBA") {
        float4 r;
        switch (k) {
            case K_F1: r = float4(f[0], f[0], f[0], 1); break;
            case K_F2: r = float4(f[0], f[1], 0, 1); break;
            case K_F3: r = float4(f[0], f[1], f[2], 1); break;
            case K_F4: r = float4(f[0], f[1], f[2], f[3]); break;
            case K_SHADER: r = float4(sh->emission, 1); break;
        }
        std::memcpy(dst, &r, sizeof(r));
    } else if (type == "VALUE") {
        float r;
        switch (k) {
            case K_F1: r = f[0]; break;
            case K_F3: r = (f[0] + f[1] + f[2]) / 3; break;
            case K_F4: r = f[3] * (f[0] + f[1] + f[2]) / 3; break;
            default: throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "VALUE() of this kind"};
        }
        if (dstKind == K_F1) std::memcpy(dst, &r, sizeof(r));
        else if (dstKind == K_F3) { float3 b(r); std::memcpy(dst, &b, sizeof(b)); }
        else if (dstKind == K_F4) { float4 b(r); std::memcpy(dst, &b, sizeof(b)); }
    } else if (type == "SHADER") {
        UberShader m;
        switch (k) {
            case K_SHADER: m = *sh; break;
            case K_F1: m.emission = float3(f[0]); break;
            case K_F2: m.emission = float3(f[0], f[1], 0); break;
            case K_F3: m.emission = float3(f[0], f[1], f[2]); break;
            case K_F4: m.emission = float3(f[0], f[1], f[2]); break;
        }
        *static_cast<UberShader *>(dst) = m;
    }
}

MaterialProgram::MaterialProgram(const rmd_material &m, const std::vector<std::string> &textureNames,
                                 const std::vector<int> &textureChannels) {
    static std::atomic<uint64_t> nextSerial{1};
    serial_ = nextSerial.fetch_add(1);
    name_ = m.name ? m.name : "";
    std::map<std::string, const rmd_node *> nodes;
    for (int i = 0; i < m.num_nodes; i++) nodes[m.nodes[i].name ? m.nodes[i].name : ""] = &m.nodes[i];
    std::map<std::string, int> state;  // 1 = pending, 2 = emitted
    std::map<std::string, int> stepIndex;

    // MaterialBuilder.swift:793-825
    std::function<void(const std::string &)> emit = [&](const std::string &key) {
        auto st = state.find(key);
        if (st != state.end()) {
            if (st->second == 2) return;
            throw CodegenError{RMD_ERROR_CODEGEN_CYCLE, "cycle detected at node '" + key + "'"};
        }
        auto it = nodes.find(key);
        if (it == nodes.end()) throw CodegenError{RMD_ERROR_INVALID_ARGUMENT, "link to unknown node '" + key + "'"};
        state[key] = 1;
        const rmd_node &node = *it->second;
        Step step;
        step.proto = makeKernel(node, textureNames, textureChannels);
        void *base = step.proto->base();

        // provideDefaults, MaterialBuilder.swift:762-791
        std::string t = node.type;
        std::string defaultInput;
        MaterialProgram::Binding::Src defaultSrc = Binding::SHADING_NORMAL;
        if (t == "TEX_IMAGE") { defaultInput = "Vector"; defaultSrc = Binding::SHADING_UV; }
        else if (t == "TEX_CHECKER" || t == "TEX_NOISE" || t == "TEX_ENVIRONMENT") {
            defaultInput = "Vector"; defaultSrc = Binding::SHADING_GENERATED;
        } else if (t == "FRESNEL" || t == "LAYER_WEIGHT" || t == "BSDF_GLASS" || t == "BSDF_GLOSSY" ||
                   t == "BSDF_DIFFUSE" || t == "BSDF_PRINCIPLED" || t == "BSDF_TRANSLUCENT" ||
                   t == "BSDF_REFRACTION" || t == "BSDF_ANISOTROPIC" || t == "BSDF_VELVET" || t == "BUMP") {
            defaultInput = "Normal"; defaultSrc = Binding::SHADING_NORMAL;
        }
        std::map<std::string, Binding> inputs;  // keyed by field identifier, last assignment wins
        if (!defaultInput.empty()) {
            bool found = false;
            for (int i = 0; i < node.num_inputs; i++)
                if (node.inputs[i].name && defaultInput == node.inputs[i].name) found = true;
            if (!found)
                throw CodegenError{RMD_ERROR_INVALID_ARGUMENT, "node '" + key + "' lacks input '" + defaultInput + "'"};
            auto fd = step.proto->field(makeIdentifier(defaultInput));
            if (!fd) throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "no field for default input"};
            Binding b;
            b.src = defaultSrc;
            b.dst_offset = fd->offset;
            b.dst_kind = fd->kind;
            b.in_type = "VECTOR";
            inputs[fd->name] = b;
        }
        std::vector<const rmd_node_input *> sorted;
        for (int i = 0; i < node.num_inputs; i++) sorted.push_back(&node.inputs[i]);
        std::sort(sorted.begin(), sorted.end(), [](const rmd_node_input *a, const rmd_node_input *b) {
            return std::string(a->name) < std::string(b->name);
        });
        for (const rmd_node_input *in : sorted) {
            std::string fieldName = makeIdentifier(in->name);
            bool linked = in->link_node != nullptr || in->num_links > 0;
            if (in->num_links > 1) throw CodegenError{RMD_ERROR_CODEGEN_MULTI_INPUT, "multi-input link detected"};
            if (!linked) {
                bool isDefault = (!defaultInput.empty() && defaultInput == in->name);
                if (isDefault || in->num_values <= 0) continue;  // value cleared by provideDefaults / no value
                auto fd = step.proto->field(fieldName);
                if (!fd)  // the generated Metal would not compile: the struct has no such field
                    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED,
                                       "node '" + key + "' has no input field '" + fieldName + "'"};
                // MaterialBuilder.swift:110-121: TYPE(literal)
                std::string ty = in->type ? in->type : "VALUE";
                Kind litKind = in->num_values == 1 ? K_F1 : (Kind)std::min(4, in->num_values);
                checkAssignable(ty, fd->kind, fieldName);
                coerce(ty, litKind, in->values, fd->kind, (char *)base + fd->offset);
                inputs.erase(fd->name);
            } else {
                std::string src = in->link_node;
                emit(src);
                auto fd = step.proto->field(fieldName);
                if (!fd)
                    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED,
                                       "node '" + key + "' has no input field '" + fieldName + "'"};
                int si = stepIndex.at(src);
                std::string outName = makeIdentifier(in->link_socket ? in->link_socket : "");
                auto sfd = steps_[si].proto->field(outName);
                if (!sfd)
                    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED,
                                       "node '" + src + "' has no output '" + outName + "'"};
                Binding b;
                b.src = Binding::LINK;
                b.dst_offset = fd->offset;
                b.dst_kind = fd->kind;
                b.in_type = in->type ? in->type : "VALUE";
                checkAssignable(b.in_type, fd->kind, fieldName);
                if (b.in_type == "VALUE" && sfd->kind == K_F2)
                    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "VALUE() of a float2 output"};
                b.src_node = si;
                b.src_offset = sfd->offset;
                b.src_kind = sfd->kind;
                inputs[fd->name] = b;
            }
        }
        for (auto &kv : inputs) step.links.push_back(kv.second);
        stepIndex[key] = (int)steps_.size();
        steps_.push_back(std::move(step));
        state[key] = 2;
    };
    // MaterialBuilder.swift:684-691
    for (auto &kv : nodes)
        if (isOutput(kv.second->type)) emit(kv.first);

    // hasSurfaceEmission (Rayjay Material.hasSurfaceEmission, source absent): an
    // Emission node reachable from an output, or a Principled node whose
    // emission colour and strength are both linked or non-zero.
    for (auto &kv : stepIndex) {
        const rmd_node &n = *nodes[kv.first];
        std::string t = n.type;
        if (t == "EMISSION") hasEmission_ = true;
        if (t == "BSDF_PRINCIPLED") {
            bool colorOn = false, strengthOn = false;
            for (int i = 0; i < n.num_inputs; i++) {
                const rmd_node_input &in = n.inputs[i];
                std::string nm = in.name;
                bool linked = in.link_node != nullptr;
                if (nm == "Emission")
                    colorOn = linked || (in.num_values >= 3 && (in.values[0] != 0 || in.values[1] != 0 || in.values[2] != 0));
                if (nm == "Emission Strength") strengthOn = linked || (in.num_values >= 1 && in.values[0] != 0);
            }
            if (colorOn && strengthOn) hasEmission_ = true;
        }
    }
}

void MaterialProgram::run(const SceneData &ctx, ShadingContext &shading) const {
    // Per-thread node instances of each program.  Keyed by serial, not by
    // address: a program built after another was destroyed may reuse its
    // address, and must not inherit its node instances.
    thread_local std::map<uint64_t, std::vector<std::unique_ptr<NodeImpl>>> cache;
    if (cache.size() > 1024 && !cache.count(serial_)) cache.clear();
    auto &inst = cache[serial_];
    if (inst.size() != steps_.size()) {
        inst.clear();
        for (auto &s : steps_) inst.push_back(s.proto->clone());
    }
    for (size_t i = 0; i < steps_.size(); i++) {
        const Step &s = steps_[i];
        NodeImpl &n = *inst[i];
        n.copy_from(*s.proto);
        char *base = (char *)n.base();
        for (const Binding &b : s.links) {
            switch (b.src) {
                case Binding::LINK:
                    coerce(b.in_type, b.src_kind, (char *)inst[b.src_node]->base() + b.src_offset, b.dst_kind,
                           base + b.dst_offset);
                    break;
                case Binding::SHADING_UV: coerce("VECTOR", K_F3, &shading.uv, b.dst_kind, base + b.dst_offset); break;
                case Binding::SHADING_GENERATED:
                    coerce("VECTOR", K_F3, &shading.generated, b.dst_kind, base + b.dst_offset);
                    break;
                case Binding::SHADING_NORMAL:
                    coerce("VECTOR", K_F3, &shading.normal, b.dst_kind, base + b.dst_offset);
                    break;
                default: break;
            }
        }
        n.compute(ctx, shading);
    }
}

}  // namespace orc
