// Cycles node library of the reference (raymond/device/nodes/nodes.hpp) for the
// NVRTC material module: the same struct names, template parameters, field
// names and `compute(ctx, shading)` contract, so that generated material code
// has the shape MaterialBuilder.swift emits (`Kernel<params> n_x{}; n_x.field =
// TYPE(...); n_x.compute(ctx, shading);`).
#pragma once
#include "noise.cuh"
#include "scene.cuh"

namespace rmd {

RMD_HD float luminance(float3 c) { return dot(make_float3(0.2126f, 0.7152f, 0.0722f), c); }  // color.hpp:3-6

// color.hpp:9-72
RMD_HD float3 rgb2hsv(float3 rgb) {
    const float cmax = fmaxf(rgb.x, fmaxf(rgb.y, rgb.z));
    const float cmin = fminf(rgb.x, fminf(rgb.y, rgb.z));
    const float cdelta = cmax - cmin;
    float h = 0.0f, s = 0.0f, v = cmax;
    if (cmax != 0.0f) s = cdelta / cmax;
    if (s != 0.0f) {
        const float3 c = (f3(cmax) - rgb) / cdelta;
        if (rgb.x == cmax) h = 0.0f + c.z - c.y;
        else if (rgb.y == cmax) h = 2.0f + c.x - c.z;
        else h = 4.0f + c.y - c.x;
        h /= 6.0f;
        if (h < 0.0f) h += 1.0f;
    }
    return make_float3(h, s, v);
}
RMD_HD float3 hsv2rgb(float3 hsv) {
    float h = hsv.x;
    const float s = hsv.y, v = hsv.z;
    if (s == 0.0f) return make_float3(v, v, v);
    if (h == 1.0f) h = 0.0f;
    h *= 6.0f;
    const float i = floorf(h);
    const float f = h - i;
    const float p = v * (1.0f - s);
    const float q = v * (1.0f - (s * f));
    const float t = v * (1.0f - (s * (1.0f - f)));
    switch ((int)i) {
        case 0: return make_float3(v, t, p);
        case 1: return make_float3(q, v, p);
        case 2: return make_float3(p, v, t);
        case 3: return make_float3(p, q, v);
        case 4: return make_float3(t, p, v);
        default: return make_float3(v, p, q);
    }
}

// ---------------------------------------------------------------- coercions (nodes.hpp:2007-2031)
RMD_HD float3 VECTOR(float v) { return f3(v); }
RMD_HD float3 VECTOR(float2 v) { return f3(v, 0.0f); }
RMD_HD float3 VECTOR(float3 v) { return v; }
RMD_HD float3 VECTOR(float4 v) { return xyz(v); }
RMD_HD float3 VECTOR(const UberShader &) { return f3(0.0f); }
RMD_HD float4 RGBA(float v) { return make_float4(v, v, v, 1.0f); }
RMD_HD float4 RGBA(float2 v) { return make_float4(v.x, v.y, 0.0f, 1.0f); }
RMD_HD float4 RGBA(float3 v) { return f4(v, 1.0f); }
RMD_HD float4 RGBA(float4 v) { return v; }
RMD_HD float4 RGBA(const UberShader &v) { return f4(v.emission, 1.0f); }
RMD_HD float VALUE(float v) { return v; }
RMD_HD float VALUE(float3 v) { return (v.x + v.y + v.z) / 3.0f; }
RMD_HD float VALUE(float4 v) { return v.w * (v.x + v.y + v.z) / 3.0f; }
RMD_HD UberShader SHADER(const UberShader &v) { return v; }
RMD_HD UberShader SHADER(float3 v) {
    UberShader m;
    m.emission = v;
    return m;
}
RMD_HD UberShader SHADER(float v) { return SHADER(f3(v)); }
RMD_HD UberShader SHADER(float2 v) { return SHADER(f3(v, 0.0f)); }
RMD_HD UberShader SHADER(float4 v) { return SHADER(xyz(v)); }

// ---------------------------------------------------------------- input nodes
struct LightPath {  // nodes.hpp:15-43
    bool isCameraRay, isReflectionRay, isTransmissionRay, isShadowRay, isDiffuseRay, isGlossyRay, isSingularRay;
    float rayLength;
    RMD_HD void compute(const Context &, const ShadingContext &sh) {
        const uint32_t f = sh.rayFlags;
        isCameraRay = (f & RayFlagsCamera) != 0;
        isReflectionRay = (f & RayFlagsReflection) != 0;
        isTransmissionRay = (f & RayFlagsTransmission) != 0;
        isShadowRay = (f & RayFlagsShadow) != 0;
        isDiffuseRay = (f & RayFlagsDiffuse) != 0;
        isGlossyRay = (f & RayFlagsGlossy) != 0;
        isSingularRay = (f & RayFlagsSingular) != 0;
        rayLength = sh.distance;
        if (isSingularRay) isGlossyRay = true;
    }
};
struct NewGeometry {  // nodes.hpp:201-221
    float3 normal, trueNormal, tangent, position, parametric, incoming, randomPerIsland;
    bool backfacing;
    RMD_HD void compute(const Context &, const ShadingContext &sh) {
        normal = sh.normal;
        trueNormal = sh.trueNormal;
        tangent = sh.tu;
        position = sh.position;
        parametric = sh.uv;
        incoming = sh.wo;
        randomPerIsland = f3(0.0f);
        backfacing = dot(sh.wo, sh.normal) < 0.0f;
    }
};
struct TextureCoordinate {  // nodes.hpp:223-237
    float3 generated, uv, object, normal, reflection;
    RMD_HD void compute(const Context &, const ShadingContext &sh) {
        uv = sh.uv;
        generated = sh.generated;
        object = sh.object;
        normal = sh.normal;
        reflection = sh.normal;
    }
};
struct UVMapCoordinate {  // nodes.hpp:239-245
    float3 uv;
    RMD_HD void compute(const Context &, const ShadingContext &sh) { uv = sh.uv; }
};
struct Value {  // nodes.hpp:1716-1719
    float value;
    RMD_HD void compute(const Context &, const ShadingContext &) {}
};
struct RGB {  // nodes.hpp:1721-1724
    float4 color;
    RMD_HD void compute(const Context &, const ShadingContext &) {}
};

// ---------------------------------------------------------------- textures
struct TexChecker {  // nodes.hpp:247-264
    float scale;
    float4 color1, color2;
    float3 vector;
    float fac;
    float4 color;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        float3 p = (vector * scale + 0.000001f) * 0.999999f;
        const int ix = (int)floorf(p.x), iy = (int)floorf(p.y), iz = (int)floorf(p.z);
        const bool which = ((ix ^ iy ^ iz) & 1) != 0;
        color = which ? color1 : color2;
        fac = which ? 1.0f : 0.0f;
    }
};

struct kTexNoise {
    enum Dimension { DIMENSION_1D, DIMENSION_2D, DIMENSION_3D, DIMENSION_4D };
};
template <int Dimension>
struct TexNoise {  // nodes.hpp:872-1011
    float detail, distortion, roughness, scale, w;
    float3 vector;
    float fac;
    float4 color;

    RMD_HD static float off1(float seed) { return 100.0f + noise::hash_float_to_float(seed) * 100.0f; }
    RMD_HD static float off2(float seed, float k) {
        return 100.0f + noise::hash_float2_to_float(make_float2(seed, k)) * 100.0f;
    }
    RMD_HD static float2 off2v(float s) { return make_float2(off2(s, 0.0f), off2(s, 1.0f)); }
    RMD_HD static float3 off3v(float s) { return make_float3(off2(s, 0.0f), off2(s, 1.0f), off2(s, 2.0f)); }
    RMD_HD static float4 off4v(float s) {
        return make_float4(off2(s, 0.0f), off2(s, 1.0f), off2(s, 2.0f), off2(s, 3.0f));
    }
    RMD_HD void compute(const Context &, const ShadingContext &) {
        const float3 p3 = this->vector * scale;
        const float ww = this->w * scale;
        if (Dimension == kTexNoise::DIMENSION_1D) {
            float p = ww;
            if (distortion != 0.0f) p += noise::snoise(p + off1(0.0f)) * distortion;
            color = make_float4(noise::fractal_noise(p, detail, roughness),
                                noise::fractal_noise(p + off1(1.0f), detail, roughness),
                                noise::fractal_noise(p + off1(2.0f), detail, roughness), 1.0f);
        } else if (Dimension == kTexNoise::DIMENSION_2D) {
            float2 p = make_float2(p3.x, p3.y);
            if (distortion != 0.0f)
                p = p + distortion * make_float2(noise::snoise(p + off2v(0.0f)), noise::snoise(p + off2v(1.0f)));
            color = make_float4(noise::fractal_noise(p, detail, roughness),
                                noise::fractal_noise(p + off2v(2.0f), detail, roughness),
                                noise::fractal_noise(p + off2v(3.0f), detail, roughness), 1.0f);
        } else if (Dimension == kTexNoise::DIMENSION_3D) {
            float3 p = p3;
            if (distortion != 0.0f)
                p += distortion * make_float3(noise::snoise(p + off3v(0.0f)), noise::snoise(p + off3v(1.0f)),
                                              noise::snoise(p + off3v(2.0f)));
            color = make_float4(noise::fractal_noise(p, detail, roughness),
                                noise::fractal_noise(p + off3v(3.0f), detail, roughness),
                                noise::fractal_noise(p + off3v(4.0f), detail, roughness), 1.0f);
        } else {
            float4 p = f4(p3, ww);
            if (distortion != 0.0f)
                p = p + distortion * make_float4(noise::snoise(p + off4v(0.0f)), noise::snoise(p + off4v(1.0f)),
                                                 noise::snoise(p + off4v(2.0f)), noise::snoise(p + off4v(3.0f)));
            color = make_float4(noise::fractal_noise(p, detail, roughness),
                                noise::fractal_noise(p + off4v(4.0f), detail, roughness),
                                noise::fractal_noise(p + off4v(5.0f), detail, roughness), 1.0f);
        }
        fac = color.x;
    }
};

struct ColorRampElement {
    float position;
    float4 color;
};
template <int NumElements>
struct ColorRamp {  // nodes.hpp:1013-1046
    float fac;
    float4 color;
    ColorRampElement elements[NumElements];
    RMD_HD void compute(const Context &, const ShadingContext &) {
        if (fac < elements[0].position) {
            color = elements[0].color;
            return;
        }
        if (fac > elements[NumElements - 1].position) {
            color = elements[NumElements - 1].color;
            return;
        }
        for (int i = 1; i < NumElements; ++i) {
            if (elements[i].position >= fac) {
                const ColorRampElement a = elements[i - 1], b = elements[i];
                float v = (fac - a.position) / (b.position - a.position);
                color = (1.0f - v) * a.color + v * b.color;
                return;
            }
        }
    }
};

// ---------------------------------------------------------------- converters
struct kColorMix {
    enum BlendType {
        BLEND_TYPE_MIX, BLEND_TYPE_ADD, BLEND_TYPE_MULTIPLY, BLEND_TYPE_SCREEN, BLEND_TYPE_OVERLAY,
        BLEND_TYPE_SUB, BLEND_TYPE_COLOR, BLEND_TYPE_LIGHTEN, BLEND_TYPE_DARKEN, BLEND_TYPE_VALUE
    };
};
template <int BlendType, bool Clamp>
struct ColorMix {  // nodes.hpp:1319-1385
    float4 color1, color2;
    float fac;
    float4 color;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        switch (BlendType) {
            case kColorMix::BLEND_TYPE_MIX: color = lerp(color1, color2, fac); break;
            case kColorMix::BLEND_TYPE_ADD: color = color1 + fac * color2; break;
            case kColorMix::BLEND_TYPE_SUB: color = color1 - fac * color2; break;
            case kColorMix::BLEND_TYPE_MULTIPLY: color = color1 * lerp(f4(1.0f), color2, fac); break;
            case kColorMix::BLEND_TYPE_SCREEN: color = f4(1.0f) - (f4(1.0f) - fac * color1) * (f4(1.0f) - color1); break;
            case kColorMix::BLEND_TYPE_OVERLAY: {
                color = color1;
                float *c = &color.x;
                const float *c2 = &color2.x;
                for (int d = 0; d < 3; d++) {
                    if (c[d] < 0.5f) c[d] *= 1.0f - fac + 2.0f * fac * c2[d];
                    else c[d] = 1.0f - (1.0f - fac + 2.0f * fac * (1.0f - c2[d])) * (1.0f - c[d]);
                }
                break;
            }
            case kColorMix::BLEND_TYPE_COLOR: {
                color = color1;
                const float3 hsv2 = rgb2hsv(xyz(color2));
                if (hsv2.y == 0.0f) {
                    color = color1;
                } else {
                    float3 hsv = rgb2hsv(xyz(color1));
                    hsv.x = hsv2.x;
                    hsv.y = hsv2.y;
                    color = lerp(color1, f4(hsv2rgb(hsv), color2.w), fac);
                }
                break;
            }
            case kColorMix::BLEND_TYPE_LIGHTEN: color = lerp(color1, vmax(color1, color2), fac); break;
            case kColorMix::BLEND_TYPE_DARKEN: color = lerp(color1, vmin(color1, color2), fac); break;
            case kColorMix::BLEND_TYPE_VALUE: {
                float3 hsv = rgb2hsv(xyz(color1));
                hsv.z = rgb2hsv(xyz(color2)).z;
                color = lerp(color1, f4(hsv2rgb(hsv), color2.w), fac);
                break;
            }
        }
        if (Clamp) color = saturate(color);
    }
};
struct kMix {
    enum FactorMode { FACTOR_MODE_UNIFORM, FACTOR_MODE_NON_UNIFORM };
};
template <bool ClampFactor, bool ClampResult, int FactorMode>
struct Mix {  // nodes.hpp:1940-1974
    float4 a_Color, b_Color, result_Color;
    float a_Float, b_Float, result_Float;
    float3 a_Vector, b_Vector, result_Vector;
    float factor_Float;
    float3 factor_Vector;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        if (ClampFactor) {
            factor_Float = saturate(factor_Float);
            factor_Vector = saturate(factor_Vector);
        }
        if (FactorMode == kMix::FACTOR_MODE_UNIFORM) result_Vector = lerp(a_Vector, b_Vector, factor_Float);
        else result_Vector = a_Vector + (b_Vector - a_Vector) * factor_Vector;
        result_Float = lerp(a_Float, b_Float, factor_Float);
        result_Color = lerp(a_Color, b_Color, factor_Float);
        if (ClampResult) result_Color = saturate(result_Color);
    }
};
struct kMath {
    enum Operation {
        OPERATION_ADD, OPERATION_SUBTRACT, OPERATION_MULTIPLY, OPERATION_DIVIDE, OPERATION_MULTIPLY_ADD,
        OPERATION_POWER, OPERATION_MINIMUM, OPERATION_MAXIMUM, OPERATION_TANGENT, OPERATION_LESS_THAN,
        OPERATION_GREATER_THAN, OPERATION_MODULO
    };
};
template <int Operation, bool Clamp>
struct Math {  // nodes.hpp:1145-1193
    float value, value_001, value_002;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        switch (Operation) {
            case kMath::OPERATION_ADD: value = value + value_001; break;
            case kMath::OPERATION_SUBTRACT: value = value - value_001; break;
            case kMath::OPERATION_MULTIPLY: value = value * value_001; break;
            case kMath::OPERATION_DIVIDE: value = value_001 == 0.0f ? 0.0f : value / value_001; break;
            case kMath::OPERATION_MULTIPLY_ADD: value = value * value_001 + value_002; break;
            case kMath::OPERATION_POWER: value = powf(value, value_001); break;
            case kMath::OPERATION_MINIMUM: value = fminf(value, value_001); break;
            case kMath::OPERATION_MAXIMUM: value = fmaxf(value, value_001); break;
            case kMath::OPERATION_TANGENT: value = tanf(value); break;
            case kMath::OPERATION_LESS_THAN: value = value < value_001 ? 1.0f : 0.0f; break;
            case kMath::OPERATION_GREATER_THAN: value = value > value_001 ? 1.0f : 0.0f; break;
            case kMath::OPERATION_MODULO: value = fmodf(value, value_001); break;
        }
        if (Clamp) value = saturate(value);
    }
};
struct kVectorMath {
    enum Operation {
        OPERATION_ADD, OPERATION_SUBTRACT, OPERATION_MULTIPLY, OPERATION_MULTIPLY_ADD, OPERATION_NORMALIZE,
        OPERATION_SCALE, OPERATION_MINIMUM, OPERATION_LENGTH, OPERATION_DOT_PRODUCT
    };
};
template <int Operation>
struct VectorMath {  // nodes.hpp:165-199
    float scale, value;
    float3 vector, vector_001, vector_002;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        switch (Operation) {
            case kVectorMath::OPERATION_ADD: vector = vector + vector_001; break;
            case kVectorMath::OPERATION_SUBTRACT: vector = vector - vector_001; break;
            case kVectorMath::OPERATION_MULTIPLY: vector = vector * vector_001; break;
            case kVectorMath::OPERATION_MULTIPLY_ADD: vector = vector * vector_001 + vector_002; break;
            case kVectorMath::OPERATION_NORMALIZE: vector = normalize(vector); break;
            case kVectorMath::OPERATION_SCALE: vector = vector * scale; break;
            case kVectorMath::OPERATION_MINIMUM: vector = vmin(vector, vector_001); break;
            case kVectorMath::OPERATION_LENGTH: value = length(vector); break;
            case kVectorMath::OPERATION_DOT_PRODUCT: vector = f3(dot(vector, vector_001)); break;
        }
    }
};
struct SeparateVector {  // nodes.hpp:266-275
    float3 vector;
    float x, y, z;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        x = vector.x;
        y = vector.y;
        z = vector.z;
    }
};
struct CombineVector {  // nodes.hpp:277-284
    float x, y, z;
    float3 vector;
    RMD_HD void compute(const Context &, const ShadingContext &) { vector = make_float3(x, y, z); }
};
struct kMapRange {
    enum DataType { DATA_TYPE_FLOAT };
    enum InterpolationType { INTERPOLATION_TYPE_LINEAR };
};
template <bool Clamp, int DataType, int InterpolationType>
struct MapRange {  // nodes.hpp:314-344
    float fromMin, fromMax, toMin, toMax, steps;
    float3 steps_Float3, from_Min_Float3, from_Max_Float3, to_Min_Float3, to_Max_Float3;
    float value;
    float3 vector;
    float result;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        float v = (value - fromMin) / (fromMax - fromMin);
        if (Clamp) v = saturate(v);
        result = lerp(toMin, toMax, v);
    }
};
struct RGBToBW {  // nodes.hpp:1726-1734
    float4 color;
    float val;
    RMD_HD void compute(const Context &, const ShadingContext &) { val = luminance(xyz(color)); }
};
struct ColorInvert {  // nodes.hpp:1387-1394
    float4 color;
    float fac;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        const float3 c = xyz(color) - fac * (2.0f * xyz(color) - f3(1.0f));
        color = f4(c, color.w);
    }
};
// Metal's linear sampler with address::repeat over normalized coordinates
// (the sampler of nodes.hpp:517): texel centres at (i + 1/2) / size, the four
// nearest texels wrapped around the image and blended bilinearly, in FP32.
RMD_HD int wrapTexel(float i, int n) {
    const float m = i - floorf(i / (float)n) * (float)n;  // in [0, n] up to rounding
    const int k = (int)m;
    return k < 0 ? 0 : (k >= n ? n - 1 : k);
}
RMD_HD float4 sampleLinearRepeat(const TextureView &t, float2 uv) {
    const float x = uv.x * (float)t.width - 0.5f, y = uv.y * (float)t.height - 0.5f;
    const float x0f = floorf(x), y0f = floorf(y);
    const float ax = x - x0f, ay = y - y0f;
    const int x0 = wrapTexel(x0f, t.width), y0 = wrapTexel(y0f, t.height);
    const int x1 = x0 + 1 == t.width ? 0 : x0 + 1, y1 = y0 + 1 == t.height ? 0 : y0 + 1;
    const float4 *row0 = t.texels + (size_t)y0 * t.width, *row1 = t.texels + (size_t)y1 * t.width;
    const float4 top = lerp(row0[x0], row0[x1], ax), bottom = lerp(row1[x0], row1[x1], ax);
    return lerp(top, bottom, ay);
}

// color.hpp:74-78
RMD_HD float3 xyz_to_rgb(float3 c) {
    return make_float3(3.240479f * c.x + -1.537150f * c.y + -0.498535f * c.z,
                       -0.969256f * c.x + 1.875991f * c.y + 0.041556f * c.z,
                       0.055648f * c.x + -0.204043f * c.y + 1.057311f * c.z);
}

struct kTexImage {
    enum Interpolation { INTERPOLATION_LINEAR };
    enum Projection { PROJECTION_FLAT, PROJECTION_BOX, PROJECTION_EQUIRECTANGULAR, PROJECTION_MIRROR_BALL };
    enum Extension { EXTENSION_REPEAT };
    enum Alpha { ALPHA_STRAIGHT };
    enum ColorSpace {
        COLOR_SPACE_LINEAR,
        COLOR_SPACE_SRGB,
        COLOR_SPACE_NON_COLOR,
        COLOR_SPACE_RAW,
        COLOR_SPACE_XYZ,
        COLOR_SPACE_FILMIC_LOG
    };
    enum PixelFormat { PIXEL_FORMAT_R, PIXEL_FORMAT_RGBA };
};
// nodes.hpp:486-564 (the image and environment texture nodes): project the
// vector (flat: (x, 1 - y); equirectangular: the sphere to the unit square;
// box and mirror ball are not implemented there and read (0, 0)), sample with
// repeat, a single-channel image as grey, then decode the colour space.
template <int TextureIndex, kTexImage::Interpolation Interp, kTexImage::Projection Projection,
          kTexImage::Extension Extension, kTexImage::Alpha Alpha, kTexImage::ColorSpace ColorSpace,
          kTexImage::PixelFormat PixelFormat>
struct TexImage {
    float3 vector;
    float4 color;
    float alpha;
    RMD_HD static float srgbToLinear(float c) {  // nodes.hpp:556-562
        if (c < 0.04045f) return c < 0.0f ? 0.0f : c * (1.0f / 12.92f);
        return powf((c + 0.055f) * (1.0f / 1.055f), 2.4f);
    }
    RMD_HD void compute(const Context &ctx, const ShadingContext &) {
        float2 projected = make_float2(0.0f, 0.0f);
        if (Projection == kTexImage::PROJECTION_FLAT) projected = make_float2(vector.x, 1.0f - vector.y);
        else if (Projection == kTexImage::PROJECTION_EQUIRECTANGULAR) projected = warp::equirectSphereToSquare(vector);
        color = sampleLinearRepeat(ctx.textures[TextureIndex], projected);
        alpha = color.w;
        if (PixelFormat == kTexImage::PIXEL_FORMAT_R) color = make_float4(color.x, color.x, color.x, 1.0f);
        if (ColorSpace == kTexImage::COLOR_SPACE_SRGB)
            color = make_float4(srgbToLinear(color.x), srgbToLinear(color.y), srgbToLinear(color.z), color.w);
        else if (ColorSpace == kTexImage::COLOR_SPACE_XYZ)
            color = f4(xyz_to_rgb(xyz(color)), color.w);
    }
};

// The Nishita sky (nodes.hpp:774-870): radiance of direction `dir` from the
// sky texture the scene generated for this node (rows: elevation, from the
// horizon up with sqrt spacing; columns: azimuth), the sun disc between its
// bottom and top colours with limb darkening, and below the horizon the
// horizon row fading to black by -0.4; XYZ converted to linear RGB.
// data: sun bottom and top XYZ, sun elevation, rotation, angular diameter
// (-1 without a disc), intensity.
RMD_HD float3 skyRadianceNishita(float3 dir, const float *data, const TextureView &texture) {
    const float sunElevation = data[6], sunRotation = data[7], angularDiameter = data[8], sunIntensity = data[9];
    const bool sunDisc = angularDiameter > 0.0f;
    float3 xyzc = f3(0.0f);
    const float theta = acosf(dir.z), phi = atan2f(dir.x, dir.y);  // sky_spherical_coordinates
    if (dir.z >= 0.0f) {
        const float lat = sunElevation, lon = sunRotation + 0.5f * M_PI_F;
        const float3 sunDir = make_float3(cosf(lat) * cosf(lon), cosf(lat) * sinf(lon), sinf(lat));
        const float sunAngle = 2.0f * atan2f(length(dir - sunDir), length(dir + sunDir));  // precise_angle
        const float halfAngular = angularDiameter / 2.0f;
        const float dirElevation = 0.5f * M_PI_F - theta;
        if (sunAngle < halfAngular && sunDisc) {
            const float3 bottom = make_float3(data[0], data[1], data[2]), top = make_float3(data[3], data[4], data[5]);
            if (sunElevation - halfAngular > 0.0f) {
                if (sunElevation + halfAngular > 0.0f) {
                    const float y = ((dirElevation - sunElevation) / angularDiameter) + 0.5f;
                    xyzc = (bottom + (top - bottom) * y) * sunIntensity;  // Metal mix
                }
            } else if (sunElevation + halfAngular > 0.0f) {
                const float y = dirElevation / (sunElevation + halfAngular);
                xyzc = (bottom + (top - bottom) * y) * sunIntensity;  // Metal mix
            }
            const float fraction = sunAngle / halfAngular;
            xyzc = xyzc * (1.0f - 0.6f * (1.0f - sqrtf(1.0f - fraction * fraction)));  // limb darkening
        } else {
            float x = (phi + M_PI_F + sunRotation) / (2.0f * M_PI_F);
            const float y = sqrtf(dirElevation / (0.5f * M_PI_F));
            if (x > 1.0f) x = x - 1.0f;
            xyzc = xyz(sampleLinearRepeat(texture, make_float2(x, y)));
        }
    } else if (dir.z >= -0.4f) {
        const float mul = powf(1.0f + dir.z * 2.5f, 3.0f);  // black ground fade
        float x = (phi + M_PI_F + sunRotation) / (2.0f * M_PI_F);
        if (x > 1.0f) x = x - 1.0f;
        xyzc = xyz(sampleLinearRepeat(texture, make_float2(x, 1e-3f))) * mul;
    }
    return xyz_to_rgb(xyzc);
}

// TexNishita (nodes.hpp:857-870); the texture slot holds the sky texture the
// scene generated from the node's parameters (MaterialBuilder.swift:350-388)
template <int TextureIndex>
struct TexNishita {
    float scale;
    float3 vector;
    float4 color;
    float data[10];
    RMD_HD void compute(const Context &ctx, const ShadingContext &shading) {
        color = f4(scale * skyRadianceNishita(shading.wo * make_float3(1.0f, -1.0f, -1.0f), data,
                                              ctx.textures[TextureIndex]),
                   1.0f);
    }
};

struct kMapping {
    enum Type { TYPE_MAPPING };  // the exporter writes the node's type, MAPPING, for every vector type
};
// nodes.hpp:346-364: vector = R(rotation) (vector * scale) + location, R the
// XYZ Euler rotation of math.hpp:46-68 (Cycles' node_mapping.osl)
template <kMapping::Type Type>
struct Mapping {
    float3 scale, rotation, location, vector;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        float sx, cx, sy, cy, sz, cz;
        sincosf(rotation.x, &sx, &cx);
        sincosf(rotation.y, &sy, &cy);
        sincosf(rotation.z, &sz, &cz);
        float3x3 r;
        r.c[0] = make_float3(cy * cz, cy * sz, -sy);
        r.c[1] = make_float3(sy * sx * cz - cx * sz, sy * sx * sz + cx * cz, cy * sx);
        r.c[2] = make_float3(sy * cx * cz + sx * sz, sy * cx * sz - sx * cz, cy * cx);
        vector = r * (vector * scale) + location;
    }
};

struct kNormalMap {
    enum Space { SPACE_TANGENT, SPACE_WORLD };
};
// nodes.hpp:1060-1097: the colour as a normal, blended towards +z by
// strength, in the shading point's (tu, tv, normal) frame (tangent space) or
// as it is (world space)
template <kNormalMap::Space Space>
struct NormalMap {
    float4 color;
    float strength;
    float3 normal;
    RMD_HD void compute(const Context &, const ShadingContext &sh) {
        const float s = fmaxf(strength, 0.0f);
        float3 n = normalize(2.0f * xyz(color) - f3(1.0f));
        n = normalize(s * n + (1.0f - s) * make_float3(0.0f, 0.0f, 1.0f));
        if (Space == kNormalMap::SPACE_TANGENT) n = sh.tu * n.x + sh.tv * n.y + sh.normal * n.z;
        normal = n;
    }
};

struct HueSaturation {  // nodes.hpp:1261-1277
    float4 color;
    float fac, hue, saturation, value;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        float3 hsv = rgb2hsv(xyz(color));
        hsv.x = fmodf(hsv.x + hue + 0.5f, 1.0f);
        hsv.y = saturate(hsv.y * saturation);
        hsv.z *= value;
        const float3 rgb = hsv2rgb(hsv);
        const float3 result = make_float3(fmaxf(rgb.x, 0.0f), fmaxf(rgb.y, 0.0f), fmaxf(rgb.z, 0.0f));
        color = f4(lerp(xyz(color), result, fac), color.w);
    }
};

struct BrightnessContrast {  // nodes.hpp:1279-1290 (alpha included, as there)
    float bright, contrast;
    float4 color;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        const float a = 1.0f + contrast, b = bright - contrast / 2.0f;
        color = make_float4(fmaxf(a * color.x + b, 0.0f), fmaxf(a * color.y + b, 0.0f), fmaxf(a * color.z + b, 0.0f),
                            fmaxf(a * color.w + b, 0.0f));
    }
};

// Blackbody colour: Cycles' piecewise fit over 800..12000 K, a / t + b t + c
// for red and green and a cubic in t for blue, one coefficient row per
// temperature band (the table of nodes.hpp:1421-1449, which must be the same
// numbers for the colours to match).
struct BlackbodyFit {
    float r[7][3], g[7][3], b[7][4];
};
__constant__ const BlackbodyFit kBlackbodyFit = {
    {{1.61919106e+03f, -2.05010916e-03f, 5.02995757e+00f},
     {2.48845471e+03f, -1.11330907e-03f, 3.22621544e+00f},
     {3.34143193e+03f, -4.86551192e-04f, 1.76486769e+00f},
     {4.09461742e+03f, -1.27446582e-04f, 7.25731635e-01f},
     {4.67028036e+03f, 2.91258199e-05f, 1.26703442e-01f},
     {4.59509185e+03f, 2.87495649e-05f, 1.50345020e-01f},
     {3.78717450e+03f, 9.35907826e-06f, 3.99075871e-01f}},
    {{-4.88999748e+02f, 6.04330754e-04f, -7.55807526e-02f},
     {-7.55994277e+02f, 3.16730098e-04f, 4.78306139e-01f},
     {-1.02363977e+03f, 1.20223470e-04f, 9.36662319e-01f},
     {-1.26571316e+03f, 4.87340896e-06f, 1.27054498e+00f},
     {-1.42529332e+03f, -4.01150431e-05f, 1.43972784e+00f},
     {-1.17554822e+03f, -2.16378048e-05f, 1.30408023e+00f},
     {-5.00799571e+02f, -4.59832026e-06f, 1.09098763e+00f}},
    {{5.96945309e-11f, -4.85742887e-08f, -9.70622247e-05f, -4.07936148e-03f},
     {2.40430366e-11f, 5.55021075e-08f, -1.98503712e-04f, 2.89312858e-02f},
     {-1.40949732e-11f, 1.89878968e-07f, -3.56632824e-04f, 9.10767778e-02f},
     {-3.61460868e-11f, 2.84822009e-07f, -4.93211319e-04f, 1.56723440e-01f},
     {-1.97075738e-11f, 1.75359352e-07f, -2.50542825e-04f, -2.22783266e-02f},
     {-1.61997957e-13f, -1.64216008e-08f, 3.86216271e-04f, -7.38077418e-01f},
     {6.72650283e-13f, -2.73078809e-08f, 4.24098264e-04f, -7.52335691e-01f}}};

struct Blackbody {  // nodes.hpp:1451-1495: the fit's colour divided by its luminance
    float temperature;
    float4 color;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        float3 c;
        const float t = temperature;
        if (t >= 12000.0f) {
            c = make_float3(0.8262954810464208f, 0.9945080501520986f, 1.566307710274283f);
        } else if (t < 800.0f) {
            c = make_float3(5.413294490189271f, -0.20319390035873933f, -0.0822535242887164f);
        } else {
            const int i = t >= 6365.0f ? 6 : t >= 3315.0f ? 5 : t >= 1902.0f ? 4 : t >= 1449.0f ? 3 :
                          t >= 1167.0f ? 2 : t >= 965.0f ? 1 : 0;
            const float *r = kBlackbodyFit.r[i], *g = kBlackbodyFit.g[i], *b = kBlackbodyFit.b[i];
            const float inv = 1.0f / t;
            c = make_float3(r[0] * inv + r[1] * t + r[2], g[0] * inv + g[1] * t + g[2],
                            ((b[0] * t + b[1]) * t + b[2]) * t + b[3]);
        }
        color = f4(c / luminance(c), 1.0f);
    }
};

struct Gamma {  // nodes.hpp:1292-1302
    float4 color;
    float gamma;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        if (gamma == 0.0f) {
            color.x = color.y = color.z = 1.0f;
        } else {
            if (color.x > 0.0f) color.x = powf(color.x, gamma);
            if (color.y > 0.0f) color.y = powf(color.y, gamma);
            if (color.z > 0.0f) color.z = powf(color.z, gamma);
        }
    }
};
struct Fresnel {  // nodes.hpp:1112-1126
    float ior;
    float3 normal;
    float fac;
    RMD_HD void compute(const Context &, const ShadingContext &sh) {
        const float cosI = dot(sh.wo, normal);
        const bool backfacing = cosI < 0.0f;
        float eta = fmaxf(ior, 1e-5f);
        eta = backfacing ? 1.0f / eta : eta;
        fac = fresnelDielectricCos(cosI, eta);
    }
};
struct LayerWeight {  // nodes.hpp:1689-1714
    float blend;
    float3 normal;
    float fresnel, facing;
    RMD_HD void compute(const Context &, const ShadingContext &sh) {
        const bool backfacing = dot(sh.wo, normal) < 0.0f;
        const float cosI = dot(sh.wo, normal);
        float eta = fmaxf(1.0f - blend, 1e-5f);
        eta = backfacing ? eta : 1.0f / eta;
        fresnel = fresnelDielectricCos(cosI, eta);
        facing = fabsf(cosI);
        if (blend != 0.5f) {
            float b = clampf(blend, 0.0f, 1.0f - 1e-5f);
            b = (b < 0.5f) ? 2.0f * b : 0.5f / (1.0f - b);
            facing = powf(facing, b);
        }
        facing = 1.0f - facing;
    }
};

// ---------------------------------------------------------------- shaders
struct Emission {  // nodes.hpp:1396-1407
    float4 color;
    float strength, weight;
    UberShader emission;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        emission.lobeProbabilities[0] = 1.0f;
        emission.emission = xyz(color) * strength;
    }
};
struct Background {  // nodes.hpp:1409-1419
    float4 color;
    float strength, weight;
    UberShader background;
    RMD_HD void compute(const Context &, const ShadingContext &) { background.emission = xyz(color) * strength; }
};
struct kBsdfPrincipled {
    enum Distribution { DISTRIBUTION_GGX };
    enum SubsurfaceMethod { SUBSURFACE_METHOD_BURLEY, SUBSURFACE_METHOD_RANDOM_WALK, SUBSURFACE_METHOD_RANDOM_WALK_FIXED_RADIUS };
};
template <int Distribution, int SubsurfaceMethod>
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

    RMD_HD void compute(const Context &, const ShadingContext &) {
        clearcoatRoughness = fmaxf(clearcoatRoughness, 1e-4f);
        roughness = fmaxf(roughness, 1e-4f);
        const float diffuseWeight = (1.0f - saturate(transmission)) * (1.0f - saturate(metallic));
        const float transmissionWeight = saturate(transmission) * (1.0f - saturate(metallic));
        const float specularWeight = 1.0f - transmissionWeight;
        const float3 base = xyz(baseColor);
        const float lum = luminance(base);
        const float3 tintColor = lum > 0.0f ? base * (1.0f / lum) : f3(1.0f);
        const float3 sheenColor = lerp(f3(1.0f), tintColor, sheenTint);
        const float3 specularColor = lerp(f3(1.0f), tintColor, specularTint);
        const float3 Cspec0 = lerp(specular * 0.08f * specularColor, base, metallic);
        const float aspect = sqrtf(1.0f - 0.9f * anisotropic);
        const float r2 = square(roughness);
        bsdf.diffuse = Diffuse{diffuseWeight * base, diffuseWeight * sheen * sheenColor, roughness, false};
        bsdf.specular = Specular{r2 / aspect, r2 * aspect, Cspec0, (2.0f / (1.0f - sqrtf(0.08f * specular))) - 1.0f,
                                 specularWeight};
        bsdf.transmission = Transmission{r2,
                                         square(1.0f - (1.0f - roughness) * (1.0f - transmissionRoughness)),
                                         base,
                                         lerp(f3(1.0f), base, specularTint),
                                         ior,
                                         transmissionWeight,
                                         false};
        bsdf.clearcoat = Clearcoat{square(clearcoatRoughness), clearcoat};
        bsdf.lobeProbabilities[0] = diffuseWeight;
        bsdf.lobeProbabilities[1] = specularWeight;
        bsdf.lobeProbabilities[2] = transmissionWeight;
        bsdf.lobeProbabilities[3] = clearcoat * 0.25f;
        float weightsSum = 0.0f;
        for (int i = 0; i < 4; i++) weightsSum += bsdf.lobeProbabilities[i];
        for (int i = 0; i < 4; i++) bsdf.lobeProbabilities[i] /= weightsSum;
        bsdf.alpha = alpha;
        bsdf.normal = normal;
        bsdf.emission = alpha * xyz(emission) * emissionStrength;
    }
};
struct BsdfDiffuse {  // nodes.hpp:1809-1827
    float4 color;
    float3 normal;
    float roughness, weight;
    UberShader bsdf;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        bsdf.diffuse = Diffuse{xyz(color), f3(0.0f), roughness, false};
        bsdf.normal = normal;
        bsdf.lobeProbabilities[0] = 1.0f;
    }
};
struct kBsdfGlossy {
    enum Distribution { DISTRIBUTION_GGX };
};
template <int Distribution>
struct BsdfGlossy {  // nodes.hpp:1534-1567
    float4 color;
    float3 normal;
    float roughness, weight;
    UberShader bsdf;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        const float a = square(fmaxf(roughness, 1e-4f));
        bsdf.specular = Specular{a, a, xyz(color), 1.45f, 1.0f};
        bsdf.lobeProbabilities[1] = 1.0f;
        bsdf.normal = normal;
    }
};
struct kBsdfGlass {
    enum Distribution { DISTRIBUTION_GGX };
};
template <int Distribution>
struct BsdfGlass {  // nodes.hpp:1497-1532
    float4 color;
    float ior;
    float3 normal;
    float roughness, weight;
    UberShader bsdf;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        const float a = square(fmaxf(roughness, 1e-4f));
        bsdf.transmission = Transmission{a, a, xyz(color), xyz(color), ior, 1.0f, false};
        bsdf.lobeProbabilities[2] = 1.0f;
        bsdf.normal = normal;
    }
};
struct BsdfTransparent {  // nodes.hpp:1797-1807
    float4 color;
    float weight;
    UberShader bsdf;
    RMD_HD void compute(const Context &, const ShadingContext &) {
        bsdf.alpha = 0.0f;
        bsdf.alphaWeight = xyz(color);
    }
};
struct AddShader {  // nodes.hpp:1895-1911
    UberShader shader, shader_001;
    RMD_HD void compute(const Context &, ShadingContext &sh) {
        const float3 em = shader_001.emission + shader.emission;
        if (sh.rnd.x < 0.5f) {
            sh.rnd.x /= 0.5f;
            shader = shader_001;
        } else {
            sh.rnd.x = 2.0f * (sh.rnd.x - 0.5f);
        }
        shader.emission = em;
        shader.weight *= 2.0f;
    }
};
struct MixShader {  // nodes.hpp:1916-1931
    float fac;
    UberShader shader, shader_001;
    RMD_HD void compute(const Context &, ShadingContext &sh) {
        const float3 em = fac * shader_001.emission + (1.0f - fac) * shader.emission;
        if (sh.rnd.x < fac) {
            sh.rnd.x /= fac;
            shader = shader_001;
        } else {
            sh.rnd.x = (sh.rnd.x - fac) / (1.0f - fac);
        }
        shader.emission = em;
    }
};
struct OutputMaterial {  // nodes.hpp:1976-1986
    float3 displacement;
    float thickness;
    UberShader surface, volume;
    RMD_HD void compute(const Context &, ShadingContext &sh) { sh.material = surface; }
};
struct OutputWorld {  // nodes.hpp:1988-1995
    float thickness;
    UberShader surface;
    RMD_HD void compute(const Context &, ShadingContext &sh) { sh.material = surface; }
};
struct OutputLight {  // nodes.hpp:1997-2005
    UberShader surface;
    RMD_HD void compute(const Context &, ShadingContext &sh) {
        sh.material.alpha = 0.0f;
        sh.material.emission = surface.emission;
    }
};

}  // namespace rmd
