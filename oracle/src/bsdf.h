// Oracle (test infrastructure only): the reference's Principled "UberShader"
// BSDF, restated from raymond/device/bsdf/** and raymond/device/utils/{math,warp}.hpp.
#pragma once
#include "vec.h"

namespace orc {

enum RayFlags : uint8_t {  // bridge/Ray.hpp:6-15
    RayFlagsCamera = 1 << 0,
    RayFlagsReflection = 1 << 1,
    RayFlagsTransmission = 1 << 2,
    RayFlagsShadow = 1 << 3,
    RayFlagsVolume = 1 << 4,
    RayFlagsDiffuse = 1 << 5,
    RayFlagsGlossy = 1 << 6,
    RayFlagsSingular = 1 << 7,
};

// ---------------------------------------------------------------- utils/math.hpp
// math.hpp:4-14 ("Building an Orthonormal Basis, Revisited", Duff et al. 2017)
inline float3x3 buildOrthonormalBasis(float3 n) {
    const float sign = std::copysign(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    float3x3 frame;
    frame[0] = float3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    frame[1] = float3(b, sign + n.y * n.y * a, -n.y);
    frame[2] = n;
    return frame;
}
inline float safe_sqrtf(float f) { return std::sqrt(std::max(f, 0.0f)); }   // math.hpp:16
inline float sqr(float f) { return f * f; }                                  // math.hpp:17
inline float safe_sqrt(float v) { return v <= 0 ? 0.0f : std::sqrt(v); }     // math.hpp:23
inline float lerp(float a, float b, float v) { return (1 - v) * a + v * b; } // math.hpp:29-30
inline float3 lerp(float3 a, float3 b, float v) { return (1 - v) * a + v * b; }
inline float4 lerp(float4 a, float4 b, float v) { return (1 - v) * a + v * b; }
inline float square(float v) { return v * v; }                               // math.hpp:35-36
inline float mean(float3 v) { return (v.x + v.y + v.z) / 3; }                // math.hpp:41

// math.hpp:73-119 (from Cycles kernel_montecarlo.h)
inline float3 ensure_valid_reflection(float3 Ng, float3 I, float3 N) {
    float3 R = 2 * dot(N, I) * N - I;
    float threshold = std::min(0.9f * dot(Ng, I), 0.01f);
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
        float2 N1 = float2(safe_sqrtf(1.0f - N1_z2), safe_sqrtf(N1_z2));
        float2 N2 = float2(safe_sqrtf(1.0f - N2_z2), safe_sqrtf(N2_z2));
        float R1 = 2 * (N1.x * Ix + N1.y * Iz) * N1.y - Iz;
        float R2 = 2 * (N2.x * Ix + N2.y * Iz) * N2.y - Iz;
        valid1 = (R1 >= 1e-5f);
        valid2 = (R2 >= 1e-5f);
        if (valid1 && valid2) {
            N_new = (R1 < R2) ? N1 : N2;
        } else {
            N_new = (R1 > R2) ? N1 : N2;
        }
    } else if (valid1 || valid2) {
        float Nz2 = valid1 ? N1_z2 : N2_z2;
        N_new = float2(safe_sqrtf(1.0f - Nz2), safe_sqrtf(Nz2));
    } else {
        return Ng;
    }
    return N_new.x * X + N_new.y * Ng;
}

// ---------------------------------------------------------------- utils/warp.hpp
namespace warp {
// warp.hpp:12-20
inline float3 uniformSquareToSphere(float2 uv) {
    float z = 1 - 2 * uv.y;
    float r = safe_sqrt(1 - z * z);
    float phi = 2 * M_PI_F * uv.x;
    return float3(r * std::cos(phi), r * std::sin(phi), z);
}
// warp.hpp:22-26
inline float2 uniformSphereToSquare(float3 v) {
    float y = (1 - v.z) / 2;
    float x = std::atan2(v.y, v.x) / (2 * M_PI_F);
    return float2(x < 0 ? x + 1 : x, y);
}
inline float uniformSquareToSpherePdf() { return 1 / (4 * M_PI_F); }  // warp.hpp:28-30
// warp.hpp:33-39
inline float2 uniformSquareToDisk(float2 uv) {
    float phi = 2 * M_PI_F * uv.x;
    float r = std::sqrt(uv.y);
    return float2(r * std::cos(phi), r * std::sin(phi));
}
// warp.hpp:46-54
inline float3 uniformSquareToCosineWeightedHemisphere(float2 rnd) {
    float cosTheta = std::sqrt(rnd.x);
    float sinTheta = std::sqrt(1 - square(cosTheta));
    float phi = 2 * M_PI_F * rnd.y;
    return float3(sinTheta * std::cos(phi), sinTheta * std::sin(phi), cosTheta);
}
// warp.hpp:56-59
inline float2 uniformSquareToTriangleBarycentric(float2 rnd) {
    float x = std::sqrt(rnd.x);
    return float2(1 - x, x * rnd.y);
}
}  // namespace warp

// ---------------------------------------------------------------- bsdf/*
// ShadingFrame.hpp:3-27
namespace frame {
inline float cosTheta(float3 w) { return w.z; }
inline float cosTheta2(float3 w) { return square(w.z); }
inline bool sameHemisphere(float3 wi, float3 wo) { return cosTheta(wi) * cosTheta(wo) > 0; }
inline float cosPhiSinTheta(float3 w) { return w.x; }
inline float sinPhiSinTheta(float3 w) { return w.y; }
inline float tanTheta2(float3 w) {
    const float cos2 = cosTheta2(w);
    return (1 - cos2) / cos2;
}
}  // namespace frame

// BsdfSample.hpp:3-16
struct BsdfSample {
    float pdf = 0;
    float3 wi;
    float3 weight;
    uint8_t flags = 0;
    static BsdfSample invalid() {
        BsdfSample r;
        r.pdf = 0;
        r.weight = float3(0.0f);
        r.flags = 0;
        return r;
    }
};

// fresnel.hpp:3-6
inline float schlickWeight(float cosTheta) {
    float m = saturate(1 - cosTheta);
    return (m * m) * (m * m) * m;
}
// fresnel.hpp:43-53
inline float fresnelDielectricCos(float cosi, float eta) {
    float c = std::fabs(cosi);
    float g = eta * eta - 1 + c * c;
    if (g > 0) {
        g = std::sqrt(g);
        float A = (g - c) / (g + c);
        float B = (c * (g + c) - 1) / (c * (g - c) + 1);
        return 0.5f * A * A * (1 + B * B);
    }
    return 1.0f;
}
// fresnel.hpp:55-64
inline float3 interpolateFresnel(float3 wi, float3 wh, float ior, float F0, float3 cspec0) {
    float F0_norm = 1 / (1 - F0);
    float FH = (fresnelDielectricCos(dot(wi, wh), ior) - F0) * F0_norm;
    return cspec0 * (1 - FH) + float3(1.0f) * FH;
}
inline float3 fresnelReflectionColor(float3 wi, float3 wh, float ior, float3 Cspec0) {
    float F0 = fresnelDielectricCos(1, ior);
    return interpolateFresnel(wi, wh, ior, F0, Cspec0);
}

// microfacet.hpp:55-67
inline float anisotropicSmithG1(float3 w, float3 wh, float ax, float ay) {
    if (dot(w, wh) * frame::cosTheta(w) * frame::cosTheta(wh) <= 0) return 0;
    if (std::fabs(frame::cosTheta(w)) >= 1) return 1;
    const float a2tanTheta2 =
        (square(ax * frame::cosPhiSinTheta(w)) + square(ay * frame::sinPhiSinTheta(w))) / frame::cosTheta2(w);
    return 2 / (1 + std::sqrt(1 + a2tanTheta2));
}
// microfacet.hpp:39-48
inline float smithG1(float3 w, float3 wh, float a) {
    if (dot(w, wh) * frame::cosTheta(w) * frame::cosTheta(wh) <= 0) return 0;
    if (std::fabs(frame::cosTheta(w)) >= 1) return 1;
    const float a2tanTheta2 = square(a) * frame::tanTheta2(w);
    return 2 / (1 + std::sqrt(1 + a2tanTheta2));
}
// microfacet.hpp:73-79
inline float anisotropicGGX(float3 wh, float ax, float ay) {
    float nDotH = frame::cosTheta(wh);
    float a = frame::cosPhiSinTheta(wh) / ax;
    float b = frame::sinPhiSinTheta(wh) / ay;
    float c = square(a) + square(b) + square(nDotH);
    return 1 / (M_PI_F * ax * ay * square(c));
}
// microfacet.hpp:87-108 (Heitz 2018 VNDF sampling)
inline float3 sampleGGXVNDF(float2 rnd, float ax, float ay, float3 wo) {
    float sgn = signf(frame::cosTheta(wo));
    float3 Vh = sgn * normalize(float3(ax * wo.x, ay * wo.y, wo.z));
    float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    float3 T1 = lensq > 0 ? float3(-Vh.y, Vh.x, 0) * (1.0f / std::sqrt(lensq)) : float3(1, 0, 0);
    float3 T2 = cross(Vh, T1);
    float r = std::sqrt(rnd.x);
    float phi = 2.0f * M_PI_F * rnd.y;
    float t1 = r * std::cos(phi);
    float t2 = r * std::sin(phi);
    float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * std::sqrt(1.0f - t1 * t1) + s * t2;
    float3 Nh = t1 * T1 + t2 * T2 + std::sqrt(std::max(0.0f, 1.0f - t1 * t1 - t2 * t2)) * Vh;
    float3 Ne = normalize(float3(ax * Nh.x, ay * Nh.y, std::max(0.f, Nh.z)));
    return sgn * Ne;
}

// lobes/Diffuse.hpp:14-96
struct Diffuse {
    float3 diffuseWeight = float3(0.0f);
    float3 sheenWeight = float3(0.0f);
    float roughness = 0;
    bool translucent = false;

    float3 evaluate(float3 wo, float3 wi, float &pdf) const {
        if (frame::sameHemisphere(wi, wo) == translucent) {
            pdf = 0;
            return float3(0.0f);
        }
        const float NdotL = std::fabs(frame::cosTheta(wi));
        pdf = M_1_PI_F * NdotL;
        const float NdotV = std::fabs(frame::cosTheta(wo));
        const float LdotV = dot(wi, wo);
        const float FL = schlickWeight(NdotL);
        const float FV = schlickWeight(NdotV);
        const float lambertian = (1.0f - 0.5f * FV) * (1.0f - 0.5f * FL);
        const float LH2 = LdotV + 1;
        const float RR = roughness * LH2;
        const float retroReflection = RR * (FL + FV + FL * FV * (RR - 1.0f));
        const float3 wh = normalize(wo + wi);
        const float LdotH = std::fabs(dot(wh, wi));
        const float sheen = schlickWeight(LdotH);
        return pdf * (diffuseWeight * (lambertian + retroReflection) + sheenWeight * (M_PI_F * sheen));
    }
    BsdfSample sample(float2 rnd, float3 wo) const {
        BsdfSample result;
        result.wi = warp::uniformSquareToCosineWeightedHemisphere(rnd);
        if (!frame::sameHemisphere(result.wi, wo)) result.wi *= -1.0f;
        const float NdotL = std::fabs(frame::cosTheta(result.wi));
        result.pdf = M_1_PI_F * NdotL;
        if (!(result.pdf > 0)) return BsdfSample::invalid();
        const float NdotV = std::fabs(frame::cosTheta(wo));
        const float LdotV = dot(result.wi, wo);
        const float FL = schlickWeight(NdotL);
        const float FV = schlickWeight(NdotV);
        const float lambertian = (1.0f - 0.5f * FV) * (1.0f - 0.5f * FL);
        const float LH2 = LdotV + 1;
        const float RR = roughness * LH2;
        const float retroReflection = RR * (FL + FV + FL * FV * (RR - 1.0f));
        const float3 wh = normalize(wo + result.wi);
        const float LdotH = std::fabs(dot(wh, result.wi));
        const float sheen = schlickWeight(LdotH);
        result.weight = diffuseWeight * (lambertian + retroReflection) + sheenWeight * (M_PI_F * sheen);
        if (translucent) {
            result.wi = -result.wi;
            result.flags = RayFlagsTransmission | RayFlagsDiffuse;
        } else {
            result.flags = RayFlagsReflection | RayFlagsDiffuse;
        }
        return result;
    }
};

// lobes/Specular.hpp:15-67 (evaluate omits `weight`, sample includes it: kept)
struct Specular {
    float alphaX = 0;
    float alphaY = 0;
    float3 Cspec0;
    float ior = 0;
    float weight = 0;

    float3 evaluate(float3 wo, float3 wi, float &pdf) const {
        const float3 wh = normalize(wi + wo);
        pdf = anisotropicGGX(wh, alphaX, alphaY) * anisotropicSmithG1(wo, wh, alphaX, alphaY) *
              std::fabs(dot(wo, wh) / frame::cosTheta(wo));
        if (!(pdf > 0)) {
            pdf = 0;
            return float3(0.0f);
        }
        pdf *= 1 / std::fabs(4 * dot(wo, wh));
        const float3 F = fresnelReflectionColor(wi, wh, ior, Cspec0);
        const float G = anisotropicSmithG1(wi, wh, alphaX, alphaY) * anisotropicSmithG1(wo, wh, alphaX, alphaY);
        const float D = anisotropicGGX(wh, alphaX, alphaY);
        return F * D * G / std::fabs(4 * frame::cosTheta(wo));
    }
    BsdfSample sample(float2 rnd, float3 wo) const {
        BsdfSample result;
        const float3 wh = sampleGGXVNDF(rnd, alphaX, alphaY, wo);
        result.pdf = anisotropicGGX(wh, alphaX, alphaY) * anisotropicSmithG1(wo, wh, alphaX, alphaY) *
                     std::fabs(dot(wo, wh) / frame::cosTheta(wo));
        if (!(result.pdf > 0)) return BsdfSample::invalid();
        result.wi = reflect(-wo, wh);
        if (!frame::sameHemisphere(result.wi, wo)) return BsdfSample::invalid();
        result.pdf *= 1 / std::fabs(4 * dot(wo, wh));
        const float3 F = fresnelReflectionColor(result.wi, wh, ior, Cspec0);
        const float Gi = anisotropicSmithG1(result.wi, wh, alphaX, alphaY);
        result.weight = weight * F * Gi;
        result.flags = RayFlagsReflection | RayFlagsGlossy;
        return result;
    }
};

// lobes/Transmission.hpp:15-123
struct Transmission {
    float reflectionAlpha = 0;
    float transmissionAlpha = 0;
    float3 baseColor;
    float3 Cspec0;
    float ior = 0;
    float weight = 0;
    bool onlyRefract = false;

    float3 evaluate(float3 wo, float3 wi, float &pdf) const {
        const bool isReflection = frame::sameHemisphere(wi, wo);
        if (onlyRefract && isReflection) {
            pdf = 0;
            return float3(0.0f);
        }
        const float eta = frame::cosTheta(wo) > 0 ? ior : 1 / ior;
        const float3 wh = isReflection ? normalize(wi + wo) : normalize(wi * eta + wo);
        const float alpha = isReflection ? reflectionAlpha : transmissionAlpha;
        pdf = anisotropicGGX(wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha) *
              std::fabs(dot(wo, wh) / frame::cosTheta(wo));
        if (!(pdf > 0)) {
            pdf = 0;
            return float3(0.0f);
        }
        const float Gi = anisotropicSmithG1(wi, wh, alpha, alpha);
        const float Fr = onlyRefract ? 0 : fresnelDielectricCos(frame::cosTheta(wo), eta);
        if (isReflection) {
            pdf *= Fr;
            pdf *= 1 / std::fabs(4 * dot(wo, wh));
            const float3 F = fresnelReflectionColor(wi, wh, eta, Cspec0);
            return pdf * weight * F * Gi;
        } else {
            pdf *= 1 - Fr;
            pdf *= std::fabs(dot(wi, wh) / square(dot(wi, wh) + dot(wh, wo) / eta));
            return pdf * weight * baseColor * Gi;
        }
    }
    BsdfSample sample(float2 rnd, float3 wo) const {
        BsdfSample result;
        float eta = frame::cosTheta(wo) > 0 ? ior : 1 / ior;
        const float Fr = onlyRefract ? 0 : fresnelDielectricCos(frame::cosTheta(wo), eta);
        const bool isReflection = rnd.x < Fr;
        const float alpha = isReflection ? reflectionAlpha : transmissionAlpha;
        const float3 wh = sampleGGXVNDF(rnd, alpha, alpha, wo);
        result.pdf = anisotropicGGX(wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha) *
                     std::fabs(dot(wo, wh) / frame::cosTheta(wo));
        if (isReflection) {
            rnd.x /= Fr;
            if (!(result.pdf > 0)) return BsdfSample::invalid();
            result.wi = reflect(-wo, wh);
            if (!frame::sameHemisphere(result.wi, wo)) return BsdfSample::invalid();
            result.pdf *= Fr;
            result.pdf *= 1 / std::fabs(4 * dot(wo, wh));
            const float3 F = fresnelReflectionColor(result.wi, wh, eta, Cspec0);
            const float Gi = anisotropicSmithG1(result.wi, wh, alpha, alpha);
            result.weight = weight * F * Gi;
            result.flags = RayFlagsReflection | RayFlagsGlossy;
            return result;
        } else {
            rnd.x = (rnd.x - Fr) / (1 - Fr);
            if (!(result.pdf > 0)) return BsdfSample::invalid();
            result.wi = refract(-wo, wh, 1 / eta);
            if (frame::sameHemisphere(result.wi, wo)) return BsdfSample::invalid();
            result.pdf *= 1 - Fr;
            result.pdf *= std::fabs(dot(result.wi, wh) / square(dot(result.wi, wh) + dot(wh, wo) / eta));
            const float Gi = anisotropicSmithG1(result.wi, wh, alpha, alpha);
            result.weight = weight * baseColor * Gi;
            result.flags = RayFlagsTransmission | RayFlagsGlossy;
            return result;
        }
    }
};

// lobes/Clearcoat.hpp:15-63
struct Clearcoat {
    float alpha = 0;
    float weight = 0;

    float3 evaluate(float3 wo, float3 wi, float &pdf) const {
        const float3 wh = normalize(wi + wo);
        pdf = anisotropicGGX(wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha) *
              std::fabs(dot(wo, wh) / frame::cosTheta(wo));
        if (!(pdf > 0)) {
            pdf = 0;
            return float3(0.0f);
        }
        pdf *= 1 / std::fabs(4 * dot(wo, wh));
        const float3 F = fresnelReflectionColor(wi, wh, 1.5f, float3(0.04f));
        const float G = anisotropicSmithG1(wi, wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha);
        const float D = anisotropicGGX(wh, alpha, alpha);
        return 0.25f * F * D * G / std::fabs(4 * frame::cosTheta(wo));
    }
    BsdfSample sample(float2 rnd, float3 wo) const {
        BsdfSample result;
        const float3 wh = sampleGGXVNDF(rnd, alpha, alpha, wo);
        result.pdf = anisotropicGGX(wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha) *
                     std::fabs(dot(wo, wh) / frame::cosTheta(wo));
        if (!(result.pdf > 0)) return BsdfSample::invalid();
        result.wi = reflect(-wo, wh);
        if (!frame::sameHemisphere(result.wi, wo)) return BsdfSample::invalid();
        result.pdf *= 1 / std::fabs(4 * dot(wo, wh));
        const float3 F = fresnelReflectionColor(result.wi, wh, 1.5f, float3(0.04f));
        const float Gi = smithG1(result.wi, wh, alpha);
        result.weight = 0.25f * weight * F * Gi;
        result.flags = RayFlagsReflection | RayFlagsGlossy;
        return result;
    }
};

// UberShader.hpp:10-146
struct UberShader {
    float3 normal;
    float lobeProbabilities[4] = {0, 0, 0, 0};
    Diffuse diffuse;
    Specular specular;
    Transmission transmission;
    Clearcoat clearcoat;
    float alpha = 1;
    float3 alphaWeight = float3(1.0f);
    float3 emission = float3(0.0f);
    float weight = 1;

    // UberShader.hpp:43-83
    float3 evaluate(float3 wo, float3 wi, float3 shNormal, float3 geoNormal, float &pdf, bool isLocal = false) const {
        pdf = 0;
        if (!isLocal) {
            float3x3 worldToShadingFrame = buildOrthonormalBasis(shNormal);
            const float woDotGeoN = dot(wo, geoNormal);
            wo = wo * worldToShadingFrame;
            const float woDotShN = wo.z;
            if (woDotShN * woDotGeoN < 0) return float3(0.0f);
            const float wiDotGeoN = dot(wi, geoNormal);
            wi = wi * worldToShadingFrame;
            const float wiDotShN = wi.z;
            if (wiDotShN * wiDotGeoN < 0) return float3(0.0f);
        }
        float3 value(0.0f);
        float lobePdf;
        if (lobeProbabilities[0] > 0) {
            value += diffuse.evaluate(wo, wi, lobePdf);
            pdf += lobeProbabilities[0] * lobePdf;
        }
        if (lobeProbabilities[1] > 0) {
            value += specular.evaluate(wo, wi, lobePdf);
            pdf += lobeProbabilities[1] * lobePdf;
        }
        if (lobeProbabilities[2] > 0) {
            value += transmission.evaluate(wo, wi, lobePdf);
            pdf += lobeProbabilities[2] * lobePdf;
        }
        if (lobeProbabilities[3] > 0) {
            value += clearcoat.evaluate(wo, wi, lobePdf);
            pdf += lobeProbabilities[3] * lobePdf;
        }
        pdf *= alpha;
        value *= this->weight * alpha;
        return value;
    }

    // UberShader.hpp:85-145
    BsdfSample sample(float3 rnd, float3 wo, float3 shNormal, float3 geoNormal, uint8_t previousFlags) const {
        if (rnd.x < alpha) {
            rnd.x /= alpha;
        } else {
            BsdfSample s;
            s.weight = alphaWeight * weight;
            s.wi = -wo;
            s.pdf = 1;
            s.flags = (uint8_t)(previousFlags | RayFlagsSingular);
            return s;
        }
        float3x3 worldToShadingFrame = buildOrthonormalBasis(shNormal);
        const float woDotGeoN = dot(wo, geoNormal);
        wo = wo * worldToShadingFrame;
        const float woDotShN = wo.z;
        if (woDotShN * woDotGeoN < 0) return BsdfSample::invalid();

        int selectedLobe;
        BsdfSample s;
        float2 rndyz = rnd.yz();
        if (rnd.x < lobeProbabilities[0]) {
            selectedLobe = 0;
            s = diffuse.sample(rndyz, wo);
        } else if (rnd.x < (lobeProbabilities[0] + lobeProbabilities[1])) {
            selectedLobe = 1;
            s = specular.sample(rndyz, wo);
        } else if (rnd.x < (lobeProbabilities[0] + lobeProbabilities[1] + lobeProbabilities[2])) {
            selectedLobe = 2;
            s = transmission.sample(rndyz, wo);
        } else {
            selectedLobe = 3;
            s = clearcoat.sample(rndyz, wo);
        }
        if (!std::isfinite(lobeProbabilities[selectedLobe])) return BsdfSample::invalid();
        if (lobeProbabilities[selectedLobe] < 1) {
            s.weight = evaluate(wo, s.wi, shNormal, geoNormal, s.pdf, true);
            s.weight /= s.pdf;
        } else {
            s.pdf *= alpha;
            s.weight *= this->weight * alpha;
        }
        const float wiDotShN = s.wi.z;
        s.wi = s.wi * transpose(worldToShadingFrame);
        const float wiDotGeoN = dot(s.wi, geoNormal);
        if (wiDotShN * wiDotGeoN < 0) return BsdfSample::invalid();
        return s;
    }
};

}  // namespace orc
