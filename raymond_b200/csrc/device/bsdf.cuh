// The reference's Principled "UberShader" (raymond/device/bsdf/**): four lobes
// (diffuse + sheen, anisotropic GGX specular, rough dielectric transmission,
// GTR1/GGX clearcoat), alpha / null scattering, evaluate and sample.
#pragma once
#include "rt_math.cuh"

namespace rmd {

enum : uint8_t {  // RayFlags, bridge/Ray.hpp:6-15
    RayFlagsCamera = 1 << 0,
    RayFlagsReflection = 1 << 1,
    RayFlagsTransmission = 1 << 2,
    RayFlagsShadow = 1 << 3,
    RayFlagsVolume = 1 << 4,
    RayFlagsDiffuse = 1 << 5,
    RayFlagsGlossy = 1 << 6,
    RayFlagsSingular = 1 << 7,
};

namespace frame {  // ShadingFrame.hpp:3-27
RMD_HD float cosTheta(float3 w) { return w.z; }
RMD_HD float cosTheta2(float3 w) { return square(w.z); }
RMD_HD bool sameHemisphere(float3 wi, float3 wo) { return cosTheta(wi) * cosTheta(wo) > 0.0f; }
RMD_HD float tanTheta2(float3 w) {
    const float cos2 = cosTheta2(w);
    return (1.0f - cos2) / cos2;
}
}  // namespace frame

struct BsdfSample {  // BsdfSample.hpp:3-16
    float pdf;
    float3 wi;
    float3 weight;
    uint8_t flags;
    RMD_HD static BsdfSample invalid() {
        BsdfSample r;
        r.pdf = 0.0f;
        r.wi = f3(0.0f);
        r.weight = f3(0.0f);
        r.flags = 0;
        return r;
    }
};

// fresnel.hpp:3-64
RMD_HD float schlickWeight(float cosTheta) {
    float m = saturate(1.0f - cosTheta);
    return (m * m) * (m * m) * m;
}
RMD_HD float fresnelDielectricCos(float cosi, float eta) {
    float c = fabsf(cosi);
    float g = eta * eta - 1.0f + c * c;
    if (g > 0.0f) {
        g = sqrtf(g);
        float A = (g - c) / (g + c);
        float B = (c * (g + c) - 1.0f) / (c * (g - c) + 1.0f);
        return 0.5f * A * A * (1.0f + B * B);
    }
    return 1.0f;
}
RMD_HD float3 fresnelReflectionColor(float3 wi, float3 wh, float ior, float3 Cspec0) {
    float F0 = fresnelDielectricCos(1.0f, ior);
    float F0_norm = 1.0f / (1.0f - F0);
    float FH = (fresnelDielectricCos(dot(wi, wh), ior) - F0) * F0_norm;
    return Cspec0 * (1.0f - FH) + f3(1.0f) * FH;
}

// microfacet.hpp:39-108
RMD_HD float smithG1(float3 w, float3 wh, float a) {
    if (dot(w, wh) * frame::cosTheta(w) * frame::cosTheta(wh) <= 0.0f) return 0.0f;
    if (fabsf(frame::cosTheta(w)) >= 1.0f) return 1.0f;
    const float a2tanTheta2 = square(a) * frame::tanTheta2(w);
    return 2.0f / (1.0f + sqrtf(1.0f + a2tanTheta2));
}
RMD_HD float anisotropicSmithG1(float3 w, float3 wh, float ax, float ay) {
    if (dot(w, wh) * frame::cosTheta(w) * frame::cosTheta(wh) <= 0.0f) return 0.0f;
    if (fabsf(frame::cosTheta(w)) >= 1.0f) return 1.0f;
    const float a2tanTheta2 = (square(ax * w.x) + square(ay * w.y)) / frame::cosTheta2(w);
    return 2.0f / (1.0f + sqrtf(1.0f + a2tanTheta2));
}
RMD_HD float anisotropicGGX(float3 wh, float ax, float ay) {
    float a = wh.x / ax;
    float b = wh.y / ay;
    float c = square(a) + square(b) + square(wh.z);
    return 1.0f / (M_PI_F * ax * ay * square(c));
}
RMD_HD float3 sampleGGXVNDF(float2 rnd, float ax, float ay, float3 wo) {
    float sgn = signf(frame::cosTheta(wo));
    float3 Vh = sgn * normalize(make_float3(ax * wo.x, ay * wo.y, wo.z));
    float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    float3 T1 = lensq > 0.0f ? make_float3(-Vh.y, Vh.x, 0.0f) * (1.0f / sqrtf(lensq)) : make_float3(1.0f, 0.0f, 0.0f);
    float3 T2 = cross(Vh, T1);
    float r = sqrtf(rnd.x);
    float s_, c_;
    sincosf(2.0f * M_PI_F * rnd.y, &s_, &c_);
    float t1 = r * c_;
    float t2 = r * s_;
    float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
    float3 Nh = t1 * T1 + t2 * T2 + sqrtf(fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2)) * Vh;
    float3 Ne = normalize(make_float3(ax * Nh.x, ay * Nh.y, fmaxf(0.0f, Nh.z)));
    return sgn * Ne;
}

// lobes/Diffuse.hpp:14-96
struct Diffuse {
    float3 diffuseWeight;
    float3 sheenWeight;
    float roughness;
    bool translucent;

    RMD_HD float3 value(float3 wo, float3 wi, float NdotL) const {
        const float NdotV = fabsf(frame::cosTheta(wo));
        const float LdotV = dot(wi, wo);
        const float FL = schlickWeight(NdotL);
        const float FV = schlickWeight(NdotV);
        const float lambertian = (1.0f - 0.5f * FV) * (1.0f - 0.5f * FL);
        const float LH2 = LdotV + 1.0f;
        const float RR = roughness * LH2;
        const float retroReflection = RR * (FL + FV + FL * FV * (RR - 1.0f));
        const float3 wh = normalize(wo + wi);
        const float LdotH = fabsf(dot(wh, wi));
        const float sheen = schlickWeight(LdotH);
        return diffuseWeight * (lambertian + retroReflection) + sheenWeight * (M_PI_F * sheen);
    }
    RMD_HD float3 evaluate(float3 wo, float3 wi, float &pdf) const {
        if (frame::sameHemisphere(wi, wo) == translucent) {
            pdf = 0.0f;
            return f3(0.0f);
        }
        const float NdotL = fabsf(frame::cosTheta(wi));
        pdf = M_1_PI_F * NdotL;
        return pdf * value(wo, wi, NdotL);
    }
    RMD_HD BsdfSample sample(float2 rnd, float3 wo) const {
        BsdfSample result;
        result.wi = warp::uniformSquareToCosineWeightedHemisphere(rnd);
        if (!frame::sameHemisphere(result.wi, wo)) result.wi *= -1.0f;
        const float NdotL = fabsf(frame::cosTheta(result.wi));
        result.pdf = M_1_PI_F * NdotL;
        if (!(result.pdf > 0.0f)) return BsdfSample::invalid();
        result.weight = value(wo, result.wi, NdotL);
        if (translucent) {
            result.wi = -result.wi;
            result.flags = RayFlagsTransmission | RayFlagsDiffuse;
        } else {
            result.flags = RayFlagsReflection | RayFlagsDiffuse;
        }
        return result;
    }
};

// lobes/Specular.hpp:15-67 (evaluate omits `weight`, sample applies it: kept)
struct Specular {
    float alphaX;
    float alphaY;
    float3 Cspec0;
    float ior;
    float weight;

    RMD_HD float3 evaluate(float3 wo, float3 wi, float &pdf) const {
        const float3 wh = normalize(wi + wo);
        pdf = anisotropicGGX(wh, alphaX, alphaY) * anisotropicSmithG1(wo, wh, alphaX, alphaY) *
              fabsf(dot(wo, wh) / frame::cosTheta(wo));
        if (!(pdf > 0.0f)) {
            pdf = 0.0f;
            return f3(0.0f);
        }
        pdf *= 1.0f / fabsf(4.0f * dot(wo, wh));
        const float3 F = fresnelReflectionColor(wi, wh, ior, Cspec0);
        const float G = anisotropicSmithG1(wi, wh, alphaX, alphaY) * anisotropicSmithG1(wo, wh, alphaX, alphaY);
        const float D = anisotropicGGX(wh, alphaX, alphaY);
        return F * D * G / fabsf(4.0f * frame::cosTheta(wo));
    }
    RMD_HD BsdfSample sample(float2 rnd, float3 wo) const {
        BsdfSample result;
        const float3 wh = sampleGGXVNDF(rnd, alphaX, alphaY, wo);
        result.pdf = anisotropicGGX(wh, alphaX, alphaY) * anisotropicSmithG1(wo, wh, alphaX, alphaY) *
                     fabsf(dot(wo, wh) / frame::cosTheta(wo));
        if (!(result.pdf > 0.0f)) return BsdfSample::invalid();
        result.wi = reflect(-wo, wh);
        if (!frame::sameHemisphere(result.wi, wo)) return BsdfSample::invalid();
        result.pdf *= 1.0f / fabsf(4.0f * dot(wo, wh));
        const float3 F = fresnelReflectionColor(result.wi, wh, ior, Cspec0);
        const float Gi = anisotropicSmithG1(result.wi, wh, alphaX, alphaY);
        result.weight = weight * F * Gi;
        result.flags = RayFlagsReflection | RayFlagsGlossy;
        return result;
    }
};

// lobes/Transmission.hpp:15-123
struct Transmission {
    float reflectionAlpha;
    float transmissionAlpha;
    float3 baseColor;
    float3 Cspec0;
    float ior;
    float weight;
    bool onlyRefract;

    RMD_HD float3 evaluate(float3 wo, float3 wi, float &pdf) const {
        const bool isReflection = frame::sameHemisphere(wi, wo);
        if (onlyRefract && isReflection) {
            pdf = 0.0f;
            return f3(0.0f);
        }
        const float eta = frame::cosTheta(wo) > 0.0f ? ior : 1.0f / ior;
        const float3 wh = isReflection ? normalize(wi + wo) : normalize(wi * eta + wo);
        const float alpha = isReflection ? reflectionAlpha : transmissionAlpha;
        pdf = anisotropicGGX(wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha) *
              fabsf(dot(wo, wh) / frame::cosTheta(wo));
        if (!(pdf > 0.0f)) {
            pdf = 0.0f;
            return f3(0.0f);
        }
        const float Gi = anisotropicSmithG1(wi, wh, alpha, alpha);
        const float Fr = onlyRefract ? 0.0f : fresnelDielectricCos(frame::cosTheta(wo), eta);
        if (isReflection) {
            pdf *= Fr;
            pdf *= 1.0f / fabsf(4.0f * dot(wo, wh));
            const float3 F = fresnelReflectionColor(wi, wh, eta, Cspec0);
            return pdf * weight * F * Gi;
        }
        pdf *= 1.0f - Fr;
        pdf *= fabsf(dot(wi, wh) / square(dot(wi, wh) + dot(wh, wo) / eta));
        return pdf * weight * baseColor * Gi;
    }
    RMD_HD BsdfSample sample(float2 rnd, float3 wo) const {
        BsdfSample result;
        float eta = frame::cosTheta(wo) > 0.0f ? ior : 1.0f / ior;
        const float Fr = onlyRefract ? 0.0f : fresnelDielectricCos(frame::cosTheta(wo), eta);
        const bool isReflection = rnd.x < Fr;
        const float alpha = isReflection ? reflectionAlpha : transmissionAlpha;
        const float3 wh = sampleGGXVNDF(rnd, alpha, alpha, wo);
        result.pdf = anisotropicGGX(wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha) *
                     fabsf(dot(wo, wh) / frame::cosTheta(wo));
        if (!(result.pdf > 0.0f)) return BsdfSample::invalid();
        if (isReflection) {
            result.wi = reflect(-wo, wh);
            if (!frame::sameHemisphere(result.wi, wo)) return BsdfSample::invalid();
            result.pdf *= Fr;
            result.pdf *= 1.0f / fabsf(4.0f * dot(wo, wh));
            const float3 F = fresnelReflectionColor(result.wi, wh, eta, Cspec0);
            const float Gi = anisotropicSmithG1(result.wi, wh, alpha, alpha);
            result.weight = weight * F * Gi;
            result.flags = RayFlagsReflection | RayFlagsGlossy;
            return result;
        }
        result.wi = refract(-wo, wh, 1.0f / eta);
        if (frame::sameHemisphere(result.wi, wo)) return BsdfSample::invalid();
        result.pdf *= 1.0f - Fr;
        result.pdf *= fabsf(dot(result.wi, wh) / square(dot(result.wi, wh) + dot(wh, wo) / eta));
        const float Gi = anisotropicSmithG1(result.wi, wh, alpha, alpha);
        result.weight = weight * baseColor * Gi;
        result.flags = RayFlagsTransmission | RayFlagsGlossy;
        return result;
    }
};

// lobes/Clearcoat.hpp:15-63
struct Clearcoat {
    float alpha;
    float weight;

    RMD_HD float3 evaluate(float3 wo, float3 wi, float &pdf) const {
        const float3 wh = normalize(wi + wo);
        pdf = anisotropicGGX(wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha) *
              fabsf(dot(wo, wh) / frame::cosTheta(wo));
        if (!(pdf > 0.0f)) {
            pdf = 0.0f;
            return f3(0.0f);
        }
        pdf *= 1.0f / fabsf(4.0f * dot(wo, wh));
        const float3 F = fresnelReflectionColor(wi, wh, 1.5f, f3(0.04f));
        const float G = anisotropicSmithG1(wi, wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha);
        const float D = anisotropicGGX(wh, alpha, alpha);
        return 0.25f * F * D * G / fabsf(4.0f * frame::cosTheta(wo));
    }
    RMD_HD BsdfSample sample(float2 rnd, float3 wo) const {
        BsdfSample result;
        const float3 wh = sampleGGXVNDF(rnd, alpha, alpha, wo);
        result.pdf = anisotropicGGX(wh, alpha, alpha) * anisotropicSmithG1(wo, wh, alpha, alpha) *
                     fabsf(dot(wo, wh) / frame::cosTheta(wo));
        if (!(result.pdf > 0.0f)) return BsdfSample::invalid();
        result.wi = reflect(-wo, wh);
        if (!frame::sameHemisphere(result.wi, wo)) return BsdfSample::invalid();
        result.pdf *= 1.0f / fabsf(4.0f * dot(wo, wh));
        const float3 F = fresnelReflectionColor(result.wi, wh, 1.5f, f3(0.04f));
        const float Gi = smithG1(result.wi, wh, alpha);
        result.weight = 0.25f * weight * F * Gi;
        result.flags = RayFlagsReflection | RayFlagsGlossy;
        return result;
    }
};

// UberShader.hpp:10-146.  Default-constructed state equals the reference's
// default member initializers (zero lobes, alpha 1, weight 1, no emission).
struct UberShader {
    float3 normal = {0.0f, 0.0f, 0.0f};
    float lobeProbabilities[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    Diffuse diffuse = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, 0.0f, false};
    Specular specular = {0.0f, 0.0f, {0.0f, 0.0f, 0.0f}, 0.0f, 0.0f};
    Transmission transmission = {0.0f, 0.0f, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, 0.0f, 0.0f, false};
    Clearcoat clearcoat = {0.0f, 0.0f};
    float alpha = 1.0f;
    float3 alphaWeight = {1.0f, 1.0f, 1.0f};
    float3 emission = {0.0f, 0.0f, 0.0f};
    float weight = 1.0f;

    // UberShader.hpp:43-83 (wo, wi already in the shading frame)
    RMD_HD float3 evaluateLocal(float3 wo, float3 wi, float &pdf) const {
        pdf = 0.0f;
        float3 value = f3(0.0f);
        float lobePdf;
        if (lobeProbabilities[0] > 0.0f) {
            value += diffuse.evaluate(wo, wi, lobePdf);
            pdf += lobeProbabilities[0] * lobePdf;
        }
        if (lobeProbabilities[1] > 0.0f) {
            value += specular.evaluate(wo, wi, lobePdf);
            pdf += lobeProbabilities[1] * lobePdf;
        }
        if (lobeProbabilities[2] > 0.0f) {
            value += transmission.evaluate(wo, wi, lobePdf);
            pdf += lobeProbabilities[2] * lobePdf;
        }
        if (lobeProbabilities[3] > 0.0f) {
            value += clearcoat.evaluate(wo, wi, lobePdf);
            pdf += lobeProbabilities[3] * lobePdf;
        }
        pdf *= alpha;
        value *= this->weight * alpha;
        return value;
    }
    RMD_HD float3 evaluate(float3 wo, float3 wi, float3 shNormal, float3 geoNormal, float &pdf) const {
        pdf = 0.0f;
        float3x3 f = buildOrthonormalBasis(shNormal);
        const float woDotGeoN = dot(wo, geoNormal);
        wo = toLocal(f, wo);
        if (wo.z * woDotGeoN < 0.0f) return f3(0.0f);
        const float wiDotGeoN = dot(wi, geoNormal);
        wi = toLocal(f, wi);
        if (wi.z * wiDotGeoN < 0.0f) return f3(0.0f);
        return evaluateLocal(wo, wi, pdf);
    }
    // UberShader.hpp:85-145
    RMD_HD BsdfSample sample(float3 rnd, float3 wo, float3 shNormal, float3 geoNormal, uint8_t previousFlags) const {
        if (rnd.x < alpha) {
            rnd.x /= alpha;
        } else {
            BsdfSample s;
            s.weight = alphaWeight * weight;
            s.wi = -wo;
            s.pdf = 1.0f;
            s.flags = (uint8_t)(previousFlags | RayFlagsSingular);
            return s;
        }
        float3x3 f = buildOrthonormalBasis(shNormal);
        const float woDotGeoN = dot(wo, geoNormal);
        wo = toLocal(f, wo);
        if (wo.z * woDotGeoN < 0.0f) return BsdfSample::invalid();
        float p0 = lobeProbabilities[0], p1 = lobeProbabilities[1], p2 = lobeProbabilities[2];
        float2 rnd2 = make_float2(rnd.y, rnd.z);
        float selected;
        BsdfSample s;
        if (rnd.x < p0) {
            selected = p0;
            s = diffuse.sample(rnd2, wo);
        } else if (rnd.x < (p0 + p1)) {
            selected = p1;
            s = specular.sample(rnd2, wo);
        } else if (rnd.x < (p0 + p1 + p2)) {
            selected = p2;
            s = transmission.sample(rnd2, wo);
        } else {
            selected = lobeProbabilities[3];
            s = clearcoat.sample(rnd2, wo);
        }
        if (!is_finite(selected)) return BsdfSample::invalid();
        if (selected < 1.0f) {
            s.weight = evaluateLocal(wo, s.wi, s.pdf);
            s.weight = s.weight / s.pdf;
        } else {
            s.pdf *= alpha;
            s.weight *= this->weight * alpha;
        }
        const float wiDotShN = s.wi.z;
        s.wi = toWorld(f, s.wi);
        const float wiDotGeoN = dot(s.wi, geoNormal);
        if (wiDotShN * wiDotGeoN < 0.0f) return BsdfSample::invalid();
        return s;
    }
};

}  // namespace rmd
