// Scene data as the device sees it (the reference's `Context` argument
// buffer, raymond/device/Context.hpp:15-26, re-laid out for 16-byte loads),
// the shading context (ShadingContext.hpp/.metal) and the light samplers
// (raymond/device/lights/*).  shadeSurface / shadeLight are defined by the
// NVRTC-compiled material module (the JIT switch tables of
// MaterialBuilder.swift:289-300).
#pragma once
#include "bsdf.cuh"
#include "prng.cuh"

namespace rmd {

// bridge/PerInstanceData.hpp:6-20
struct PerInstanceData {
    uint32_t vertexOffset, faceOffset, lightFaceOffset, lightFaceCount;
    uint32_t lightIndex, visibility, triOffset, pad;
    float4 boundsMin;   // xyz
    float4 boundsSize;  // xyz
    float4 pointTransform[4];   // columns
    float4 normalTransform[3];  // columns (xyz)
};

struct LightInfo {  // bridge/lights/LightInfo.hpp
    uint32_t shaderIndex, castsShadows, usesMIS, pad;
};
struct AreaLight {  // bridge/lights/AreaLight.hpp
    LightInfo info;
    float4 transform[3];  // float3x4 columns
    float4 color;         // w: isCircular
};
struct PointLight {  // bridge/lights/PointLight.hpp
    LightInfo info;
    float4 locationRadius;
    float4 color;
};
struct SunLight {  // bridge/lights/SunLight.hpp
    LightInfo info;
    float4 directionCosAngle;
    float4 color;
};
struct SpotLight {  // bridge/lights/SpotLight.hpp
    LightInfo info;
    float4 locationRadius;
    float4 directionSpotSize;
    float4 colorSpotBlend;
};
struct ShapeLight {  // bridge/lights/ShapeLight.hpp
    uint32_t instanceIndex;
    float emissiveArea;
};

// One texture of the scene, RGBA floats row by row from the top of the image
// (single-channel images as (r, 0, 0, 1), RGB with alpha 1).
struct TextureView {
    const float4 *texels;
    int width, height, channels, pad;
};

struct Context {
    const float4 *vertices;  // object space, xyz
    const float4 *normals;   // xyz
    const float2 *texcoords;
    const uint4 *faces;      // xyz: vertex indices, w: material index
    const PerInstanceData *instances;
    const float *lightFaces;
    const float *envPdfs;
    const float *envMipmap;
    const AreaLight *areaLights;
    const PointLight *pointLights;
    const SunLight *sunLights;
    const SpotLight *spotLights;
    const ShapeLight *shapeLights;
    const uint2 *surfaceTable;     // per surface material: (function group, parameter offset)
    const uint2 *lightTable;       // per light material
    const float *materialParams;   // hoisted node-graph literals
    int numLightsTotal, numAreaLights, numPointLights, numSunLights;
    int numSpotLights, numShapeLights, envResolution;
    uint32_t worldShader;
    // bridge/Camera.hpp
    float4 cameraTransform[4];
    float nearClip, farClip, focalLength, pad;
    float2 shift;
    const TextureView *textures;  // the scene's textures, then a 1 x 1 zero texture for missing files
    int numTextures, pad2;
};

struct LightSample {  // lights/LightSample.hpp:6-34
    bool isLight;
    bool canBeHit;
    bool castsShadows;
    uint32_t shaderIndex;
    float3 weight;
    float pdf;
    float3 direction;
    float distance;
};

struct ShadingContext {  // ShadingContext.hpp:7-32
    float3 uv, position, generated, object, normal, trueNormal, tu, tv, rnd, wo;
    float distance;
    uint32_t rayFlags;
    UberShader material;
    RMD_HD float geometryTerm() const { return fabsf(dot(wo, trueNormal)) / square(distance); }
};

RMD_HD float3 mul3(const float4 *cols, float3 v) {  // float3x3 (xyz of 3 columns) * v
    return xyz(cols[0]) * v.x + xyz(cols[1]) * v.y + xyz(cols[2]) * v.z;
}
RMD_HD float3 mulPoint(const float4 *cols, float3 p) {  // (float4x4 * float4(p, 1)).xyz
    float4 r = cols[0] * p.x + cols[1] * p.y + cols[2] * p.z + cols[3] * 1.0f;
    return xyz(r);
}

// ShadingContext.metal:4-47
RMD_HD void buildShading(ShadingContext &sh, const Context &ctx, const PerInstanceData &inst, uint32_t prim,
                         float2 bary, float distance, uint32_t &shaderIndex) {
    const uint32_t faceIndex = inst.faceOffset + prim;
    const uint4 face = ctx.faces[faceIndex];
    const uint32_t i0 = inst.vertexOffset + face.x, i1 = inst.vertexOffset + face.y, i2 = inst.vertexOffset + face.z;
    const float2 Tc = ctx.texcoords[i2];
    const float2 T0 = ctx.texcoords[i0] - Tc;
    const float2 T1 = ctx.texcoords[i1] - Tc;
    sh.uv = f3(T0 * bary.x + T1 * bary.y + Tc, 0.0f);
    const float3 Pc = xyz(ctx.vertices[i2]);
    const float3 P0 = xyz(ctx.vertices[i0]) - Pc;
    const float3 P1 = xyz(ctx.vertices[i1]) - Pc;
    sh.trueNormal = normalize(mul3(inst.normalTransform, cross(P0, P1)));
    const float3 localP = P0 * bary.x + P1 * bary.y + Pc;
    sh.object = localP;
    const float3 d = localP - xyz(inst.boundsMin);
    const float3 s = xyz(inst.boundsSize);
    sh.generated = make_float3(s.x == 0.0f ? 0.5f : d.x / s.x, s.y == 0.0f ? 0.5f : d.y / s.y,
                               s.z == 0.0f ? 0.5f : d.z / s.z);
    sh.position = mulPoint(inst.pointTransform, localP);
    const float u = bary.x, v = bary.y, w = 1.0f - u - v;
    const float3 n = xyz(ctx.normals[i0]) * u + xyz(ctx.normals[i1]) * v + xyz(ctx.normals[i2]) * w;
    sh.normal = normalize(mul3(inst.normalTransform, n));
    sh.tu = normalize(mul3(inst.normalTransform, P0 * T1.y + P1 * (-T0.y)));
    sh.tv = normalize(mul3(inst.normalTransform, P0 * (-T1.x) + P1 * T0.x));
    sh.distance = distance;
    shaderIndex = face.w;
}

// defined by the material module
__device__ void shadeSurface(uint32_t shaderIndex, const Context &ctx, ShadingContext &shading);
__device__ void shadeLight(uint32_t shaderIndex, const Context &ctx, ShadingContext &shading);

// ---------------------------------------------------------------- world light
// WorldLight.hpp:14-17
RMD_HD float worldLightPdf(const Context &ctx, float3 wo) {
    const float2 sq = warp::uniformSphereToSquare(wo);
    const uint32_t res = (uint32_t)ctx.envResolution;
    const uint32_t px = ((uint32_t)((float)res * sq.x)) % res;
    const uint32_t py = ((uint32_t)((float)res * sq.y)) % res;
    return ctx.envPdfs[py * res + px];
}
// WorldLight.hpp:19-62
RMD_HD float3 worldLightSample(const Context &ctx, float2 uv, float &pdf) {
    int cur = 1;
    int sx = 0, sy = 0;
    const float *level = ctx.envMipmap;
    while (cur < ctx.envResolution) {
        const int off = 4 * (sy * cur + sx);
        level += cur * cur;
        sx *= 2;
        sy *= 2;
        cur *= 2;
        const float topLeft = level[off + 0];
        const float topRight = level[off + 1];
        const float bottomLeft = level[off + 2];
        const float leftProb = topLeft + bottomLeft;
        float topProb;
        if (uv.x < leftProb) {
            const float invProb = 1.0f / leftProb;
            uv.x *= invProb;
            topProb = topLeft * invProb;
        } else {
            const float invProb = 1.0f / (1.0f - leftProb);
            uv.x = (uv.x - leftProb) * invProb;
            topProb = topRight * invProb;
            sx += 1;
        }
        if (uv.y < topProb) {
            uv.y /= topProb;
        } else {
            uv.y = (uv.y - topProb) / (1.0f - topProb);
            sy += 1;
        }
    }
    pdf = ctx.envPdfs[sy * ctx.envResolution + sx];
    uv = (make_float2((float)sx, (float)sy) + uv) / (float)ctx.envResolution;
    return warp::uniformSquareToSphere(uv);
}

// Lights.hpp:33-41
RMD_HD float lightsShapePdf(const Context &ctx, const PerInstanceData &inst, const ShadingContext &sh) {
    const float sel = 1.0f / (float)ctx.numLightsTotal;
    if (inst.lightIndex >= (uint32_t)ctx.numShapeLights) return 0.0f;
    return sel * (1.0f / (sh.geometryTerm() * ctx.shapeLights[inst.lightIndex].emissiveArea));
}
RMD_HD float lightsEnvmapPdf(const Context &ctx, float3 wo) {
    const float sel = 1.0f / (float)ctx.numLightsTotal;
    return sel * worldLightPdf(ctx, wo);
}
// Lights.metal:6-15
__device__ __forceinline__ void evaluateEnvironment(const Context &ctx, ShadingContext &sh) {
    sh.position = sh.wo;
    sh.normal = sh.wo;
    sh.trueNormal = sh.wo;
    sh.generated = -sh.wo;
    sh.object = -sh.wo;
    sh.uv = f3(0.0f);
    shadeLight(ctx.worldShader, ctx, sh);
}

RMD_HD void initLightSample(LightSample &s, const LightInfo &info) {
    s.isLight = true;
    s.shaderIndex = info.shaderIndex;
    s.canBeHit = info.usesMIS != 0;
    s.castsShadows = info.castsShadows != 0;
}

// SpotLight.metal:9-20
RMD_HD float spotLightAttenuation(float3 dir, float spotAngle, float spotSmooth, float3 N) {
    float attenuation = dot(dir, N);
    if (attenuation <= spotAngle) {
        attenuation = 0.0f;
    } else {
        float t = attenuation - spotAngle;
        if (t < spotSmooth && spotSmooth != 0.0f) attenuation *= smoothstep(0.0f, spotSmooth, t);
    }
    return attenuation;
}
// ShapeLight.metal:14-28
RMD_HD int upperBound(const float *buf, int count, float value) {
    int left = 0, right = count;
    while (left < right) {
        int c = (left + right) / 2;
        if (value >= buf[c]) left = c + 1;
        else right = c;
    }
    return left;
}

// Lights.hpp:43-93 with the per-type samplers of lights/*.metal inlined.  Of the
// caller's shading context only the position and ray flags are read (the
// reference copies just these two into lightShading, Lights.hpp:47-49).
static __device__ __noinline__ LightSample lightsSample(const Context &ctx, float3 position, uint32_t rayFlags,
                                                       PrngState &prng) {
    int sampled = prng.sampleInt(ctx.numLightsTotal);
    LightSample s;
    s.isLight = false;
    s.canBeHit = false;
    s.castsShadows = false;
    s.shaderIndex = 0;
    s.pdf = 0.0f;
    s.weight = f3(0.0f);
    s.direction = f3(0.0f);
    s.distance = 0.0f;
    ShadingContext ls;
    ls.uv = ls.generated = ls.object = ls.normal = ls.trueNormal = ls.tu = ls.tv = ls.rnd = ls.wo = f3(0.0f);
    ls.distance = 0.0f;
    ls.rayFlags = rayFlags;
    ls.position = position;
    if (sampled == 0) {  // Lights.hpp:98-116
        s.direction = worldLightSample(ctx, prng.sample2d(), s.pdf);
        s.distance = inf_f();
        s.shaderIndex = ctx.worldShader;
        s.castsShadows = true;
        s.canBeHit = true;
        s.isLight = true;
        ls.position = -s.direction;
        ls.normal = -s.direction;
        ls.trueNormal = -s.direction;
        ls.generated = s.direction;
        ls.object = s.direction;
        ls.uv = f3(0.0f);
        s.weight = f3(1.0f / s.pdf);
    } else if ((sampled -= 1) < ctx.numAreaLights) {  // AreaLight.metal:7-38
        const AreaLight &l = ctx.areaLights[sampled];
        float2 uv = prng.sample2d();
        if (l.color.w != 0.0f) uv = warp::uniformSquareToDisk(uv) / 2.0f + 0.5f;
        float3x4 tr;
        tr.c[0] = l.transform[0];
        tr.c[1] = l.transform[1];
        tr.c[2] = l.transform[2];
        const float3 point = f4(uv - 0.5f, 0.0f, 1.0f) * tr;
        const float3 normal = normalize(f4(0.0f, 0.0f, 1.0f, 0.0f) * tr);
        initLightSample(s, l.info);
        s.direction = point - ls.position;
        const float lensqr = length_squared(s.direction);
        s.distance = sqrtf(lensqr);
        ls.normal = -normal;
        ls.trueNormal = -normal;
        ls.position = point;
        ls.generated = point;
        ls.uv = f3(uv, 0.0f);
        const float G = saturate(dot(normal, s.direction)) / lensqr;
        s.direction /= s.distance;
        s.weight = xyz(l.color) * G * 0.25f;
        s.pdf = 1.0f;
    } else if ((sampled -= ctx.numAreaLights) < ctx.numPointLights) {  // PointLight.metal:9-40
        const PointLight &l = ctx.pointLights[sampled];
        const float3 loc = xyz(l.locationRadius);
        const float radius = l.locationRadius.w;
        const float3 lightN = normalize(ls.position - loc);
        float3 point = loc;
        if (radius > 0.0f) {
            float3x3 basis = buildOrthonormalBasis(lightN);
            point += radius * (basis * f3(warp::uniformSquareToDisk(prng.sample2d()), 0.0f));
        }
        initLightSample(s, l.info);
        s.direction = point - ls.position;
        const float lensqr = length_squared(s.direction);
        s.distance = sqrtf(lensqr);
        s.direction /= s.distance;
        ls.normal = -s.direction;
        ls.trueNormal = -s.direction;
        ls.position = point;
        ls.generated = point;
        ls.uv = f3(warp::uniformSphereToSquare(-s.direction), 0.0f);
        const float G = 1.0f / lensqr;
        s.weight = xyz(l.color) * G * (M_1_PI_F * 0.25f);
        s.pdf = 1.0f;
    } else if ((sampled -= ctx.numPointLights) < ctx.numSunLights) {  // SunLight.metal:9-37
        const SunLight &l = ctx.sunLights[sampled];
        const float2 rnd = prng.sample2d();
        const float cosTheta = 1.0f - rnd.y * (1.0f - l.directionCosAngle.w);
        const float sinTheta = sqrtf(saturate(1.0f - cosTheta * cosTheta));
        float sinPhi, cosPhi;
        sincosf(2.0f * M_PI_F * rnd.x, &sinPhi, &cosPhi);
        const float3x3 fr = buildOrthonormalBasis(xyz(l.directionCosAngle));
        const float3 point = fr * make_float3(sinTheta * sinPhi, sinTheta * cosPhi, cosTheta);
        initLightSample(s, l.info);
        s.direction = point;
        s.distance = inf_f();
        ls.normal = -s.direction;
        ls.trueNormal = -s.direction;
        ls.position = -s.direction;
        ls.generated = -s.direction;
        ls.uv = f3(warp::uniformSphereToSquare(-s.direction), 0.0f);
        s.weight = xyz(l.color);
        s.pdf = 1.0f;
    } else if ((sampled -= ctx.numSunLights) < ctx.numSpotLights) {  // SpotLight.metal:22-54
        const SpotLight &l = ctx.spotLights[sampled];
        const float3 loc = xyz(l.locationRadius);
        const float radius = l.locationRadius.w;
        const float3 lightN = normalize(ls.position - loc);
        float3 point = loc;
        if (radius > 0.0f) {
            float3x3 basis = buildOrthonormalBasis(lightN);
            point += radius * (basis * f3(warp::uniformSquareToDisk(prng.sample2d()), 0.0f));
        }
        initLightSample(s, l.info);
        s.direction = point - ls.position;
        const float lensqr = length_squared(s.direction);
        s.distance = sqrtf(lensqr);
        s.direction /= s.distance;
        ls.normal = -s.direction;
        ls.trueNormal = -s.direction;
        ls.position = point;
        ls.generated = point;
        ls.uv = f3(warp::uniformSphereToSquare(-s.direction), 0.0f);
        const float G = 1.0f / lensqr;
        const float att = spotLightAttenuation(xyz(l.directionSpotSize), l.directionSpotSize.w, l.colorSpotBlend.w,
                                               s.direction);
        s.weight = att * xyz(l.colorSpotBlend) * G * (M_1_PI_F * 0.25f);
        s.pdf = 1.0f;
    } else if ((sampled -= ctx.numSpotLights) < ctx.numShapeLights) {  // ShapeLight.metal:30-66
        const ShapeLight &l = ctx.shapeLights[sampled];
        const PerInstanceData &inst = ctx.instances[l.instanceIndex];
        const uint32_t prim =
            (uint32_t)upperBound(ctx.lightFaces + inst.lightFaceOffset, (int)inst.lightFaceCount, prng.sample());
        const float2 bary = warp::uniformSquareToTriangleBarycentric(prng.sample2d());
        s.canBeHit = true;
        s.castsShadows = true;
        const float3 origin = ls.position;
        uint32_t shaderIndex;
        buildShading(ls, ctx, inst, prim, bary, 0.0f, shaderIndex);
        s.shaderIndex = shaderIndex;
        s.direction = ls.position - origin;
        const float lensqr = length_squared(s.direction);
        s.distance = sqrtf(lensqr);
        s.direction /= s.distance;
        ls.wo = -s.direction;
        ls.distance = s.distance;
        const float G = ls.geometryTerm();
        s.weight = f3(G * l.emissiveArea);
        s.pdf = 1.0f / (G * l.emissiveArea);
    } else {
        return s;  // LightSample::invalid()
    }
    ls.wo = -s.direction;
    if (any_nonzero(s.weight)) {
        if (s.isLight) shadeLight(s.shaderIndex, ctx, ls);
        else shadeSurface(s.shaderIndex, ctx, ls);
        s.weight *= ls.material.emission;
    }
    s.weight *= (float)ctx.numLightsTotal;
    s.pdf /= (float)ctx.numLightsTotal;
    const float survival = saturate(4.0f * mean(s.weight));
    if (survival < 1.0f) {
        if (prng.sample() < survival) s.weight /= survival;
        else s.weight = f3(0.0f);
    }
    return s;
}

}  // namespace rmd
