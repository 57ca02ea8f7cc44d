// Oracle (test infrastructure only): shading context, lights and the
// environment importance map, restated from the reference device library.
#include "scene.h"

#include "nodes.h"

namespace orc {

// ShadingContext.metal:4-47
void buildShadingContext(ShadingContext &sh, const SceneData &ctx, const PerInstanceData &instance,
                         const Intersection &isect, uint16_t &shaderIndex) {
    const float2 barycentric = isect.coordinates;
    const uint32_t faceIndex = instance.faceOffset + isect.primitiveIndex;
    const uint32_t idx0 = instance.vertexOffset + ctx.vertexIndices[3 * faceIndex + 0];
    const uint32_t idx1 = instance.vertexOffset + ctx.vertexIndices[3 * faceIndex + 1];
    const uint32_t idx2 = instance.vertexOffset + ctx.vertexIndices[3 * faceIndex + 2];

    const float2 Tc = ctx.texcoords[idx2];
    const float2 T0 = ctx.texcoords[idx0] - Tc;  // T.columns[0]
    const float2 T1 = ctx.texcoords[idx1] - Tc;  // T.columns[1]
    sh.uv = float3(T0 * barycentric.x + T1 * barycentric.y + Tc, 0);

    const float3 Pc = ctx.vertices[idx2];
    const float3 P0 = ctx.vertices[idx0] - Pc;
    const float3 P1 = ctx.vertices[idx1] - Pc;
    sh.trueNormal = normalize(instance.normalTransform * cross(P0, P1));

    const float3 localP = P0 * barycentric.x + P1 * barycentric.y + Pc;
    sh.object = localP;
    const float3 d = localP - instance.boundsMin;
    const float3 s = instance.boundsSize;
    sh.generated = float3(s.x == 0 ? 0.5f : d.x / s.x, s.y == 0 ? 0.5f : d.y / s.y, s.z == 0 ? 0.5f : d.z / s.z);
    sh.position = (instance.pointTransform * float4(localP, 1)).xyz();

    // math.hpp:121-128 interpolate(a, b, c, bary) = a*u + b*v + c*(1-u-v)
    const float u = barycentric.x, v = barycentric.y, w = 1.0f - u - v;
    const float3 n = ctx.vertexNormals[idx0] * u + ctx.vertexNormals[idx1] * v + ctx.vertexNormals[idx2] * w;
    sh.normal = normalize(instance.normalTransform * n);

    // T[1][1] = T1.y, T[0][1] = T0.y, T[1][0] = T1.x, T[0][0] = T0.x
    sh.tu = normalize(instance.normalTransform * (P0 * T1.y + P1 * (-T0.y)));
    sh.tv = normalize(instance.normalTransform * (P0 * (-T1.x) + P1 * T0.x));
    sh.distance = isect.distance;
    shaderIndex = ctx.materials[faceIndex];
}

// The JIT's shadeSurface / shadeLight switch tables (MaterialBuilder.swift:289-300):
// an index without a material leaves the shading context untouched.
void shadeSurface(uint16_t i, const SceneData &ctx, ShadingContext &sh) {
    if (i < ctx.surfaceShaders.size() && ctx.surfaceShaders[i]) ctx.surfaceShaders[i]->run(ctx, sh);
}
void shadeLight(uint16_t i, const SceneData &ctx, ShadingContext &sh) {
    if (i < ctx.lightShaders.size() && ctx.lightShaders[i]) ctx.lightShaders[i]->run(ctx, sh);
}

// ---------------------------------------------------------------- lights
// WorldLight.hpp:14-17
float worldLightPdf(const SceneData &ctx, float3 wo) {
    const float2 sq = warp::uniformSphereToSquare(wo);
    const uint32_t res = (uint32_t)ctx.envResolution;
    uint32_t px = ((uint32_t)(float(res) * sq.x)) % res;
    uint32_t py = ((uint32_t)(float(res) * sq.y)) % res;
    return ctx.envPdfs[py * res + px];
}
// WorldLight.hpp:19-62
float3 worldLightSample(const SceneData &ctx, float2 uv, float &pdf) {
    int currentResolution = 1;
    int sx = 0, sy = 0;
    const float *currentLevel = ctx.envMipmap.data();
    while (currentResolution < ctx.envResolution) {
        const int currentOffset = 4 * (sy * currentResolution + sx);
        currentLevel += currentResolution * currentResolution;
        sx *= 2;
        sy *= 2;
        currentResolution *= 2;
        const float topLeft = currentLevel[currentOffset + 0];
        const float topRight = currentLevel[currentOffset + 1];
        const float bottomLeft = currentLevel[currentOffset + 2];
        const float leftProb = topLeft + bottomLeft;
        float topProb;
        if (uv.x < leftProb) {
            const float invProb = 1 / leftProb;
            uv.x *= invProb;
            topProb = topLeft * invProb;
        } else {
            const float invProb = 1 / (1 - leftProb);
            uv.x = (uv.x - leftProb) * invProb;
            topProb = topRight * invProb;
            sx += 1;
        }
        if (uv.y < topProb) {
            uv.y /= topProb;
        } else {
            uv.y = (uv.y - topProb) / (1 - topProb);
            sy += 1;
        }
    }
    pdf = ctx.envPdfs[sy * ctx.envResolution + sx];
    uv = (float2((float)sx, (float)sy) + uv) / (float)ctx.envResolution;
    return warp::uniformSquareToSphere(uv);
}

// Lights.hpp:33-36
float lightsShapePdf(const SceneData &ctx, const PerInstanceData &instance, const ShadingContext &sh) {
    const float selectionProbability = 1 / float(ctx.numLightsTotal);
    if (instance.lightIndex >= ctx.shapeLights.size()) return 0;  // no shape light registered
    const ShapeLight &l = ctx.shapeLights[instance.lightIndex];
    return selectionProbability * (1 / (sh.geometryTerm() * l.emissiveArea));  // ShapeLight.metal:10-12
}
// Lights.hpp:38-41
float lightsEnvmapPdf(const SceneData &ctx, float3 wo) {
    const float selectionProbability = 1 / float(ctx.numLightsTotal);
    return selectionProbability * worldLightPdf(ctx, wo);
}
// Lights.metal:6-15
void evaluateEnvironment(const SceneData &ctx, ShadingContext &sh) {
    sh.position = sh.wo;
    sh.normal = sh.wo;
    sh.trueNormal = sh.wo;
    sh.generated = -sh.wo;
    sh.object = -sh.wo;
    sh.uv = float3(0.0f);
    shadeLight(ctx.worldShaderIndex, ctx, sh);
}

// Lights.hpp:98-116
static LightSample sampleEnvmap(const SceneData &ctx, ShadingContext &sh, PrngState &prng) {
    LightSample s;
    s.direction = worldLightSample(ctx, prng.sample2d(), s.pdf);
    s.distance = INF;
    s.shaderIndex = ctx.worldShaderIndex;
    s.castsShadows = true;
    s.canBeHit = true;
    s.isLight = true;
    sh.position = -s.direction;
    sh.normal = -s.direction;
    sh.trueNormal = -s.direction;
    sh.generated = s.direction;
    sh.object = s.direction;
    sh.uv = float3(0.0f);
    s.weight = float3(1 / s.pdf);
    return s;
}
// AreaLight.metal:7-38
static LightSample sampleArea(const AreaLight &l, ShadingContext &sh, PrngState &prng) {
    float2 uv = prng.sample2d();
    if (l.isCircular) uv = warp::uniformSquareToDisk(uv) / 2 + 0.5f;
    const float3 point = float4(uv - 0.5f, 0, 1) * l.transform;
    const float3 normal = normalize(float4(0, 0, 1, 0) * l.transform);
    LightSample s(l.info);
    s.direction = point - sh.position;
    const float lensqr = length_squared(s.direction);
    s.distance = std::sqrt(lensqr);
    sh.normal = -normal;
    sh.trueNormal = -normal;
    sh.position = point;
    sh.generated = point;
    sh.uv = float3(uv, 0);
    const float G = saturate(dot(normal, s.direction)) / lensqr;
    s.direction /= s.distance;
    s.weight = l.color * G * 0.25f;
    s.pdf = 1;
    return s;
}
// PointLight.metal:9-40
static LightSample samplePoint(const PointLight &l, ShadingContext &sh, PrngState &prng) {
    const float3 lightN = normalize(sh.position - l.location);
    float3 point = l.location;
    if (l.radius > 0) {
        float3x3 basis = buildOrthonormalBasis(lightN);
        point += l.radius * (basis * float3(warp::uniformSquareToDisk(prng.sample2d()), 0));
    }
    LightSample s(l.info);
    s.direction = point - sh.position;
    const float lensqr = length_squared(s.direction);
    s.distance = std::sqrt(lensqr);
    s.direction /= s.distance;
    sh.normal = -s.direction;
    sh.trueNormal = -s.direction;
    sh.position = point;
    sh.generated = point;
    sh.uv = float3(warp::uniformSphereToSquare(-s.direction), 0);
    const float G = 1 / lensqr;
    s.weight = l.color * G * (M_1_PI_F * 0.25f);
    s.pdf = 1;
    return s;
}
// SunLight.metal:9-37
static LightSample sampleSun(const SunLight &l, ShadingContext &sh, PrngState &prng) {
    const float2 rnd = prng.sample2d();
    const float cosTheta = 1 - rnd.y * (1 - l.cosAngle);
    const float sinTheta = std::sqrt(saturate(1 - cosTheta * cosTheta));
    const float phi = 2 * M_PI_F * rnd.x;
    const float sinPhi = std::sin(phi), cosPhi = std::cos(phi);
    const float3x3 fr = buildOrthonormalBasis(l.direction);
    const float3 point = fr * float3(sinTheta * sinPhi, sinTheta * cosPhi, cosTheta);
    LightSample s(l.info);
    s.direction = point;
    s.distance = INF;
    sh.normal = -s.direction;
    sh.trueNormal = -s.direction;
    sh.position = -s.direction;
    sh.generated = -s.direction;
    sh.uv = float3(warp::uniformSphereToSquare(-s.direction), 0);
    s.weight = l.color;
    s.pdf = 1;
    return s;
}
// SpotLight.metal:9-20
static float spotLightAttenuation(float3 dir, float spotAngle, float spotSmooth, float3 N) {
    float attenuation = dot(dir, N);
    if (attenuation <= spotAngle) {
        attenuation = 0.0f;
    } else {
        float t = attenuation - spotAngle;
        if (t < spotSmooth && spotSmooth != 0.0f) attenuation *= smoothstep(0, spotSmooth, t);
    }
    return attenuation;
}
// SpotLight.metal:22-54
static LightSample sampleSpot(const SpotLight &l, ShadingContext &sh, PrngState &prng) {
    const float3 lightN = normalize(sh.position - l.location);
    float3 point = l.location;
    if (l.radius > 0) {
        float3x3 basis = buildOrthonormalBasis(lightN);
        point += l.radius * (basis * float3(warp::uniformSquareToDisk(prng.sample2d()), 0));
    }
    LightSample s(l.info);
    s.direction = point - sh.position;
    const float lensqr = length_squared(s.direction);
    s.distance = std::sqrt(lensqr);
    s.direction /= s.distance;
    sh.normal = -s.direction;
    sh.trueNormal = -s.direction;
    sh.position = point;
    sh.generated = point;
    sh.uv = float3(warp::uniformSphereToSquare(-s.direction), 0);
    const float G = 1 / lensqr;
    const float attenuation = spotLightAttenuation(l.direction, l.spotSize, l.spotBlend, s.direction);
    s.weight = attenuation * l.color * G * (M_1_PI_F * 0.25f);
    s.pdf = 1;
    return s;
}
// ShapeLight.metal:14-28
static int upper_bound(const float *buffer, int count, float value) {
    int left = 0, right = count;
    while (left < right) {
        int candidate = (left + right) / 2;
        if (value >= buffer[candidate]) left = candidate + 1;
        else right = candidate;
    }
    return left;
}
// ShapeLight.metal:30-66
static LightSample sampleShape(const SceneData &ctx, const ShapeLight &l, ShadingContext &sh, PrngState &prng) {
    const PerInstanceData &instance = ctx.perInstanceData[l.instanceIndex];
    Intersection isect;
    isect.primitiveIndex =
        (uint32_t)upper_bound(ctx.lightFaces.data() + instance.lightFaceOffset, (int)instance.lightFaceCount,
                              prng.sample());
    isect.coordinates = warp::uniformSquareToTriangleBarycentric(prng.sample2d());
    LightSample s;
    s.canBeHit = true;
    s.castsShadows = true;
    const float3 origin = sh.position;
    buildShadingContext(sh, ctx, instance, isect, s.shaderIndex);
    s.direction = sh.position - origin;
    const float lensqr = length_squared(s.direction);
    s.distance = std::sqrt(lensqr);
    s.direction /= s.distance;
    sh.wo = -s.direction;
    sh.distance = s.distance;
    const float G = sh.geometryTerm();
    s.weight = float3(G * l.emissiveArea);
    s.pdf = 1 / (G * l.emissiveArea);
    return s;
}

// Lights.hpp:43-93
LightSample lightsSample(const SceneData &ctx, const ShadingContext &shading, PrngState &prng) {
    int sampled = prng.sampleInt(ctx.numLightsTotal);
    LightSample s;
    ShadingContext lightShading;
    lightShading.rayFlags = shading.rayFlags;
    lightShading.position = shading.position;
    const int nArea = (int)ctx.areaLights.size(), nPoint = (int)ctx.pointLights.size();
    const int nSun = (int)ctx.sunLights.size(), nSpot = (int)ctx.spotLights.size();
    const int nShape = (int)ctx.shapeLights.size();
    if (sampled == 0) {
        s = sampleEnvmap(ctx, lightShading, prng);
    } else if ((sampled -= 1) < nArea) {
        s = sampleArea(ctx.areaLights[sampled], lightShading, prng);
    } else if ((sampled -= nArea) < nPoint) {
        s = samplePoint(ctx.pointLights[sampled], lightShading, prng);
    } else if ((sampled -= nPoint) < nSun) {
        s = sampleSun(ctx.sunLights[sampled], lightShading, prng);
    } else if ((sampled -= nSun) < nSpot) {
        s = sampleSpot(ctx.spotLights[sampled], lightShading, prng);
    } else if ((sampled -= nSpot) < nShape) {
        s = sampleShape(ctx, ctx.shapeLights[sampled], lightShading, prng);
    } else {
        return LightSample::invalid();
    }
    lightShading.wo = -s.direction;
    if (any_nonzero(s.weight)) {
        if (s.isLight) shadeLight(s.shaderIndex, ctx, lightShading);
        else shadeSurface(s.shaderIndex, ctx, lightShading);
        s.weight *= lightShading.material.emission;
    }
    s.weight *= (float)ctx.numLightsTotal;
    s.pdf /= (float)ctx.numLightsTotal;
    const float survivalProbability = saturate(4 * mean(s.weight));
    if (survivalProbability < 1) {
        if (prng.sample() < survivalProbability) s.weight /= survivalProbability;
        else s.weight = float3(0.0f);
    }
    return s;
}

// ---------------------------------------------------------------- envmap
// build.metal:4-51, reduce.metal:3-24, normalize.metal:4-11, driven as
// LightBuilder.swift:83-167.
void buildEnvironmentMap(SceneData &ctx, int exponent) {
    const int resolution = 1 << exponent;
    size_t mipmapSize = 0;
    for (int e = 0; e <= exponent; e++) mipmapSize += (size_t)1 << (2 * e);
    ctx.envResolution = resolution;
    ctx.envMipmap.assign(mipmapSize, 0.0f);
    ctx.envPdfs.assign((size_t)resolution * resolution, 0.0f);
    const size_t lastLevelOffset = mipmapSize - (size_t)resolution * resolution;
    float *finest = ctx.envMipmap.data() + lastLevelOffset;

#pragma omp parallel for schedule(dynamic, 16)
    for (int ty = 0; ty < resolution; ty++) {
        for (int tx = 0; tx < resolution; tx++) {
            const int rayIndex = ty * resolution + tx;
            float value = 0;
            const int numSamples = 64;
            for (int sampleIndex = 0; sampleIndex < numSamples; sampleIndex++) {
                PrngState prng = PrngState::tea((uint32_t)sampleIndex, (uint32_t)rayIndex);
                float2 projected = (float2((float)tx, (float)ty) + prng.sample2d()) / float2((float)resolution);
                float3 wo = warp::uniformSquareToSphere(projected);
                ShadingContext sh;
                sh.rayFlags = 0;
                sh.rnd = prng.sample3d();
                sh.wo = -wo;
                evaluateEnvironment(ctx, sh);
                value += mean(sh.material.emission);
            }
            value /= numSamples;
            value += 1e-8f;
            const uint32_t qx = tx / 2, qy = ty / 2, qw = resolution / 2;
            const uint32_t quadIndex = qy * qw + qx;
            const uint32_t outputIndex = 4 * quadIndex + (tx & 1) + 2 * (ty & 1);
            // at resolution 1 (exponent 0) the quad layout degenerates to index 0
            if (resolution == 1) finest[0] = value;
            else finest[outputIndex] = value;
            ctx.envPdfs[(size_t)ty * resolution + tx] = value;
        }
    }
    size_t bufferOffset = lastLevelOffset;
    for (int e = exponent - 1; e >= 0; e--) {
        const int cur = 1 << e;
        bufferOffset -= (size_t)cur * cur;
        float *mip = ctx.envMipmap.data() + bufferOffset;
        const int gridLength = cur * cur;
        for (int ty = 0; ty < cur; ty++) {
            for (int tx = 0; tx < cur; tx++) {
                const int inputIndex = ty * cur + tx;
                float sum = 0;
                for (int i = 0; i < 4; ++i) sum += mip[gridLength + 4 * inputIndex + i];
                for (int i = 0; i < 4; ++i) mip[gridLength + 4 * inputIndex + i] /= sum;
                const uint32_t qx = tx / 2, qy = ty / 2, qw = cur / 2;
                const uint32_t outputIndex = cur == 1 ? 0 : 4 * (qy * qw + qx) + (tx & 1) + 2 * (ty & 1);
                mip[outputIndex] = sum;
            }
        }
    }
    const float sum = ctx.envMipmap[0];
    const uint32_t gridSize = (uint32_t)resolution * (uint32_t)resolution;
    const float scale = (float)gridSize * warp::uniformSquareToSpherePdf() / sum;
    for (size_t i = 0; i < ctx.envPdfs.size(); i++) ctx.envPdfs[i] *= scale;
}

}  // namespace orc
