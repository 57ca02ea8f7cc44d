// Oracle (test infrastructure only): scene data the reference's device code
// reads through `Context` (raymond/device/Context.hpp:15-26), the shading
// context (raymond/device/ShadingContext.hpp:7-32) and the light records
// (raymond/bridge/lights/*.hpp, raymond/device/lights/*).
#pragma once
#include <memory>
#include <string>
#include <vector>
#include "bsdf.h"
#include "prng.h"

namespace orc {

// bridge/PerInstanceData.hpp:6-20
struct PerInstanceData {
    uint32_t vertexOffset = 0;
    uint32_t faceOffset = 0;
    uint32_t lightFaceOffset = 0;
    uint32_t lightFaceCount = 0;
    uint32_t lightIndex = 0xffffffffu;
    float3 boundsMin;
    float3 boundsSize;
    float4x4 pointTransform;
    float3x3 normalTransform;
    uint8_t visibility = 0;
    // oracle bookkeeping (not in the reference struct)
    uint32_t shape = 0;
};

struct LightInfo {  // bridge/lights/LightInfo.hpp:5-9
    uint16_t shaderIndex = 0;
    bool castsShadows = true;
    bool usesMIS = false;
};
struct AreaLight {  // bridge/lights/AreaLight.hpp
    LightInfo info;
    float3x4 transform;
    float3 color;
    bool isCircular = false;
};
struct PointLight {  // bridge/lights/PointLight.hpp
    LightInfo info;
    float3 location;
    float radius = 0;
    float3 color;
};
struct SunLight {  // bridge/lights/SunLight.hpp
    LightInfo info;
    float3 direction;
    float cosAngle = 1;
    float3 color;
};
struct SpotLight {  // bridge/lights/SpotLight.hpp
    LightInfo info;
    float3 location;
    float3 direction;
    float radius = 0;
    float3 color;
    float spotSize = 0;
    float spotBlend = 0;
};
struct ShapeLight {  // bridge/lights/ShapeLight.hpp
    uint32_t instanceIndex = 0;
    float emissiveArea = 0;
};

// LightSample.hpp:6-34
struct LightSample {
    bool isLight = false;
    uint16_t shaderIndex = 0;
    bool canBeHit = false;
    bool castsShadows = false;
    float3 weight;
    float pdf = 0;
    float3 direction;
    float distance = 0;
    LightSample() = default;
    explicit LightSample(const LightInfo &info) {
        isLight = true;
        shaderIndex = info.shaderIndex;
        canBeHit = info.usesMIS;
        castsShadows = info.castsShadows;
    }
    static LightSample invalid() {
        LightSample r;
        r.pdf = 0;
        r.weight = float3(0.0f);
        return r;
    }
};

// ShadingContext.hpp:7-32
struct ShadingContext {
    float3 uv, position, generated, object, normal, trueNormal, tu, tv, rnd, wo;
    float distance = 0;
    uint8_t rayFlags = 0;
    UberShader material;
    float geometryTerm() const { return std::fabs(dot(wo, trueNormal)) / square(distance); }
};

struct Intersection {  // bridge/Ray.hpp:41-46
    float distance = -1;
    uint32_t primitiveIndex = 0;
    uint32_t instanceIndex = 0;
    float2 coordinates;
};

class MaterialProgram;  // nodes.h
class Bvh;              // bvh.h

// A texture as the oracle samples it: RGBA floats from the top row (a
// single-channel image as (r, 0, 0, 1), RGB with alpha 1).
struct Texture {
    int width = 1, height = 1, channels = 1;
    std::vector<float4> texels{float4(0, 0, 0, 1)};
};

struct SceneData {
    // Context.hpp:15-26
    std::vector<float3> vertices;
    std::vector<uint32_t> vertexIndices;  // 3 per face
    std::vector<float3> vertexNormals;
    std::vector<float2> texcoords;
    std::vector<PerInstanceData> perInstanceData;
    std::vector<uint16_t> materials;
    // camera (bridge/Camera.hpp)
    float4x4 cameraTransform;
    float nearClip = 0.1f, farClip = 100.0f, focalLength = 2.5f;
    float2 shift;
    // Lights.hpp:16-31
    int numLightsTotal = 1;
    std::vector<float> lightFaces;
    uint16_t worldShaderIndex = 0;
    int envResolution = 0;
    std::vector<float> envPdfs, envMipmap;
    std::vector<AreaLight> areaLights;
    std::vector<PointLight> pointLights;
    std::vector<SunLight> sunLights;
    std::vector<SpotLight> spotLights;
    std::vector<ShapeLight> shapeLights;
    // JIT tables (MaterialBuilder.swift:289-300)
    std::vector<std::unique_ptr<MaterialProgram>> surfaceShaders;
    std::vector<std::unique_ptr<MaterialProgram>> lightShaders;
    std::unique_ptr<Bvh> bvh;
    // Context.hpp:25 (textures): the scene's, then a 1 x 1 zero texture for missing files
    std::vector<Texture> textures;
};

// ShadingContext.metal:4-47
void buildShadingContext(ShadingContext &sh, const SceneData &ctx, const PerInstanceData &instance,
                         const Intersection &isect, uint16_t &shaderIndex);
// shading.hpp:11-12 (the JIT switch tables)
void shadeSurface(uint16_t shaderIndex, const SceneData &ctx, ShadingContext &sh);
void shadeLight(uint16_t shaderIndex, const SceneData &ctx, ShadingContext &sh);

// Lights.hpp:33-93, Lights.metal:6-15, WorldLight.hpp:14-62
float lightsShapePdf(const SceneData &ctx, const PerInstanceData &instance, const ShadingContext &sh);
float lightsEnvmapPdf(const SceneData &ctx, float3 wo);
LightSample lightsSample(const SceneData &ctx, const ShadingContext &sh, PrngState &prng);
void evaluateEnvironment(const SceneData &ctx, ShadingContext &sh);
float worldLightPdf(const SceneData &ctx, float3 wo);
float3 worldLightSample(const SceneData &ctx, float2 uv, float &pdf);
// kernels/envmap/{build,reduce,normalize}.metal driven as LightBuilder.swift:83-167
void buildEnvironmentMap(SceneData &ctx, int exponent);

}  // namespace orc
