// Oracle (test infrastructure only): scene building (SceneLoader /
// ShapeBuilder / EntityBuilder / LightBuilder) and the wavefront frame loop
// of Renderer.execute with the generateRays / handleIntersections /
// handleShadowRays kernels, restated for the host.
#include <atomic>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>

#include "sky.h"
#endif

#include "../oracle.h"
#include "bvh.h"
#include "nodes.h"
#include "noise.h"
#include "scene.h"

using namespace orc;

struct oracle_scene {
    SceneData data;
    uint64_t triangles = 0;
};

namespace {

constexpr float eps = 0.001f;  // device/constants.hpp:3

// bridge/Ray.hpp:17-29
struct Ray {
    float3 origin;
    float minDistance = 0;
    float3 direction;
    float maxDistance = 0;
    PrngState prng;
    float3 weight;
    uint16_t x = 0, y = 0;
    uint16_t depth = 0;
    uint8_t flags = 0;
    float bsdfPdf = 0;
};
// bridge/Ray.hpp:31-39
struct ShadowRay {
    float3 origin;
    float minDistance = 0;
    float3 direction;
    float maxDistance = 0;
    float3 weight;
    uint16_t x = 0, y = 0;
};

float3x3 inverseTranspose3(const float4x4 &m) {
    // columns of the upper 3x3
    float3 a(m.c[0].x, m.c[0].y, m.c[0].z), b(m.c[1].x, m.c[1].y, m.c[1].z), c(m.c[2].x, m.c[2].y, m.c[2].z);
    // inverse(M)^T = cofactor(M) / det(M); cofactor columns are cross products of the other columns
    float3 r0 = cross(b, c), r1 = cross(c, a), r2 = cross(a, b);
    float det = dot(a, r0);
    float3x3 it;
    it.c[0] = r0 / det;
    it.c[1] = r1 / det;
    it.c[2] = r2 / det;
    return it;
}
float3x3 inner3x3(const float4x4 &m) {
    float3x3 r;
    for (int i = 0; i < 3; i++) r.c[i] = float3(m.c[i].x, m.c[i].y, m.c[i].z);
    return r;
}
float4x4 toMatrix(const float *m) {
    float4x4 r;
    for (int c = 0; c < 4; c++) r.c[c] = float4(m[4 * c + 0], m[4 * c + 1], m[4 * c + 2], m[4 * c + 3]);
    return r;
}

// host/lights/distribution.m:7-39
float buildLightDistribution(const float3x3 &normalTransform, const uint32_t *indices, const float3 *vertices,
                             uint32_t faceCount, float *output) {
    double accumulatedArea = 0;
    for (uint32_t i = 0; i < faceCount; i++) {
        float3 v0 = vertices[indices[3 * i + 0]];
        float3 v1 = vertices[indices[3 * i + 1]];
        float3 v2 = vertices[indices[3 * i + 2]];
        float3 tn = cross(normalTransform * (v2 - v0), normalTransform * (v2 - v1));
        float area = length(tn) / 2;
        output[i] = (float)(accumulatedArea += area);
    }
    for (uint32_t i = 0; i < faceCount; i++) output[i] = (float)(output[i] / accumulatedArea);
    return (float)accumulatedArea;
}

// generate.metal:88-91 with 8x8 threadgroups (Renderer.swift:536-538)
inline uint32_t blockLinearIndex(uint32_t x, uint32_t y, uint32_t W, uint32_t H) {
    uint32_t gx = x / 8, gy = y / 8, tx = x % 8, ty = y % 8;
    uint32_t awx = std::min(8u, W - gx * 8), awy = std::min(8u, H - gy * 8);
    return tx + ty * awx + gx * 8 * awy + gy * 8 * W;
}

// intersection.metal:14-20
inline float computeMisWeight(float pdf, float other) {
    pdf *= pdf;
    if (std::isinf(pdf)) return 1;
    other *= other;
    return pdf / (pdf + other);
}

template <typename FilmT>
struct Film {
    uint32_t W, H;
    std::vector<FilmT> rgba;
    void add(uint32_t x, uint32_t y, float3 c) {
        FilmT *p = &rgba[4 * ((size_t)y * W + x)];
        p[0] += (FilmT)c.x;
        p[1] += (FilmT)c.y;
        p[2] += (FilmT)c.z;
        p[3] += (FilmT)1;
    }
};

template <typename FilmT>
struct Frame {
    const SceneData &ctx;
    const oracle_settings &st;
    Film<FilmT> &film;
    std::vector<Ray> rays[2];
    std::vector<ShadowRay> shadowRays;
    std::vector<Intersection> intersections;
    std::atomic<uint32_t> nextCount{0}, shadowCount{0};
    std::atomic<uint64_t> segments{0}, shadows{0};

    Frame(const SceneData &c, const oracle_settings &s, Film<FilmT> &f) : ctx(c), st(s), film(f) {
        size_t n = s.pixels ? (size_t)s.num_pixels : (size_t)s.width * s.height;
        rays[0].resize(n);
        rays[1].resize(n);
        shadowRays.resize(n);
        intersections.resize(n);
    }

    void trace(const Ray &r, Intersection &isect) const {  // raytrace.metal:11-50
        HitRecord h;
        if (ctx.bvh->intersect(r.origin, r.direction, r.minDistance, r.maxDistance, h)) {
            isect.distance = h.t;
            isect.coordinates = float2(h.b0, h.b1);
            isect.instanceIndex = h.instance;
            isect.primitiveIndex = h.prim;
        } else {
            isect.distance = -1;
        }
    }

    // generate.metal:72-121 (pinhole branch) + :165-191 (fused trace)
    // `slot`: position in the ray arrays (the ray index when every pixel is traced)
    void generate(uint32_t x, uint32_t y, uint64_t sampleIndex, uint32_t slot) {
        const uint32_t W = st.width, H = st.height;
        const uint32_t rayIndex = blockLinearIndex(x, y, W, H);
        Ray ray;
        if (st.rng == RMD_RNG_TEA) ray.prng = PrngState::tea((uint32_t)(sampleIndex + 1), rayIndex);
        else ray.prng = PrngState::pcg(st.seed, sampleIndex * (uint64_t)W * H + (uint64_t)y * W + x);
        ray.minDistance = ctx.nearClip;
        ray.maxDistance = ctx.farClip;
        ray.flags = RayFlagsCamera;
        ray.depth = 0;
        ray.bsdfPdf = INF;
        ray.x = (uint16_t)x;
        ray.y = (uint16_t)y;
        const float2 jittered = float2((float)x, (float)y) + ray.prng.sample2d();
        const float2 uv = float2(+1, -1) * ((jittered / float2((float)W, (float)H) + ctx.shift) * 2.0f - 1.0f);
        const float aspect = float(H) / float(W);
        ray.origin = (ctx.cameraTransform * float4(0, 0, 0, 1.f)).xyz();
        ray.direction = normalize((ctx.cameraTransform * float4(uv.x, uv.y * aspect, -ctx.focalLength, 0)).xyz());
        ray.weight = float3(1.0f);
        rays[0][slot] = ray;
        trace(ray, intersections[slot]);
    }

    // intersection.metal:22-211
    void handleIntersection(uint32_t rayIndex, int cur, bool lastDepth) {
        const Ray &ray = rays[cur][rayIndex];
        const bool needsToCollectEmission = std::isinf(ray.bsdfPdf) || st.sampling_mode != RMD_SAMPLING_NEE;
        const Intersection &isect = intersections[rayIndex];
        PrngState prng = ray.prng;
        ShadingContext shading;
        shading.rayFlags = ray.flags;
        shading.rnd = prng.sample3d();
        shading.wo = -ray.direction;
        if (isect.distance <= 0.0f) {
            if (needsToCollectEmission) {
                const float misWeight = (st.sampling_mode == RMD_SAMPLING_BSDF) || std::isinf(ray.bsdfPdf)
                                            ? 1.0f
                                            : computeMisWeight(ray.bsdfPdf, lightsEnvmapPdf(ctx, ray.direction));
                evaluateEnvironment(ctx, shading);
                film.add(ray.x, ray.y, misWeight * ray.weight * shading.material.emission);
            }
            return;
        }
        segments++;
        const PerInstanceData &instance = ctx.perInstanceData[isect.instanceIndex];
        uint16_t shaderIndex;
        buildShadingContext(shading, ctx, instance, isect, shaderIndex);
        if (instance.visibility & ray.flags) shadeSurface(shaderIndex, ctx, shading);
        else shading.material.alpha = 0;

        if (needsToCollectEmission && mean(shading.material.emission) != 0) {
            const float misWeight = (st.sampling_mode == RMD_SAMPLING_BSDF) || std::isinf(ray.bsdfPdf)
                                        ? 1.0f
                                        : computeMisWeight(ray.bsdfPdf, lightsShapePdf(ctx, instance, shading));
            film.add(ray.x, ray.y, misWeight * ray.weight * shading.material.emission);
        }

        float3 shNormal;
        if (all_zero(shading.material.normal)) {
            shNormal = shading.trueNormal;
        } else {
            float3 geoNormal = shading.trueNormal;
            if (dot(geoNormal, shading.wo) < 0) geoNormal *= -1.0f;
            shNormal = ensure_valid_reflection(geoNormal, shading.wo, shading.material.normal);
        }

        if (st.sampling_mode != RMD_SAMPLING_BSDF) {
            LightSample neeSample = lightsSample(ctx, shading, prng);
            float bsdfPdf;
            float3 bsdf =
                shading.material.evaluate(shading.wo, neeSample.direction, shNormal, shading.trueNormal, bsdfPdf);
            float3 contribution = neeSample.weight * bsdf * ray.weight;
            if (neeSample.castsShadows) {
                const float misWeight = st.sampling_mode == RMD_SAMPLING_NEE || !neeSample.canBeHit
                                            ? 1.0f
                                            : computeMisWeight(neeSample.pdf, bsdfPdf);
                const float3 neeWeight = misWeight * contribution;
                if (isfinite3(neeWeight) && any_nonzero(neeWeight) && !lastDepth) {
                    // shadow rays of the last pass are never traced (Renderer.swift:623-625)
                    uint32_t idx = shadowCount++;
                    ShadowRay &sr = shadowRays[idx];
                    sr.origin = shading.position;
                    sr.direction = neeSample.direction;
                    sr.minDistance = eps;
                    sr.maxDistance = neeSample.distance - eps;
                    sr.weight = neeWeight;
                    sr.x = ray.x;
                    sr.y = ray.y;
                }
            } else {
                film.add(ray.x, ray.y, ray.weight * contribution);
            }
        }

        BsdfSample sample = shading.material.sample(shading.rnd, -ray.direction, shNormal, shading.trueNormal, ray.flags);
        float3 weight = ray.weight * sample.weight;
        float meanWeight = mean(weight);
        if (!std::isfinite(meanWeight)) return;
        float survivalProb = std::min(meanWeight, 1.f);
        if (prng.sample() < survivalProb) {
            if (lastDepth) return;  // next rays of the last pass are never traced
            uint32_t idx = nextCount++;
            Ray &nextRay = rays[cur ^ 1][idx];
            nextRay.origin = shading.position;
            nextRay.flags = sample.flags;
            nextRay.depth = (uint16_t)(ray.depth + 1);
            nextRay.direction = sample.wi;
            nextRay.minDistance = eps;
            nextRay.maxDistance = INF;
            nextRay.weight = weight * (1 / survivalProb);
            nextRay.x = ray.x;
            nextRay.y = ray.y;
            nextRay.prng = prng;
            nextRay.bsdfPdf = sample.pdf;
        }
    }

    // raytraceAny (raytrace.metal:52-85) fused with handleShadowRays (shadow.metal:6-29)
    void handleShadow(uint32_t i) {
        const ShadowRay &sr = shadowRays[i];
        shadows++;
        if (!ctx.bvh->occluded(sr.origin, sr.direction, sr.minDistance, sr.maxDistance))
            film.add(sr.x, sr.y, sr.weight);
    }

    // Renderer.swift:480-696, one frame
    void run(uint64_t sampleIndex) {
        const uint32_t W = st.width, H = st.height;
        uint32_t count;
        if (st.pixels) {
#pragma omp parallel for schedule(dynamic, 256)
            for (int64_t i = 0; i < (int64_t)st.num_pixels; i++)
                generate(st.pixels[i] % W, st.pixels[i] / W, sampleIndex, (uint32_t)i);
            count = (uint32_t)st.num_pixels;
        } else {
#pragma omp parallel for schedule(dynamic, 4)
            for (int y = 0; y < (int)H; y++)
                for (uint32_t x = 0; x < W; x++)
                    generate(x, (uint32_t)y, sampleIndex, blockLinearIndex(x, (uint32_t)y, W, H));
            count = W * H;
        }
        int cur = 0;
        for (uint32_t depth = 0; depth < st.max_depth; depth++) {
            const bool isMaxDepth = depth + 1 == st.max_depth;
            if (depth > 0) {
#pragma omp parallel for schedule(dynamic, 256)
                for (int i = 0; i < (int)count; i++) trace(rays[cur][i], intersections[i]);
            }
            nextCount = 0;
            shadowCount = 0;
#pragma omp parallel for schedule(dynamic, 256)
            for (int i = 0; i < (int)count; i++) handleIntersection((uint32_t)i, cur, isMaxDepth);
            if (isMaxDepth) break;
            const uint32_t ns = shadowCount;
#pragma omp parallel for schedule(dynamic, 256)
            for (int i = 0; i < (int)ns; i++) handleShadow((uint32_t)i);
            count = nextCount;
            cur ^= 1;
            if (count == 0) break;
        }
    }
};

void fail(char *err, int errlen, const std::string &msg) {
    if (err && errlen > 0) {
        std::strncpy(err, msg.c_str(), (size_t)errlen - 1);
        err[errlen - 1] = 0;
    }
}

}  // namespace

// ---------------------------------------------------------------- scene
extern "C" int oracle_scene_create(const rmd_scene_desc *d, oracle_scene **out, char *err, int errlen) {
    if (!d || !out) return RMD_ERROR_INVALID_ARGUMENT;
    auto s = std::make_unique<oracle_scene>();
    SceneData &ctx = s->data;
    // the textures (RGBA floats, integers normalised), then the 1 x 1 zero texture
    std::vector<std::string> texNames;
    std::vector<int> texChannels;
    for (int i = 0; i < d->num_textures; i++) {
        const rmd_texture &t = d->textures[i];
        Texture tex;
        tex.width = (int)t.width;
        tex.height = (int)t.height;
        tex.channels = (int)t.channels;
        tex.texels.assign((size_t)t.width * t.height, float4(0, 0, 0, 1));
        for (size_t p = 0; p < tex.texels.size(); p++)
            for (uint32_t c = 0; c < t.channels; c++) {
                const size_t k = p * t.channels + c;
                float v;
                if (t.format == RMD_TEXTURE_U8) v = (float)static_cast<const uint8_t *>(t.data)[k] / 255.0f;
                else if (t.format == RMD_TEXTURE_U16) v = (float)static_cast<const uint16_t *>(t.data)[k] / 65535.0f;
                else v = static_cast<const float *>(t.data)[k];
                tex.texels[p][c] = v;
            }
        ctx.textures.push_back(std::move(tex));
        texNames.push_back(t.name ? t.name : "");
        texChannels.push_back((int)t.channels);
    }
    // the sky textures of the TEX_SKY nodes (SkyLoader.generate, MaterialBuilder.swift:350-372), one per
    // distinct set of parameters, after the scene's images
    try {
        auto addSkies = [&](const rmd_material *mats, int count) {
            for (int m = 0; m < count; m++)
                for (int k = 0; k < mats[m].num_nodes; k++) {
                    const rmd_node &n = mats[m].nodes[k];
                    if (!n.type || std::string(n.type) != "TEX_SKY") continue;
                    const SkyParams p = skyParams(n);
                    const std::string key = skyTextureKey(p);
                    if (std::find(texNames.begin(), texNames.end(), key) != texNames.end()) continue;
                    Texture tex;
                    tex.width = tex.height = 512;
                    tex.channels = 4;
                    tex.texels = oracle_sky::skyTexture(512, 512, p.elevation, p.altitude, p.air, p.dust, p.ozone);
                    ctx.textures.push_back(std::move(tex));
                    texNames.push_back(key);
                    texChannels.push_back(4);
                }
        };
        addSkies(d->surface_materials, d->num_surface_materials);
        addSkies(d->light_materials, d->num_light_materials);
    } catch (const CodegenError &e) {
        fail(err, errlen, e.message);
        return e.status;
    }
    ctx.textures.push_back(Texture());
    try {
        // MaterialBuilder: shadeSurface / shadeLight tables
        for (int i = 0; i < d->num_surface_materials; i++)
            ctx.surfaceShaders.push_back(
                std::make_unique<MaterialProgram>(d->surface_materials[i], texNames, texChannels));
        for (int i = 0; i < d->num_light_materials; i++)
            ctx.lightShaders.push_back(std::make_unique<MaterialProgram>(d->light_materials[i], texNames, texChannels));
    } catch (const CodegenError &e) {
        fail(err, errlen, e.message);
        return e.status;
    }
    // ShapeBuilder.build (ShapeBuilder.swift:251-298)
    struct ShapeInfo {
        uint32_t vertexOffset, faceOffset, faceCount;
        float3 boundsMin, boundsMax;
        bool hasEmission;
    };
    std::vector<ShapeInfo> shapes;
    for (int si = 0; si < d->num_shapes; si++) {
        const rmd_shape &sh = d->shapes[si];
        ShapeInfo info;
        info.vertexOffset = (uint32_t)ctx.vertices.size();
        info.faceOffset = (uint32_t)(ctx.vertexIndices.size() / 3);
        info.faceCount = sh.num_faces;
        // PLYReader.m:119-122: the first vertex only updates the minimum (else-if)
        info.boundsMin = float3(INF);
        info.boundsMax = float3(-INF);
        for (uint32_t v = 0; v < sh.num_vertices; v++) {
            float3 p(sh.vertices[3 * v], sh.vertices[3 * v + 1], sh.vertices[3 * v + 2]);
            for (int j = 0; j < 3; j++) {
                if (p[j] < info.boundsMin[j]) info.boundsMin[j] = p[j];
                else if (p[j] > info.boundsMax[j]) info.boundsMax[j] = p[j];
            }
            ctx.vertices.push_back(p);
            ctx.vertexNormals.push_back(float3(sh.normals[3 * v], sh.normals[3 * v + 1], sh.normals[3 * v + 2]));
            ctx.texcoords.push_back(float2(sh.texcoords[2 * v], sh.texcoords[2 * v + 1]));
        }
        info.hasEmission = false;
        for (uint32_t f = 0; f < sh.num_faces; f++) {
            for (int j = 0; j < 3; j++) {
                if (sh.indices[3 * f + j] >= sh.num_vertices) {
                    fail(err, errlen, "vertex index out of range");
                    return RMD_ERROR_INVALID_ARGUMENT;
                }
                ctx.vertexIndices.push_back(sh.indices[3 * f + j]);
            }
            uint16_t m = sh.materials[f];
            if (m >= ctx.surfaceShaders.size()) {
                fail(err, errlen, "face material out of range");
                return RMD_ERROR_INVALID_ARGUMENT;
            }
            ctx.materials.push_back(m);
            if (ctx.surfaceShaders[m]->hasSurfaceEmission()) info.hasEmission = true;
        }
        shapes.push_back(info);
    }
    // EntityBuilder.build (EntityBuilder.swift:79-141) + LightBuilder.add(shapeLight:)
    uint32_t lightFaceOffset = 0;
    struct PendingShapeLight {
        uint32_t instance, shape;
        float3x3 transform;
        uint32_t lightFaceOffset;
    };
    std::vector<PendingShapeLight> pending;
    std::vector<Bvh::Tri> tris;
    for (int ei = 0; ei < d->num_entities; ei++) {
        const rmd_entity &e = d->entities[ei];
        if (e.shape >= shapes.size()) {
            fail(err, errlen, "entity shape out of range");
            return RMD_ERROR_INVALID_ARGUMENT;
        }
        const ShapeInfo &si = shapes[e.shape];
        PerInstanceData inst;
        inst.pointTransform = toMatrix(e.matrix);
        inst.normalTransform = inverseTranspose3(inst.pointTransform);
        inst.vertexOffset = si.vertexOffset;
        inst.faceOffset = si.faceOffset;
        inst.boundsMin = si.boundsMin;
        inst.boundsSize = si.boundsMax - si.boundsMin;
        inst.visibility = (uint8_t)e.visibility;
        inst.shape = e.shape;
        if (si.hasEmission) {
            inst.lightIndex = (uint32_t)pending.size();
            inst.lightFaceOffset = lightFaceOffset;
            inst.lightFaceCount = si.faceCount;
            pending.push_back({(uint32_t)ei, e.shape, inner3x3(inst.pointTransform), lightFaceOffset});
            lightFaceOffset += si.faceCount;
        }
        ctx.perInstanceData.push_back(inst);
        for (uint32_t f = 0; f < si.faceCount; f++) {
            Bvh::Tri t;
            float3 v[3];
            for (int j = 0; j < 3; j++) {
                float3 p = ctx.vertices[si.vertexOffset + ctx.vertexIndices[3 * (si.faceOffset + f) + j]];
                v[j] = (inst.pointTransform * float4(p, 1)).xyz();
            }
            t.v0 = v[0];
            t.v1 = v[1];
            t.v2 = v[2];
            t.instance = (uint32_t)ei;
            t.prim = f;
            tris.push_back(t);
        }
    }
    s->triangles = tris.size();
    ctx.bvh = std::make_unique<Bvh>();
    ctx.bvh->build(std::move(tris));
    // LightBuilder.build (LightBuilder.swift:179-281)
    ctx.lightFaces.assign(lightFaceOffset, 0.0f);
    for (auto &p : pending) {
        const ShapeInfo &si = shapes[p.shape];
        ShapeLight sl;
        sl.instanceIndex = p.instance;
        sl.emissiveArea =
            buildLightDistribution(p.transform, ctx.vertexIndices.data() + 3 * (size_t)si.faceOffset,
                                   ctx.vertices.data() + si.vertexOffset, si.faceCount,
                                   ctx.lightFaces.data() + p.lightFaceOffset);
        ctx.shapeLights.push_back(sl);
    }
    auto info = [](const rmd_light_info &i) {
        LightInfo r;
        r.shaderIndex = i.shader_index;
        r.castsShadows = i.casts_shadows != 0;
        r.usesMIS = i.uses_mis != 0;
        return r;
    };
    for (int i = 0; i < d->num_area_lights; i++) {
        const rmd_area_light &l = d->area_lights[i];
        AreaLight a;
        a.info = info(l.info);
        for (int c = 0; c < 3; c++)
            a.transform.c[c] = float4(l.transform[4 * c], l.transform[4 * c + 1], l.transform[4 * c + 2],
                                      l.transform[4 * c + 3]);
        a.color = float3(l.color[0], l.color[1], l.color[2]);
        a.isCircular = l.is_circular != 0;
        ctx.areaLights.push_back(a);
    }
    for (int i = 0; i < d->num_point_lights; i++) {
        const rmd_point_light &l = d->point_lights[i];
        PointLight p;
        p.info = info(l.info);
        p.location = float3(l.location[0], l.location[1], l.location[2]);
        p.radius = l.radius;
        p.color = float3(l.color[0], l.color[1], l.color[2]);
        ctx.pointLights.push_back(p);
    }
    for (int i = 0; i < d->num_sun_lights; i++) {
        const rmd_sun_light &l = d->sun_lights[i];
        SunLight p;
        p.info = info(l.info);
        p.direction = float3(l.direction[0], l.direction[1], l.direction[2]);
        p.cosAngle = l.cos_angle;
        p.color = float3(l.color[0], l.color[1], l.color[2]);
        ctx.sunLights.push_back(p);
    }
    for (int i = 0; i < d->num_spot_lights; i++) {
        const rmd_spot_light &l = d->spot_lights[i];
        SpotLight p;
        p.info = info(l.info);
        p.location = float3(l.location[0], l.location[1], l.location[2]);
        p.direction = float3(l.direction[0], l.direction[1], l.direction[2]);
        p.radius = l.radius;
        p.color = float3(l.color[0], l.color[1], l.color[2]);
        p.spotSize = l.spot_size;
        p.spotBlend = l.spot_blend;
        ctx.spotLights.push_back(p);
    }
    ctx.numLightsTotal = 1 + (int)ctx.areaLights.size() + (int)ctx.pointLights.size() + (int)ctx.sunLights.size() +
                         (int)ctx.spotLights.size() + (int)ctx.shapeLights.size();
    ctx.worldShaderIndex = d->world_shader;
    // camera
    ctx.cameraTransform = toMatrix(d->camera.transform);
    ctx.nearClip = d->camera.near_clip;
    ctx.farClip = d->camera.far_clip;
    ctx.focalLength = d->camera.focal_length;
    ctx.shift = float2(d->camera.shift[0], d->camera.shift[1]);
    // LightBuilder.prepareEnvironmentMapSampling
    int exponent = d->envmap_exponent;
    if (exponent < 0 || exponent > 12) {
        fail(err, errlen, "envmap_exponent out of range");
        return RMD_ERROR_INVALID_ARGUMENT;
    }
    buildEnvironmentMap(ctx, exponent);
    *out = s.release();
    return 0;
}

extern "C" void oracle_scene_destroy(oracle_scene *s) { delete s; }

// Per surface material: 1 if it emits (Material.hasSurfaceEmission), which makes
// a shape carrying it a shape light.
extern "C" int oracle_surface_emissive(const oracle_scene *s, uint8_t *out) {
    for (size_t i = 0; i < s->data.surfaceShaders.size(); i++) out[i] = s->data.surfaceShaders[i]->hasSurfaceEmission();
    return (int)s->data.surfaceShaders.size();
}

// Renderer.updateProjection / scene.camera (Renderer.swift:749-755)
extern "C" int oracle_scene_set_camera(oracle_scene *s, const rmd_camera *c) {
    if (!s || !c) return RMD_ERROR_INVALID_ARGUMENT;
    s->data.cameraTransform = toMatrix(c->transform);
    s->data.nearClip = c->near_clip;
    s->data.farClip = c->far_clip;
    s->data.focalLength = c->focal_length;
    s->data.shift = float2(c->shift[0], c->shift[1]);
    return 0;
}

extern "C" int oracle_scene_info(const oracle_scene *s, uint64_t *triangles, int32_t *num_lights_total,
                                 int32_t *num_shape_lights) {
    if (triangles) *triangles = s->triangles;
    if (num_lights_total) *num_lights_total = s->data.numLightsTotal;
    if (num_shape_lights) *num_shape_lights = (int32_t)s->data.shapeLights.size();
    return 0;
}

template <typename FilmT>
static void renderFrames(oracle_scene *s, const oracle_settings *st, double *film_rgb, uint64_t *stats) {
    Film<FilmT> film;
    film.W = st->width;
    film.H = st->height;
    film.rgba.assign(4 * (size_t)st->width * st->height, (FilmT)0);
    uint64_t segs = 0, shadows = 0;
    for (uint32_t f = 0; f < st->spp; f++) {
        Frame<FilmT> frame(s->data, *st, film);
        frame.run((uint64_t)st->first_sample + f);
        segs += frame.segments;
        shadows += frame.shadows;
    }
    for (size_t p = 0; p < (size_t)st->width * st->height; p++)
        for (int c = 0; c < 3; c++) film_rgb[3 * p + c] = (double)film.rgba[4 * p + c];
    if (stats) {
        stats[0] = (uint64_t)st->spp * (st->pixels ? st->num_pixels : (uint64_t)st->width * st->height);
        stats[1] = segs;
        stats[2] = shadows;
    }
}

extern "C" int oracle_render(oracle_scene *s, const oracle_settings *st, double *film_rgb, uint64_t *stats) {
    if (!s || !st || !film_rgb || st->width == 0 || st->height == 0 || st->width > 65535 || st->height > 65535 ||
        st->max_depth == 0)
        return RMD_ERROR_INVALID_ARGUMENT;
    if (st->pixels) {  // each pixel once, inside the image
        std::vector<uint8_t> seen((size_t)st->width * st->height, 0);
        for (uint64_t i = 0; i < st->num_pixels; i++) {
            const uint32_t p = st->pixels[i];
            if (p >= seen.size() || seen[p]) return RMD_ERROR_INVALID_ARGUMENT;
            seen[p] = 1;
        }
    }
#ifdef _OPENMP
    if (st->threads > 0) omp_set_num_threads(st->threads);
#endif
    if (st->film_fp64) renderFrames<double>(s, st, film_rgb, stats);
    else renderFrames<float>(s, st, film_rgb, stats);
    return 0;
}

// ------------------------------------------------------------- film read-out
// normalizeImage.metal:11-19, the Hable filmic curve with its six constants
static float3 tonemapHablePartial(float3 x) {
    const float hA = 0.15f, hB = 0.50f, hC = 0.10f, hD = 0.20f, hE = 0.02f, hF = 0.30f;
    return ((x * (hA * x + float3(hC * hB)) + float3(hD * hE)) / (x * (hA * x + float3(hB)) + float3(hD * hF))) -
           float3(hE / hF);
}

extern "C" void oracle_normalize_image(const float *film, uint32_t width, uint32_t height, float exposure,
                                       int32_t accumulate, uint32_t frame_index, uint32_t tonemapping, float *out) {
    const size_t n = (size_t)width * height;
    for (size_t i = 0; i < n; i++) {
        // normalizeImage.metal:45-46
        float3 c = exposure * float3(film[4 * i], film[4 * i + 1], film[4 * i + 2]);
        if (accumulate) c = c / float3((float)(frame_index + 1));
        if (tonemapping == RMD_TONEMAP_HABLE) {  // :21-28, exposure bias 2 and white point 11.2
            const float3 curr = tonemapHablePartial(c * 2.0f);
            const float3 whiteScale = float3(1.0f) / tonemapHablePartial(float3(11.2f));
            c = curr * whiteScale;
        } else if (tonemapping == RMD_TONEMAP_ACES) {  // :30-37, Narkowicz's fit
            const float tA = 2.51f, tB = 0.03f, tC = 2.43f, tD = 0.59f, tE = 0.14f;
            c = (c * (tA * c + float3(tB))) / (c * (tC * c + float3(tD)) + float3(tE));
            // saturate: fmax/fmin semantics, so an overflow's NaN becomes 0
            c = float3(std::fmin(std::fmax(c.x, 0.0f), 1.0f), std::fmin(std::fmax(c.y, 0.0f), 1.0f),
                       std::fmin(std::fmax(c.z, 0.0f), 1.0f));
        }
        out[4 * i] = c.x;
        out[4 * i + 1] = c.y;
        out[4 * i + 2] = c.z;
        out[4 * i + 3] = 1.0f;
    }
}

// ---------------------------------------------------------------- sky hooks
extern "C" void oracle_sky_texture(int32_t width, int32_t height, float sun_elevation, float altitude, float air,
                                   float dust, float ozone, float *rgba) {
    const std::vector<float4> t = oracle_sky::skyTexture(width, height, sun_elevation, altitude, air, dust, ozone);
    std::memcpy(rgba, t.data(), t.size() * sizeof(float4));
}

extern "C" void oracle_sky_data(float sun_elevation, float sun_rotation, int32_t sun_disc, float sun_size,
                                float sun_intensity, float altitude, float air, float dust, float *data10) {
    oracle_sky::skyData(sun_elevation, sun_rotation, sun_disc != 0, sun_size, sun_intensity, altitude, air, dust,
                        data10);
}

// ---------------------------------------------------------------- unit hooks
extern "C" void oracle_prng(int32_t mode, uint64_t a, uint64_t b, int32_t n, float *out) {
    PrngState p = mode == RMD_RNG_TEA ? PrngState::tea((uint32_t)a, (uint32_t)b) : PrngState::pcg(a, b);
    for (int i = 0; i < n; i++) out[i] = p.sample();
}

extern "C" int oracle_trace(const oracle_scene *s, const float *rays, int32_t n, int32_t any, float *out,
                            uint32_t *instances) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; i++) {
        const float *r = rays + 8 * (size_t)i;
        float3 o(r[0], r[1], r[2]), d(r[4], r[5], r[6]);
        float *w = out + 4 * (size_t)i;
        if (any == 1) {
            w[0] = s->data.bvh->occluded(o, d, r[3], r[7]) ? 1.0f : -1.0f;
            w[1] = w[2] = w[3] = 0;
            if (instances) instances[i] = 0;
        } else {
            HitRecord h;
            if (s->data.bvh->intersect(o, d, r[3], r[7], h, any == 2)) {
                w[0] = h.t;
                w[1] = h.b0;
                w[2] = h.b1;
                w[3] = uint_as_float(h.prim);
                if (instances) instances[i] = h.instance;
            } else {
                w[0] = -1;
                w[1] = w[2] = w[3] = 0;
                if (instances) instances[i] = 0xffffffffu;
            }
        }
    }
    return 0;
}

extern "C" void oracle_fractal_noise3(const float *p, int32_t n, float detail, float roughness, float *out) {
    for (int i = 0; i < n; i++)
        out[i] = noise::fractal_noise(float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), detail, roughness);
}

// record: position, normal, trueNormal, generated, uv, wo, wi, rnd (8 x float3), rayFlags, tangent tu (3) = 28 floats
// out: emission(3), eval(3), evalPdf, sample wi(3), sample weight(3), sample pdf, sample flags, alpha = 16 floats
extern "C" int oracle_material_eval(const oracle_scene *s, int32_t material, const float *records, int32_t n,
                                    float *out) {
    if (material < 0 || material >= (int)s->data.surfaceShaders.size()) return RMD_ERROR_INVALID_ARGUMENT;
    for (int i = 0; i < n; i++) {
        const float *r = records + 28 * (size_t)i;
        auto v3 = [&](int k) { return float3(r[3 * k], r[3 * k + 1], r[3 * k + 2]); };
        ShadingContext sh;
        sh.position = v3(0);
        sh.normal = v3(1);
        sh.trueNormal = v3(2);
        sh.generated = v3(3);
        sh.uv = v3(4);
        sh.wo = v3(5);
        float3 wi = v3(6);
        sh.rnd = v3(7);
        sh.rayFlags = (uint8_t)r[24];
        sh.object = sh.generated;
        sh.tu = float3(r[25], r[26], r[27]);  // the tangent frame: tu given, tv = normal x tu
        sh.tv = cross(sh.normal, sh.tu);
        shadeSurface((uint16_t)material, s->data, sh);
        float3 shNormal;
        if (all_zero(sh.material.normal)) {
            shNormal = sh.trueNormal;
        } else {
            float3 geoNormal = sh.trueNormal;
            if (dot(geoNormal, sh.wo) < 0) geoNormal *= -1.0f;
            shNormal = ensure_valid_reflection(geoNormal, sh.wo, sh.material.normal);
        }
        float pdf;
        float3 f = sh.material.evaluate(sh.wo, wi, shNormal, sh.trueNormal, pdf);
        BsdfSample bs = sh.material.sample(sh.rnd, sh.wo, shNormal, sh.trueNormal, sh.rayFlags);
        float *o = out + 16 * (size_t)i;
        o[0] = sh.material.emission.x; o[1] = sh.material.emission.y; o[2] = sh.material.emission.z;
        o[3] = f.x; o[4] = f.y; o[5] = f.z; o[6] = pdf;
        o[7] = bs.wi.x; o[8] = bs.wi.y; o[9] = bs.wi.z;
        o[10] = bs.weight.x; o[11] = bs.weight.y; o[12] = bs.weight.z;
        o[13] = bs.pdf; o[14] = (float)bs.flags; o[15] = sh.material.alpha;
    }
    return 0;
}
