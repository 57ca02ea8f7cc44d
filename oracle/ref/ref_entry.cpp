// C entry points into the reference's own device code, built for the host
// (see Makefile).  TEST INFRASTRUCTURE ONLY: the pinning tests run these
// beside the oracle's restatement on the same inputs.
//
// Compiled from the reference: PrngState, utils (noise, warp, math, color),
// the BSDF lobes and UberShader, the node library, ShadingContext::build, the
// lights (Lights, Area/Point/Sun/Spot/Shape lights, the world light), and the
// kernels raytrace / raytraceAny, handleIntersections, handleShadowRays and
// the environment-map build / reduce / normalize.  Restated here (their
// sources need what this build lacks: Swift, Apple's intersector, the lore
// lens library): the host scheduling of Renderer.execute, the scene set-up of
// ShapeBuilder / EntityBuilder / LightBuilder, the pinhole camera of
// generateRays, and the intersector itself (the oracle's BVH, ref_bvh.cpp).
#include <vector>

#include <metal_stdlib>
using namespace metal;

#include <bridge/PrngState.hpp>
#include "PrngState.cpp"
#include <device/utils/noise.hpp>
#include <device/bsdf/UberShader.hpp>
#include <device/nodes/nodes.hpp>
#include <device/ShadingContext.metal>
#include <device/lights/Lights.metal>
#include <device/lights/AreaLight.metal>
#include <device/lights/PointLight.metal>
#include <device/lights/SunLight.metal>
#include <device/lights/SpotLight.metal>
#include <device/lights/ShapeLight.metal>
#include <device/kernels/shading/raytrace.metal>
#include <device/kernels/shading/intersection.metal>
#include <device/kernels/shading/shadow.metal>
#include <device/kernels/envmap/build.metal>
#include <device/kernels/envmap/reduce.metal>
#include <device/kernels/envmap/normalize.metal>
#include <device/kernels/utils/normalizeImage.metal>

#include <memory>
#include <string>
#include <vector>

#include "../../include/raymond.h"

// generated material functions (gen_materials.py), one table per scene
struct RefMaterialTable {
    const char *name;
    void (*surface)(MaterialIndex, device Context &, thread ShadingContext &);
    void (*light)(MaterialIndex, device Context &, thread ShadingContext &);
    int numSurface, numLight;
};
#include "materials.inc"

static const RefMaterialTable *g_table = nullptr;  // the scene being set up or rendered

static const RefMaterialTable *findTable(const char *name) {
    for (int i = 0; i < kNumRefMaterialTables; i++)
        if (std::string(kRefMaterialTables[i].name) == name) return &kRefMaterialTables[i];
    return nullptr;
}

// the JIT's entry points (device/shading.hpp), bound to the active table
void shadeSurface(MaterialIndex shaderIndex, device Context &ctx, thread ShadingContext &shading) {
    g_table->surface(shaderIndex, ctx, shading);
}
void shadeLight(MaterialIndex shaderIndex, device Context &ctx, thread ShadingContext &shading) {
    g_table->light(shaderIndex, ctx, shading);
}

extern "C" {
void *refbvh_build(const float *tris, const uint32_t *instance, const uint32_t *prim, size_t n);
void refbvh_destroy(void *b);
int refbvh_intersect(const void *b, const float *o, const float *d, float tmin, float tmax, int any, float *t,
                     uint32_t *instance, uint32_t *prim, float *b0, float *b1);
}

// Apple's intersector, on the oracle's BVH.  A hit reports the distance,
// instance and primitive and the barycentric weights of v1 and v2 (Metal's
// triangle_barycentric_coord; raytrace.metal turns them back into (w0, w1));
// a miss reports distance -1.
namespace metal {
namespace raytracing {
intersection_result hostIntersect(const void *bvh, const ray &r, bool any) {
    intersection_result res;
    if (!bvh) return res;
    const float o[3] = {r.origin.x, r.origin.y, r.origin.z};
    const float d[3] = {r.direction.x, r.direction.y, r.direction.z};
    float t = -1, b0 = 0, b1 = 0;
    uint32_t inst = 0, prim = 0;
    if (refbvh_intersect(bvh, o, d, r.min_distance, r.max_distance, any ? 1 : 0, &t, &inst, &prim, &b0, &b1)) {
        res.distance = t;
        res.instance_id = inst;
        res.primitive_id = prim;
        res.triangle_barycentric_coord = float2(b1, 1.0f - b0 - b1);
    }
    return res;
}
}  // namespace raytracing
}  // namespace metal

namespace {

struct RefScene {
    const RefMaterialTable *table = nullptr;
    std::vector<Vertex> vertices;
    std::vector<Normal> normals;
    std::vector<TexCoord> texcoords;
    std::vector<IndexTriplet> indices;
    std::vector<MaterialIndex> materials;
    std::vector<PerInstanceData> instances;
    std::vector<AreaLight> areaLights;
    std::vector<PointLight> pointLights;
    std::vector<SunLight> sunLights;
    std::vector<SpotLight> spotLights;
    std::vector<ShapeLight> shapeLights;
    std::vector<float> lightFaces, envPdfs, envMipmap;
    Context ctx;
    instance_acceleration_structure accel;
    ~RefScene() {
        if (accel.bvh) refbvh_destroy(const_cast<void *>(accel.bvh));
    }
};

float4x4 matrix4(const float *m) {  // column-major
    return float4x4(float4(m[0], m[1], m[2], m[3]), float4(m[4], m[5], m[6], m[7]),
                    float4(m[8], m[9], m[10], m[11]), float4(m[12], m[13], m[14], m[15]));
}
float3x3 inner3x3(const float4x4 &m) { return float3x3(m[0].xyz, m[1].xyz, m[2].xyz); }
float3x3 inverse3x3(const float3x3 &m) {
    const float3 a = m[0], b = m[1], c = m[2];
    const float3 r0 = cross(b, c), r1 = cross(c, a), r2 = cross(a, b);
    const float invDet = 1.0f / dot(a, r0);
    return transpose(float3x3(r0 * invDet, r1 * invDet, r2 * invDet));
}

// distribution.m:7-39: per-face cumulative area of a shape light, in double
float buildLightDistribution(float3x3 transform, const IndexTriplet *indices, const Vertex *vertices,
                             uint32_t faceCount, float *output) {
    double accumulated = 0;
    for (uint32_t i = 0; i < faceCount; i++) {
        const IndexTriplet idx = indices[i];
        const float3 v0 = vertices[idx.x], v1 = vertices[idx.y], v2 = vertices[idx.z];
        const float3 tn = cross(transform * (v2 - v0), transform * (v2 - v1));
        const float area = length(tn) / 2;
        output[i] = (float)(accumulated += area);
    }
    for (uint32_t i = 0; i < faceCount; i++) output[i] = (float)(output[i] / accumulated);
    return (float)accumulated;
}

}  // namespace

extern "C" {

void ref_prng_tea(uint32_t a, uint32_t b, int n, float *out) {
    PrngState p(a, b);
    for (int i = 0; i < n; i++) out[i] = p.sample();
}

void ref_fractal_noise3(const float *p, int n, float detail, float roughness, float *out) {
    for (int i = 0; i < n; i++) out[i] = fractal_noise(float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), detail, roughness);
}

int ref_num_materials() { return findTable("pin")->numSurface; }

// One material of pin_materials.py on shading records, evaluated and sampled
// the way handleIntersections does (intersection.metal:100-104,135-144,149-185).
// Record (28 floats): position, normal, trueNormal, generated, uv, wo, wi, rnd
// (float3 each), rayFlags, tangent tu (bitangent normal x tu).  Output (16 floats): emission, evaluate
// value, evaluate pdf, sampled wi, sampled weight, sampled pdf, sampled flags,
// alpha.
// The pinning materials' textures: slot `slot` becomes a w x h RGBA float
// image (copied), as the reference's Context.textures holds them.
static std::vector<float4> g_textureData[NUMBER_OF_TEXTURES];
static Context g_materialCtx;
int ref_set_texture(int slot, const float *rgba, int w, int h) {
    if (slot < 0 || slot >= NUMBER_OF_TEXTURES || w <= 0 || h <= 0) return 1;
    g_textureData[slot].resize((size_t)w * h);
    for (size_t i = 0; i < g_textureData[slot].size(); i++)
        g_textureData[slot][i] = float4(rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2], rgba[4 * i + 3]);
    g_materialCtx.textures[slot].data = g_textureData[slot].data();
    g_materialCtx.textures[slot].width = (uint)w;
    g_materialCtx.textures[slot].height = (uint)h;
    return 0;
}

int ref_material_eval(int material, const float *records, int n, float *out) {
    const RefMaterialTable *table = findTable("pin");
    if (material < 0 || material >= table->numSurface) return 1;
    g_table = table;
    Context &ctx = g_materialCtx;  // the pinned nodes read only its textures
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
        const float3 wi = v3(6);
        sh.rnd = v3(7);
        sh.rayFlags = RayFlags((uint8_t)r[24]);
        sh.object = sh.generated;
        sh.tu = float3(r[25], r[26], r[27]);  // the tangent frame: tu given, tv = normal x tu
        sh.tv = cross(sh.normal, sh.tu);
        sh.distance = 0;
        shadeSurface((MaterialIndex)material, ctx, sh);
        float3 shNormal;
        if (all(sh.material.normal == 0)) {
            shNormal = sh.trueNormal;
        } else {
            float3 geoNormal = sh.trueNormal;
            if (dot(geoNormal, sh.wo) < 0) geoNormal *= -1;
            shNormal = ensure_valid_reflection(geoNormal, sh.wo, sh.material.normal);
        }
        float pdf;
        const float3 f = sh.material.evaluate(sh.wo, wi, shNormal, sh.trueNormal, pdf);
        const BsdfSample bs = sh.material.sample(sh.rnd, sh.wo, shNormal, sh.trueNormal, sh.rayFlags);
        float *o = out + 16 * (size_t)i;
        o[0] = sh.material.emission.x; o[1] = sh.material.emission.y; o[2] = sh.material.emission.z;
        o[3] = f.x; o[4] = f.y; o[5] = f.z; o[6] = pdf;
        o[7] = bs.wi.x; o[8] = bs.wi.y; o[9] = bs.wi.z;
        o[10] = bs.weight.x; o[11] = bs.weight.y; o[12] = bs.weight.z;
        o[13] = bs.pdf; o[14] = (float)bs.flags; o[15] = sh.material.alpha;
    }
    return 0;
}

// Scene set-up as ShapeBuilder / EntityBuilder / LightBuilder do it
// (ShapeBuilder.swift:251-298, EntityBuilder.swift:79-141,
// LightBuilder.swift:83-167,179-281).  `table` names the generated material
// table of this scene; emissive[m] says whether surface material m emits
// (a shape with such a face becomes a shape light).
void *ref_scene_create(const rmd_scene_desc *d, const char *table, const uint8_t *emissive) {
    auto s = std::make_unique<RefScene>();
    s->table = findTable(table);
    if (!s->table) return nullptr;
    g_table = s->table;
    struct ShapeInfo {
        uint32_t vertexOffset, faceOffset, faceCount;
        float3 boundsMin, boundsMax;
        bool hasEmission;
    };
    std::vector<ShapeInfo> shapes;
    for (int si = 0; si < d->num_shapes; si++) {
        const rmd_shape &sh = d->shapes[si];
        ShapeInfo info;
        info.vertexOffset = (uint32_t)s->vertices.size();
        info.faceOffset = (uint32_t)s->indices.size();
        info.faceCount = sh.num_faces;
        info.boundsMin = float3(INFINITY);
        info.boundsMax = float3(-INFINITY);
        for (uint32_t v = 0; v < sh.num_vertices; v++) {
            const float3 p(sh.vertices[3 * v], sh.vertices[3 * v + 1], sh.vertices[3 * v + 2]);
            for (int j = 0; j < 3; j++) {  // PLYReader.m:119-122 (else-if)
                if (p[j] < info.boundsMin[j]) info.boundsMin[j] = p[j];
                else if (p[j] > info.boundsMax[j]) info.boundsMax[j] = p[j];
            }
            s->vertices.push_back(p);
            s->normals.push_back(float3(sh.normals[3 * v], sh.normals[3 * v + 1], sh.normals[3 * v + 2]));
            s->texcoords.push_back(float2(sh.texcoords[2 * v], sh.texcoords[2 * v + 1]));
        }
        info.hasEmission = false;
        for (uint32_t f = 0; f < sh.num_faces; f++) {
            IndexTriplet t;
            t.x = sh.indices[3 * f];
            t.y = sh.indices[3 * f + 1];
            t.z = sh.indices[3 * f + 2];
            s->indices.push_back(t);
            s->materials.push_back(sh.materials[f]);
            if (emissive[sh.materials[f]]) info.hasEmission = true;
        }
        shapes.push_back(info);
    }
    std::vector<float> tris;
    std::vector<uint32_t> triInstance, triPrim;
    uint32_t lightFaceOffset = 0;
    struct PendingLight {
        uint32_t instance, shape, lightFaceOffset;
        float3x3 transform;
    };
    std::vector<PendingLight> pending;
    for (int ei = 0; ei < d->num_entities; ei++) {
        const rmd_entity &e = d->entities[ei];
        const ShapeInfo &si = shapes[e.shape];
        const float4x4 transform = matrix4(e.matrix);
        PerInstanceData inst;
        inst.vertexOffset = si.vertexOffset;
        inst.faceOffset = si.faceOffset;
        inst.lightIndex = 0xFFFFFFFFu;  // LightIndex.max
        inst.lightFaceOffset = 0;
        inst.lightFaceCount = 0;
        if (si.hasEmission) {
            inst.lightIndex = (uint32_t)pending.size();
            inst.lightFaceOffset = lightFaceOffset;
            inst.lightFaceCount = si.faceCount;
            pending.push_back({(uint32_t)ei, e.shape, lightFaceOffset, inner3x3(transform)});
            lightFaceOffset += si.faceCount;
        }
        inst.boundsMin = si.boundsMin;
        inst.boundsSize = si.boundsMax - si.boundsMin;
        inst.pointTransform = transform;
        inst.normalTransform = transpose(inverse3x3(inner3x3(transform)));
        inst.visibility = RayFlags(e.visibility);
        s->instances.push_back(inst);
        for (uint32_t f = 0; f < si.faceCount; f++) {
            const IndexTriplet &t = s->indices[si.faceOffset + f];
            for (uint32_t k : {t.x, t.y, t.z}) {
                const float4 p = transform * float4(s->vertices[si.vertexOffset + k], 1.0f);
                tris.push_back(p.x);
                tris.push_back(p.y);
                tris.push_back(p.z);
            }
            triInstance.push_back((uint32_t)ei);
            triPrim.push_back(f);
        }
    }
    if (!triPrim.empty()) s->accel.bvh = refbvh_build(tris.data(), triInstance.data(), triPrim.data(), triPrim.size());
    s->lightFaces.assign(std::max<uint32_t>(1, lightFaceOffset), 0.0f);
    for (const PendingLight &p : pending) {
        const ShapeInfo &si = shapes[p.shape];
        ShapeLight l;
        l.instanceIndex = p.instance;
        l.emissiveArea = buildLightDistribution(p.transform, s->indices.data() + si.faceOffset,
                                                s->vertices.data() + si.vertexOffset, si.faceCount,
                                                s->lightFaces.data() + p.lightFaceOffset);
        s->shapeLights.push_back(l);
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
            a.transform[c] = float4(l.transform[4 * c], l.transform[4 * c + 1], l.transform[4 * c + 2],
                                    l.transform[4 * c + 3]);
        a.color = float3(l.color[0], l.color[1], l.color[2]);
        a.isCircular = l.is_circular != 0;
        s->areaLights.push_back(a);
    }
    for (int i = 0; i < d->num_point_lights; i++) {
        const rmd_point_light &l = d->point_lights[i];
        PointLight p;
        p.info = info(l.info);
        p.location = float3(l.location[0], l.location[1], l.location[2]);
        p.radius = l.radius;
        p.color = float3(l.color[0], l.color[1], l.color[2]);
        s->pointLights.push_back(p);
    }
    for (int i = 0; i < d->num_sun_lights; i++) {
        const rmd_sun_light &l = d->sun_lights[i];
        SunLight p;
        p.info = info(l.info);
        p.direction = float3(l.direction[0], l.direction[1], l.direction[2]);
        p.cosAngle = l.cos_angle;
        p.color = float3(l.color[0], l.color[1], l.color[2]);
        s->sunLights.push_back(p);
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
        s->spotLights.push_back(p);
    }
    Context &c = s->ctx;
    c.vertices = s->vertices.data();
    c.vertexIndices = s->indices.data();
    c.vertexNormals = s->normals.data();
    c.texcoords = s->texcoords.data();
    c.perInstanceData = s->instances.data();
    c.materials = s->materials.data();
    c.camera.transform = matrix4(d->camera.transform);
    c.camera.nearClip = d->camera.near_clip;
    c.camera.farClip = d->camera.far_clip;
    c.camera.focalLength = d->camera.focal_length;
    c.camera.shift = float2(d->camera.shift[0], d->camera.shift[1]);
    Lights &L = c.lights;
    L.numAreaLights = (int)s->areaLights.size();
    L.numPointLights = (int)s->pointLights.size();
    L.numSunLights = (int)s->sunLights.size();
    L.numSpotLights = (int)s->spotLights.size();
    L.numShapeLights = (int)s->shapeLights.size();
    L.numLightsTotal = 1 + L.numAreaLights + L.numPointLights + L.numSunLights + L.numSpotLights + L.numShapeLights;
    L.lightFaces = s->lightFaces.data();
    L.areaLights = s->areaLights.data();
    L.pointLights = s->pointLights.data();
    L.sunLights = s->sunLights.data();
    L.spotLights = s->spotLights.data();
    L.shapeLights = s->shapeLights.data();
    // prepareEnvironmentMapSampling (LightBuilder.swift:83-167)
    const int exponent = d->envmap_exponent;
    const int resolution = 1 << exponent;
    size_t mipmapSize = 0;
    for (int e = 0; e <= exponent; e++) mipmapSize += (size_t)1 << (2 * e);
    s->envMipmap.assign(mipmapSize, 0.0f);
    s->envPdfs.assign((size_t)resolution * resolution, 0.0f);
    L.worldLight.shaderIndex = d->world_shader;
    L.worldLight.resolution = resolution;
    L.worldLight.pdfs = s->envPdfs.data();
    L.worldLight.mipmap = s->envMipmap.data();
    size_t bufferOffset = mipmapSize - (size_t)resolution * resolution;
#pragma omp parallel for schedule(dynamic, 8)
    for (int ty = 0; ty < resolution; ty++)
        for (int tx = 0; tx < resolution; tx++)
            buildEnvironmentMap(c, s->envMipmap.data() + bufferOffset, s->envPdfs.data(), uint2(tx, ty),
                                uint2(resolution, resolution));
    for (int e = exponent - 1; e >= 0; e--) {
        const int cur = 1 << e;
        bufferOffset -= (size_t)cur * cur;
        for (int ty = 0; ty < cur; ty++)
            for (int tx = 0; tx < cur; tx++)
                reduceEnvironmentMap(s->envMipmap.data() + bufferOffset, uint2(tx, ty), uint2(cur, cur));
    }
    for (int i = 0; i < resolution * resolution; i++)
        normalizeEnvironmentMap(s->envMipmap[0], s->envPdfs.data(), (uint)i, (uint)(resolution * resolution));
    return s.release();
}

void ref_scene_destroy(void *s) { delete static_cast<RefScene *>(s); }

// Renderer.execute (Renderer.swift:480-696) for `frames` frames of one sample
// each: generateRays (pinhole branch, generate.metal:88-121,165-191), then per
// depth raytrace, handleIntersections, raytraceAny and handleShadowRays, with
// the frame's randomSeed = first_frame + frame + 1 (Renderer.swift:438-443).
// Each kernel's threads run as the iterations of an OpenMP loop; within one
// depth every pixel has at most one ray, so film writes never collide.
// film: W*H float4, accumulated (rgb sums, write count in w).
int ref_render(void *scene, uint32_t W, uint32_t H, uint32_t frames, uint32_t maxDepth, uint32_t samplingMode,
               uint32_t firstFrame, float *film) {
    RefScene *s = static_cast<RefScene *>(scene);
    g_table = s->table;
    Context &ctx = s->ctx;
    const uint32_t N = W * H;
    std::vector<Ray> rays(2 * (size_t)N);
    std::vector<ShadowRay> shadowRays(N);
    std::vector<Intersection> intersections(N);
    texture2d<float, access::read_write> image;
    image.data = reinterpret_cast<float4 *>(film);
    image.width = W;
    image.height = H;
    Uniforms uniforms{};
    uniforms.numLensSurfaces = 0;
    uniforms.accumulate = true;
    uniforms.samplingMode = SamplingMode(samplingMode);
    for (uint32_t frame = 0; frame < frames; frame++) {
        uniforms.frameIndex = firstFrame + frame;
        uniforms.randomSeed = firstFrame + frame + 1;
        // generateRays, pinhole: block-linear index over 8x8 threadgroups
#pragma omp parallel for schedule(static)
        for (uint32_t y = 0; y < H; y++) {
            for (uint32_t x = 0; x < W; x++) {
                const uint32_t gx = x / 8, gy = y / 8;
                const uint32_t awx = std::min(8u, W - gx * 8), awy = std::min(8u, H - gy * 8);
                const int rayIndex = (int)((x % 8) + (y % 8) * awx + gx * 8 * awy + gy * 8 * W);
                Ray ray;
                ray.prng = PrngState(uniforms.randomSeed, rayIndex);
                ray.minDistance = ctx.camera.nearClip;
                ray.maxDistance = ctx.camera.farClip;
                ray.flags = RayFlagsCamera;
                ray.depth = 0;
                ray.bsdfPdf = INFINITY;
                ray.x = x;
                ray.y = y;
                const float2 jittered = float2(float(x), float(y)) + ray.prng.sample2d();
                const float2 uv = float2(+1, -1) * ((jittered / float2(float(W), float(H)) + ctx.camera.shift) * 2.0f - 1.0f);
                const float aspect = float(H) / float(W);
                ray.origin = (ctx.camera.transform * float4(0, 0, 0, 1.f)).xyz;
                ray.direction =
                    normalize((ctx.camera.transform * float4(uv.x, uv.y * aspect, -ctx.camera.focalLength, 0)).xyz);
                ray.weight = 1;
                rays[rayIndex] = ray;
            }
        }
        uint rayCount[64] = {};  // per depth, as the reference's rayCountBuffer
        uint shadowCount[64] = {};
        rayCount[0] = N;
#pragma omp parallel for schedule(dynamic, 256)
        for (uint i = 0; i < N; i++) raytrace(rays.data(), rayCount[0], intersections.data(), s->accel, i);
        size_t cur = 0, next = N;
        for (uint32_t depth = 0; depth < maxDepth && depth < 63; depth++) {
            const bool isMaxDepth = depth + 1 == maxDepth;
            uint n = rayCount[depth];
            if (depth > 0) {
#pragma omp parallel for schedule(dynamic, 256)
                for (uint i = 0; i < n; i++) raytrace(rays.data() + cur, n, intersections.data(), s->accel, i);
            }
#pragma omp parallel for schedule(dynamic, 256)
            for (uint i = 0; i < n; i++)
                handleIntersections(image, s->accel, intersections.data(), rays.data() + cur, rays.data() + next,
                                    shadowRays.data(), rayCount[depth], rayCount[depth + 1], shadowCount[depth],
                                    uniforms, ctx, i);
            if (isMaxDepth) break;
            uint ns = shadowCount[depth];
#pragma omp parallel for schedule(dynamic, 256)
            for (uint i = 0; i < ns; i++) raytraceAny(shadowRays.data(), ns, intersections.data(), s->accel, i);
#pragma omp parallel for schedule(dynamic, 256)
            for (uint i = 0; i < ns; i++) handleShadowRays(image, intersections.data(), shadowRays.data(), ns, i);
            std::swap(cur, next);
        }
    }
    return 0;
}

// normalizeImage (kernels/utils/normalizeImage.metal:39-59) over a W*H float4
// film with the given Uniforms fields; out: W*H float4.
int ref_normalize_image(const float *film, uint32_t W, uint32_t H, float exposure, uint32_t accumulate,
                        uint32_t frameIndex, uint32_t tonemapping, float *out) {
    texture2d<float, access::read> input;
    input.data = reinterpret_cast<float4 *>(const_cast<float *>(film));
    input.width = W;
    input.height = H;
    texture2d<float, access::write> output;
    output.data = reinterpret_cast<float4 *>(out);
    output.width = W;
    output.height = H;
    Uniforms uniforms{};
    uniforms.exposure = exposure;
    uniforms.accumulate = accumulate != 0;
    uniforms.frameIndex = frameIndex;
    uniforms.tonemapping = Tonemapping(tonemapping);
    for (uint32_t y = 0; y < H; y++)
        for (uint32_t x = 0; x < W; x++) normalizeImage(uniforms, input, output, uint2(x, y));
    return 0;
}

}  // extern "C"
