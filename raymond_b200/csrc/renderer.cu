// C ABI of include/raymond.h: scene building (SceneLoader / ShapeBuilder /
// EntityBuilder / LightBuilder / MaterialBuilder of the reference) and the
// persistent wavefront render loop that replaces Renderer.execute.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/raymond.h"
#include "../../include/raymond_testing.h"
#include "bvh_build.h"
#include "bvh_gpu.h"
#include "codegen.h"
#include "exr.h"
#include "device/wavefront.cuh"
#include "guide.h"
#include "jit.h"
#include "kernels.h"
#include "scene_view.h"

using namespace rmd;

// The host-facing records keep the layout of the reference's DEVICE_STRUCTs
// (raymond/bridge/Camera.hpp, PerInstanceData.hpp, Uniforms.hpp, lights/ *.hpp)
// as Swift and Metal lay them out: float3 16 bytes aligned to 16, float2 8
// aligned to 8, bool one byte.
static_assert(sizeof(rmd_camera) == 96 && alignof(rmd_camera) == 16, "Camera.hpp layout");
static_assert(offsetof(rmd_camera, near_clip) == 64 && offsetof(rmd_camera, far_clip) == 68 &&
                  offsetof(rmd_camera, focal_length) == 72 && offsetof(rmd_camera, shift) == 80,
              "Camera.hpp layout");
static_assert(sizeof(rmd_light_info) == 4 && offsetof(rmd_light_info, casts_shadows) == 2 &&
                  offsetof(rmd_light_info, uses_mis) == 3,
              "LightInfo.hpp layout");
static_assert(sizeof(rmd_area_light) == 96 && offsetof(rmd_area_light, transform) == 16 &&
                  offsetof(rmd_area_light, color) == 64 && offsetof(rmd_area_light, is_circular) == 80,
              "AreaLight.hpp layout");
static_assert(sizeof(rmd_point_light) == 64 && offsetof(rmd_point_light, location) == 16 &&
                  offsetof(rmd_point_light, radius) == 32 && offsetof(rmd_point_light, color) == 48,
              "PointLight.hpp layout");
static_assert(sizeof(rmd_sun_light) == 64 && offsetof(rmd_sun_light, direction) == 16 &&
                  offsetof(rmd_sun_light, cos_angle) == 32 && offsetof(rmd_sun_light, color) == 48,
              "SunLight.hpp layout");
static_assert(sizeof(rmd_spot_light) == 96 && offsetof(rmd_spot_light, location) == 16 &&
                  offsetof(rmd_spot_light, direction) == 32 && offsetof(rmd_spot_light, radius) == 48 &&
                  offsetof(rmd_spot_light, color) == 64 && offsetof(rmd_spot_light, spot_size) == 80 &&
                  offsetof(rmd_spot_light, spot_blend) == 84,
              "SpotLight.hpp layout");
static_assert(sizeof(rmd_per_instance_data) == 192 && offsetof(rmd_per_instance_data, light_index) == 16 &&
                  offsetof(rmd_per_instance_data, bounds_min) == 32 &&
                  offsetof(rmd_per_instance_data, bounds_size) == 48 &&
                  offsetof(rmd_per_instance_data, point_transform) == 64 &&
                  offsetof(rmd_per_instance_data, normal_transform) == 128 &&
                  offsetof(rmd_per_instance_data, visibility) == 176,
              "PerInstanceData.hpp layout");
static_assert(sizeof(rmd_uniforms) == 64 && offsetof(rmd_uniforms, accumulate) == 12 &&
                  offsetof(rmd_uniforms, lens_spectral) == 13 && offsetof(rmd_uniforms, sensor_scale) == 16 &&
                  offsetof(rmd_uniforms, exposure) == 28 && offsetof(rmd_uniforms, sampling_mode) == 44 &&
                  offsetof(rmd_uniforms, tonemapping) == 48 && offsetof(rmd_uniforms, output_channel) == 60,
              "Uniforms.hpp layout");

namespace {

thread_local std::string g_lastError;

rmd_status fail(rmd_status s, const std::string &msg) {
    g_lastError = msg;
    return s;
}

#define RMD_CUDA(expr)                                                                                      \
    do {                                                                                                    \
        cudaError_t e_ = (expr);                                                                            \
        if (e_ != cudaSuccess)                                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? RMD_ERROR_OUT_OF_MEMORY : RMD_ERROR_CUDA,         \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                               \
    } while (0)

// Device buffer owned by a scene or renderer.
// Register budget of the shading kernel before autotuning: at least this many
// 128-thread blocks per SM (measured best on the 1080p benchmark scene: 5-6);
// RMD_SHADE_MIN_BLOCKS overrides it.
static int defaultShadeMinBlocks() {
    const char *e = std::getenv("RMD_SHADE_MIN_BLOCKS");
    const int v = e ? std::atoi(e) : 5;
    return v >= 1 && v <= 16 ? v : 5;
}

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n) {
        release();
        bytes = n;
        if (n == 0) return cudaSuccess;
        return cudaMalloc(&ptr, n);
    }
    void adopt(void *p, size_t n) {  // takes ownership of a cudaMalloc'd block
        release();
        ptr = p;
        bytes = n;
    }
    cudaError_t upload(const void *src, size_t n, cudaStream_t s) {
        cudaError_t e = alloc(n);
        if (e != cudaSuccess || n == 0) return e;
        e = cudaMemcpyAsync(ptr, src, n, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        return cudaStreamSynchronize(s);
    }
    template <class T>
    T *as() const {
        return static_cast<T *>(ptr);
    }
};

struct HostMat4 {
    float c[4][4];  // columns
};

}  // namespace

struct rmd_context {
    int device = 0;
    int smCount = 148;
    cudaStream_t stream = nullptr;
    uint32_t bvhBuilder = RMD_BVH_HOST;  // builder of the scenes created next
};

struct rmd_scene {
    rmd_context *ctx = nullptr;
    Context dctx{};  // device view
    DevBuf vertices, normals, texcoords, faces, instances, lightFaces, envPdfs, envMipmap;
    DevBuf areaLights, pointLights, sunLights, spotLights, shapeLights;
    DevBuf surfaceTable, lightTable, materialParams;
    DevBuf bvhNodes, bvhTris;
    DevBuf textureTexels, textureViews;  // RGBA float texels of all textures; one TextureView each
    rmdhost::JitModule jit;   // default variant (envmap build, test hooks, default shade kernel)
    std::string moduleSource;
    // shading kernels by shadeVariantKey(minimum blocks per SM, guide code);
    // `jit` is the default budget without the guide's code
    std::map<int, std::unique_ptr<rmdhost::JitModule>> variants;
    uint64_t triangles = 0, bvhNodeCount = 0;
    std::vector<rmd_per_instance_data> instanceRecords;  // EntityBuilder's records, bridge layout
    rmd_bvh_stats bvhStats{};  // builder, build time and levels; SAH cost computed when first asked
    bool bvhSahKnown = false;
    float boundsMin[3] = {0, 0, 0}, boundsMax[3] = {1, 1, 1};  // world-space triangle bounds
    int numSurface = 0, numLight = 0;
    int shadeBlocks = 0, traceBlocks = 0, regenBlocks = 0;
    int defaultMinBlocks = 1;
    bool ownsModule = true;  // false for the scenes of a batch (the batch owns the shared module)
    ~rmd_scene() {
        for (auto &kv : variants) rmdhost::unloadModule(*kv.second);
        if (ownsModule) rmdhost::unloadModule(jit);
    }
};

// Learned path guiding of one renderer or batch: the network and the
// per-path buffers of its pool.
struct GuideState {
    rmd_guide_settings settings{};
    rmd_guide_stats stats{};
    rmdhost::GuideNet net;
    DevBuf mixtures, features, rec, finRec, shRec, records;
    uint32_t pathCapacity = 0;    // paths the mixtures / pending-record buffers hold
    uint32_t recordCapacity = 0;  // nonzero-target records the replay ring holds
    bool initialised = false;
    float3 frameMin = {0, 0, 0}, frameInvExtent = {1, 1, 1};  // position encoding frame (scene bounds)
};

struct rmd_renderer {
    rmd_scene *scene = nullptr;
    uint32_t width = 0, height = 0, capacity = 0;
    // launch choices (rmd_renderer_autotune)
    cudaKernel_t shade = nullptr;
    int shadeBlocks = 0;
    int shadeMinBlocks = 1;
    bool shadeGuided = false;  // the shading kernel carries the guide's sampling and training code
    int traceBlocksPerSm = 12;
    DevBuf pool;  // path state, finish list and shadow rays (carvePathPool)
    DevBuf counters, film, film64, resolve;
    Counters *hostCounters = nullptr;  // pinned
    Context dctx{};
    uint64_t samples = 0;     // samples accumulated in the film (what normalisation divides by)
    uint64_t nextSample = 0;  // sample index a render continues at (first_sample < 0)
    rmd_stats stats{};
    cudaEvent_t ev[4] = {};
    std::vector<cudaEvent_t> stageEvents;  // recorded between the stage kernels
    std::vector<int> stageOf;              // stage of the interval that ends at each event
    GuideState guide;  // learned path guiding
    ~rmd_renderer() {
        if (hostCounters) cudaFreeHost(hostCounters);
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        for (auto &e : stageEvents) cudaEventDestroy(e);
    }
    // records event i on `st`, closing an interval of stage `stage`
    cudaError_t stageEvent(size_t i, int stage, cudaStream_t st) {
        while (stageEvents.size() <= i) {
            cudaEvent_t e;
            cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) return err;
            stageEvents.push_back(e);
            stageOf.push_back(0);
        }
        stageOf[i] = stage;
        return cudaEventRecord(stageEvents[i], st);
    }
};

// Many scenes and views traced by one wavefront (one pool, one launch per
// stage), the whole render one CUDA-graph launch whose while loop the device
// drives.
struct rmd_batch {
    rmd_context *ctx = nullptr;
    std::vector<std::unique_ptr<rmd_scene>> scenes;
    rmdhost::JitModule jit;  // the merged material module of all scenes (batch shading kernel)
    std::string moduleSource;
    std::map<int, std::unique_ptr<rmdhost::JitModule>> variants;  // shading kernels by shadeVariantKey
    std::vector<rmd_batch_view> views;
    std::vector<uint32_t> offsets;  // film pixel offset of each view
    uint32_t totalPixels = 0;
    DevBuf viewTable, pool, counters, film, film64, resolve;
    Counters *hostCounters = nullptr;
    uint32_t capacity = 0;
    cudaKernel_t shade = nullptr;
    int shadeBlocks = 0, shadeMinBlocks = 1, defaultMinBlocks = 1, traceBlocksPerSm = 12;
    bool shadeGuided = false;
    bool useGraph = true;
    GuideState guide;  // learned path guiding (all views of one scene)
    int guideScene = -1;
    uint64_t samples = 0;     // samples of every view accumulated in the films
    uint64_t nextSample = 0;  // sample index a render continues at (first_sample < 0)
    rmd_stats stats{};
    cudaEvent_t ev[2] = {};
    // the instantiated render graph and the settings it was captured for
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    std::vector<uint64_t> graphKey;
    ~rmd_batch() {
        if (graphExec) cudaGraphExecDestroy(graphExec);
        if (graph) cudaGraphDestroy(graph);
        if (hostCounters) cudaFreeHost(hostCounters);
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        scenes.clear();  // before the module their envmaps were built with goes
        for (auto &kv : variants) rmdhost::unloadModule(*kv.second);
        rmdhost::unloadModule(jit);
    }
};

// --------------------------------------------------------------------- helpers
namespace {

// column-major 4x4 from the C ABI
HostMat4 toMat(const float *m) {
    HostMat4 r;
    for (int c = 0; c < 4; c++)
        for (int k = 0; k < 4; k++) r.c[c][k] = m[4 * c + k];
    return r;
}

// (M * float4(p, 1)).xyz in the same association order as the device code
void transformPoint(const HostMat4 &M, const float *p, float *out) {
    for (int k = 0; k < 3; k++) {
        float a = M.c[0][k] * p[0];
        float b = M.c[1][k] * p[1];
        float c = M.c[2][k] * p[2];
        float d = M.c[3][k] * 1.0f;
        out[k] = ((a + b) + c) + d;
    }
}

// inverse-transpose of the upper 3x3 (EntityBuilder.swift:98), columns
void inverseTranspose3(const HostMat4 &M, float out[3][3]) {
    const float *a = M.c[0], *b = M.c[1], *c = M.c[2];
    auto cross = [](const float *u, const float *v, float *r) {
        r[0] = u[1] * v[2] - u[2] * v[1];
        r[1] = u[2] * v[0] - u[0] * v[2];
        r[2] = u[0] * v[1] - u[1] * v[0];
    };
    float r0[3], r1[3], r2[3];
    cross(b, c, r0);
    cross(c, a, r1);
    cross(a, b, r2);
    const float det = a[0] * r0[0] + a[1] * r0[1] + a[2] * r0[2];
    for (int k = 0; k < 3; k++) {
        out[0][k] = r0[k] / det;
        out[1][k] = r1[k] / det;
        out[2][k] = r2[k] / det;
    }
}

// host/lights/distribution.m:7-39 (area CDF over all faces of the shape, accumulated in double)
float buildLightDistribution(const HostMat4 &M, const uint32_t *idx, const float *verts, uint32_t faceCount,
                             float *output) {
    double acc = 0;
    auto mul = [&](const float *v, float *r) {  // inner3x3 * v
        for (int k = 0; k < 3; k++) r[k] = M.c[0][k] * v[0] + M.c[1][k] * v[1] + M.c[2][k] * v[2];
    };
    for (uint32_t i = 0; i < faceCount; i++) {
        const float *v0 = verts + 3 * idx[3 * i], *v1 = verts + 3 * idx[3 * i + 1], *v2 = verts + 3 * idx[3 * i + 2];
        float e0[3], e1[3], a[3], b[3];
        for (int k = 0; k < 3; k++) {
            e0[k] = v2[k] - v0[k];
            e1[k] = v2[k] - v1[k];
        }
        mul(e0, a);
        mul(e1, b);
        const float tn[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        const float area = std::sqrt(tn[0] * tn[0] + tn[1] * tn[1] + tn[2] * tn[2]) / 2;
        output[i] = (float)(acc += area);
    }
    for (uint32_t i = 0; i < faceCount; i++) output[i] = (float)(output[i] / acc);
    return (float)acc;
}

rmd_status buildEnvironmentMap(rmd_scene *s, int exponent) {
    cudaStream_t st = s->ctx->stream;
    const int res = 1 << exponent;
    size_t mipSize = 0;
    for (int e = 0; e <= exponent; e++) mipSize += (size_t)1 << (2 * e);
    RMD_CUDA(s->envMipmap.alloc(mipSize * sizeof(float)));
    RMD_CUDA(s->envPdfs.alloc((size_t)res * res * sizeof(float)));
    s->dctx.envResolution = res;
    s->dctx.envMipmap = s->envMipmap.as<float>();
    s->dctx.envPdfs = s->envPdfs.as<float>();
    const size_t lastLevel = mipSize - (size_t)res * res;
    float *finest = s->envMipmap.as<float>() + lastLevel;
    float *pdfs = s->envPdfs.as<float>();
    void *args[] = {&s->dctx, &finest, &pdfs, (void *)&res};
    dim3 b(8, 8), g((res + 7) / 8, (res + 7) / 8);
    RMD_CUDA(cudaLaunchKernel((const void *)s->jit.envmapBuild, g, b, args, 0, st));
    size_t off = lastLevel;
    for (int e = exponent - 1; e >= 0; e--) {
        const int cur = 1 << e;
        off -= (size_t)cur * cur;
        RMD_CUDA(rmdLaunchEnvmapReduce(s->envMipmap.as<float>() + off, cur, st));
    }
    RMD_CUDA(rmdLaunchEnvmapNormalize(s->envMipmap.as<float>(), pdfs, (uint32_t)res * (uint32_t)res, st));
    RMD_CUDA(cudaStreamSynchronize(st));
    return RMD_OK;
}

int occupancyBlocks(const void *fn, int threads, int smCount) {
    int perSm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, threads, 0) != cudaSuccess || perSm <= 0) perSm = 4;
    return perSm * smCount;
}

}  // namespace

namespace rmdhost {
bool sceneView(const rmd_scene *s, SceneView &v) {
    if (!s) return false;
    v.ctx = s->dctx;
    v.nodes = s->bvhNodes.as<WideNode>();
    v.tris = s->bvhTris.as<float4>();
    v.shade = s->jit.shade;
    v.shadeBlocks = s->shadeBlocks;
    v.stream = s->ctx->stream;
    v.device = s->ctx->device;
    v.smCount = s->ctx->smCount;
    return true;
}
rmd_status setLastError(rmd_status status, const char *msg) { return fail(status, msg); }
}  // namespace rmdhost

// --------------------------------------------------------------------- C ABI
extern "C" {

// shading-kernel variants (defined with the autotuner)
static rmd_status ensureVariants(rmd_scene *s, const std::vector<int> &minBlocks, bool guided);
static void selectShade(rmd_renderer *r, int mb, bool guided);

const char *rmd_last_error(void) { return g_lastError.c_str(); }
const char *rmd_version(void) { return "raymond_b200 0.1 (sm_100a)"; }

rmd_status rmd_context_create(int32_t device, rmd_context **out) {
    if (!out) return fail(RMD_ERROR_INVALID_ARGUMENT, "out is NULL");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(RMD_ERROR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= count) return fail(RMD_ERROR_INVALID_ARGUMENT, "device index out of range");
    auto c = std::make_unique<rmd_context>();
    c->device = device;
    RMD_CUDA(cudaSetDevice(device));
    RMD_CUDA(cudaDeviceGetAttribute(&c->smCount, cudaDevAttrMultiProcessorCount, device));
    RMD_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const rmd_status ns = rmdhost::noallocSetup(device);
    if (ns != RMD_OK) {
        cudaStreamDestroy(c->stream);
        return ns;
    }
    *out = c.release();
    return RMD_OK;
}

void rmd_context_destroy(rmd_context *c) {
    if (!c) return;
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static rmd_status validateSceneDesc(const rmd_scene_desc *d) {
    if (d->num_surface_materials < 0 || d->num_light_materials <= 0 || d->num_shapes < 0 || d->num_entities < 0)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid counts (at least the world material is required)");
    if (d->world_shader >= d->num_light_materials) return fail(RMD_ERROR_INVALID_ARGUMENT, "world_shader out of range");
    if (d->envmap_exponent < 0 || d->envmap_exponent > 12)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "envmap_exponent out of range (0..12)");
    if (d->num_textures < 0 || (d->num_textures > 0 && !d->textures))
        return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid texture list");
    for (int i = 0; i < d->num_textures; i++) {
        const rmd_texture &t = d->textures[i];
        if (!t.name || !t.data || t.width == 0 || t.height == 0 || t.width > 65536 || t.height > 65536 ||
            (t.channels != 1 && t.channels != 3 && t.channels != 4) || t.format > RMD_TEXTURE_F32)
            return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid texture " + std::to_string(i));
    }
    return RMD_OK;
}

// The textures as the device reads them: RGBA floats (a single-channel
// image as (r, 0, 0, 1), RGB with alpha 1, integers normalised), then a
// 1 x 1 zero single-channel texture, the slot of files that are missing.
static rmd_status uploadTextures(const rmd_texture *textures, int count, rmd_scene *s, cudaStream_t st) {
    std::vector<float4> texels;
    std::vector<TextureView> views;
    std::vector<size_t> offsets;
    std::vector<std::pair<size_t, int>> skies;  // (texel offset, texture index) of generated sky textures
    for (int i = 0; i < count; i++) {
        const rmd_texture &t = textures[i];
        offsets.push_back(texels.size());
        const size_t n = (size_t)t.width * t.height;
        texels.resize(texels.size() + n);
        float4 *out = texels.data() + offsets.back();
        if (!t.data) {  // a sky texture, filled on the device below
            skies.push_back({offsets.back(), i});
            views.push_back(TextureView{nullptr, (int)t.width, (int)t.height, (int)t.channels, 0});
            continue;
        }
        for (size_t p = 0; p < n; p++) {
            float v[4] = {0.0f, 0.0f, 0.0f, 1.0f};
            for (uint32_t c = 0; c < t.channels; c++) {
                const size_t k = p * t.channels + c;
                if (t.format == RMD_TEXTURE_U8) v[c] = (float)static_cast<const uint8_t *>(t.data)[k] / 255.0f;
                else if (t.format == RMD_TEXTURE_U16) v[c] = (float)static_cast<const uint16_t *>(t.data)[k] / 65535.0f;
                else v[c] = static_cast<const float *>(t.data)[k];
            }
            out[p] = make_float4(v[0], v[1], v[2], v[3]);
        }
        views.push_back(TextureView{nullptr, (int)t.width, (int)t.height, (int)t.channels, 0});
    }
    offsets.push_back(texels.size());
    texels.push_back(make_float4(0.0f, 0.0f, 0.0f, 1.0f));
    views.push_back(TextureView{nullptr, 1, 1, 1, 0});
    RMD_CUDA(s->textureTexels.upload(texels.data(), texels.size() * sizeof(float4), st));
    for (const auto &sky : skies) {  // the Nishita sky textures of the scene's TEX_SKY nodes
        float v[5];
        if (!rmdhost::parseSkyTextureName(textures[sky.second].name, v))
            return fail(RMD_ERROR_INVALID_ARGUMENT, "texture " + std::to_string(sky.second) + " has no data");
        RMD_CUDA(rmdLaunchSkyTexture(s->textureTexels.as<float4>() + sky.first, textures[sky.second].width,
                                     textures[sky.second].height, v[0], v[1], v[2], v[3], v[4], st));
    }
    for (size_t i = 0; i < views.size(); i++) views[i].texels = s->textureTexels.as<float4>() + offsets[i];
    RMD_CUDA(s->textureViews.upload(views.data(), views.size() * sizeof(TextureView), st));
    s->dctx.textures = s->textureViews.as<TextureView>();
    s->dctx.numTextures = (int)views.size();
    return RMD_OK;
}

// Everything of a scene but its material module: geometry, BVH, lights,
// material tables and the device Context.  `mod` is the generated module
// that holds this scene's materials from index surfaceBase / lightBase on
// (0 for a scene of its own; the scene's slice of a module shared by the
// scenes of a batch).
static rmd_status buildSceneData(rmd_context *ctx, const rmd_scene_desc *d, rmd_scene *s,
                                 const rmdhost::GeneratedModule &mod, int surfaceBase, int lightBase,
                                 const rmd_texture *textures, int numTextures) {
    cudaStream_t st = ctx->stream;
    s->ctx = ctx;
    s->numSurface = d->num_surface_materials;
    s->numLight = d->num_light_materials;

    // ShapeBuilder.build (ShapeBuilder.swift:251-298)
    struct ShapeInfo {
        uint32_t vertexOffset, faceOffset, faceCount;
        float boundsMin[3], boundsMax[3];
        bool hasEmission;
    };
    std::vector<ShapeInfo> shapes;
    std::vector<float4> verts, norms;
    std::vector<float2> uvs;
    std::vector<uint4> faces;
    std::vector<float> vertsPacked;  // for the light CDF
    std::vector<uint32_t> idxPacked;
    for (int si = 0; si < d->num_shapes; si++) {
        const rmd_shape &sh = d->shapes[si];
        if ((sh.num_vertices && (!sh.vertices || !sh.normals || !sh.texcoords)) ||
            (sh.num_faces && (!sh.indices || !sh.materials)))
            return fail(RMD_ERROR_INVALID_ARGUMENT, "shape " + std::to_string(si) + " has NULL arrays");
        ShapeInfo info{};
        info.vertexOffset = (uint32_t)verts.size();
        info.faceOffset = (uint32_t)faces.size();
        info.faceCount = sh.num_faces;
        for (int k = 0; k < 3; k++) {
            info.boundsMin[k] = INFINITY;
            info.boundsMax[k] = -INFINITY;
        }
        for (uint32_t v = 0; v < sh.num_vertices; v++) {
            const float *p = sh.vertices + 3 * v;
            for (int k = 0; k < 3; k++) {  // PLYReader.m:119-122 (else-if: the first vertex never raises the max)
                if (p[k] < info.boundsMin[k]) info.boundsMin[k] = p[k];
                else if (p[k] > info.boundsMax[k]) info.boundsMax[k] = p[k];
            }
            verts.push_back(make_float4(p[0], p[1], p[2], 0.0f));
            vertsPacked.insert(vertsPacked.end(), p, p + 3);
            const float *n = sh.normals + 3 * v;
            norms.push_back(make_float4(n[0], n[1], n[2], 0.0f));
            uvs.push_back(make_float2(sh.texcoords[2 * v], sh.texcoords[2 * v + 1]));
        }
        info.hasEmission = false;
        for (uint32_t f = 0; f < sh.num_faces; f++) {
            const uint32_t *ix = sh.indices + 3 * f;
            if (ix[0] >= sh.num_vertices || ix[1] >= sh.num_vertices || ix[2] >= sh.num_vertices)
                return fail(RMD_ERROR_INVALID_ARGUMENT, "vertex index out of range in shape " + std::to_string(si));
            const uint16_t m = sh.materials[f];
            if (m >= d->num_surface_materials)
                return fail(RMD_ERROR_INVALID_ARGUMENT, "face material out of range in shape " + std::to_string(si));
            faces.push_back(make_uint4(ix[0], ix[1], ix[2], m));
            idxPacked.insert(idxPacked.end(), ix, ix + 3);
            if (mod.surfaceEmissive[surfaceBase + m]) info.hasEmission = true;
        }
        shapes.push_back(info);
    }

    // EntityBuilder.build (EntityBuilder.swift:79-141), flattened into one BVH
    std::vector<PerInstanceData> insts;
    std::vector<float> t0, t1, t2;
    std::vector<uint32_t> triInst, triPrim;
    struct PendingLight {
        uint32_t instance, shape;
        HostMat4 M;
        uint32_t lightFaceOffset;
    };
    std::vector<PendingLight> pending;
    uint32_t lightFaceOffset = 0;
    for (int ei = 0; ei < d->num_entities; ei++) {
        const rmd_entity &e = d->entities[ei];
        if (e.shape >= (uint32_t)d->num_shapes) return fail(RMD_ERROR_INVALID_ARGUMENT, "entity shape out of range");
        const ShapeInfo &si = shapes[e.shape];
        const HostMat4 M = toMat(e.matrix);
        PerInstanceData inst{};
        inst.vertexOffset = si.vertexOffset;
        inst.faceOffset = si.faceOffset;
        inst.visibility = e.visibility;
        inst.lightIndex = 0xffffffffu;
        inst.triOffset = (uint32_t)triInst.size();
        inst.boundsMin = make_float4(si.boundsMin[0], si.boundsMin[1], si.boundsMin[2], 0.0f);
        inst.boundsSize = make_float4(si.boundsMax[0] - si.boundsMin[0], si.boundsMax[1] - si.boundsMin[1],
                                      si.boundsMax[2] - si.boundsMin[2], 0.0f);
        for (int c = 0; c < 4; c++) inst.pointTransform[c] = make_float4(M.c[c][0], M.c[c][1], M.c[c][2], M.c[c][3]);
        float nt[3][3];
        inverseTranspose3(M, nt);
        for (int c = 0; c < 3; c++) inst.normalTransform[c] = make_float4(nt[c][0], nt[c][1], nt[c][2], 0.0f);
        if (si.hasEmission) {
            inst.lightIndex = (uint32_t)pending.size();
            inst.lightFaceOffset = lightFaceOffset;
            inst.lightFaceCount = si.faceCount;
            pending.push_back({(uint32_t)ei, e.shape, M, lightFaceOffset});
            lightFaceOffset += si.faceCount;
        }
        insts.push_back(inst);
        for (uint32_t f = 0; f < si.faceCount; f++) {
            const uint4 fc = faces[si.faceOffset + f];
            const uint32_t vi[3] = {fc.x, fc.y, fc.z};
            float w[3][3];
            for (int j = 0; j < 3; j++) {
                const float4 p = verts[si.vertexOffset + vi[j]];
                const float pp[3] = {p.x, p.y, p.z};
                transformPoint(M, pp, w[j]);
            }
            t0.insert(t0.end(), w[0], w[0] + 3);
            t1.insert(t1.end(), w[1], w[1] + 3);
            t2.insert(t2.end(), w[2], w[2] + 3);
            triInst.push_back((uint32_t)ei);
            triPrim.push_back(f);
        }
    }
    s->triangles = triInst.size();
    if (!t0.empty()) {
        for (int k = 0; k < 3; k++) {
            s->boundsMin[k] = INFINITY;
            s->boundsMax[k] = -INFINITY;
        }
        for (const std::vector<float> *t : {&t0, &t1, &t2})
            for (size_t i = 0; i < t->size(); i++) {
                s->boundsMin[i % 3] = std::min(s->boundsMin[i % 3], (*t)[i]);
                s->boundsMax[i % 3] = std::max(s->boundsMax[i % 3], (*t)[i]);
            }
    }
    // ShapeBuilder / EntityBuilder acceleration structures: one BVH over the
    // flattened world-space triangles, built on the host or on the device
    rmdhost::GpuWideBvh bvh;
    const auto buildStart = std::chrono::steady_clock::now();
    s->bvhStats.builder = ctx->bvhBuilder;
    if (ctx->bvhBuilder == RMD_BVH_GPU) {
        DevBuf d0, d1, d2, dInst, dPrim;
        RMD_CUDA(d0.upload(t0.data(), t0.size() * sizeof(float), st));
        RMD_CUDA(d1.upload(t1.data(), t1.size() * sizeof(float), st));
        RMD_CUDA(d2.upload(t2.data(), t2.size() * sizeof(float), st));
        RMD_CUDA(dInst.upload(triInst.data(), triInst.size() * sizeof(uint32_t), st));
        RMD_CUDA(dPrim.upload(triPrim.data(), triPrim.size() * sizeof(uint32_t), st));
        rmdhost::GpuBvhResult g;
        const cudaError_t e = rmdhost::buildWideBvhGpu(d0.as<float>(), d1.as<float>(), d2.as<float>(),
                                                       dInst.as<uint32_t>(), dPrim.as<uint32_t>(),
                                                       (uint32_t)std::min<size_t>(triInst.size(), 0xffffffffu), st, g);
        s->bvhNodes.adopt(g.nodes, g.nodeCount * sizeof(rmdhost::GpuWideNode));
        s->bvhTris.adopt(g.tris, triInst.size() * 12 * sizeof(float));
        if (e != cudaSuccess) {
            if (!g.error.empty()) return fail(RMD_ERROR_INVALID_ARGUMENT, "device BVH build: " + g.error);
            RMD_CUDA(e);
        }
        s->bvhNodeCount = g.nodeCount;
        s->bvhStats.levels = g.levels;
        s->bvhStats.cluster_iterations = g.clusterIterations;
    } else {
        rmdhost::buildWideBvh(t0, t1, t2, triInst, triPrim, bvh);
        s->bvhNodeCount = bvh.nodes.size();
    }
    s->bvhStats.build_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - buildStart).count();

    // LightBuilder.build (LightBuilder.swift:179-281)
    std::vector<float> lightFaces(std::max<uint32_t>(1, lightFaceOffset), 0.0f);
    std::vector<ShapeLight> shapeLights;
    for (auto &p : pending) {
        const ShapeInfo &si = shapes[p.shape];
        ShapeLight sl;
        sl.instanceIndex = p.instance;
        sl.emissiveArea = buildLightDistribution(p.M, idxPacked.data() + 3 * (size_t)si.faceOffset,
                                                 vertsPacked.data() + 3 * (size_t)si.vertexOffset, si.faceCount,
                                                 lightFaces.data() + p.lightFaceOffset);
        shapeLights.push_back(sl);
    }
    auto info = [](const rmd_light_info &i) {
        LightInfo r{};
        r.shaderIndex = i.shader_index;
        r.castsShadows = i.casts_shadows;
        r.usesMIS = i.uses_mis;
        return r;
    };
    std::vector<AreaLight> areas;
    for (int i = 0; i < d->num_area_lights; i++) {
        const rmd_area_light &l = d->area_lights[i];
        AreaLight a{};
        a.info = info(l.info);
        for (int c = 0; c < 3; c++)
            a.transform[c] = make_float4(l.transform[4 * c], l.transform[4 * c + 1], l.transform[4 * c + 2],
                                         l.transform[4 * c + 3]);
        a.color = make_float4(l.color[0], l.color[1], l.color[2], l.is_circular ? 1.0f : 0.0f);
        areas.push_back(a);
    }
    std::vector<PointLight> points;
    for (int i = 0; i < d->num_point_lights; i++) {
        const rmd_point_light &l = d->point_lights[i];
        PointLight p{};
        p.info = info(l.info);
        p.locationRadius = make_float4(l.location[0], l.location[1], l.location[2], l.radius);
        p.color = make_float4(l.color[0], l.color[1], l.color[2], 0.0f);
        points.push_back(p);
    }
    std::vector<SunLight> suns;
    for (int i = 0; i < d->num_sun_lights; i++) {
        const rmd_sun_light &l = d->sun_lights[i];
        SunLight p{};
        p.info = info(l.info);
        p.directionCosAngle = make_float4(l.direction[0], l.direction[1], l.direction[2], l.cos_angle);
        p.color = make_float4(l.color[0], l.color[1], l.color[2], 0.0f);
        suns.push_back(p);
    }
    std::vector<SpotLight> spots;
    for (int i = 0; i < d->num_spot_lights; i++) {
        const rmd_spot_light &l = d->spot_lights[i];
        SpotLight p{};
        p.info = info(l.info);
        p.locationRadius = make_float4(l.location[0], l.location[1], l.location[2], l.radius);
        p.directionSpotSize = make_float4(l.direction[0], l.direction[1], l.direction[2], l.spot_size);
        p.colorSpotBlend = make_float4(l.color[0], l.color[1], l.color[2], l.spot_blend);
        spots.push_back(p);
    }
    auto checkShader = [&](const rmd_light_info &i) { return i.shader_index < d->num_light_materials; };
    for (int i = 0; i < d->num_area_lights; i++)
        if (!checkShader(d->area_lights[i].info)) return fail(RMD_ERROR_INVALID_ARGUMENT, "area light shader index");
    for (int i = 0; i < d->num_point_lights; i++)
        if (!checkShader(d->point_lights[i].info)) return fail(RMD_ERROR_INVALID_ARGUMENT, "point light shader index");
    for (int i = 0; i < d->num_sun_lights; i++)
        if (!checkShader(d->sun_lights[i].info)) return fail(RMD_ERROR_INVALID_ARGUMENT, "sun light shader index");
    for (int i = 0; i < d->num_spot_lights; i++)
        if (!checkShader(d->spot_lights[i].info)) return fail(RMD_ERROR_INVALID_ARGUMENT, "spot light shader index");

    // material tables
    std::vector<uint2> stab, ltab;
    for (int i = surfaceBase; i < surfaceBase + d->num_surface_materials; i++)
        stab.push_back(make_uint2(mod.surface.group[i], mod.surface.offset[i]));
    for (int i = lightBase; i < lightBase + d->num_light_materials; i++)
        ltab.push_back(make_uint2(mod.light.group[i], mod.light.offset[i]));
    const std::vector<float> params = mod.params.empty() ? std::vector<float>{0.0f} : mod.params;
    if (stab.empty()) stab.push_back(make_uint2(0, 0));

    // uploads
    RMD_CUDA(s->vertices.upload(verts.data(), verts.size() * sizeof(float4), st));
    RMD_CUDA(s->normals.upload(norms.data(), norms.size() * sizeof(float4), st));
    RMD_CUDA(s->texcoords.upload(uvs.data(), uvs.size() * sizeof(float2), st));
    RMD_CUDA(s->faces.upload(faces.data(), faces.size() * sizeof(uint4), st));
    RMD_CUDA(s->instances.upload(insts.data(), insts.size() * sizeof(PerInstanceData), st));
    s->instanceRecords.assign(insts.size(), rmd_per_instance_data{});
    for (size_t i = 0; i < insts.size(); i++) {
        const PerInstanceData &p = insts[i];
        rmd_per_instance_data &o = s->instanceRecords[i];
        o.vertex_offset = p.vertexOffset;
        o.face_offset = p.faceOffset;
        o.light_face_offset = p.lightFaceOffset;
        o.light_face_count = p.lightFaceCount;
        o.light_index = p.lightIndex;
        std::memcpy(o.bounds_min, &p.boundsMin, 3 * sizeof(float));
        std::memcpy(o.bounds_size, &p.boundsSize, 3 * sizeof(float));
        std::memcpy(o.point_transform, p.pointTransform, 16 * sizeof(float));
        for (int c = 0; c < 3; c++) std::memcpy(o.normal_transform + 4 * c, &p.normalTransform[c], 3 * sizeof(float));
        o.visibility = (uint8_t)p.visibility;
    }
    RMD_CUDA(s->lightFaces.upload(lightFaces.data(), lightFaces.size() * sizeof(float), st));
    RMD_CUDA(s->areaLights.upload(areas.data(), areas.size() * sizeof(AreaLight), st));
    RMD_CUDA(s->pointLights.upload(points.data(), points.size() * sizeof(PointLight), st));
    RMD_CUDA(s->sunLights.upload(suns.data(), suns.size() * sizeof(SunLight), st));
    RMD_CUDA(s->spotLights.upload(spots.data(), spots.size() * sizeof(SpotLight), st));
    RMD_CUDA(s->shapeLights.upload(shapeLights.data(), shapeLights.size() * sizeof(ShapeLight), st));
    RMD_CUDA(s->surfaceTable.upload(stab.data(), stab.size() * sizeof(uint2), st));
    RMD_CUDA(s->lightTable.upload(ltab.data(), ltab.size() * sizeof(uint2), st));
    RMD_CUDA(s->materialParams.upload(params.data(), params.size() * sizeof(float), st));
    if (ctx->bvhBuilder != RMD_BVH_GPU) {
        RMD_CUDA(s->bvhNodes.upload(bvh.nodes.data(), bvh.nodes.size() * sizeof(rmdhost::GpuWideNode), st));
        RMD_CUDA(s->bvhTris.upload(bvh.tris.data(), bvh.tris.size() * sizeof(float), st));
    }
    if (s->triangles) {  // the traversal kernels read three rotated copies of each triangle (device/traverse.cuh)
        DevBuf rotated;
        RMD_CUDA(rotated.alloc(s->triangles * TRI_FLOAT4 * sizeof(float4)));
        RMD_CUDA(rmdLaunchRotateTriangles(s->bvhTris.as<float4>(), rotated.as<float4>(), (uint32_t)s->triangles, st));
        RMD_CUDA(cudaStreamSynchronize(st));
        s->bvhTris.adopt(rotated.ptr, rotated.bytes);
        rotated.ptr = nullptr;
        rotated.bytes = 0;
    }

    Context &c = s->dctx;
    c.vertices = s->vertices.as<float4>();
    c.normals = s->normals.as<float4>();
    c.texcoords = s->texcoords.as<float2>();
    c.faces = s->faces.as<uint4>();
    c.instances = s->instances.as<PerInstanceData>();
    c.lightFaces = s->lightFaces.as<float>();
    c.areaLights = s->areaLights.as<AreaLight>();
    c.pointLights = s->pointLights.as<PointLight>();
    c.sunLights = s->sunLights.as<SunLight>();
    c.spotLights = s->spotLights.as<SpotLight>();
    c.shapeLights = s->shapeLights.as<ShapeLight>();
    c.surfaceTable = s->surfaceTable.as<uint2>();
    c.lightTable = s->lightTable.as<uint2>();
    c.materialParams = s->materialParams.as<float>();
    c.numAreaLights = (int)areas.size();
    c.numPointLights = (int)points.size();
    c.numSunLights = (int)suns.size();
    c.numSpotLights = (int)spots.size();
    c.numShapeLights = (int)shapeLights.size();
    c.numLightsTotal = 1 + c.numAreaLights + c.numPointLights + c.numSunLights + c.numSpotLights + c.numShapeLights;
    c.worldShader = d->world_shader;
    for (int k = 0; k < 4; k++)
        c.cameraTransform[k] = make_float4(d->camera.transform[4 * k], d->camera.transform[4 * k + 1],
                                           d->camera.transform[4 * k + 2], d->camera.transform[4 * k + 3]);
    c.nearClip = d->camera.near_clip;
    c.farClip = d->camera.far_clip;
    c.focalLength = d->camera.focal_length;
    c.shift = make_float2(d->camera.shift[0], d->camera.shift[1]);
    rmd_status tr = uploadTextures(textures, numTextures, s, st);
    if (tr != RMD_OK) return tr;

    s->defaultMinBlocks = defaultShadeMinBlocks();
    return RMD_OK;
}

rmd_status rmd_scene_create(rmd_context *ctx, const rmd_scene_desc *d, rmd_scene **out) {
    if (!ctx || !d || !out) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    rmd_status r = validateSceneDesc(d);
    if (r != RMD_OK) return r;
    RMD_CUDA(cudaSetDevice(ctx->device));
    auto s = std::make_unique<rmd_scene>();
    // MaterialBuilder.build: generate and JIT-compile the material module
    rmdhost::GeneratedModule mod;
    rmdhost::SceneTextures tex;
    try {
        const bool hoist = std::getenv("RMD_NO_HOIST") == nullptr;
        tex = rmdhost::sceneTextures(d);
        mod = rmdhost::generateModule(d->surface_materials, d->num_surface_materials, d->light_materials,
                                      d->num_light_materials, hoist,
                                      rmdhost::TextureTable::of(tex.list.data(), (int)tex.list.size()));
    } catch (const rmdhost::CodegenError &e) {
        return fail(e.status, e.message);
    }
    if ((r = buildSceneData(ctx, d, s.get(), mod, 0, 0, tex.list.data(), (int)tex.list.size())) != RMD_OK) return r;
    const std::string err = rmdhost::compileModule(
        mod.source, s->jit, {"-DRMD_SHADE_MIN_BLOCKS=" + std::to_string(s->defaultMinBlocks), "-DRMD_PLAIN_SHADE"});
    if (!err.empty()) return fail(RMD_ERROR_NVRTC, err);
    s->moduleSource = mod.source;
    if ((r = buildEnvironmentMap(s.get(), d->envmap_exponent)) != RMD_OK) return r;
    s->shadeBlocks = occupancyBlocks((const void *)s->jit.shade, 128, ctx->smCount);
    *out = s.release();
    return RMD_OK;
}

void rmd_scene_destroy(rmd_scene *s) { delete s; }

rmd_status rmd_context_set_bvh_builder(rmd_context *ctx, uint32_t builder) {
    if (!ctx) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL context");
    if (builder != RMD_BVH_HOST && builder != RMD_BVH_GPU) return fail(RMD_ERROR_INVALID_ARGUMENT, "unknown BVH builder");
    ctx->bvhBuilder = builder;
    return RMD_OK;
}

rmd_status rmd_scene_bvh_stats(rmd_scene *s, rmd_bvh_stats *out) {
    if (!s || !out) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (!s->bvhSahKnown) {
        std::vector<rmdhost::GpuWideNode> nodes(s->bvhNodeCount);
        if (!nodes.empty()) {
            RMD_CUDA(cudaSetDevice(s->ctx->device));
            RMD_CUDA(cudaMemcpy(nodes.data(), s->bvhNodes.ptr, nodes.size() * sizeof(rmdhost::GpuWideNode),
                                cudaMemcpyDeviceToHost));
        }
        uint32_t levels = 0;
        s->bvhStats.sah_cost = rmdhost::wideBvhSahCost(nodes.data(), nodes.size(), levels);
        s->bvhStats.levels = levels;
        s->bvhSahKnown = true;
    }
    *out = s->bvhStats;
    out->nodes = s->bvhNodeCount;
    return RMD_OK;
}

rmd_status rmd_scene_info(const rmd_scene *s, uint64_t *triangles, uint64_t *bvh_nodes, int32_t *num_lights_total) {
    if (!s) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL scene");
    if (triangles) *triangles = s->triangles;
    if (bvh_nodes) *bvh_nodes = s->bvhNodeCount;
    if (num_lights_total) *num_lights_total = s->dctx.numLightsTotal;
    return RMD_OK;
}

rmd_status rmd_scene_instance_data(const rmd_scene *s, rmd_per_instance_data *out, int32_t capacity, int32_t *count) {
    if (!s || (capacity > 0 && !out) || capacity < 0) return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid argument");
    const size_t n = std::min<size_t>((size_t)capacity, s->instanceRecords.size());
    if (n) std::memcpy(out, s->instanceRecords.data(), n * sizeof(rmd_per_instance_data));
    if (count) *count = (int32_t)s->instanceRecords.size();
    return RMD_OK;
}

static rmd_status ensureGuideBuffers(rmd_renderer *r);
static void guideFrame(const rmd_scene *s, float3 &lo, float3 &invExtent);

static rmd_status allocatePool(rmd_renderer *r) {
    RMD_CUDA(r->pool.alloc(pathPoolBytes(r->capacity)));
    RMD_CUDA(r->counters.alloc(sizeof(Counters)));
    RMD_CUDA(cudaMemset(r->counters.ptr, 0, sizeof(Counters)));
    return ensureGuideBuffers(r);
}

// points a pool of `capacity` paths at the guide's buffers
static void applyGuide(const GuideState &g, uint32_t capacity, PathPool &pool) {
    if (g.settings.training && g.pathCapacity >= capacity) {
        pool.s[0].rec = g.rec.as<float4>();
        pool.s[1].rec = g.rec.as<float4>() + 4 * (size_t)capacity;
        pool.finRec = g.finRec.as<float4>();
        pool.shRec = g.settings.skip_light_records ? nullptr : g.shRec.as<float4>();
        pool.records = g.records.as<GuideRecord>();
        pool.recordCapacity = g.recordCapacity;
    }
    if (g.settings.sampling && g.pathCapacity >= capacity) {
        pool.guide = g.mixtures.as<GuideMixture>();
        pool.guideFeat = g.features.as<uint4>();
        pool.guideMin = g.frameMin;
        pool.guideInvExtent = g.frameInvExtent;
    }
}

static PathPool poolView(rmd_renderer *r) {
    PathPool pool = carvePathPool(r->pool.ptr, r->capacity);
    applyGuide(r->guide, r->capacity, pool);
    return pool;
}

// frame of the guide's position encoding: the scene bounds, slightly padded
static void guideFrame(const rmd_scene *s, float3 &lo, float3 &invExtent) {
    float l[3], inv[3];
    for (int k = 0; k < 3; k++) {
        const float pad = 1e-3f * std::max(1.0f, s->boundsMax[k] - s->boundsMin[k]);
        l[k] = s->boundsMin[k] - pad;
        inv[k] = 1.0f / (s->boundsMax[k] - s->boundsMin[k] + 2.0f * pad);
    }
    lo = make_float3(l[0], l[1], l[2]);
    invExtent = make_float3(inv[0], inv[1], inv[2]);
}

// (re)allocates the guide's buffers for a pool of `capacity` paths
static rmd_status guideBuffers(GuideState &g, uint32_t capacity, Counters *counters) {
    if (!g.settings.sampling && !g.settings.training) return RMD_OK;
    if (g.pathCapacity < capacity) {
        g.pathCapacity = 0;
        g.mixtures.release();
        g.features.release();
        g.rec.release();
        g.finRec.release();
        g.shRec.release();
    }
    if (g.settings.sampling && !g.mixtures.ptr) {
        RMD_CUDA(g.mixtures.alloc((size_t)capacity * sizeof(GuideMixture)));
        RMD_CUDA(g.features.alloc((size_t)capacity * sizeof(uint4)));
    }
    if (g.settings.training && !g.rec.ptr) {
        RMD_CUDA(g.rec.alloc((size_t)capacity * 2 * 4 * sizeof(float4)));
        RMD_CUDA(g.finRec.alloc((size_t)capacity * 4 * sizeof(float4)));
        RMD_CUDA(g.shRec.alloc((size_t)capacity * 2 * sizeof(float4)));
    }
    g.pathCapacity = capacity;
    const uint32_t want = g.settings.replay_records;
    if (g.settings.training && g.recordCapacity != want) {
        g.recordCapacity = 0;
        RMD_CUDA(g.records.alloc((size_t)want * sizeof(GuideRecord)));
        g.recordCapacity = want;
        RMD_CUDA(cudaMemset(&counters->numRecords, 0, 2 * sizeof(uint32_t)));
    }
    return RMD_OK;
}

static rmd_status ensureGuideBuffers(rmd_renderer *r) {
    return guideBuffers(r->guide, r->capacity, r->counters.as<Counters>());
}

// Adam steps due after a counter check: one per `batch_size` samples (times
// steps_per_batch), each on records drawn from the replay ring.
static rmd_status guideTrainStep(GuideState &guide, const Counters &h, Counters *cnt, const GuideNetView &net,
                                 int trainBlocks, cudaStream_t st, uint64_t &trainSteps) {
    if (!guide.settings.training || h.numSamples < guide.settings.batch_size) return RMD_OK;
    const uint32_t stored = std::min(h.numRecords, guide.recordCapacity);
    const uint32_t steps = h.numSamples / guide.settings.batch_size * guide.settings.steps_per_batch;
    if (steps > 0 && stored > 0) {
        RMD_CUDA(rmdLaunchGuideTrain(guide.records.as<GuideRecord>(), stored, guide.settings.step_records,
                                     (uint32_t)guide.net.steps + 1u, steps, net, guide.net.scratch, trainBlocks,
                                     guide.settings.learning_rate, guide.net.steps + 1, &cnt->errors, st));
        guide.net.steps += (int)steps;
        trainSteps += steps;
        guide.stats.steps += steps;
    }
    RMD_CUDA(cudaMemsetAsync(&cnt->numSamples, 0, sizeof(uint32_t), st));
    guide.stats.samples += h.numSamples;
    guide.stats.records = h.numRecords;
    return RMD_OK;
}

static rmd_status guideReadLoss(GuideState &guide) {
    float loss = 0;
    RMD_CUDA(cudaMemcpy(&loss, guide.net.scratch + 1, sizeof(float), cudaMemcpyDeviceToHost));
    guide.stats.last_loss = loss;
    return RMD_OK;
}

// rmd_renderer_set_guide / rmd_batch_set_guide
static rmd_status setGuide(GuideState &g, const rmd_guide_settings *settings, cudaStream_t stream, Counters *counters) {
    const uint32_t ring = settings->replay_records;
    if (settings->sampling > 1 || settings->training > 1 || settings->reset > 1 || settings->learning_rate < 0.0f ||
        !std::isfinite(settings->learning_rate) || settings->batch_size > (1u << 26) ||
        (settings->batch_size != 0 && settings->batch_size < 16) || settings->step_records > (1u << 24) ||
        settings->steps_per_batch > 1024 || settings->skip_light_records > 1 || settings->guided_depth > 65535 ||
        (ring != 0 && (ring < 1024 || ring > (1u << 26) || (ring & (ring - 1)) != 0)))
        return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid guide settings");
    rmd_guide_settings next = *settings;
    if (next.batch_size == 0) next.batch_size = 1u << 20;
    if (next.learning_rate == 0.0f) next.learning_rate = 1e-3f;
    if (next.step_records == 0) next.step_records = 1u << 13;
    if (next.replay_records == 0) next.replay_records = 1u << 18;
    if (next.steps_per_batch == 0) next.steps_per_batch = 8;
    if (next.guided_depth == 0) next.guided_depth = 65535;
    if (!g.net.allocated()) RMD_CUDA(g.net.allocate());
    if (!g.initialised || next.reset) {
        std::vector<float> params(GUIDE_PARAMS);
        rmdhost::GuideNet::initParams(params.data(), next.seed);
        RMD_CUDA(g.net.setParams(params.data(), stream));
        g.initialised = true;
        g.stats = rmd_guide_stats{};
        // records gathered by an earlier network are dropped with it
        RMD_CUDA(cudaMemset(&counters->numRecords, 0, 2 * sizeof(uint32_t)));
    }
    next.reset = 0;
    g.settings = next;
    return RMD_OK;
}

static rmd_status guideParams(GuideState &g, float *params, int32_t write, cudaStream_t stream) {
    if (!g.net.allocated()) RMD_CUDA(g.net.allocate());
    if (write) {
        for (int i = 0; i < GUIDE_PARAMS; i++)
            if (!std::isfinite(params[i])) return fail(RMD_ERROR_INVALID_ARGUMENT, "non-finite guide parameter");
        RMD_CUDA(g.net.setParams(params, stream));
        g.initialised = true;
        g.stats = rmd_guide_stats{};
    } else {
        if (!g.initialised) return fail(RMD_ERROR_INVALID_ARGUMENT, "the guide has not been set up");
        RMD_CUDA(g.net.getParams(params, stream));
    }
    return RMD_OK;
}

rmd_status rmd_renderer_set_size(rmd_renderer *r, uint32_t width, uint32_t height) {
    if (!r || width == 0 || height == 0 || width > 65535 || height > 65535)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid renderer size");
    RMD_CUDA(cudaSetDevice(r->scene->ctx->device));
    r->width = width;
    r->height = height;
    RMD_CUDA(r->film.alloc((size_t)width * height * sizeof(float4)));
    r->film64.release();
    RMD_CUDA(r->resolve.alloc((size_t)width * height * 4 * sizeof(float)));  // RGB or RGBA (rmd_film_normalize)
    return rmd_renderer_reset(r);
}

rmd_status rmd_renderer_create(rmd_scene *scene, uint32_t width, uint32_t height, uint32_t pool_size,
                               rmd_renderer **out) {
    if (!scene || !out) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    RMD_CUDA(cudaSetDevice(scene->ctx->device));
    auto r = std::make_unique<rmd_renderer>();
    r->scene = scene;
    r->dctx = scene->dctx;
    r->shade = scene->jit.shade;
    r->shadeBlocks = scene->shadeBlocks;
    r->shadeMinBlocks = scene->defaultMinBlocks;
    r->capacity = pool_size ? pool_size : (1u << 21);
    rmd_status st = allocatePool(r.get());
    if (st != RMD_OK) return st;
    RMD_CUDA(cudaMallocHost((void **)&r->hostCounters, sizeof(Counters)));
    for (auto &e : r->ev) RMD_CUDA(cudaEventCreate(&e));
    st = rmd_renderer_set_size(r.get(), width, height);
    if (st != RMD_OK) return st;
    *out = r.release();
    return RMD_OK;
}

void rmd_renderer_destroy(rmd_renderer *r) { delete r; }

rmd_status rmd_renderer_reset(rmd_renderer *r) {
    if (!r) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL renderer");
    cudaStream_t st = r->scene->ctx->stream;
    RMD_CUDA(cudaMemsetAsync(r->film.ptr, 0, r->film.bytes, st));
    if (r->film64.ptr) RMD_CUDA(cudaMemsetAsync(r->film64.ptr, 0, r->film64.bytes, st));
    RMD_CUDA(cudaStreamSynchronize(st));
    r->samples = 0;
    r->nextSample = 0;
    return RMD_OK;
}

rmd_status rmd_renderer_set_camera(rmd_renderer *r, const rmd_camera *cam) {
    if (!r || !cam) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    Context &c = r->dctx;
    for (int k = 0; k < 4; k++)
        c.cameraTransform[k] = make_float4(cam->transform[4 * k], cam->transform[4 * k + 1], cam->transform[4 * k + 2],
                                           cam->transform[4 * k + 3]);
    c.nearClip = cam->near_clip;
    c.farClip = cam->far_clip;
    c.focalLength = cam->focal_length;
    c.shift = make_float2(cam->shift[0], cam->shift[1]);
    return rmd_renderer_reset(r);
}

rmd_status rmd_render_frame(rmd_renderer *r, const rmd_uniforms *u, uint32_t max_depth) {
    if (!r || !u) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (u->num_lens_surfaces != 0) return fail(RMD_ERROR_INVALID_ARGUMENT, "lens cameras are not supported");
    if (u->random_seed == 0) return fail(RMD_ERROR_INVALID_ARGUMENT, "random_seed must be >= 1");
    if (u->sampling_mode > 2 || u->output_channel != RMD_OUTPUT_IMAGE)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid uniforms");
    if (!u->accumulate) {  // generate.metal:103-106 clears each pixel before the frame adds to it
        const rmd_status st = rmd_renderer_reset(r);
        if (st != RMD_OK) return st;
    }
    rmd_render_settings s{};
    s.spp = 1;
    s.max_depth = max_depth;
    s.sampling_mode = u->sampling_mode;
    s.rng = RMD_RNG_TEA;
    s.first_sample = (int64_t)u->random_seed - 1;  // TEA seeds sample k with k + 1
    return rmd_render(r, &s);
}

rmd_status rmd_film_normalize(rmd_renderer *r, const rmd_uniforms *u, float *rgba) {
    if (!r || !u || !rgba) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (u->tonemapping > 2) return fail(RMD_ERROR_INVALID_ARGUMENT, "tonemapping out of range");
    cudaStream_t st = r->scene->ctx->stream;
    const uint32_t n = r->width * r->height;
    const float div = u->accumulate ? (float)u->frame_index + 1.0f : 1.0f;
    RMD_CUDA(rmdLaunchFilmResolve(r->film.as<float4>(), r->film64.as<double>(), 0, r->resolve.as<float>(), n,
                                  u->exposure, div, u->tonemapping, 4, st));
    RMD_CUDA(cudaMemcpyAsync(rgba, r->resolve.ptr, (size_t)n * 4 * sizeof(float), cudaMemcpyDeviceToHost, st));
    RMD_CUDA(cudaStreamSynchronize(st));
    return RMD_OK;
}

rmd_status rmd_render(rmd_renderer *r, const rmd_render_settings *s) {
    if (!r || !s) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (s->max_depth == 0 || s->max_depth > 65535 || s->sampling_mode > 2 || s->rng > 1)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid render settings");
    rmd_scene *scene = r->scene;
    rmd_context *ctx = scene->ctx;
    RMD_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const uint64_t numPixels = (uint64_t)r->width * r->height;
    const uint64_t firstSample = s->first_sample >= 0 ? (uint64_t)s->first_sample : r->nextSample;
    const uint64_t numPaths = (uint64_t)s->spp * numPixels;
    if (firstSample + s->spp > 0xffffffffull) return fail(RMD_ERROR_INVALID_ARGUMENT, "sample index overflow");
    if (s->film_fp64 && !r->film64.ptr) {
        RMD_CUDA(r->film64.alloc(numPixels * 3 * sizeof(double)));
        RMD_CUDA(cudaMemsetAsync(r->film64.ptr, 0, r->film64.bytes, st));
    }
    std::memset(&r->stats, 0, sizeof(r->stats));
    r->stats.pool_size = r->capacity;
    if (numPaths == 0) return RMD_OK;

    FrameParams fp{};
    fp.width = r->width;
    fp.height = r->height;
    fp.numPixels = (uint32_t)numPixels;
    fp.maxDepth = s->max_depth;
    fp.samplingMode = s->sampling_mode;
    fp.rngMode = s->rng;
    fp.seed = s->seed;
    fp.filmFp64 = s->film_fp64 ? 1 : 0;
    fp.film = r->film.as<float4>();
    fp.film64 = r->film64.as<double>();
    Counters *cnt = r->counters.as<Counters>();
    const uint64_t firstPath = firstSample * numPixels;

    ShadeParams sp;
    sp.ctx = r->dctx;
    sp.counters = cnt;
    void *shadeArgs[] = {&sp};
    const int tb = ctx->smCount * r->traceBlocksPerSm;
    const int rb = std::min<int>((r->capacity + 255) / 256, ctx->smCount * 8);

    // guiding
    auto &guide = r->guide;
    const bool guideSampling = guide.settings.sampling != 0;
    const bool guideTraining = guide.settings.training != 0;
    if (r->shadeGuided != (guideSampling || guideTraining)) {  // the shading kernel with or without the guide's code
        rmd_status vs = ensureVariants(scene, {r->shadeMinBlocks}, guideSampling || guideTraining);
        if (vs != RMD_OK) return vs;
        selectShade(r, r->shadeMinBlocks, guideSampling || guideTraining);
    }
    const int sb = r->shadeBlocks;
    GuideNetView net{};
    if (guideSampling || guideTraining) {
        rmd_status gs = ensureGuideBuffers(r);
        if (gs != RMD_OK) return gs;
        guideFrame(scene, guide.frameMin, guide.frameInvExtent);
        const float3 lo = guide.frameMin, inv = guide.frameInvExtent;
        net = guide.net.view(lo, inv);
        fp.guideDepth = guideSampling ? guide.settings.guided_depth : 0u;
        fp.guideSceneMin = lo;
        fp.guideSceneInvExtent = inv;
    }
    const PathPool pool = poolView(r);
    sp.pool = pool;
    sp.fp = fp;
    const int guideBlocks = ctx->smCount;  // the inference kernel: one CTA of 4 pipelines per SM (shared memory)
    const int trainBlocks = ctx->smCount;
    const uint32_t batch = guide.settings.batch_size;
    uint64_t trainSteps = 0;

    enum { STAGE_FILM, STAGE_TRACE, STAGE_GUIDE, STAGE_SHADE, STAGE_SHADOW, STAGE_TRAIN, STAGES };
    RMD_CUDA(cudaEventRecord(r->ev[0], st));
    RMD_CUDA(rmdLaunchFrameInit(pool, cnt, firstPath, firstPath + numPaths, st));
    // every path needs at most max_depth iterations after it is generated, and
    // each iteration generates min(capacity, remaining) paths
    const uint64_t maxIters = ((numPaths + r->capacity - 1) / r->capacity + 1) * ((uint64_t)s->max_depth + 1) + 8;
    uint64_t it = 0;
    uint32_t cur = 0;
    bool done = false;
    size_t evi = 0;
    RMD_CUDA(r->stageEvent(evi++, STAGE_FILM, st));
    while (!done) {
        for (int k = 0; k < 4; k++, it++) {
            RMD_CUDA(rmdLaunchFilmRegen(r->dctx, pool, fp, cnt, cur, rb, st));
            RMD_CUDA(r->stageEvent(evi++, STAGE_FILM, st));
            RMD_CUDA(rmdLaunchTraceClosest(scene->bvhNodes.as<WideNode>(), scene->bvhTris.as<float4>(), pool, cnt, cur, tb, st));
            RMD_CUDA(r->stageEvent(evi++, STAGE_TRACE, st));
            if (guideSampling) {
                RMD_CUDA(rmdLaunchGuideInfer(r->dctx, pool, cnt, cur, fp.guideDepth, net, pool.guide, guideBlocks, st));
                RMD_CUDA(r->stageEvent(evi++, STAGE_GUIDE, st));
            }
            sp.cur = cur;
            RMD_CUDA(cudaLaunchKernel((const void *)r->shade, dim3(sb), dim3(128), shadeArgs, 0, st));
            RMD_CUDA(r->stageEvent(evi++, STAGE_SHADE, st));
            RMD_CUDA(rmdLaunchTraceShadow(scene->bvhNodes.as<WideNode>(), scene->bvhTris.as<float4>(), pool, cnt, cur, tb, st));
            RMD_CUDA(r->stageEvent(evi++, STAGE_SHADOW, st));
            cur ^= 1u;
        }
        RMD_CUDA(cudaMemcpyAsync(r->hostCounters, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        RMD_CUDA(cudaStreamSynchronize(st));
        const Counters &h = *r->hostCounters;
        if (h.errors) {
            r->stats.errors = h.errors;
            if (h.errors & ERR_GUIDE_TIMEOUT)
                return fail(RMD_ERROR_WATCHDOG, "guide inference: a tensor-core wait expired (device error flags " +
                                                    std::to_string(h.errors) + ")");
            return fail(RMD_ERROR_QUEUE_OVERFLOW, "device error flags " + std::to_string(h.errors));
        }
        if (guideTraining && h.numSamples >= batch) {
            rmd_status gs = guideTrainStep(guide, h, cnt, net, trainBlocks, st, trainSteps);
            if (gs != RMD_OK) return gs;
            RMD_CUDA(r->stageEvent(evi++, STAGE_TRAIN, st));
        }
        if (h.pathsDone >= numPaths) done = true;
        else if (it > maxIters) return fail(RMD_ERROR_WATCHDOG, "render did not drain in the iteration bound");
    }
    RMD_CUDA(cudaEventRecord(r->ev[1], st));
    RMD_CUDA(cudaEventSynchronize(r->ev[1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, r->ev[0], r->ev[1]);
    double stage[STAGES] = {};
    for (size_t i = 1; i < evi; i++) {
        float t = 0;
        cudaEventElapsedTime(&t, r->stageEvents[i - 1], r->stageEvents[i]);
        stage[r->stageOf[i]] += t;
    }
    if (trainSteps) {
        rmd_status gs = guideReadLoss(guide);
        if (gs != RMD_OK) return gs;
    }
    const Counters &h = *r->hostCounters;
    r->stats.paths = h.pathsDone;
    r->stats.segments = h.segments;
    r->stats.rays = h.rays;
    r->stats.shadow_rays = h.shadowRays;
    r->stats.invalid_samples = h.invalid;
    r->stats.iterations = it;
    r->stats.ms_total = ms;
    r->stats.ms_film = stage[STAGE_FILM];
    r->stats.ms_trace = stage[STAGE_TRACE];
    r->stats.ms_shade = stage[STAGE_SHADE];
    r->stats.ms_shadow = stage[STAGE_SHADOW];
    r->stats.ms_guide = stage[STAGE_GUIDE] + stage[STAGE_TRAIN];
    r->stats.ms_guide_train = stage[STAGE_TRAIN];
    r->samples += s->spp;
    r->nextSample = std::max<uint64_t>(r->nextSample, firstSample + s->spp);
    return RMD_OK;
}

rmd_status rmd_film_read(rmd_renderer *r, float *rgb, int32_t normalize, uint32_t tonemapping, float exposure) {
    if (!r || !rgb) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (tonemapping > 2) return fail(RMD_ERROR_INVALID_ARGUMENT, "tonemapping out of range");
    cudaStream_t st = r->scene->ctx->stream;
    const uint32_t n = r->width * r->height;
    float ex = 1.0f, div = 1.0f;
    uint32_t tm = 0;
    if (normalize) {
        ex = exposure;
        div = (float)std::max<uint64_t>(1, r->samples);
        tm = tonemapping;
    }
    RMD_CUDA(rmdLaunchFilmResolve(r->film.as<float4>(), r->film64.as<double>(), 0, r->resolve.as<float>(), n, ex, div,
                                  tm, 3, st));
    RMD_CUDA(cudaMemcpyAsync(rgb, r->resolve.ptr, (size_t)n * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    RMD_CUDA(cudaStreamSynchronize(st));
    return RMD_OK;
}

static rmd_status saveExr(const char *path, const std::vector<float> &rgb, uint32_t w, uint32_t h, float norm,
                          uint64_t samples, uint32_t compression) {
    if (!path) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL path");
    if (compression > RMD_EXR_ZIP) return fail(RMD_ERROR_INVALID_ARGUMENT, "unknown EXR compression");
    if (!(norm > 0.0f)) norm = 1.0f / (float)std::max<uint64_t>(1, samples);
    const std::string err =
        rmdhost::writeExrFilm(path, rgb.data(), w, h, norm, (rmdhost::ExrCompression)compression);
    if (!err.empty()) return fail(RMD_ERROR_INVALID_ARGUMENT, "EXR: " + err);
    return RMD_OK;
}

rmd_status rmd_film_save_exr(rmd_renderer *r, const char *path, float normalized_by, uint32_t compression) {
    if (!r) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL renderer");
    std::vector<float> rgb((size_t)r->width * r->height * 3);
    const rmd_status st = rmd_film_read(r, rgb.data(), 0, 0, 1.0f);
    if (st != RMD_OK) return st;
    return saveExr(path, rgb, r->width, r->height, normalized_by, r->samples, compression);
}

rmd_status rmd_test_exr_write(const char *path, const float *rgb, int32_t width, int32_t height, float normalized_by,
                              uint32_t compression) {
    if (!rgb || width <= 0 || height <= 0) return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid image");
    const std::vector<float> v(rgb, rgb + (size_t)width * height * 3);
    return saveExr(path, v, (uint32_t)width, (uint32_t)height, normalized_by, 1, compression);
}

rmd_status rmd_film_read_f64(rmd_renderer *r, double *rgb) {
    if (!r || !rgb) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (!r->film64.ptr) return fail(RMD_ERROR_INVALID_ARGUMENT, "no double-precision film (render with film_fp64)");
    cudaStream_t st = r->scene->ctx->stream;
    RMD_CUDA(cudaMemcpyAsync(rgb, r->film64.ptr, r->film64.bytes, cudaMemcpyDeviceToHost, st));
    RMD_CUDA(cudaStreamSynchronize(st));
    return RMD_OK;
}

rmd_status rmd_film_samples(const rmd_renderer *r, uint64_t *samples) {
    if (!r || !samples) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    *samples = r->samples;
    return RMD_OK;
}

rmd_status rmd_film_device(rmd_renderer *r, float **film, uint64_t *num_pixels) {
    if (!r || !film) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    *film = r->film.as<float>();
    if (num_pixels) *num_pixels = (uint64_t)r->width * r->height;
    return RMD_OK;
}

rmd_status rmd_film_set_samples(rmd_renderer *r, uint64_t samples) {
    if (!r) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL renderer");
    r->samples = samples;
    return RMD_OK;
}

rmd_status rmd_renderer_stats(const rmd_renderer *r, rmd_stats *out) {
    if (!r || !out) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    *out = r->stats;
    return RMD_OK;
}

// --------------------------------------------------------------------- autotuner
// Shading-kernel variants: a register budget (minimum 128-thread blocks per
// SM) and whether the kernel carries the guide's sampling and training code;
// renderers and batches that do not guide run the kernel without it.
static int shadeVariantKey(int minBlocks, bool guided) { return minBlocks | (guided ? 0x100 : 0); }
static std::vector<std::string> shadeDefines(int minBlocks, bool guided) {
    std::vector<std::string> d = {"-DRMD_SHADE_MIN_BLOCKS=" + std::to_string(minBlocks)};
    if (!guided) d.push_back("-DRMD_PLAIN_SHADE");
    return d;
}

static rmd_status ensureVariants(rmd_scene *s, const std::vector<int> &minBlocks, bool guided) {
    std::vector<int> missing;
    for (int mb : minBlocks)
        if ((guided || mb != s->defaultMinBlocks) && !s->variants.count(shadeVariantKey(mb, guided)))
            missing.push_back(mb);
    // NVRTC is thread-safe: compile the missing variants in parallel, load them serially
    std::vector<std::vector<char>> cubins(missing.size());
    std::vector<std::string> errs(missing.size()), logs(missing.size());
    std::vector<std::thread> th;
    for (size_t i = 0; i < missing.size(); i++) {
        th.emplace_back([&, i] {
            bool cached = false;
            errs[i] = rmdhost::compileCubin(s->moduleSource, cubins[i], logs[i], cached,
                                            shadeDefines(missing[i], guided));
        });
    }
    for (auto &t : th) t.join();
    for (size_t i = 0; i < missing.size(); i++) {
        if (!errs[i].empty()) return fail(RMD_ERROR_NVRTC, errs[i]);
        auto m = std::make_unique<rmdhost::JitModule>();
        RMD_CUDA(cudaLibraryLoadData(&m->library, cubins[i].data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
        RMD_CUDA(cudaLibraryGetKernel(&m->shade, m->library, "rmd_shade"));
        s->variants[shadeVariantKey(missing[i], guided)] = std::move(m);
    }
    return RMD_OK;
}

// the variant must have been compiled (ensureVariants)
static void selectShade(rmd_renderer *r, int mb, bool guided) {
    rmd_scene *s = r->scene;
    cudaKernel_t k = !guided && mb == s->defaultMinBlocks ? s->jit.shade : s->variants.at(shadeVariantKey(mb, guided))->shade;
    r->shade = k;
    r->shadeMinBlocks = mb;
    r->shadeGuided = guided;
    r->shadeBlocks = occupancyBlocks((const void *)k, 128, s->ctx->smCount);
}

static bool guideActive(const GuideState &g) { return g.settings.sampling || g.settings.training; }

rmd_status rmd_renderer_autotune(rmd_renderer *r, const rmd_render_settings *settings, rmd_tune_result *out) {
    if (!r || !settings) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    rmd_scene *s = r->scene;
    const std::vector<int> mbs = {1, 3, 4, 5, 6, 8, 10, 12, 16};
    const bool guided = guideActive(r->guide);
    rmd_status st = ensureVariants(s, mbs, guided);
    if (st != RMD_OK) return st;
    // pool sizes tried: half, twice and four times the current one
    const uint32_t cap0 = r->capacity;
    std::vector<uint32_t> caps;
    const uint64_t candidates[3] = {(uint64_t)cap0 / 2, 2 * (uint64_t)cap0, 4 * (uint64_t)cap0};
    for (uint64_t cap : candidates)
        if (cap >= (1u << 16) && cap <= (1ull << 30)) caps.push_back((uint32_t)cap);
    // calibration: enough paths for several generations of the largest pool
    // tried (a pool drained once measures its tail, not its throughput), at
    // most the caller's samples
    rmd_render_settings cal = *settings;
    cal.film_fp64 = 0;
    const uint64_t pixels = (uint64_t)r->width * r->height;
    const uint64_t maxCap = std::max<uint64_t>(cap0, caps.empty() ? 0 : *std::max_element(caps.begin(), caps.end()));
    cal.spp = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(settings->spp, (4ull * maxCap + pixels - 1) / pixels));
    cal.first_sample = 1u << 30;  // a sample range the caller does not use
    auto trial = [&](double &ms) -> rmd_status {
        double best = 1e30;
        for (int rep = 0; rep < 2; rep++) {
            rmd_status e = rmd_render(r, &cal);
            if (e != RMD_OK) return e;
            best = std::min(best, r->stats.ms_total);
        }
        ms = best;
        return RMD_OK;
    };
    rmd_tune_result res{};
    double base = 0;
    if ((st = trial(base)) != RMD_OK) return st;
    res.ms_default = base;
    // 1) shading kernel register budget
    int bestMb = r->shadeMinBlocks;
    double bestMs = base;
    for (int mb : mbs) {
        if (mb == r->shadeMinBlocks) continue;
        selectShade(r, mb, guided);
        double ms;
        if ((st = trial(ms)) != RMD_OK) return st;
        if (ms < bestMs) {
            bestMs = ms;
            bestMb = mb;
        }
    }
    selectShade(r, bestMb, guided);
    // 2) traversal blocks per SM
    int bestTb = r->traceBlocksPerSm;
    for (int tb : {4, 8, 12, 16}) {
        r->traceBlocksPerSm = tb;
        double ms;
        if ((st = trial(ms)) != RMD_OK) return st;
        if (ms < bestMs) {
            bestMs = ms;
            bestTb = tb;
        }
    }
    r->traceBlocksPerSm = bestTb;
    // 3) paths in flight (queue sizes)
    uint32_t bestCap = cap0;
    for (uint32_t cap : caps) {
        size_t freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess || pathPoolBytes(cap) > freeB / 2) continue;
        r->capacity = cap;
        if ((st = allocatePool(r)) != RMD_OK) return st;
        double ms;
        if ((st = trial(ms)) != RMD_OK) return st;
        if (ms < bestMs) {
            bestMs = ms;
            bestCap = cap;
        }
    }
    if (r->capacity != bestCap) {
        r->capacity = bestCap;
        if ((st = allocatePool(r)) != RMD_OK) return st;
    }
    res.shade_min_blocks = (uint32_t)r->shadeMinBlocks;
    res.trace_blocks_per_sm = (uint32_t)r->traceBlocksPerSm;
    res.pool_size = r->capacity;
    res.ms_best = bestMs;
    res.calibration_spp = cal.spp;
    if (out) *out = res;
    return rmd_renderer_reset(r);
}

rmd_status rmd_renderer_set_tuning(rmd_renderer *r, const rmd_tune_result *t) {
    if (!r || !t) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (t->shade_min_blocks < 1 || t->shade_min_blocks > 16 || t->trace_blocks_per_sm < 1 ||
        t->trace_blocks_per_sm > 32 || (t->pool_size != 0 && t->pool_size < 1024))
        return fail(RMD_ERROR_INVALID_ARGUMENT, "tuning out of range");
    RMD_CUDA(cudaSetDevice(r->scene->ctx->device));
    const int mb = (int)t->shade_min_blocks;
    rmd_status st = ensureVariants(r->scene, {mb}, r->shadeGuided);
    if (st != RMD_OK) return st;
    selectShade(r, mb, r->shadeGuided);
    r->traceBlocksPerSm = (int)t->trace_blocks_per_sm;
    if (t->pool_size != 0 && t->pool_size != r->capacity) {
        r->capacity = t->pool_size;
        if ((st = allocatePool(r)) != RMD_OK) return st;
    }
    return RMD_OK;
}

// --------------------------------------------------------------------- guiding
rmd_status rmd_renderer_set_guide(rmd_renderer *r, const rmd_guide_settings *settings) {
    if (!r || !settings) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    RMD_CUDA(cudaSetDevice(r->scene->ctx->device));
    rmd_status st = setGuide(r->guide, settings, r->scene->ctx->stream, r->counters.as<Counters>());
    if (st != RMD_OK) return st;
    return ensureGuideBuffers(r);
}

rmd_status rmd_renderer_guide_stats(const rmd_renderer *r, rmd_guide_stats *out) {
    if (!r || !out) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    *out = r->guide.stats;
    return RMD_OK;
}

rmd_status rmd_renderer_guide_params(rmd_renderer *r, float *params, int32_t write) {
    if (!r || !params || write < 0 || write > 1) return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid argument");
    RMD_CUDA(cudaSetDevice(r->scene->ctx->device));
    return guideParams(r->guide, params, write, r->scene->ctx->stream);
}

// --------------------------------------------------------------------- test hooks
rmd_status rmd_test_prng(uint32_t mode, uint64_t a, uint64_t b, int32_t n, float *out) {
    if (!out || n < 0) return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid arguments");
    float *d = nullptr;
    RMD_CUDA(cudaMalloc(&d, std::max<int>(1, n) * sizeof(float)));
    cudaError_t e = rmdLaunchDebugPrng(mode, a, b, n, d, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(RMD_ERROR_CUDA, cudaGetErrorString(e));
    return RMD_OK;
}

rmd_status rmd_test_trace(const rmd_scene *s, const float *rays, int32_t n, int32_t any, float *out,
                          uint32_t *instances) {
    if (!s || !rays || !out || !instances || n < 0) return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid arguments");
    DevBuf dr, dout, dinst, derr;
    RMD_CUDA(dr.upload(rays, (size_t)n * 8 * sizeof(float), s->ctx->stream));
    RMD_CUDA(dout.alloc((size_t)std::max(1, n) * 4 * sizeof(float)));
    RMD_CUDA(dinst.alloc((size_t)std::max(1, n) * sizeof(uint32_t)));
    RMD_CUDA(derr.alloc(sizeof(uint32_t)));
    RMD_CUDA(cudaMemset(derr.ptr, 0, sizeof(uint32_t)));
    if (n > 0)
        RMD_CUDA(rmdLaunchDebugTrace(s->bvhNodes.as<WideNode>(), s->bvhTris.as<float4>(), dr.as<float>(), n, any,
                                     dout.as<float>(), dinst.as<uint32_t>(), derr.as<uint32_t>(), s->ctx->stream));
    RMD_CUDA(cudaStreamSynchronize(s->ctx->stream));
    RMD_CUDA(cudaMemcpy(out, dout.ptr, (size_t)n * 4 * sizeof(float), cudaMemcpyDeviceToHost));
    RMD_CUDA(cudaMemcpy(instances, dinst.ptr, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return RMD_OK;
}

rmd_status rmd_test_bvh_read(const rmd_scene *s, void *nodes, uint64_t max_nodes, float *tris, uint64_t max_triangles) {
    if (!s) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL scene");
    if ((nodes && max_nodes < s->bvhNodeCount) || (tris && max_triangles < s->triangles))
        return fail(RMD_ERROR_INVALID_ARGUMENT, "output buffers too small");
    RMD_CUDA(cudaSetDevice(s->ctx->device));
    if (nodes && s->bvhNodeCount)
        RMD_CUDA(cudaMemcpy(nodes, s->bvhNodes.ptr, s->bvhNodeCount * sizeof(rmdhost::GpuWideNode),
                            cudaMemcpyDeviceToHost));
    if (tris && s->triangles)  // copy 2 of each triangle: the builders' (v0, v1, v2) in world coordinates
        RMD_CUDA(cudaMemcpy2D(tris, 3 * sizeof(float4), static_cast<const float4 *>(s->bvhTris.ptr) + 6,
                              TRI_FLOAT4 * sizeof(float4), 3 * sizeof(float4), s->triangles, cudaMemcpyDeviceToHost));
    return RMD_OK;
}

rmd_status rmd_test_material_eval(const rmd_scene *s, int32_t material, const float *records, int32_t n, float *out) {
    if (!s || !records || !out || n < 0 || material < 0 || material >= s->numSurface)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid arguments");
    DevBuf din, dout;
    RMD_CUDA(din.upload(records, (size_t)n * 28 * sizeof(float), s->ctx->stream));
    RMD_CUDA(dout.alloc((size_t)std::max(1, n) * 16 * sizeof(float)));
    Context c = s->dctx;
    unsigned m = (unsigned)material;
    const float *pin = din.as<float>();
    float *pout = dout.as<float>();
    int nn = n;
    void *args[] = {&c, &m, &pin, &pout, &nn};
    if (n > 0)
        RMD_CUDA(cudaLaunchKernel((const void *)s->jit.materialEval, dim3((n + 127) / 128), dim3(128), args, 0,
                                  s->ctx->stream));
    RMD_CUDA(cudaStreamSynchronize(s->ctx->stream));
    RMD_CUDA(cudaMemcpy(out, dout.ptr, (size_t)n * 16 * sizeof(float), cudaMemcpyDeviceToHost));
    return RMD_OK;
}

rmd_status rmd_test_generate_source(const rmd_scene_desc *d, int32_t hoist, char *buf, int64_t buflen,
                                    int64_t *needed) {
    if (!d) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL desc");
    try {
        const rmdhost::SceneTextures tex = rmdhost::sceneTextures(d);
        rmdhost::GeneratedModule mod =
            rmdhost::generateModule(d->surface_materials, d->num_surface_materials, d->light_materials,
                                    d->num_light_materials, hoist != 0,
                                    rmdhost::TextureTable::of(tex.list.data(), (int)tex.list.size()));
        if (needed) *needed = (int64_t)mod.source.size() + 1;
        if (buf && buflen > 0) {
            const size_t n = std::min<size_t>((size_t)buflen - 1, mod.source.size());
            std::memcpy(buf, mod.source.data(), n);
            buf[n] = 0;
        }
    } catch (const rmdhost::CodegenError &e) {
        return fail(e.status, e.message);
    }
    return RMD_OK;
}

rmd_status rmd_test_jit_compile(const rmd_scene_desc *d, int32_t hoist, char *log, int64_t loglen,
                                int64_t *cubin_bytes) {
    if (!d) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL desc");
    std::string msg;
    try {
        const rmdhost::SceneTextures tex = rmdhost::sceneTextures(d);
        rmdhost::GeneratedModule mod =
            rmdhost::generateModule(d->surface_materials, d->num_surface_materials, d->light_materials,
                                    d->num_light_materials, hoist != 0,
                                    rmdhost::TextureTable::of(tex.list.data(), (int)tex.list.size()));
        std::vector<char> cubin;
        bool cached = false;
        std::string err = rmdhost::compileCubin(mod.source, cubin, msg, cached,
                                                {"-DRMD_SHADE_MIN_BLOCKS=" + std::to_string(defaultShadeMinBlocks())});
        if (cubin_bytes) *cubin_bytes = (int64_t)cubin.size();
        if (!err.empty()) {
            if (log && loglen > 0) {
                const size_t n = std::min<size_t>((size_t)loglen - 1, err.size());
                std::memcpy(log, err.data(), n);
                log[n] = 0;
            }
            return fail(RMD_ERROR_NVRTC, err);
        }
    } catch (const rmdhost::CodegenError &e) {
        return fail(e.status, e.message);
    }
    if (log && loglen > 0) {
        const size_t n = std::min<size_t>((size_t)loglen - 1, msg.size());
        std::memcpy(log, msg.data(), n);
        log[n] = 0;
    }
    return RMD_OK;
}

// --------------------------------------------------------------------- batches
static rmd_status batchAllocatePool(rmd_batch *b) {
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    b->graphKey.clear();
    RMD_CUDA(b->pool.alloc(pathPoolBytes(b->capacity)));
    RMD_CUDA(b->counters.alloc(sizeof(Counters)));
    RMD_CUDA(cudaMemset(b->counters.ptr, 0, sizeof(Counters)));
    return guideBuffers(b->guide, b->capacity, b->counters.as<Counters>());
}

static PathPool batchPoolView(const rmd_batch *b) {
    PathPool pool = carvePathPool(b->pool.ptr, b->capacity);
    pool.views = b->viewTable.as<BatchView>();
    pool.numViews = (uint32_t)b->views.size();
    applyGuide(b->guide, b->capacity, pool);
    return pool;
}

// the variant must have been compiled (batchEnsureVariants)
static void batchSelectShade(rmd_batch *b, int mb, bool guided) {
    cudaKernel_t k = !guided && mb == b->defaultMinBlocks ? b->jit.shade : b->variants.at(shadeVariantKey(mb, guided))->shade;
    b->shade = k;
    b->shadeMinBlocks = mb;
    b->shadeGuided = guided;
    b->shadeBlocks = occupancyBlocks((const void *)k, 128, b->ctx->smCount);
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    b->graphKey.clear();
}

static rmd_status batchEnsureVariants(rmd_batch *b, const std::vector<int> &minBlocks, bool guided) {
    for (int mb : minBlocks) {
        const int key = shadeVariantKey(mb, guided);
        if ((!guided && mb == b->defaultMinBlocks) || b->variants.count(key)) continue;
        auto m = std::make_unique<rmdhost::JitModule>();
        std::vector<std::string> defines = shadeDefines(mb, guided);
        defines.push_back("-DRMD_BATCH");
        const std::string err = rmdhost::compileModule(b->moduleSource, *m, defines);
        if (!err.empty()) return fail(RMD_ERROR_NVRTC, err);
        b->variants[key] = std::move(m);
    }
    return RMD_OK;
}

rmd_status rmd_batch_create(rmd_context *ctx, const rmd_scene_desc *descs, int32_t numScenes,
                            const rmd_batch_view *views, int32_t numViews, uint32_t poolSize, uint32_t flags,
                            rmd_batch **out) {
    if (!ctx || !descs || !views || !out || numScenes <= 0 || numViews <= 0)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument or empty batch");
    if (numViews > 256) return fail(RMD_ERROR_INVALID_ARGUMENT, "at most 256 views per batch");
    if (flags & ~RMD_BATCH_NO_GRAPH) return fail(RMD_ERROR_INVALID_ARGUMENT, "unknown batch flags");
    uint64_t total = 0;
    for (int v = 0; v < numViews; v++) {
        const rmd_batch_view &bv = views[v];
        if (bv.scene < 0 || bv.scene >= numScenes || bv.width == 0 || bv.height == 0 || bv.width > 65535 ||
            bv.height > 65535)
            return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid batch view " + std::to_string(v));
        total += (uint64_t)bv.width * bv.height;
    }
    if (total > 0x7fffffffull) return fail(RMD_ERROR_INVALID_ARGUMENT, "batch films exceed 2^31 pixels");
    for (int i = 0; i < numScenes; i++) {
        rmd_status r = validateSceneDesc(&descs[i]);
        if (r != RMD_OK) return fail(r, "scene " + std::to_string(i) + ": " + g_lastError);
    }
    RMD_CUDA(cudaSetDevice(ctx->device));
    auto b = std::make_unique<rmd_batch>();
    b->ctx = ctx;
    b->useGraph = !(flags & RMD_BATCH_NO_GRAPH);
    // one material module for all scenes: their materials concatenated
    std::vector<rmd_material> surf, light;
    std::vector<int> surfBase, lightBase;
    for (int i = 0; i < numScenes; i++) {
        surfBase.push_back((int)surf.size());
        lightBase.push_back((int)light.size());
        surf.insert(surf.end(), descs[i].surface_materials, descs[i].surface_materials + descs[i].num_surface_materials);
        light.insert(light.end(), descs[i].light_materials, descs[i].light_materials + descs[i].num_light_materials);
    }
    // The scenes' textures in one table (slots are baked into the shared
    // module; an image two scenes pass under the same name is stored once).
    // Each scene's materials resolve file names against its own textures.
    std::vector<rmd_texture> texUnion;
    std::vector<rmdhost::TextureTable> sceneTables(numScenes);
    std::vector<rmdhost::SceneTextures> sceneTex(numScenes);  // images and generated skies (names live here)
    try {
        for (int i = 0; i < numScenes; i++) sceneTex[i] = rmdhost::sceneTextures(&descs[i]);
    } catch (const rmdhost::CodegenError &e) {
        return fail(e.status, e.message);
    }
    for (int i = 0; i < numScenes; i++) {
        rmdhost::TextureTable &t = sceneTables[i];
        for (const rmd_texture &x : sceneTex[i].list) {
            auto same = std::find_if(texUnion.begin(), texUnion.end(), [&](const rmd_texture &u) {
                return std::strcmp(u.name, x.name) == 0 && u.data == x.data && u.width == x.width &&
                       u.height == x.height && u.channels == x.channels && u.format == x.format;
            });
            t.names.push_back(x.name);
            t.channels.push_back(x.channels);
            t.slots.push_back((uint32_t)(same - texUnion.begin()));
            if (same == texUnion.end()) texUnion.push_back(x);
        }
    }
    std::vector<const rmdhost::TextureTable *> surfTables, lightTables;
    for (int i = 0; i < numScenes; i++) {
        sceneTables[i].missingSlot = (uint32_t)texUnion.size();  // the zero texture after the union
        surfTables.insert(surfTables.end(), descs[i].num_surface_materials, &sceneTables[i]);
        lightTables.insert(lightTables.end(), descs[i].num_light_materials, &sceneTables[i]);
    }
    rmdhost::GeneratedModule mod;
    try {
        mod = rmdhost::generateModule(surf.data(), (int)surf.size(), light.data(), (int)light.size(), true,
                                      rmdhost::TextureTable(), surfTables, lightTables);
    } catch (const rmdhost::CodegenError &e) {
        return fail(e.status, e.message);
    }
    b->defaultMinBlocks = defaultShadeMinBlocks();
    const std::string err = rmdhost::compileModule(
        mod.source, b->jit, {"-DRMD_SHADE_MIN_BLOCKS=" + std::to_string(b->defaultMinBlocks), "-DRMD_PLAIN_SHADE", "-DRMD_BATCH"});
    if (!err.empty()) return fail(RMD_ERROR_NVRTC, err);
    b->moduleSource = mod.source;
    for (int i = 0; i < numScenes; i++) {
        auto sc = std::make_unique<rmd_scene>();
        rmd_status r = buildSceneData(ctx, &descs[i], sc.get(), mod, surfBase[i], lightBase[i], texUnion.data(),
                                      (int)texUnion.size());
        if (r != RMD_OK) return r;
        sc->jit = b->jit;  // the batch's module builds the scene's environment map
        sc->ownsModule = false;
        if ((r = buildEnvironmentMap(sc.get(), descs[i].envmap_exponent)) != RMD_OK) return r;
        b->scenes.push_back(std::move(sc));
    }
    // views: their scene's context with the view's camera, in film order
    std::vector<BatchView> table(numViews);
    uint32_t offset = 0;
    for (int v = 0; v < numViews; v++) {
        const rmd_batch_view &bv = views[v];
        const rmd_scene *sc = b->scenes[bv.scene].get();
        BatchView &t = table[v];
        t.ctx = sc->dctx;
        for (int k = 0; k < 4; k++)
            t.ctx.cameraTransform[k] = make_float4(bv.camera.transform[4 * k], bv.camera.transform[4 * k + 1],
                                                   bv.camera.transform[4 * k + 2], bv.camera.transform[4 * k + 3]);
        t.ctx.nearClip = bv.camera.near_clip;
        t.ctx.farClip = bv.camera.far_clip;
        t.ctx.focalLength = bv.camera.focal_length;
        t.ctx.shift = make_float2(bv.camera.shift[0], bv.camera.shift[1]);
        t.nodes = sc->bvhNodes.ptr;
        t.tris = sc->bvhTris.as<float4>();
        t.width = bv.width;
        t.height = bv.height;
        t.numPixels = bv.width * bv.height;
        t.pixelOffset = offset;
        b->views.push_back(bv);
        b->offsets.push_back(offset);
        offset += t.numPixels;
    }
    b->totalPixels = offset;
    RMD_CUDA(b->viewTable.upload(table.data(), table.size() * sizeof(BatchView), ctx->stream));
    RMD_CUDA(b->film.alloc((size_t)offset * sizeof(float4)));
    RMD_CUDA(cudaMemset(b->film.ptr, 0, b->film.bytes));
    RMD_CUDA(b->resolve.alloc((size_t)offset * 3 * sizeof(float)));
    b->capacity = poolSize ? poolSize : (1u << 21);
    if (b->capacity > BATCH_MAX_CAPACITY) return fail(RMD_ERROR_INVALID_ARGUMENT, "batch pools hold at most 2^22 paths");
    rmd_status r = batchAllocatePool(b.get());
    if (r != RMD_OK) return r;
    RMD_CUDA(cudaMallocHost((void **)&b->hostCounters, sizeof(Counters)));
    for (auto &e : b->ev) RMD_CUDA(cudaEventCreate(&e));
    batchSelectShade(b.get(), b->defaultMinBlocks, false);
    *out = b.release();
    return RMD_OK;
}

void rmd_batch_destroy(rmd_batch *b) { delete b; }

rmd_status rmd_batch_reset(rmd_batch *b) {
    if (!b) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL batch");
    cudaStream_t st = b->ctx->stream;
    RMD_CUDA(cudaMemsetAsync(b->film.ptr, 0, b->film.bytes, st));
    if (b->film64.ptr) RMD_CUDA(cudaMemsetAsync(b->film64.ptr, 0, b->film64.bytes, st));
    RMD_CUDA(cudaStreamSynchronize(st));
    b->samples = 0;
    b->nextSample = 0;
    return RMD_OK;
}

// Records the render's wavefront loop on `st`: host-driven (counter checks
// every 4 iterations) or, with `handle`, as the body of a graph while loop
// (2 iterations and the condition kernel).
static rmd_status batchEnqueueIterations(rmd_batch *b, const PathPool &pool, const FrameParams &fp, ShadeParams &sp,
                                         const GuideNetView &net, int iterations, cudaStream_t st) {
    Counters *cnt = b->counters.as<Counters>();
    const int tb = b->ctx->smCount * b->traceBlocksPerSm;
    const int rb = std::min<int>((b->capacity + 255) / 256, b->ctx->smCount * 8);
    void *shadeArgs[] = {&sp};
    for (int k = 0; k < iterations; k++) {
        const uint32_t cur = (uint32_t)k & 1u;
        RMD_CUDA(rmdLaunchFilmRegen(b->scenes[0]->dctx, pool, fp, cnt, cur, rb, st));
        RMD_CUDA(rmdLaunchTraceClosest(nullptr, nullptr, pool, cnt, cur, tb, st));
        if (pool.guide)
            RMD_CUDA(rmdLaunchGuideInfer(b->scenes[0]->dctx, pool, cnt, cur, fp.guideDepth, net, pool.guide,
                                         b->ctx->smCount, st));
        sp.cur = cur;
        RMD_CUDA(cudaLaunchKernel((const void *)b->shade, dim3(b->shadeBlocks), dim3(128), shadeArgs, 0, st));
        RMD_CUDA(rmdLaunchTraceShadow(nullptr, nullptr, pool, cnt, cur, tb, st));
    }
    return RMD_OK;
}

rmd_status rmd_batch_render(rmd_batch *b, const rmd_render_settings *s) {
    if (!b || !s) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (s->max_depth == 0 || s->max_depth > 65535 || s->sampling_mode > 2 || s->rng > 1)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid render settings");
    rmd_context *ctx = b->ctx;
    RMD_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const uint64_t firstSample = s->first_sample >= 0 ? (uint64_t)s->first_sample : b->nextSample;
    if (firstSample + s->spp > BATCH_SAMPLE_MASK)
        return fail(RMD_ERROR_INVALID_ARGUMENT, "batch sample index beyond 2^24");
    const uint64_t numPaths = (uint64_t)s->spp * b->totalPixels;
    if (s->film_fp64 && !b->film64.ptr) {
        RMD_CUDA(b->film64.alloc((size_t)b->totalPixels * 3 * sizeof(double)));
        RMD_CUDA(cudaMemsetAsync(b->film64.ptr, 0, b->film64.bytes, st));
    }
    std::memset(&b->stats, 0, sizeof(b->stats));
    b->stats.pool_size = b->capacity;
    if (numPaths == 0) return RMD_OK;
    FrameParams fp{};
    fp.width = 0;  // per view (BatchView)
    fp.height = 0;
    fp.numPixels = b->totalPixels;
    fp.maxDepth = s->max_depth;
    fp.samplingMode = s->sampling_mode;
    fp.rngMode = s->rng;
    fp.seed = s->seed;
    fp.filmFp64 = s->film_fp64 ? 1 : 0;
    fp.film = b->film.as<float4>();
    fp.film64 = b->film64.as<double>();
    // guiding (all views of one scene)
    GuideState &guide = b->guide;
    if (b->shadeGuided != guideActive(guide)) {  // the shading kernel with or without the guide's code
        rmd_status vs = batchEnsureVariants(b, {b->shadeMinBlocks}, guideActive(guide));
        if (vs != RMD_OK) return vs;
        batchSelectShade(b, b->shadeMinBlocks, guideActive(guide));
    }
    GuideNetView net{};
    if (guide.settings.sampling || guide.settings.training) {
        rmd_status gs = guideBuffers(guide, b->capacity, b->counters.as<Counters>());
        if (gs != RMD_OK) return gs;
        net = guide.net.view(guide.frameMin, guide.frameInvExtent);
        fp.guideDepth = guide.settings.sampling ? guide.settings.guided_depth : 0u;
        fp.guideSceneMin = guide.frameMin;
        fp.guideSceneInvExtent = guide.frameInvExtent;
    }
    const PathPool pool = batchPoolView(b);
    Counters *cnt = b->counters.as<Counters>();
    ShadeParams sp;
    sp.ctx = b->scenes[0]->dctx;  // per path from its view
    sp.pool = pool;
    sp.fp = fp;
    sp.counters = cnt;
    const uint64_t firstPath = firstSample * b->totalPixels;
    const uint64_t maxIters = ((numPaths + b->capacity - 1) / b->capacity + 1) * ((uint64_t)s->max_depth + 1) + 8;
    if (maxIters > 0xffffffffull) return fail(RMD_ERROR_INVALID_ARGUMENT, "render too long for one call");

    RMD_CUDA(cudaEventRecord(b->ev[0], st));
    RMD_CUDA(rmdLaunchFrameInit(pool, cnt, firstPath, firstPath + numPaths, st));
    uint64_t iterations = 0, trainSteps = 0;
    // training steps run between counter checks, so a training batch uses the host-driven loop
    if (b->useGraph && !guide.settings.training) {
        // the graph depends on everything but the sample range (frame init sets that)
        const std::vector<uint64_t> key = {s->max_depth, s->sampling_mode, s->rng, s->seed, (uint64_t)fp.filmFp64,
                                           maxIters, (uint64_t)b->capacity, (uint64_t)b->shadeMinBlocks,
                                           (uint64_t)b->traceBlocksPerSm, (uint64_t)fp.guideDepth};
        if (!b->graphExec || b->graphKey != key) {
            if (b->graphExec) cudaGraphExecDestroy(b->graphExec);
            if (b->graph) cudaGraphDestroy(b->graph);
            b->graphExec = nullptr;
            b->graph = nullptr;
            RMD_CUDA(cudaGraphCreate(&b->graph, 0));
            cudaGraphConditionalHandle handle;
            RMD_CUDA(cudaGraphConditionalHandleCreate(&handle, b->graph, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t loop;
            RMD_CUDA(cudaGraphAddNode(&loop, b->graph, nullptr, 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            // the body: two iterations (both parities) and the condition kernel
            RMD_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            rmd_status e = batchEnqueueIterations(b, pool, fp, sp, net, 2, st);
            cudaError_t ce = e == RMD_OK ? rmdLaunchLoopCondition(cnt, handle, 2, (uint32_t)maxIters, st) : cudaSuccess;
            cudaGraph_t captured = nullptr;
            cudaError_t endErr = cudaStreamEndCapture(st, &captured);
            if (e != RMD_OK) return e;
            RMD_CUDA(ce);
            RMD_CUDA(endErr);
            RMD_CUDA(cudaGraphInstantiate(&b->graphExec, b->graph, 0));
            b->graphKey = key;
        }
        RMD_CUDA(cudaGraphLaunch(b->graphExec, st));
        RMD_CUDA(cudaMemcpyAsync(b->hostCounters, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        RMD_CUDA(cudaStreamSynchronize(st));
        const Counters &h = *b->hostCounters;
        iterations = h.loopIterations;
        if (h.errors) {
            b->stats.errors = h.errors;
            return fail(h.errors & ERR_LOOP_BOUND ? RMD_ERROR_WATCHDOG : RMD_ERROR_QUEUE_OVERFLOW,
                        "device error flags " + std::to_string(h.errors));
        }
    } else {
        bool done = false;
        while (!done) {
            rmd_status e = batchEnqueueIterations(b, pool, fp, sp, net, 4, st);
            if (e != RMD_OK) return e;
            iterations += 4;
            RMD_CUDA(cudaMemcpyAsync(b->hostCounters, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
            RMD_CUDA(cudaStreamSynchronize(st));
            const Counters &h = *b->hostCounters;
            if (h.errors) {
                b->stats.errors = h.errors;
                return fail(RMD_ERROR_QUEUE_OVERFLOW, "device error flags " + std::to_string(h.errors));
            }
            if ((e = guideTrainStep(guide, h, cnt, net, b->ctx->smCount, st, trainSteps)) != RMD_OK) return e;
            if (h.pathsDone >= numPaths) done = true;
            else if (iterations > maxIters) return fail(RMD_ERROR_WATCHDOG, "render did not drain in the iteration bound");
        }
    }
    RMD_CUDA(cudaEventRecord(b->ev[1], st));
    RMD_CUDA(cudaEventSynchronize(b->ev[1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
    const Counters &h = *b->hostCounters;
    b->stats.paths = h.pathsDone;
    b->stats.segments = h.segments;
    b->stats.rays = h.rays;
    b->stats.shadow_rays = h.shadowRays;
    b->stats.invalid_samples = h.invalid;
    b->stats.iterations = iterations;
    b->stats.ms_total = ms;
    b->samples += s->spp;
    b->nextSample = std::max<uint64_t>(b->nextSample, firstSample + s->spp);
    if (trainSteps) return guideReadLoss(guide);
    return RMD_OK;
}

rmd_status rmd_batch_set_guide(rmd_batch *b, const rmd_guide_settings *settings) {
    if (!b || !settings) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    const int scene = b->views[0].scene;
    for (const auto &v : b->views)
        if (v.scene != scene)
            return fail(RMD_ERROR_INVALID_ARGUMENT, "guiding needs every view of the batch on one scene");
    RMD_CUDA(cudaSetDevice(b->ctx->device));
    rmd_status st = setGuide(b->guide, settings, b->ctx->stream, b->counters.as<Counters>());
    if (st != RMD_OK) return st;
    b->guideScene = scene;
    guideFrame(b->scenes[scene].get(), b->guide.frameMin, b->guide.frameInvExtent);
    if (b->graphExec) {  // the graph gains or loses the inference launches
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    b->graphKey.clear();
    return guideBuffers(b->guide, b->capacity, b->counters.as<Counters>());
}

rmd_status rmd_batch_guide_stats(const rmd_batch *b, rmd_guide_stats *out) {
    if (!b || !out) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    *out = b->guide.stats;
    return RMD_OK;
}

rmd_status rmd_batch_film_read(rmd_batch *b, int32_t view, float *rgb, int32_t normalize, uint32_t tonemapping,
                               float exposure) {
    if (!b || !rgb || view < 0 || view >= (int32_t)b->views.size()) return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid argument");
    if (tonemapping > 2) return fail(RMD_ERROR_INVALID_ARGUMENT, "tonemapping out of range");
    cudaStream_t st = b->ctx->stream;
    const uint32_t n = b->views[view].width * b->views[view].height, off = b->offsets[view];
    float ex = 1.0f, div = 1.0f;
    uint32_t tm = 0;
    if (normalize) {
        ex = exposure;
        div = (float)std::max<uint64_t>(1, b->samples);
        tm = tonemapping;
    }
    RMD_CUDA(rmdLaunchFilmResolve(b->film.as<float4>() + off, b->film64.ptr ? b->film64.as<double>() + 3 * (size_t)off : nullptr,
                                  0, b->resolve.as<float>(), n, ex, div, tm, 3, st));
    RMD_CUDA(cudaMemcpyAsync(rgb, b->resolve.ptr, (size_t)n * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    RMD_CUDA(cudaStreamSynchronize(st));
    return RMD_OK;
}

rmd_status rmd_batch_film_save_exr(rmd_batch *b, int32_t view, const char *path, float normalized_by,
                                   uint32_t compression) {
    if (!b || view < 0 || view >= (int32_t)b->views.size()) return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid argument");
    const uint32_t w = b->views[view].width, h = b->views[view].height;
    std::vector<float> rgb((size_t)w * h * 3);
    const rmd_status st = rmd_batch_film_read(b, view, rgb.data(), 0, 0, 1.0f);
    if (st != RMD_OK) return st;
    return saveExr(path, rgb, w, h, normalized_by, b->samples, compression);
}

rmd_status rmd_batch_film_read_f64(rmd_batch *b, int32_t view, double *rgb) {
    if (!b || !rgb || view < 0 || view >= (int32_t)b->views.size()) return fail(RMD_ERROR_INVALID_ARGUMENT, "invalid argument");
    if (!b->film64.ptr) return fail(RMD_ERROR_INVALID_ARGUMENT, "no double-precision film (render with film_fp64)");
    cudaStream_t st = b->ctx->stream;
    const size_t n = (size_t)b->views[view].width * b->views[view].height;
    RMD_CUDA(cudaMemcpyAsync(rgb, b->film64.as<double>() + 3 * (size_t)b->offsets[view], n * 3 * sizeof(double),
                             cudaMemcpyDeviceToHost, st));
    RMD_CUDA(cudaStreamSynchronize(st));
    return RMD_OK;
}

rmd_status rmd_batch_stats(const rmd_batch *b, rmd_stats *out) {
    if (!b || !out) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    *out = b->stats;
    return RMD_OK;
}

rmd_status rmd_batch_autotune(rmd_batch *b, const rmd_render_settings *settings, rmd_tune_result *out) {
    if (!b || !settings) return fail(RMD_ERROR_INVALID_ARGUMENT, "NULL argument");
    const std::vector<int> mbs = {1, 3, 4, 5, 6, 8, 10, 12, 16};
    const bool guided = guideActive(b->guide);
    rmd_status st = batchEnsureVariants(b, mbs, guided);
    if (st != RMD_OK) return st;
    const uint32_t cap0 = b->capacity;
    std::vector<uint32_t> caps;  // half, twice and four times the current pool
    const uint64_t candidates[3] = {(uint64_t)cap0 / 2, 2 * (uint64_t)cap0, 4 * (uint64_t)cap0};
    for (uint64_t cap : candidates)
        if (cap >= (1u << 16) && cap <= BATCH_MAX_CAPACITY) caps.push_back((uint32_t)cap);
    rmd_render_settings cal = *settings;  // several generations of the largest pool tried
    cal.film_fp64 = 0;
    const uint64_t maxCap = std::max<uint64_t>(cap0, caps.empty() ? 0 : *std::max_element(caps.begin(), caps.end()));
    cal.spp = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(settings->spp, (4ull * maxCap + b->totalPixels - 1) / b->totalPixels));
    cal.first_sample = BATCH_SAMPLE_MASK - 2 * cal.spp;  // a sample range the caller does not use
    auto trial = [&](double &ms) -> rmd_status {
        double best = 1e30;
        for (int rep = 0; rep < 2; rep++) {
            rmd_status e = rmd_batch_render(b, &cal);
            if (e != RMD_OK) return e;
            best = std::min(best, b->stats.ms_total);
        }
        ms = best;
        return RMD_OK;
    };
    rmd_tune_result res{};
    double base = 0;
    if ((st = trial(base)) != RMD_OK) return st;
    res.ms_default = base;
    int bestMb = b->shadeMinBlocks;
    double bestMs = base;
    for (int mb : mbs) {
        if (mb == b->shadeMinBlocks) continue;
        batchSelectShade(b, mb, guided);
        double ms;
        if ((st = trial(ms)) != RMD_OK) return st;
        if (ms < bestMs) {
            bestMs = ms;
            bestMb = mb;
        }
    }
    batchSelectShade(b, bestMb, guided);
    int bestTb = b->traceBlocksPerSm;
    for (int tb : {4, 8, 12, 16}) {
        b->traceBlocksPerSm = tb;
        double ms;
        if ((st = trial(ms)) != RMD_OK) return st;
        if (ms < bestMs) {
            bestMs = ms;
            bestTb = tb;
        }
    }
    b->traceBlocksPerSm = bestTb;
    uint32_t bestCap = cap0;
    for (uint32_t cap : caps) {
        size_t freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess || pathPoolBytes(cap) > freeB / 2) continue;
        b->capacity = cap;
        if ((st = batchAllocatePool(b)) != RMD_OK) return st;
        double ms;
        if ((st = trial(ms)) != RMD_OK) return st;
        if (ms < bestMs) {
            bestMs = ms;
            bestCap = cap;
        }
    }
    if (b->capacity != bestCap) {
        b->capacity = bestCap;
        if ((st = batchAllocatePool(b)) != RMD_OK) return st;
    }
    res.shade_min_blocks = (uint32_t)b->shadeMinBlocks;
    res.trace_blocks_per_sm = (uint32_t)b->traceBlocksPerSm;
    res.pool_size = b->capacity;
    res.ms_best = bestMs;
    res.calibration_spp = cal.spp;
    if (out) *out = res;
    return rmd_batch_reset(b);
}

}  // extern "C"
