// rmd_render_noalloc: rendering without any device or host allocation.
//
// Some callers cannot allocate GPU memory when they want a frame: a plug-in
// hosted by an application that owns every device allocation and forbids new
// ones, a real-time loop that must not pay allocation latency or fragment
// the heap mid-session, or a process held to a fixed memory budget.  For
// them this entry point runs the same wavefront kernels as rmd_render, but
// the path pool, queues and counters live in one file-scope device array of
// fixed size instead of memory owned by an rmd_renderer; the caller passes
// the scene (created earlier) and its own device film.
//
// The array is defined in this file.  Host code cannot use the array's name
// as a device address: rmd_context_create looks the address up for its device
// with cudaGetSymbolAddress (noallocSetup below) and this entry point hands it
// to the kernels.  The lookup is what makes the CUDA runtime load this file's
// module, and with it reserve the array on that GPU, so with lazy module
// loading (the default since CUDA 12.2) the reservation happens when the
// context is created, not in the middle of a render.  Every context created
// refreshes the address, so contexts made after a device reset hand out the
// array's new address.  All calls share the array, so two calls whose work
// overlaps on the GPU (different streams, other threads) corrupt each other.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <algorithm>

#include "../../include/raymond.h"
#include "kernels.h"
#include "scene_view.h"

namespace {

using namespace rmd;

constexpr uint32_t kMaxPaths = RMD_NOALLOC_MAX_PATHS;
// counters (padded to 256 B), then the path pool of the largest size
constexpr size_t kCountersBytes = (sizeof(Counters) + 255) & ~size_t(255);
constexpr size_t kScratchBytes = kCountersBytes + pathPoolBytes(kMaxPaths);

static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

std::mutex g_mutex;
void *g_scratch[64] = {};  // device address of g_noallocScratch per device, set by noallocSetup

rmd_status cudaFail(cudaError_t e, const char *what) {
    std::string msg = std::string("rmd_render_noalloc: ") + what + ": " + cudaGetErrorString(e);
    return rmdhost::setLastError(RMD_ERROR_CUDA, msg.c_str());
}

}  // namespace

namespace rmdhost {

// Called by rmd_context_create with `device` current.
rmd_status noallocSetup(int device) {
    if (device < 0 || device >= 64) return RMD_OK;  // rmd_render_noalloc rejects such devices
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noallocScratch);
    if (e != cudaSuccess) return cudaFail(e, "cudaGetSymbolAddress");
    std::lock_guard<std::mutex> lock(g_mutex);
    g_scratch[device] = ptr;
    return RMD_OK;
}

}  // namespace rmdhost

extern "C" rmd_status rmd_render_noalloc(rmd_scene *scene, const rmd_camera *camera, uint32_t width, uint32_t height,
                                         const rmd_render_settings *s, float *film, uint32_t pool_size) {
    rmdhost::SceneView v;
    if (!rmdhost::sceneView(scene, v) || !camera || !s || !film)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT, "rmd_render_noalloc: NULL argument");
    if (width == 0 || height == 0 || width > 65535 || height > 65535)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT, "rmd_render_noalloc: width/height must be 1..65535");
    if (pool_size > kMaxPaths)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT,
                                     "rmd_render_noalloc: pool_size exceeds RMD_NOALLOC_MAX_PATHS (32768)");
    if (s->max_depth == 0 || s->max_depth > 65535 || s->sampling_mode > 2 || s->rng > 1 || s->film_fp64)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT,
                                     "rmd_render_noalloc: invalid settings (film_fp64 is not supported here)");
    if (s->first_sample < 0 || (uint64_t)s->first_sample + s->spp > 0xffffffffull)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT, "rmd_render_noalloc: first_sample must be >= 0");
    if (v.device < 0 || v.device >= 64)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT, "rmd_render_noalloc: device index >= 64");
    cudaError_t e = cudaSetDevice(v.device);
    if (e != cudaSuccess) return cudaFail(e, "cudaSetDevice");

    void *base;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        base = g_scratch[v.device];  // set when the scene's context was created
    }
    if (!base) return rmdhost::setLastError(RMD_ERROR_CUDA, "rmd_render_noalloc: scratch array not set up");
    const uint32_t P = pool_size ? pool_size : kMaxPaths;
    Counters *cnt = static_cast<Counters *>(base);
    const PathPool pool = carvePathPool(static_cast<unsigned char *>(base) + kCountersBytes, P);

    Context ctx = v.ctx;
    for (int k = 0; k < 4; k++)
        ctx.cameraTransform[k] = make_float4(camera->transform[4 * k], camera->transform[4 * k + 1],
                                             camera->transform[4 * k + 2], camera->transform[4 * k + 3]);
    ctx.nearClip = camera->near_clip;
    ctx.farClip = camera->far_clip;
    ctx.focalLength = camera->focal_length;
    ctx.shift = make_float2(camera->shift[0], camera->shift[1]);

    const uint64_t numPixels = (uint64_t)width * height;
    const uint64_t numPaths = (uint64_t)s->spp * numPixels;
    if (numPaths == 0) return RMD_OK;
    FrameParams fp{};
    fp.width = width;
    fp.height = height;
    fp.numPixels = (uint32_t)numPixels;
    fp.maxDepth = s->max_depth;
    fp.samplingMode = s->sampling_mode;
    fp.rngMode = s->rng;
    fp.seed = s->seed;
    fp.filmFp64 = 0;
    fp.film = reinterpret_cast<float4 *>(film);
    fp.film64 = nullptr;
    const uint64_t firstPath = (uint64_t)s->first_sample * numPixels;
    ShadeParams sp;
    sp.ctx = ctx;
    sp.pool = pool;
    sp.fp = fp;
    sp.counters = cnt;
    void *shadeArgs[] = {&sp};
    const cudaStream_t st = v.stream;
    const int tb = v.smCount * 8;
    const int rb = (int)std::min<uint32_t>((P + 255) / 256, (uint32_t)v.smCount * 8);

    if ((e = rmdLaunchFrameInit(pool, cnt, firstPath, firstPath + numPaths, st)) != cudaSuccess)
        return cudaFail(e, "frame init");
    const uint64_t maxIters = ((numPaths + P - 1) / P + 1) * ((uint64_t)s->max_depth + 1) + 8;
    uint64_t it = 0;
    uint32_t cur = 0;
    Counters h;
    while (true) {
        for (int k = 0; k < 4; k++, it++) {
            if ((e = rmdLaunchFilmRegen(ctx, pool, fp, cnt, cur, rb, st)) != cudaSuccess) return cudaFail(e, "film");
            if ((e = rmdLaunchTraceClosest(v.nodes, v.tris, pool, cnt, cur, tb, st)) != cudaSuccess)
                return cudaFail(e, "trace");
            sp.cur = cur;
            if ((e = cudaLaunchKernel((const void *)v.shade, dim3(v.shadeBlocks), dim3(128), shadeArgs, 0, st)) !=
                cudaSuccess)
                return cudaFail(e, "shade");
            if ((e = rmdLaunchTraceShadow(v.nodes, v.tris, pool, cnt, cur, tb, st)) != cudaSuccess)
                return cudaFail(e, "shadow");
            cur ^= 1u;
        }
        // pageable stack destination: no pinned staging buffer is allocated
        if ((e = cudaMemcpyAsync(&h, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return cudaFail(e, "counters");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cudaFail(e, "synchronize");
        if (h.errors) return rmdhost::setLastError(RMD_ERROR_QUEUE_OVERFLOW, "rmd_render_noalloc: device error flags");
        if (h.pathsDone >= numPaths) break;
        if (it > maxIters)
            return rmdhost::setLastError(RMD_ERROR_WATCHDOG, "rmd_render_noalloc: render did not drain");
    }
    return RMD_OK;
}
