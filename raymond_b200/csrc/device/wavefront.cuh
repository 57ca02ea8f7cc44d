// Path state, queues and counters of the persistent wavefront, shared by the
// static kernels (film / regeneration, traversal) and the NVRTC shading
// module.  One iteration is
//     film+regen -> closest-hit trace -> shade (NEE, BSDF sample) -> shadow trace
// and replaces one depth step of Renderer.execute (Renderer.swift:545-673)
// for every path in flight; finished paths are replaced by new camera
// samples, so the pool stays full until the last samples drain.
//
// Path state is kept in queue order, not in fixed slots: iteration i (parity
// p = i & 1) reads the active paths from S[p] at positions 0..n-1, and the
// shading pass writes every path it continues to the next free position of
// S[p ^ 1] (one atomic per warp), so each kernel reads and writes its path
// records with coalesced 16-byte accesses.  Paths that end go to the finish
// list with their radiance; the next film pass adds them to the film.
#pragma once
#include "guide.cuh"
#include "scene.cuh"

namespace rmd {

constexpr float SHADOW_EPS = 0.001f;  // device/constants.hpp:3

// error flags
constexpr uint32_t ERR_QUEUE_OVERFLOW = 1u;
constexpr uint32_t ERR_STACK_OVERFLOW = 2u;
constexpr uint32_t ERR_LOOP_BOUND = 4u;  // a device-driven render loop reached its iteration bound
constexpr uint32_t ERR_GUIDE_TIMEOUT = 8u;  // a guide inference CTA's tensor-core wait expired

// target of a shadow ray: position of its path in S[p ^ 1], or in the finish
// list when this bit is set
constexpr uint32_t SHADOW_TO_FINISHED = 0x80000000u;
// set beside it when the ray's light also counts towards the radiance before
// the path's guide training record (the light sample of the recorded vertex)
constexpr uint32_t SHADOW_TO_RECORD = 0x40000000u;
constexpr uint32_t SHADOW_TARGET_MASK = 0x3fffffffu;

// Queue bookkeeping without same-address atomics on the regeneration path:
// S[p] holds nQ[p] paths continued by the previous iteration followed by the
// newPaths() camera samples the film kernel of this iteration appends; the
// shading pass of parity p appends continued paths to S[p ^ 1] (nQ[p ^ 1])
// and finished ones to the finish list (nF[p]).
//
// Every counter that warps of many SMs update with atomics sits in its own
// 256-byte block, so the counters do not queue behind each other in one L2
// slice.
struct Counters {
    uint32_t nQ[2];       // continued paths at the head of each S[p]
    uint32_t padQ[62];
    uint32_t nF[2];       // finished paths written by the shading pass of parity p
    uint32_t padF[62];
    uint32_t nShadow;     // shadow rays of this iteration
    uint32_t padS[63];
    uint32_t traceWork;   // persistent closest-hit work counter
    uint32_t padT[63];
    uint32_t shadowWork;  // persistent any-hit work counter
    uint32_t padW[63];
    uint32_t nHit;        // active paths whose closest-hit ray hit a surface (front of `order`)
    uint32_t padH[63];
    uint32_t nMiss;       // ... and that missed (back of `order`)
    uint32_t padM[63];
    uint32_t numRecords;  // guide training records with a nonzero target written so far (a ring index)
    uint32_t numSamples;  // guide training samples completed since the last training step
    uint32_t padR[62];
    uint32_t errors;
    uint32_t capacity;    // paths in flight at most (size of each S[p])
    uint32_t loopIterations;  // device-driven render loop: wavefront iterations so far
    uint32_t padL;
    unsigned long long numPaths;    // paths of this render
    unsigned long long nextPath;    // next path id handed out by the film kernel
    unsigned long long endPath;     // one past the last path id of this render
    unsigned long long pathsDone;   // paths whose radiance reached the film
    unsigned long long segments;    // closest-hit rays shaded
    unsigned long long shadowRays;  // shadow rays traced
    unsigned long long rays;        // closest-hit rays traced (hits and misses)
    unsigned long long invalid;     // light and BSDF samples dropped for a non-finite weight
};


// camera samples the film kernel of this iteration appends to S[p]
__device__ __forceinline__ uint32_t newPaths(const Counters *c, uint32_t p) {
    const unsigned long long next = c->nextPath, end = c->endPath;
    if (next >= end) return 0u;
    const unsigned long long left = end - next;
    const uint32_t room = c->capacity - c->nQ[p];
    return left < (unsigned long long)room ? (uint32_t)left : room;
}
// number of active paths in S[p] after the film kernel of this iteration
__device__ __forceinline__ uint32_t activeCount(const Counters *c, uint32_t p) { return c->nQ[p] + newPaths(c, p); }

// Position in S[p] of the i-th path to shade: the closest-hit pass lists hits
// first and misses last, so shading warps see one kind or the other.
__device__ __forceinline__ uint32_t shadingOrder(const uint32_t *order, const Counters *c, uint32_t i) {
    const uint32_t nHit = c->nHit;
    return i < nHit ? order[i] : order[c->capacity - 1u - (i - nHit)];
}

// One view of a batch (many scenes and views traced by one wavefront): its
// scene's device context with the view's camera, its scene's BVH, and its
// place in the batch's film.  Paths of a batch carry the view in the top 8
// bits of their sample index and their film pixel (batch-global) in id.x.
struct BatchView {
    Context ctx;
    const void *nodes;   // the scene's wide BVH nodes (WideNode)
    const float4 *tris;  // the scene's BVH triangles
    uint32_t width, height, numPixels, pixelOffset;
};
// a batch's shadow-ray target carries the ray's view in bits 22-29 (batch
// pools hold at most 2^22 paths)
constexpr uint32_t BATCH_TARGET_BITS = 22;
constexpr uint32_t BATCH_TARGET_MASK = (1u << BATCH_TARGET_BITS) - 1u;
constexpr uint32_t BATCH_MAX_CAPACITY = 1u << BATCH_TARGET_BITS;
constexpr uint32_t BATCH_SAMPLE_BITS = 24;
constexpr uint32_t BATCH_SAMPLE_MASK = (1u << BATCH_SAMPLE_BITS) - 1u;

// One queue-ordered copy of the path state (structure of arrays).
struct PathState {
    float4 *rayO;  // origin.xyz, tmin
    float4 *rayD;  // direction.xyz, tmax
    float4 *tp;    // throughput.xyz, bsdf pdf of the ray
    float4 *L;     // radiance gathered so far .xyz; .w = depth (bits 0-15) | ray flags (bits 16-23) |
                   // guide-record vertices seen (bits 24-31, training only)
    uint4 *id;     // pixel (y * width + x), sample index, packed PrngState
    float4 *rec;   // guide training: the pending record of one of the path's vertices, 4 per path
                   // (features 0-3 | features 4-6, bsdf pdf | direction, survival (0: none) |
                   //  radiance before, 1 / mean throughput at the vertex); nullptr when not training
};

struct PathPool {
    PathState s[2];
    float4 *hit;        // per active path of this iteration: t (<= 0: miss), b0, b1, primitive (bits)
    uint32_t *hitInst;  // instance index
    uint32_t *order;    // shading order: positions of hits from the front, of misses from the back
    float4 *fin;        // finished paths: radiance.xyz, pixel (bits)
    float4 *shO;        // shadow: origin.xyz, tmax
    float4 *shD;        // shadow: direction.xyz, target (bits; SHADOW_TO_FINISHED, SHADOW_TO_RECORD)
    float4 *shW;        // shadow: weight.xyz; w: 1 / mean throughput of its vertex for a light record (else 0)
    // guide training (nullptr when not training)
    float4 *finRec;       // the pending records of finished paths (4 per entry)
    float4 *shRec;        // per shadow ray: its vertex's features 0-3 | features 4-6, BSDF pdf of the ray
    GuideRecord *records; // ring of the latest records with a nonzero target (Counters::numRecords)
    uint32_t recordCapacity;  // a power of two
    GuideMixture *guide;  // guiding: the mixture of each hit of this iteration (by shading-order position), or nullptr
    uint4 *guideFeat;     // guiding: each hit's input features (7 x unorm16) and depth, by shading-order position
    float3 guideMin, guideInvExtent;  // frame of the position features
    const BatchView *views;           // batch: the views (nullptr: one scene, one view)
    uint32_t numViews;
    uint32_t capacity;
};

#ifndef __CUDACC_RTC__
// Bytes of device memory a pool of `capacity` paths takes (each array padded
// to 256 bytes), and the pool carved out of such a block.
constexpr size_t pathPoolBytes(uint32_t capacity) {
    const size_t P = capacity, pad = 255;
    const size_t per16 = (P * 16 + pad) & ~pad, per4 = (P * 4 + pad) & ~pad;
    return 2 * 5 * per16 + 5 * per16 + 2 * per4;
}
inline PathPool carvePathPool(void *base, uint32_t capacity) {
    unsigned char *p = static_cast<unsigned char *>(base);
    auto take = [&](size_t elemBytes) {
        void *r = p;
        p += ((size_t)capacity * elemBytes + 255) & ~size_t(255);
        return r;
    };
    PathPool pool;
    for (int k = 0; k < 2; k++) {
        pool.s[k].rayO = static_cast<float4 *>(take(16));
        pool.s[k].rayD = static_cast<float4 *>(take(16));
        pool.s[k].tp = static_cast<float4 *>(take(16));
        pool.s[k].L = static_cast<float4 *>(take(16));
        pool.s[k].id = static_cast<uint4 *>(take(16));
        pool.s[k].rec = nullptr;  // guiding buffers are allocated by the renderer when enabled
    }
    pool.hit = static_cast<float4 *>(take(16));
    pool.fin = static_cast<float4 *>(take(16));
    pool.shO = static_cast<float4 *>(take(16));
    pool.shD = static_cast<float4 *>(take(16));
    pool.shW = static_cast<float4 *>(take(16));
    pool.hitInst = static_cast<uint32_t *>(take(4));
    pool.order = static_cast<uint32_t *>(take(4));
    pool.finRec = nullptr;
    pool.shRec = nullptr;
    pool.records = nullptr;
    pool.recordCapacity = 0;
    pool.guide = nullptr;
    pool.guideFeat = nullptr;
    pool.guideMin = make_float3(0.0f, 0.0f, 0.0f);
    pool.guideInvExtent = make_float3(1.0f, 1.0f, 1.0f);
    pool.views = nullptr;
    pool.numViews = 0;
    pool.capacity = capacity;
    return pool;
}
#endif

struct FrameParams {
    uint32_t width, height, numPixels;
    uint32_t maxDepth, samplingMode, rngMode;
    uint64_t seed;
    int filmFp64;
    float4 *film;      // rgb sums (w unused)
    double *film64;    // rgb sums, 3 per pixel
    uint32_t guideDepth;                        // guided sampling at path depths below this (0: none)
    float3 guideSceneMin, guideSceneInvExtent;  // frame of the guide's position encoding
};

// kernel parameters of the shading megakernel (device/integrator.cuh)
struct ShadeParams {
    Context ctx;
    PathPool pool;
    FrameParams fp;
    Counters *counters;
    uint32_t cur;
};

// Appends the calling lane to a queue with one atomic per warp
// (ballot / popc / shfl), returning its position.
__device__ __forceinline__ uint32_t warpAppend(uint32_t *counter) {
    const unsigned mask = __activemask();
    const int leader = __ffs(mask) - 1;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}
// Sums v over the block and adds it to *counter with one atomic (all threads must call).
__device__ __forceinline__ void blockAdd64(unsigned long long *counter, uint32_t v) {
    __shared__ uint32_t partial[32];
    const uint32_t w = __reduce_add_sync(0xffffffffu, v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) partial[warp] = w;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        const uint32_t x = lane < nw ? partial[lane] : 0u;
        const uint32_t t = __reduce_add_sync(0xffffffffu, x);
        if (lane == 0 && t) atomicAdd(counter, (unsigned long long)t);
    }
    __syncthreads();
}
__device__ __forceinline__ void warpAdd64(unsigned long long *counter, uint32_t v) {
    const unsigned mask = __activemask();
    const int leader = __ffs(mask) - 1;
    const uint32_t total = __reduce_add_sync(mask, v);
    if ((int)(threadIdx.x & 31) == leader && total) atomicAdd(counter, (unsigned long long)total);
}

// generate.metal:88-91 with 8x8 threadgroups: block-linear ray index and its inverse
RMD_HD uint32_t blockLinearIndex(uint32_t x, uint32_t y, uint32_t W, uint32_t H) {
    const uint32_t gx = x / 8, gy = y / 8, tx = x % 8, ty = y % 8;
    const uint32_t awx = min(8u, W - gx * 8), awy = min(8u, H - gy * 8);
    return tx + ty * awx + gx * 8 * awy + gy * 8 * W;
}
RMD_HD void blockLinearToPixel(uint32_t r, uint32_t W, uint32_t H, uint32_t &x, uint32_t &y) {
    const uint32_t gy = r / (8 * W);
    uint32_t rr = r - gy * 8 * W;
    const uint32_t awy = min(8u, H - gy * 8);
    const uint32_t gx = rr / (8 * awy);
    rr -= gx * 8 * awy;
    const uint32_t awx = min(8u, W - gx * 8);
    const uint32_t ty = rr / awx, tx = rr - ty * awx;
    x = gx * 8 + tx;
    y = gy * 8 + ty;
}

// batch: the view whose pixel range holds batch pixel r (views sorted by pixelOffset)
__device__ __forceinline__ uint32_t batchViewOf(const BatchView *views, uint32_t numViews, uint32_t r) {
    uint32_t lo = 0, hi = numViews;  // views[lo].pixelOffset <= r < views[hi].pixelOffset
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (views[mid].pixelOffset <= r) lo = mid;
        else hi = mid;
    }
    return lo;
}

RMD_HD uint64_t pathSequence(uint32_t sample, uint32_t pixel, uint32_t numPixels) {
    return (uint64_t)sample * (uint64_t)numPixels + (uint64_t)pixel;
}

// generate.metal:72-121 (pinhole branch): a camera ray for (x, y, sample)
RMD_HD void cameraRay(const Context &ctx, const FrameParams &fp, uint32_t x, uint32_t y, uint32_t sample,
                      PrngState &prng, float3 &org, float3 &dir) {
    const uint32_t W = fp.width, H = fp.height;
    if (fp.rngMode == RNG_TEA) {
        prng = PrngState::tea(sample + 1u, blockLinearIndex(x, y, W, H));
    } else {
        prng = PrngState::pcg(fp.seed, pathSequence(sample, y * W + x, fp.numPixels));
    }
    const float2 jittered = make_float2((float)x, (float)y) + prng.sample2d();
    const float2 uv = make_float2(1.0f, -1.0f) * ((jittered / make_float2((float)W, (float)H) + ctx.shift) * 2.0f - 1.0f);
    const float aspect = (float)H / (float)W;
    org = xyz(ctx.cameraTransform[3]);  // (T * float4(0, 0, 0, 1)).xyz
    const float4 dd = ctx.cameraTransform[0] * uv.x + ctx.cameraTransform[1] * (uv.y * aspect) +
                      ctx.cameraTransform[2] * (-ctx.focalLength) + ctx.cameraTransform[3] * 0.0f;
    dir = normalize(xyz(dd));
}

}  // namespace rmd
