// Static sm_100a kernels of the wavefront: closest-hit and shadow traversal,
// film accumulation + path regeneration, frame set-up, the environment-map
// pyramid reductions, film read-out, and small test hooks.  The shading
// megakernel lives in the NVRTC module (device/integrator.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "device/traverse.cuh"
#include "device/wavefront.cuh"
#include "kernels.h"
#include "sky.h"

namespace rmd {

// ------------------------------------------------------------- frame set-up
__global__ void k_frame_init(Counters *cnt, uint32_t capacity, uint64_t firstPath, uint64_t endPath) {
    cnt->nQ[0] = cnt->nQ[1] = 0;
    cnt->nF[0] = cnt->nF[1] = 0;
    cnt->nShadow = 0;
    cnt->traceWork = cnt->shadowWork = 0;
    cnt->errors = 0;
    cnt->capacity = capacity;
    cnt->nHit = cnt->nMiss = 0;  // numRecords / numSamples persist across frames (the renderer resets them)
    cnt->nextPath = firstPath;
    cnt->endPath = endPath;
    cnt->numPaths = endPath - firstPath;
    cnt->loopIterations = 0;
    cnt->pathsDone = 0;
    cnt->segments = 0;
    cnt->shadowRays = 0;
    cnt->rays = 0;
    cnt->invalid = 0;
}

// ------------------------------------------------------------- film + regeneration
// Adds the radiance of every path finished by the previous iteration to the
// film (the film writes of intersection.metal:84-87,111-116,174-178 and
// shadow.metal:24-27, gathered per path) and appends the next camera samples
// (generate.metal:72-121) to S[p]: sample j takes path id nextPath + j and
// position nQ[p] + j, so no counter is contended.  BATCH: path ids run over
// the concatenated pixels of all views (fp.numPixels in total); each sample
// takes its view's camera, size and PCG stream (the view's own pixel index),
// so a view renders as it would alone.
template <bool BATCH>
__global__ void __launch_bounds__(256) k_film_regen(Context ctx, PathPool pool, FrameParams fp, Counters *cnt,
                                                    uint32_t p) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // counters of later stages of this iteration
        cnt->nQ[p ^ 1u] = 0;
        cnt->nF[p] = 0;
        cnt->nShadow = 0;
        cnt->traceWork = 0;
        cnt->shadowWork = 0;
        cnt->nHit = 0;
        cnt->nMiss = 0;
    }
    const uint32_t nFin = cnt->nF[p ^ 1u];
    const uint32_t base = cnt->nQ[p];
    const uint32_t nNew = newPaths(cnt, p);
    const unsigned long long first = cnt->nextPath;
    const PathState S = pool.s[p];
    const uint32_t n = max(nFin, nNew);
    uint32_t finished = 0, samples = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (j < nFin) {
            const float4 f = __ldcs(&pool.fin[j]);
            const uint32_t px = __float_as_uint(f.w);
            if (fp.filmFp64) {
                atomicAdd(&fp.film64[3 * (size_t)px + 0], (double)f.x);
                atomicAdd(&fp.film64[3 * (size_t)px + 1], (double)f.y);
                atomicAdd(&fp.film64[3 * (size_t)px + 2], (double)f.z);
            } else {
                atomicAdd(&fp.film[px], make_float4(f.x, f.y, f.z, 1.0f));
            }
            finished++;
            if (pool.records) {  // complete the path's guide training record
                const float4 r2 = __ldcs(&pool.finRec[4 * j + 2]);
                if (r2.w > 0.0f) {
                    samples++;  // a training sample; only nonzero targets are stored
                    const float4 r0 = __ldcs(&pool.finRec[4 * j + 0]), r1 = __ldcs(&pool.finRec[4 * j + 1]);
                    const float4 r3 = __ldcs(&pool.finRec[4 * j + 3]);
                    const float y = r2.w * r3.w * ((f.x - r3.x) + (f.y - r3.y) + (f.z - r3.z)) * (1.0f / 3.0f);
                    if (y > 0.0f && isfinite(y)) {
                        // a ring: the newest records replace the oldest
                        const uint32_t k = warpAppend(&cnt->numRecords) & (pool.recordCapacity - 1u);
                        GuideRecord g;
                        g.features[0] = r0.x; g.features[1] = r0.y; g.features[2] = r0.z; g.features[3] = r0.w;
                        g.features[4] = r1.x; g.features[5] = r1.y; g.features[6] = r1.z;
                        g.pdfBsdf = r1.w;
                        g.dir[0] = r2.x; g.dir[1] = r2.y; g.dir[2] = r2.z;
                        g.y = y;
                        pool.records[k] = g;
                    }
                }
            }
        }
        if (j < nNew) {
            const unsigned long long id = first + j;
            const uint32_t sample = (uint32_t)(id / fp.numPixels);
            const uint32_t r = (uint32_t)(id - (unsigned long long)sample * fp.numPixels);
            uint32_t x, y, pixel, sampleWord;
            PrngState prng;
            float3 org, dir;
            float nearClip, farClip;
            if constexpr (BATCH) {
                const uint32_t view = batchViewOf(pool.views, pool.numViews, r);
                const BatchView &bv = pool.views[view];
                FrameParams vf = fp;  // the view's frame
                vf.width = bv.width;
                vf.height = bv.height;
                vf.numPixels = bv.numPixels;
                blockLinearToPixel(r - bv.pixelOffset, bv.width, bv.height, x, y);
                cameraRay(bv.ctx, vf, x, y, sample, prng, org, dir);
                nearClip = bv.ctx.nearClip;
                farClip = bv.ctx.farClip;
                pixel = bv.pixelOffset + y * bv.width + x;
                sampleWord = (view << BATCH_SAMPLE_BITS) | sample;
            } else {
                blockLinearToPixel(r, fp.width, fp.height, x, y);
                cameraRay(ctx, fp, x, y, sample, prng, org, dir);
                nearClip = ctx.nearClip;
                farClip = ctx.farClip;
                pixel = y * fp.width + x;
                sampleWord = sample;
            }
            const uint32_t k = base + j;
            const uint2 rs = prng.pack();
            __stcs(&S.rayO[k], f4(org, nearClip));
            __stcs(&S.rayD[k], f4(dir, farClip));
            __stcs(&S.tp[k], make_float4(1.0f, 1.0f, 1.0f, inf_f()));
            __stcs(&S.L[k], make_float4(0.0f, 0.0f, 0.0f, __uint_as_float((uint32_t)RayFlagsCamera << 16)));
            __stcs(&S.id[k], make_uint4(pixel, sampleWord, rs.x, rs.y));
        }
    }
    blockAdd64(&cnt->pathsDone, finished);
    if (pool.records) {
        samples = __reduce_add_sync(0xffffffffu, samples);
        if ((threadIdx.x & 31) == 0 && samples) atomicAdd(&cnt->numSamples, samples);
    }
}

// ------------------------------------------------------------- traversal
// Persistent warps (Aila & Laine 2009): a warp takes 32 consecutive queue
// entries with one atomic and traces them to the end.  begin(idx, state,
// stack) starts entry idx, finish(idx, state) consumes the finished query.
// BATCH: begin() may point `nodes` / `tris` at the entry's own scene.
template <bool ANY, class Begin, class Finish>
__device__ __forceinline__ void persistentTrace(const WideNode *__restrict__ sceneNodes,
                                                const float4 *__restrict__ sceneTris, uint32_t *work, uint32_t n,
                                                uint32_t *errors, Begin begin, Finish finish) {
    TraversalState s;
    TraversalStack stack;
    const int lane = threadIdx.x & 31;
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(work, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const uint32_t idx = base + lane;
        if (idx < n) {
            const WideNode *nodes = sceneNodes;
            const float4 *tris = sceneTris;
            begin(idx, s, stack, nodes, tris);
            traverse<ANY>(s, stack, nodes, tris, errors);
            finish(idx, s, tris);
        }
    }
}

template <bool BATCH>
__global__ void __launch_bounds__(128) k_trace_closest(const WideNode *__restrict__ sceneNodes,
                                                       const float4 *__restrict__ sceneTris, PathPool pool,
                                                       Counters *cnt, uint32_t p) {
    const uint32_t n = activeCount(cnt, p);
    const PathState S = pool.s[p];
    persistentTrace<false>(
        sceneNodes, sceneTris, &cnt->traceWork, n, &cnt->errors,
        [&](uint32_t idx, TraversalState &s, TraversalStack &, const WideNode *&nodes, const float4 *&tris) {
            if constexpr (BATCH) {
                const BatchView &bv = pool.views[__ldg(&S.id[idx].y) >> BATCH_SAMPLE_BITS];
                nodes = static_cast<const WideNode *>(bv.nodes);
                tris = bv.tris;
            }
            const float4 o = __ldcs(&S.rayO[idx]);
            const float4 d = __ldcs(&S.rayD[idx]);
            beginTraversal(s, nodes, xyz(o), xyz(d), o.w, d.w);
        },
        [&](uint32_t idx, const TraversalState &s, const float4 *tris) {
            float4 hit;
            uint32_t inst;
            const bool found = closestHit(s, tris, hit, inst);
            __stcs(&pool.hit[idx], hit);
            __stcs(&pool.hitInst[idx], inst);

            if (found) pool.order[warpAppend(&cnt->nHit)] = idx;
            else pool.order[pool.capacity - 1u - warpAppend(&cnt->nMiss)] = idx;
        });
}

// raytraceAny fused with handleShadowRays (shadow.metal:6-29): an unoccluded
// shadow ray adds its weight to its path's radiance, in S[p ^ 1] for a path
// that continues and in the finish list for one that ended.  Thread 0 also
// advances nextPath past the camera samples this iteration consumed.
// BATCH: the ray's view is in bits 22-29 of its target.
template <bool BATCH>
__global__ void __launch_bounds__(128) k_trace_shadow(const WideNode *__restrict__ sceneNodes,
                                                      const float4 *__restrict__ sceneTris, PathPool pool,
                                                      Counters *cnt, uint32_t p) {
    const uint32_t n = cnt->nShadow;
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt->nextPath += newPaths(cnt, p);
    float4 *nextL = pool.s[p ^ 1u].L;
    float4 *nextRec = pool.s[p ^ 1u].rec;
    uint32_t target = 0, traced = 0;
    persistentTrace<true>(
        sceneNodes, sceneTris, &cnt->shadowWork, n, &cnt->errors,
        [&](uint32_t idx, TraversalState &s, TraversalStack &, const WideNode *&nodes, const float4 *&tris) {
            if constexpr (BATCH) {
                const uint32_t t = __float_as_uint(__ldg(&pool.shD[idx].w));
                const BatchView &bv = pool.views[(t >> BATCH_TARGET_BITS) & 0xffu];
                nodes = static_cast<const WideNode *>(bv.nodes);
                tris = bv.tris;
            }
            const float4 o = __ldcs(&pool.shO[idx]);
            const float4 d = __ldcs(&pool.shD[idx]);
            target = __float_as_uint(d.w);
            traced++;
            beginTraversal(s, nodes, xyz(o), xyz(d), SHADOW_EPS, o.w);
        },
        [&](uint32_t idx, const TraversalState &s, const float4 *) {
            // all ones: the path overflowed its queue
            if (s.hitTri >= 0 || target == 0xffffffffu) return;
            const bool finished = (target & SHADOW_TO_FINISHED) != 0u;
            const uint32_t at = target & (BATCH ? BATCH_TARGET_MASK : SHADOW_TARGET_MASK);
            float4 *dst = finished ? &pool.fin[at] : &nextL[at];
            const float4 w = __ldcs(&pool.shW[idx]);
            float4 L = *dst;
            L.x += w.x;
            L.y += w.y;
            L.z += w.z;
            *dst = L;
            if (target & SHADOW_TO_RECORD) {  // light sample of the recorded vertex: not through its sampled direction
                float4 *rec = finished ? &pool.finRec[4 * at + 3] : &nextRec[4 * at + 3];
                float4 r = *rec;
                r.x += w.x;
                r.y += w.y;
                r.z += w.z;
                *rec = r;
            }
            if (pool.shRec && w.w > 0.0f) {
                // a training record of the vertex's light sample: its direction,
                // target (MIS-weighted contribution / throughput) and features
                const float y = (w.x + w.y + w.z) * (1.0f / 3.0f) * w.w;
                if (y > 0.0f && isfinite(y)) {
                    const uint32_t k = atomicAdd(&cnt->numRecords, 1u) & (pool.recordCapacity - 1u);
                    const float4 r0 = __ldcs(&pool.shRec[2 * idx]), r1 = __ldcs(&pool.shRec[2 * idx + 1]);
                    const float4 d = __ldcs(&pool.shD[idx]);
                    GuideRecord g;
                    g.features[0] = r0.x; g.features[1] = r0.y; g.features[2] = r0.z; g.features[3] = r0.w;
                    g.features[4] = r1.x; g.features[5] = r1.y; g.features[6] = r1.z;
                    g.pdfBsdf = r1.w;
                    g.dir[0] = d.x; g.dir[1] = d.y; g.dir[2] = d.z;
                    g.y = y;
                    pool.records[k] = g;
                }
            }
        });
    blockAdd64(&cnt->shadowRays, traced);
}

// ------------------------------------------------------------- device-driven loop
// Last node of the body of a CUDA-graph while loop of `itersPerBody`
// wavefront iterations: continue while paths remain, no error was flagged
// and the iteration bound (which every render reaches only on a fault) is
// not passed.  The bound also guarantees that the loop ends.
__global__ void k_loop_condition(Counters *cnt, cudaGraphConditionalHandle handle, uint32_t itersPerBody,
                                 uint32_t maxIterations) {
    const uint32_t it = cnt->loopIterations + itersPerBody;
    cnt->loopIterations = it;
    const bool more = cnt->pathsDone < cnt->numPaths && cnt->errors == 0u && it < maxIterations;
    if (!more && cnt->pathsDone < cnt->numPaths && cnt->errors == 0u) atomicOr(&cnt->errors, ERR_LOOP_BOUND);
    cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// ------------------------------------------------------------- environment map
// kernels/envmap/reduce.metal:3-24 over one level of `cur x cur` quads.
__global__ void k_envmap_reduce(float *mip, int cur) {
    const int tx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ty = blockIdx.y * blockDim.y + threadIdx.y;
    if (tx >= cur || ty >= cur) return;
    const int inputIndex = ty * cur + tx;
    const int gridLength = cur * cur;
    float sum = 0.0f;
    for (int i = 0; i < 4; ++i) sum += mip[gridLength + 4 * inputIndex + i];
    for (int i = 0; i < 4; ++i) mip[gridLength + 4 * inputIndex + i] /= sum;
    const unsigned qx = tx / 2, qy = ty / 2, qw = cur / 2;
    const unsigned outputIndex = cur == 1 ? 0u : 4u * (qy * qw + qx) + (tx & 1) + 2u * (ty & 1);
    mip[outputIndex] = sum;
}
// kernels/envmap/normalize.metal:4-11
__global__ void k_envmap_normalize(const float *sum, float *pdfs, uint32_t gridSize) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= gridSize) return;
    const float scale = (float)gridSize * warp::uniformSquareToSpherePdf() / *sum;
    pdfs[i] *= scale;
}

// ------------------------------------------------------------- film read-out
// kernels/utils/normalizeImage.metal:11-59
__device__ float3 tonemapHablePartial(float3 x) {
    const float hA = 0.15f, hB = 0.50f, hC = 0.10f, hD = 0.20f, hE = 0.02f, hF = 0.30f;
    return ((x * (hA * x + hC * hB) + hD * hE) / (x * (hA * x + hB) + hD * hF)) - hE / hF;
}
// color = exposure * film; color /= divisor (the frame count, 1 when not
// accumulating), then the tonemap, in the reference's order of operations;
// `channels` 3 (RGB) or 4 (RGB and alpha 1, as normalizeImage writes).
__global__ void k_film_resolve(const float4 *film, const double *film64, int fp64, float *out, uint32_t numPixels,
                               float exposure, float divisor, uint32_t tonemapping, uint32_t channels) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numPixels) return;
    float3 c;
    if (fp64) c = make_float3((float)film64[3 * (size_t)i], (float)film64[3 * (size_t)i + 1], (float)film64[3 * (size_t)i + 2]);
    else c = xyz(film[i]);
    c = exposure * c;
    if (divisor != 1.0f) c = make_float3(__fdiv_rn(c.x, divisor), __fdiv_rn(c.y, divisor), __fdiv_rn(c.z, divisor));
    if (tonemapping == 1u) {
        const float3 curr = tonemapHablePartial(c * 2.0f);
        const float3 whiteScale = 1.0f / tonemapHablePartial(f3(11.2f));
        c = curr * whiteScale;
    } else if (tonemapping == 2u) {
        const float tA = 2.51f, tB = 0.03f, tC = 2.43f, tD = 0.59f, tE = 0.14f;
        c = saturate((c * (tA * c + tB)) / (c * (tC * c + tD) + tE));
    }
    float *o = out + (size_t)channels * i;
    o[0] = c.x;
    o[1] = c.y;
    o[2] = c.z;
    if (channels == 4) o[3] = 1.0f;
}

// ------------------------------------------------------------- sky texture
// SKY_nishita_skymodel_precompute_texture (host/sky/sky_nishita.cpp:295-341)
// on the device: texel (x, y) of the left half and its mirror image.
__global__ void k_sky_texture(float4 *texels, int width, int height, float sunElevation, float altitude, float air,
                              float dust, float ozone) {
    const int half = width / 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half * height) return;
    const int y = i / half, x = i - y * half;
    const rmdsky::V3 c = rmdsky::skyTexel(x, y, width, height, sunElevation, altitude, air, dust, ozone);
    const float4 v = make_float4(c.x, c.y, c.z, 1.0f);
    texels[(size_t)y * width + x] = v;
    texels[(size_t)y * width + (width - x - 1)] = v;
}

// ------------------------------------------------------------- test hooks
__global__ void k_debug_prng(uint32_t mode, uint64_t a, uint64_t b, int n, float *out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    PrngState p = mode == RNG_TEA ? PrngState::tea((uint32_t)a, (uint32_t)b) : PrngState::pcg(a, b);
    for (int i = 0; i < n; i++) out[i] = p.sample();
}
__global__ void k_debug_trace(const WideNode *nodes, const float4 *tris, const float *rays, int n, int any, float *out,
                              uint32_t *inst, uint32_t *errors) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *r = rays + 8 * (size_t)i;
    const float3 o = make_float3(r[0], r[1], r[2]), d = make_float3(r[4], r[5], r[6]);
    float4 h = make_float4(-1.0f, 0.0f, 0.0f, 0.0f);
    uint32_t id = 0;
    if (any) {
        h.x = traceAny(nodes, tris, o, d, r[3], r[7], errors) ? 1.0f : -1.0f;
    } else {
        traceClosest(nodes, tris, o, d, r[3], r[7], h, id, errors);
    }
    out[4 * (size_t)i + 0] = h.x;
    out[4 * (size_t)i + 1] = h.y;
    out[4 * (size_t)i + 2] = h.z;
    out[4 * (size_t)i + 3] = h.w;
    inst[i] = id;
}

// The traversal kernels' triangle layout from the builders' (v0, v1, v2 per
// triangle, float4 each): three copies per triangle, copy k with the
// coordinates rotated so that axis k comes last (device/traverse.cuh).
__global__ void k_rotate_triangles(const float4 *__restrict__ in, float4 *__restrict__ out, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const float4 v = in[3 * (size_t)i + j];
            out[TRI_FLOAT4 * (size_t)i + 0 + j] = make_float4(v.y, v.z, v.x, v.w);
            out[TRI_FLOAT4 * (size_t)i + 3 + j] = make_float4(v.z, v.x, v.y, v.w);
            out[TRI_FLOAT4 * (size_t)i + 6 + j] = v;
        }
    }
}

}  // namespace rmd

// ------------------------------------------------------------- launch wrappers
using namespace rmd;

cudaError_t rmdLaunchLoopCondition(Counters *cnt, cudaGraphConditionalHandle handle, uint32_t itersPerBody,
                                   uint32_t maxIterations, cudaStream_t s) {
    k_loop_condition<<<1, 1, 0, s>>>(cnt, handle, itersPerBody, maxIterations);
    return cudaGetLastError();
}

cudaError_t rmdLaunchFrameInit(const PathPool &pool, Counters *cnt, uint64_t firstPath, uint64_t endPath,
                               cudaStream_t s) {
    k_frame_init<<<1, 1, 0, s>>>(cnt, pool.capacity, firstPath, endPath);
    return cudaGetLastError();
}
cudaError_t rmdLaunchFilmRegen(const Context &ctx, const PathPool &pool, const FrameParams &fp, Counters *cnt,
                               uint32_t cur, int blocks, cudaStream_t s) {
    if (pool.views) k_film_regen<true><<<blocks, 256, 0, s>>>(ctx, pool, fp, cnt, cur);
    else k_film_regen<false><<<blocks, 256, 0, s>>>(ctx, pool, fp, cnt, cur);
    return cudaGetLastError();
}
cudaError_t rmdLaunchTraceClosest(const WideNode *nodes, const float4 *tris, const PathPool &pool, Counters *cnt,
                                  uint32_t cur, int blocks, cudaStream_t s) {
    if (pool.views) k_trace_closest<true><<<blocks, 128, 0, s>>>(nodes, tris, pool, cnt, cur);
    else k_trace_closest<false><<<blocks, 128, 0, s>>>(nodes, tris, pool, cnt, cur);
    return cudaGetLastError();
}
cudaError_t rmdLaunchTraceShadow(const WideNode *nodes, const float4 *tris, const PathPool &pool, Counters *cnt,
                                 uint32_t cur, int blocks, cudaStream_t s) {
    if (pool.views) k_trace_shadow<true><<<blocks, 128, 0, s>>>(nodes, tris, pool, cnt, cur);
    else k_trace_shadow<false><<<blocks, 128, 0, s>>>(nodes, tris, pool, cnt, cur);
    return cudaGetLastError();
}
cudaError_t rmdLaunchEnvmapReduce(float *mip, int cur, cudaStream_t s) {
    dim3 b(8, 8), g((cur + 7) / 8, (cur + 7) / 8);
    k_envmap_reduce<<<g, b, 0, s>>>(mip, cur);
    return cudaGetLastError();
}
cudaError_t rmdLaunchEnvmapNormalize(const float *sum, float *pdfs, uint32_t gridSize, cudaStream_t s) {
    k_envmap_normalize<<<(gridSize + 255) / 256, 256, 0, s>>>(sum, pdfs, gridSize);
    return cudaGetLastError();
}
cudaError_t rmdLaunchFilmResolve(const float4 *film, const double *film64, int fp64, float *out, uint32_t numPixels,
                                 float exposure, float divisor, uint32_t tonemapping, uint32_t channels, cudaStream_t s) {
    k_film_resolve<<<(numPixels + 255) / 256, 256, 0, s>>>(film, film64, fp64, out, numPixels, exposure, divisor,
                                                            tonemapping, channels);
    return cudaGetLastError();
}
cudaError_t rmdLaunchDebugPrng(uint32_t mode, uint64_t a, uint64_t b, int n, float *out, cudaStream_t s) {
    k_debug_prng<<<1, 1, 0, s>>>(mode, a, b, n, out);
    return cudaGetLastError();
}
cudaError_t rmdLaunchRotateTriangles(const float4 *in, float4 *out, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_rotate_triangles<<<std::min<uint32_t>((n + 255) / 256, 148u * 16u), 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}
cudaError_t rmdLaunchDebugTrace(const WideNode *nodes, const float4 *tris, const float *rays, int n, int any, float *out,
                                uint32_t *inst, uint32_t *errors, cudaStream_t s) {
    k_debug_trace<<<(n + 127) / 128, 128, 0, s>>>(nodes, tris, rays, n, any, out, inst, errors);
    return cudaGetLastError();
}
cudaError_t rmdLaunchSkyTexture(float4 *texels, uint32_t width, uint32_t height, float sunElevation, float altitude,
                                float air, float dust, float ozone, cudaStream_t s) {
    const uint32_t n = width / 2 * height;
    if (n == 0) return cudaSuccess;
    k_sky_texture<<<(n + 127) / 128, 128, 0, s>>>(texels, (int)width, (int)height, sunElevation, altitude, air, dust,
                                                  ozone);
    return cudaGetLastError();
}
