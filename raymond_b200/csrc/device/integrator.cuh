// The shading megakernel (handleIntersections, raymond/device/kernels/shading/
// intersection.metal:22-211) and the environment-map build kernel
// (kernels/envmap/build.metal:4-51) over the wavefront path pool.  Compiled
// by NVRTC together with the generated material functions, so shadeSurface /
// shadeLight resolve to the scene's node graphs.
#pragma once
#include "nodes.cuh"
#include "wavefront.cuh"

namespace rmd {

// intersection.metal:14-20
RMD_HD float computeMisWeight(float pdf, float other) {
    pdf *= pdf;
    if (is_inf(pdf)) return 1.0f;
    other *= other;
    return pdf / (pdf + other);
}

// One path vertex: intersection.metal:43-208 for the active path at position
// i of S[cur], the orderPos-th in shading order; returns whether a surface
// was hit (a segment was shaded).
__device__ __forceinline__ bool shadePath(const ShadeParams &p, uint32_t i, uint32_t orderPos) {
    const PathPool &pool = p.pool;
    const FrameParams &fp = p.fp;
    Counters *cnt = p.counters;
    const PathState &S = pool.s[p.cur];

    const float4 d4 = __ldcs(&S.rayD[i]);
    const float4 tp4 = __ldcs(&S.tp[i]);
    const float4 h4 = __ldcs(&pool.hit[i]);
    const float4 L4 = __ldcs(&S.L[i]);
    const uint4 id = __ldcs(&S.id[i]);
    const uint32_t meta = __float_as_uint(L4.w);
    const uint32_t pixel = id.x;
#ifdef RMD_BATCH
    // a batch path: its view (top bits of the sample word) gives the scene
    // context and the PCG stream of the view's own pixel index
    const uint32_t view = id.y >> BATCH_SAMPLE_BITS;
    const BatchView &bv = pool.views[view];
    const Context &ctx = bv.ctx;
    const uint32_t sample = id.y & BATCH_SAMPLE_MASK;
    const uint32_t seqPixel = pixel - bv.pixelOffset, numPixels = bv.numPixels;
#else
    const Context &ctx = p.ctx;
    const uint32_t sample = id.y;
    const uint32_t seqPixel = pixel, numPixels = fp.numPixels;
#endif
    float3 L = xyz(L4);
    const float3 rayDir = xyz(d4);
    const float3 rayWeight = xyz(tp4);
    const float rayBsdfPdf = tp4.w;
    const uint32_t depth = meta & 0xffffu;
    const uint32_t rayFlags = (meta >> 16) & 0xffu;
    const bool lastDepth = depth + 1u >= fp.maxDepth;
    PrngState prng = PrngState::unpack(fp.rngMode, make_uint2(id.z, id.w), pathSequence(sample, seqPixel, numPixels));
    uint32_t shadowIndex = 0xffffffffu;  // shadow ray whose target is set once the path's fate is known
    float3 shadowDir = f3(0.0f);
    float4 next[3];                      // rayO, rayD, tp of the continued path
    float L4next = 0.0f;                 // its depth | flags word
    // RMD_PLAIN_SHADE: the module of a renderer or batch that neither samples
    // from nor trains the guide, with the guide's code compiled out (a shorter
    // kernel fetches fewer instructions)
#ifdef RMD_PLAIN_SHADE
    constexpr bool kGuideCode = false;
#else
    constexpr bool kGuideCode = true;
#endif
    const bool training = kGuideCode && S.rec != nullptr;
    float4 record[4] = {f4(0.0f), f4(0.0f), f4(0.0f), f4(0.0f)};  // guide training record
    bool recorded = false;  // this vertex replaced the path's record

    const bool needsToCollectEmission = is_inf(rayBsdfPdf) || fp.samplingMode != 1u;
    ShadingContext shading;
    shading.rayFlags = rayFlags;
    shading.rnd = prng.sample3d();
    shading.wo = -rayDir;

    bool alive = false;
    if (h4.x <= 0.0f) {  // miss, intersection.metal:75-91
        if (needsToCollectEmission) {
            const float misWeight = (fp.samplingMode == 0u) || is_inf(rayBsdfPdf)
                                        ? 1.0f
                                        : computeMisWeight(rayBsdfPdf, lightsEnvmapPdf(ctx, rayDir));
            evaluateEnvironment(ctx, shading);
            L += misWeight * rayWeight * shading.material.emission;
        }
    } else {
        const PerInstanceData &inst = ctx.instances[__ldcs(&pool.hitInst[i])];
        uint32_t shaderIndex;
        buildShading(shading, ctx, inst, __float_as_uint(h4.w), make_float2(h4.y, h4.z), h4.x, shaderIndex);
        if (inst.visibility & rayFlags) shadeSurface(shaderIndex, ctx, shading);
        else shading.material.alpha = 0.0f;

        if (needsToCollectEmission && mean(shading.material.emission) != 0.0f) {
            const float misWeight = (fp.samplingMode == 0u) || is_inf(rayBsdfPdf)
                                        ? 1.0f
                                        : computeMisWeight(rayBsdfPdf, lightsShapePdf(ctx, inst, shading));
            L += misWeight * rayWeight * shading.material.emission;
        }

        float3 shNormal;
        if (all_zero(shading.material.normal)) {
            shNormal = shading.trueNormal;
        } else {
            float3 geoNormal = shading.trueNormal;
            if (dot(geoNormal, shading.wo) < 0.0f) geoNormal *= -1.0f;
            shNormal = ensure_valid_reflection(geoNormal, shading.wo, shading.material.normal);
        }

        // Guiding: directions come from the BSDF or, with probability alpha, from
        // the guide mixture of this point (one-sample MIS); the technique's pdf is
        // then alpha q + (1 - alpha) p_bsdf in every MIS weight that uses it.
        const bool guided = kGuideCode && depth < fp.guideDepth;
        const GuideMixture *gm = &pool.guide[orderPos];  // hits are shaded in order: mixture by that position
        float alpha = guided ? gm->alpha : 0.0f;
        if (guided) {
            // A warp whose lanes are all guided uses one selection probability,
            // the mean of their alphas: the technique choice below is then the
            // same on every lane and the warp does not run both techniques.  A
            // probability that does not depend on this path's own sample keeps
            // the one-sample MIS estimator unbiased.
            if (__activemask() == 0xffffffffu) {
                float sum = alpha;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
                alpha = sum * (1.0f / 32.0f);
            }
        }
        GuideFeatures gf;  // training: the guide's input features of this vertex
        const float meanThroughput = mean(rayWeight);
        if (training)
            gf = guideFeatures(shading.position, shading.trueNormal, shading.wo, fp.guideSceneMin,
                               fp.guideSceneInvExtent);

        if (fp.samplingMode != 0u) {  // NEE, intersection.metal:149-181
            LightSample nee = lightsSample(ctx, shading.position, shading.rayFlags, prng);
            float bsdfPdf;
            const float3 bsdf = shading.material.evaluate(shading.wo, nee.direction, shNormal, shading.trueNormal, bsdfPdf);
            const float neeBsdfPdf = bsdfPdf;
            if (guided) bsdfPdf = alpha * guidePdf(gm, nee.direction) + (1.0f - alpha) * bsdfPdf;
            const float3 contribution = nee.weight * bsdf * rayWeight;
            if (nee.castsShadows) {
                const float misWeight =
                    fp.samplingMode == 1u || !nee.canBeHit ? 1.0f : computeMisWeight(nee.pdf, bsdfPdf);
                const float3 neeWeight = misWeight * contribution;
                // a non-finite light sample is dropped, as the reference's
                // device code drops it, and counted
                if (!isfinite3(neeWeight)) atomicAdd(&cnt->invalid, 1ull);
                // shadow rays of the last shade pass are never traced (Renderer.swift:623-625)
                if (isfinite3(neeWeight) && any_nonzero(neeWeight) && !lastDepth) {
                    const uint32_t k = warpAppend(&cnt->nShadow);
                    if (k < pool.capacity) {
                        __stcs(&pool.shO[k], f4(shading.position, nee.distance - SHADOW_EPS));
                        // training: the light sample is a training sample of this vertex too
                        const bool neeRecord = pool.shRec && meanThroughput > 0.0f && neeBsdfPdf > 0.0f;
                        __stcs(&pool.shW[k], f4(neeWeight, neeRecord ? 1.0f / meanThroughput : 0.0f));
                        if (neeRecord) {
                            __stcs(&pool.shRec[2 * k], make_float4(gf.v[0], gf.v[1], gf.v[2], gf.v[3]));
                            __stcs(&pool.shRec[2 * k + 1], make_float4(gf.v[4], gf.v[5], gf.v[6], neeBsdfPdf));
                        }
                        shadowIndex = k;
                        shadowDir = nee.direction;
                    } else {
                        atomicOr(&cnt->errors, ERR_QUEUE_OVERFLOW);
                    }
                }
            } else {
                L += rayWeight * contribution;  // intersection.metal:172-179 (weight applied twice, as there)
            }
        }

        // BSDF sampling and Russian roulette, intersection.metal:185-208
        BsdfSample bs;
        float pdfBsdf = 0.0f;  // the BSDF's own pdf of the sampled direction
        float3 bsdfWeight;     // guided: f / pdfBsdf, the weight BSDF sampling gives the direction
        // The technique is chosen with one uniform number per warp (each lane
        // still draws its own): every path still takes the guide with its
        // probability alpha, and lanes of similar alpha stay converged.
        bool useGuide = false;
        if (guided) {
            const float own = prng.sample();
            const unsigned mask = __activemask();
            useGuide = __shfl_sync(mask, own, __ffs(mask) - 1) < alpha;
        }
        if (useGuide) {
            bs.wi = guideSample(gm, prng.sample3d());
            const float3 f = shading.material.evaluate(shading.wo, bs.wi, shNormal, shading.trueNormal, pdfBsdf);
            bs.pdf = alpha * guidePdf(gm, bs.wi) + (1.0f - alpha) * pdfBsdf;
            bs.weight = bs.pdf > 0.0f ? f * (1.0f / bs.pdf) : f3(0.0f);
            bsdfWeight = pdfBsdf > 0.0f ? f * (1.0f / pdfBsdf) : f3(0.0f);
            const bool reflect = dot(bs.wi, shading.trueNormal) * dot(shading.wo, shading.trueNormal) >= 0.0f;
            bs.flags = (uint8_t)((reflect ? RayFlagsReflection : RayFlagsTransmission) | RayFlagsGlossy);
        } else {
            bs = shading.material.sample(shading.rnd, -rayDir, shNormal, shading.trueNormal, (uint8_t)rayFlags);
            pdfBsdf = bs.pdf;
            bsdfWeight = bs.weight;
            if (guided) {
                if (bs.flags & RayFlagsSingular) {  // only the BSDF technique produces it
                    bs.weight = bs.weight * (1.0f / (1.0f - alpha));
                } else if (bs.pdf > 0.0f) {
                    const float pmix = alpha * guidePdf(gm, bs.wi) + (1.0f - alpha) * bs.pdf;
                    bs.weight = bs.weight * (bs.pdf / pmix);
                    bs.pdf = pmix;
                }
            }
        }
        const float3 weight = rayWeight * bs.weight;
        const float meanWeight = mean(weight);
        if (!is_finite(meanWeight)) atomicAdd(&cnt->invalid, 1ull);  // the path ends, as in the reference
        if (is_finite(meanWeight)) {
            // Guided, roulette keeps the path with the probability BSDF sampling
            // would give its direction, so directions the guide favours (high
            // pdf, small weight) are not culled for it
            const float survivalProb = fminf(guided ? mean(rayWeight * bsdfWeight) : meanWeight, 1.0f);
            if (prng.sample() < survivalProb && !lastDepth) {
                alive = true;
                next[0] = f4(shading.position, SHADOW_EPS);
                next[1] = f4(bs.wi, inf_f());
                next[2] = f4(weight * (1.0f / survivalProb), bs.pdf);
                // bits 24-31: eligible guide-record vertices so far
                L4next = __uint_as_float((depth + 1u) | ((uint32_t)bs.flags << 16) | (meta & 0xff000000u));
                if (training && !(bs.flags & RayFlagsSingular) && pdfBsdf > 0.0f && meanThroughput > 0.0f) {
                    // Reservoir of one over the path's eligible vertices: the n-th
                    // replaces the pending record with probability 1 / n (a hash of
                    // the path and depth, so the PCG stream is untouched).  The
                    // radiance-weighted target f Li cos / p of the sampled direction
                    // is survival * (final radiance - radiance so far) / throughput,
                    // completed when the path ends.
                    const uint32_t seen = min((meta >> 24) + 1u, 255u);
                    L4next = __uint_as_float((__float_as_uint(L4next) & 0x00ffffffu) | (seen << 24));
                    if (seen == 1u || recordHash(pixel, sample, depth) * (float)seen < 1.0f) {
                        record[0] = make_float4(gf.v[0], gf.v[1], gf.v[2], gf.v[3]);
                        record[1] = make_float4(gf.v[4], gf.v[5], gf.v[6], pdfBsdf);
                        record[2] = f4(bs.wi, survivalProb);
                        record[3] = f4(L, 1.0f / meanThroughput);
                        recorded = true;
                    }
                }
            }
        }
    }
    uint32_t target = 0xffffffffu;
    if (alive) {  // continued: next free position of S[cur ^ 1]
        const uint32_t k = warpAppend(&cnt->nQ[p.cur ^ 1u]);
        if (k < pool.capacity) {
            const PathState &N = pool.s[p.cur ^ 1u];
            const uint2 rs = prng.pack();
            __stcs(&N.rayO[k], next[0]);
            __stcs(&N.rayD[k], next[1]);
            __stcs(&N.tp[k], next[2]);
            __stcs(&N.L[k], f4(L, L4next));
            __stcs(&N.id[k], make_uint4(pixel, id.y, rs.x, rs.y));
            if (training) {
                if (!recorded && depth > 0u)
                    for (int r = 0; r < 4; r++) record[r] = __ldcs(&S.rec[4 * i + r]);
                for (int r = 0; r < 4; r++) __stcs(&N.rec[4 * k + r], record[r]);
            }
            target = k;
        } else {
            atomicOr(&cnt->errors, ERR_QUEUE_OVERFLOW);
        }
    } else {  // finished: the finish list, added to the film by the next film pass
        const uint32_t k = warpAppend(&cnt->nF[p.cur]);
        if (k < pool.capacity) {
            __stcs(&pool.fin[k], f4(L, __uint_as_float(pixel)));
            if (training) {
                if (depth > 0u)  // a finishing vertex never records
                    for (int r = 0; r < 4; r++) record[r] = __ldcs(&S.rec[4 * i + r]);
                for (int r = 0; r < 4; r++) __stcs(&pool.finRec[4 * k + r], record[r]);
            }
            target = k | SHADOW_TO_FINISHED;
        } else {
            atomicOr(&cnt->errors, ERR_QUEUE_OVERFLOW);
        }
    }
    if (shadowIndex != 0xffffffffu) {
        if (recorded && target != 0xffffffffu) target |= SHADOW_TO_RECORD;
#ifdef RMD_BATCH
        if (target != 0xffffffffu) target |= view << BATCH_TARGET_BITS;  // the shadow ray's scene
#endif
        __stcs(&pool.shD[shadowIndex], f4(shadowDir, __uint_as_float(target)));
    }
    return h4.x > 0.0f;
}

}  // namespace rmd

#ifndef RMD_SHADE_MIN_BLOCKS
#define RMD_SHADE_MIN_BLOCKS 1
#endif
extern "C" __global__ void __launch_bounds__(128, RMD_SHADE_MIN_BLOCKS) rmd_shade(const __grid_constant__ rmd::ShadeParams p) {
    const unsigned n = rmd::activeCount(p.counters, p.cur);
    unsigned segments = 0, rays = 0;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        segments += rmd::shadePath(p, rmd::shadingOrder(p.pool.order, p.counters, i), i) ? 1u : 0u;
        rays++;
    }
    rmd::blockAdd64(&p.counters->segments, segments);
    rmd::blockAdd64(&p.counters->rays, rays);
}

// kernels/envmap/build.metal:4-51 — the finest level of the importance map:
// mean of 64 world-shader evaluations per texel (+1e-8), written both as a
// pdf and into the quad-ordered mip level.
extern "C" __global__ void rmd_envmap_build(const __grid_constant__ rmd::Context ctx, float *mipmap, float *pdfs,
                                            int resolution) {
    using namespace rmd;
    const int tx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ty = blockIdx.y * blockDim.y + threadIdx.y;
    if (tx >= resolution || ty >= resolution) return;
    const int rayIndex = ty * resolution + tx;
    float value = 0.0f;
    const int numSamples = 64;
    for (int sampleIndex = 0; sampleIndex < numSamples; sampleIndex++) {
        PrngState prng = PrngState::tea((uint32_t)sampleIndex, (uint32_t)rayIndex);
        const float2 projected = (make_float2((float)tx, (float)ty) + prng.sample2d()) /
                                 make_float2((float)resolution, (float)resolution);
        const float3 wo = warp::uniformSquareToSphere(projected);
        ShadingContext sh;
        sh.uv = sh.position = sh.generated = sh.object = sh.normal = sh.trueNormal = sh.tu = sh.tv = f3(0.0f);
        sh.distance = 0.0f;
        sh.rayFlags = 0;
        sh.rnd = prng.sample3d();
        sh.wo = -wo;
        evaluateEnvironment(ctx, sh);
        value += mean(sh.material.emission);
    }
    value /= (float)numSamples;
    value += 1e-8f;
    const unsigned qx = tx / 2, qy = ty / 2, qw = resolution / 2;
    const unsigned outputIndex = resolution == 1 ? 0u : 4u * (qy * qw + qx) + (tx & 1) + 2u * (ty & 1);
    mipmap[outputIndex] = value;
    pdfs[rayIndex] = value;
}

// Test hook: shade records with one material and evaluate / sample its BSDF the
// way handleIntersections does (intersection.metal:93-185).  Record layout:
// position, normal, trueNormal, generated, uv, wo, wi, rnd (float3 each),
// rayFlags, tangent tu (bitangent normal x tu); output: emission, eval value, eval pdf, sampled wi,
// sampled weight, sampled pdf, sampled flags, alpha.
extern "C" __global__ void rmd_material_eval(const __grid_constant__ rmd::Context ctx, unsigned material,
                                             const float *records, float *out, int n) {
    using namespace rmd;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *r = records + 28 * (size_t)i;
    ShadingContext sh;
    sh.position = make_float3(r[0], r[1], r[2]);
    sh.normal = make_float3(r[3], r[4], r[5]);
    sh.trueNormal = make_float3(r[6], r[7], r[8]);
    sh.generated = make_float3(r[9], r[10], r[11]);
    sh.uv = make_float3(r[12], r[13], r[14]);
    sh.wo = make_float3(r[15], r[16], r[17]);
    const float3 wi = make_float3(r[18], r[19], r[20]);
    sh.rnd = make_float3(r[21], r[22], r[23]);
    sh.rayFlags = (unsigned)r[24];
    sh.object = sh.generated;
    sh.tu = make_float3(r[25], r[26], r[27]);  // the tangent frame: tu given, tv = normal x tu
    sh.tv = cross(sh.normal, sh.tu);
    sh.distance = 0.0f;
    shadeSurface(material, ctx, sh);
    float3 shNormal;
    if (all_zero(sh.material.normal)) {
        shNormal = sh.trueNormal;
    } else {
        float3 g = sh.trueNormal;
        if (dot(g, sh.wo) < 0.0f) g *= -1.0f;
        shNormal = ensure_valid_reflection(g, sh.wo, sh.material.normal);
    }
    float pdf;
    const float3 f = sh.material.evaluate(sh.wo, wi, shNormal, sh.trueNormal, pdf);
    const BsdfSample bs = sh.material.sample(sh.rnd, sh.wo, shNormal, sh.trueNormal, (uint8_t)sh.rayFlags);
    float *o = out + 16 * (size_t)i;
    o[0] = sh.material.emission.x; o[1] = sh.material.emission.y; o[2] = sh.material.emission.z;
    o[3] = f.x; o[4] = f.y; o[5] = f.z; o[6] = pdf;
    o[7] = bs.wi.x; o[8] = bs.wi.y; o[9] = bs.wi.z;
    o[10] = bs.weight.x; o[11] = bs.weight.y; o[12] = bs.weight.z;
    o[13] = bs.pdf; o[14] = (float)bs.flags; o[15] = sh.material.alpha;
}
