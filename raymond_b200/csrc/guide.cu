// The path-guiding network on the tensor cores: BF16 inference of the vMF
// mixtures for the hits of one wavefront iteration, and BF16 training
// (forward, loss gradient, backward, Adam) on the records the tracer
// produces.  No counterpart in the reference.
//
// Both run on the 5th-generation tensor cores (tcgen05.mma, operands in
// shared memory, FP32 accumulators in tensor memory): inference one thread per
// sample in pipelines of 128 (see the tcgen05 inference core), training one
// CTA per tile of 128 records, the weight gradients accumulated in tensor
// memory (see the tcgen05 training core).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device/guide.cuh"
#include "device/scene.cuh"
#include "device/wavefront.cuh"
#include "guide.h"

namespace rmd {
namespace {

__device__ __forceinline__ uint16_t toBf16(float x) { return (uint16_t)bf16Bits(x); }
__device__ __forceinline__ float fromBf16(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
__device__ __forceinline__ uint32_t pack2(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

__device__ __forceinline__ float sigmoid(float x) { return __fdividef(1.0f, 1.0f + __expf(-x)); }

// decoded network output of one sample
struct Decoded {
    float st[GUIDE_LOBES], sp[GUIDE_LOBES];  // sigmoids of the raw values (theta / pi, phi / 2 pi)
    float logKappa[GUIDE_LOBES];
    bool kappaClamped[GUIDE_LOBES];
    float lambda[GUIDE_LOBES];
    float alpha, alphaSig;
};

__device__ Decoded decode(const float *o) {
    Decoded d;
    float maxLogit = -1e30f;
#pragma unroll
    for (int j = 0; j < GUIDE_LOBES; j++) maxLogit = fmaxf(maxLogit, o[4 * j + 3]);
    float sum = 0.0f;
#pragma unroll
    for (int j = 0; j < GUIDE_LOBES; j++) {
        d.st[j] = sigmoid(o[4 * j + 0]);
        d.sp[j] = sigmoid(o[4 * j + 1]);
        const float lk = o[4 * j + 2];
        d.kappaClamped[j] = lk < GUIDE_LOG_KAPPA_MIN || lk > GUIDE_LOG_KAPPA_MAX;
        d.logKappa[j] = fminf(GUIDE_LOG_KAPPA_MAX, fmaxf(GUIDE_LOG_KAPPA_MIN, lk));
        d.lambda[j] = __expf(o[4 * j + 3] - maxLogit);
        sum += d.lambda[j];
    }
    const float invSum = 1.0f / sum;
    for (int j = 0; j < GUIDE_LOBES; j++) d.lambda[j] *= invSum;
    d.alphaSig = sigmoid(o[4 * GUIDE_LOBES]);
    d.alpha = GUIDE_ALPHA_MIN + (GUIDE_ALPHA_MAX - GUIDE_ALPHA_MIN) * d.alphaSig;
    return d;
}


// vMF normalisation k / (2 pi (1 - e^{-2k})) for k in [e^-3, e^5], where
// 1 - e^{-2k} >= 0.09 and needs no expm1
__device__ __forceinline__ float vmfNormPacked(float k) {
    return __fdividef(k * (0.5f / M_PI_F), 1.0f - __expf(-2.0f * k));
}

// the mean direction with the fast intrinsics: their error on [0, 2 pi]
// (~1e-6) is far below the BF16 rounding the packed mixture applies
__device__ float3 lobeMeanPacked(const Decoded &d, int j) {
    float st, ct, sp, cp;
    __sincosf(M_PI_F * d.st[j], &st, &ct);
    __sincosf(2.0f * M_PI_F * d.sp[j], &sp, &cp);
    return make_float3(st * cp, st * sp, ct);
}

__device__ GuideMixture pack(const Decoded &d) {
    GuideMixture m;
    uint32_t w[4];
    float total = 0.0f, kappa[GUIDE_LOBES];
    for (int j = 0; j < GUIDE_LOBES; j++) {
        const float3 mu = lobeMeanPacked(d, j);
        const uint32_t kb = bf16Bits(__expf(d.logKappa[j]));
        kappa[j] = bf16Lo(kb);
        total += bf16Lo(bf16Bits(d.lambda[j]));
        m.lobe[j] = make_uint2(bf16Bits(mu.x) | (bf16Bits(mu.y) << 16), bf16Bits(mu.z) | (kb << 16));
        if (j & 1) w[j >> 1] |= bf16Bits(d.lambda[j]) << 16;
        else w[j >> 1] = bf16Bits(d.lambda[j]);
    }
    const float inv = 1.0f / total;
    for (int j = 0; j < GUIDE_LOBES; j++) m.coef[j] = bf16Lo(bf16Bits(d.lambda[j])) * inv * vmfNormPacked(kappa[j]);
    m.weights = make_uint4(w[0], w[1], w[2], w[3]);
    m.alpha = d.alpha;
    m.invTotal = inv;
    m.pad[0] = m.pad[1] = 0.0f;
    return m;
}

// Loss of one sample and its gradient with respect to the 48 raw outputs
// (unused ones zero), scaled by `scale`.  Two terms, as in neural parametric
// mixtures (Dong et al. 2023): the mixture q learns the target distribution
// alone, -y log q(w); the selection probability a learns the MIS combination,
// -y log(a q(w) + (1 - a) pb), with q held fixed.  The returned loss is the
// second (the cross entropy of the distribution that is sampled).
// The gradient is written as BF16 to out[0..GUIDE_OUTPUTS) (the unused
// outputs and clamped concentrations zero), one lobe at a time, so nothing of
// it is held in an indexed local array.
// The training step's gradient is rounded to BF16, so the fast intrinsics
// (errors near 1e-6 relative on the concentrations' range [e^-3, e^5] and
// on angles in [0, 2 pi]) stand in for the precise library functions.
__device__ float lossGradient(const float *o, float3 w, float pb, float y, float scale, uint16_t *out) {
    const Decoded d = decode(o);
    float v[GUIDE_LOBES], q = 0.0f;
    float kappa[GUIDE_LOBES], cosw[GUIDE_LOBES];
#pragma unroll
    for (int j = 0; j < GUIDE_LOBES; j++) {
        const float3 mu = lobeMeanPacked(d, j);
        kappa[j] = __expf(d.logKappa[j]);
        cosw[j] = dot(mu, w);
        v[j] = vmfNormPacked(kappa[j]) * __expf(kappa[j] * (cosw[j] - 1.0f));
        q += d.lambda[j] * v[j];
    }
    const float a = d.alpha;
    const float pmix = fmaxf(a * q + (1.0f - a) * pb, 1e-20f);
    const float loss = -y * __logf(pmix);
    for (int c = 4 * GUIDE_LOBES + 1; c < GUIDE_OUTPUTS; c++) out[c] = 0;
    // selection probability: a = amin + (amax - amin) sigmoid(z)
    out[4 * GUIDE_LOBES] = toBf16(-y / pmix * scale * (q - pb) * (GUIDE_ALPHA_MAX - GUIDE_ALPHA_MIN) * d.alphaSig *
                                  (1.0f - d.alphaSig));
    const float gq = -y / fmaxf(q, 1e-20f) * scale;  // dL/dq of -y log q
#pragma unroll
    for (int j = 0; j < GUIDE_LOBES; j++) {
        // softmax weights
        out[4 * j + 3] = toBf16(gq * d.lambda[j] * (v[j] - q));
        const float gv = gq * d.lambda[j];  // dL/dv_j
        // concentration: dv/dk = v (1/k - 2 / (e^{2k} - 1) + cos - 1), dk/dlogk = k
        float gk = 0.0f;
        if (!d.kappaClamped[j]) {
            const float k = kappa[j];  // e^{2k} - 1 >= 0.105 for k >= e^-3: no cancellation to guard
            const float dlogC = __fdividef(1.0f, k) - __fdividef(2.0f, __expf(2.0f * k) - 1.0f);
            gk = gv * v[j] * (dlogC + cosw[j] - 1.0f) * k;
        }
        out[4 * j + 2] = toBf16(gk);
        // mean direction: dv/dmu = v k w; mu(theta, phi)
        const float gmu = gv * v[j] * kappa[j];
        float st, ct, sp, cp;
        __sincosf(M_PI_F * d.st[j], &st, &ct);
        __sincosf(2.0f * M_PI_F * d.sp[j], &sp, &cp);
        const float3 dmu_dtheta = make_float3(ct * cp, ct * sp, -st);
        const float3 dmu_dphi = make_float3(-st * sp, st * cp, 0.0f);
        out[4 * j + 0] = toBf16(gmu * dot(w, dmu_dtheta) * M_PI_F * d.st[j] * (1.0f - d.st[j]));
        out[4 * j + 1] = toBf16(gmu * dot(w, dmu_dphi) * 2.0f * M_PI_F * d.sp[j] * (1.0f - d.sp[j]));
    }
    return loss;
}

// A training batch: records 0..n-1 of `rec` when n covers all `total` stored
// records, else n draws (with replacement) from them by a hash of the step.
struct RecordBatch {
    const GuideRecord *rec;
    uint32_t total, n, seed;
    __device__ const GuideRecord &pick(uint32_t i) const {
        if (n >= total) return rec[i];
        uint32_t h = (i * 0x9E3779B1u) ^ (seed * 0x85EBCA77u);
        h ^= h >> 16;
        h *= 0x7feb352du;
        h ^= h >> 15;
        h *= 0x846ca68bu;
        h ^= h >> 16;
        return rec[h % total];
    }
};

// one-blob value of bin `bin` of a feature with `bins` bins
__device__ __forceinline__ float oneBlob(float v, int bins, int bin) {
    const float d = v * (float)bins - ((float)bin + 0.5f);
    const float x = fmaxf(0.0f, 1.0f - d * d);
    return x * x;
}

// ------------------------------------------------ tcgen05 inference core
// Inference on the 5th-generation tensor cores.  A CTA runs kTcPipes
// independent pipelines of 128 threads; each pipeline takes 128 samples at a
// time (M = 128), one thread per sample, and the pipelines share one copy of
// the weights in shared memory.  Each layer is tcgen05.mma (kind::f16, BF16
// operands from shared memory, FP32 accumulator in the pipeline's 64 columns
// of tensor memory) issued by the pipeline's first thread; its completion is
// committed to the pipeline's mbarrier; every thread then reads its own
// sample's row of the accumulator (tcgen05.ld, TMEM lane = sample), applies
// bias and ReLU and writes the BF16 row back to shared memory as the next
// layer's A operand.  The output layer's row stays in the thread's
// registers, so each thread decodes and packs its own sample's mixture.
// While one pipeline runs its epilogue, the tensor core serves the others.
//
// Operand layout (the canonical K-major, no-swizzle layout of the UMMA
// shared-memory descriptor): 8 x 16-byte "core matrices" (8 rows, 8 BF16
// along K); element (r, k) of a [rows][K] operand sits at byte
// (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2, SBO = K / 8 * 128.
constexpr int kTcPipes = 4;
constexpr int kTcPipeThreads = 128;
constexpr int kTcThreads = kTcPipes * kTcPipeThreads;
constexpr uint32_t kTmemCols = 64 * kTcPipes;
constexpr int kTcSpinLimit = 1 << 22;  // bounded waits: on expiry the pipeline flags an error and stops

struct TcSmem {
    uint16_t w1[GUIDE_HIDDEN * GUIDE_INPUTS];
    uint16_t w2[GUIDE_HIDDEN * GUIDE_HIDDEN];
    uint16_t w3[GUIDE_HIDDEN * GUIDE_HIDDEN];
    uint16_t w4[GUIDE_OUTPUTS * GUIDE_HIDDEN];
    uint16_t a[kTcPipes][kTcPipeThreads * GUIDE_INPUTS];  // each pipeline's A operand (inputs, then hidden)
    float b[3 * GUIDE_HIDDEN + GUIDE_OUTPUTS];
    unsigned long long mbar[kTcPipes];
    uint32_t tmemBase;
    int failed[kTcPipes];
};

__device__ __forceinline__ uint32_t smemU32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Programmatic dependent launch: a kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization may start while the
// kernel before it in the stream finishes; it waits here, before reading
// anything that kernel wrote, until that grid has completed and its writes
// are visible (no wait for a kernel launched the ordinary way).  The other
// lets the next such kernel be scheduled before this one ends.
__device__ __forceinline__ void gridDependencyWait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void gridDependentsMayLaunch() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// (lo + blo, hi + bhi) with ReLU as packed BF16 (round to nearest even), hi
// in the upper half: one paired FP32 add and one converting ReLU
__device__ __forceinline__ uint32_t biasReluBf16x2(float lo, float hi, float2 bias) {
    uint32_t r;
    asm("{\n.reg .b64 x, y;\n.reg .f32 l, h;\n"
        "mov.b64 x, {%1, %2};\nmov.b64 y, {%3, %4};\nadd.rn.f32x2 x, x, y;\nmov.b64 {l, h}, x;\n"
        "cvt.rn.relu.bf16x2.f32 %0, h, l;\n}\n"
        : "=r"(r)
        : "f"(lo), "f"(hi), "f"(bias.x), "f"(bias.y));
    return r;
}

// BF16 of a float, round to nearest even
__device__ __forceinline__ uint16_t cvtBf16(float x) {
    uint16_t r;
    asm("cvt.rn.bf16.f32 %0, %1;\n" : "=h"(r) : "f"(x));
    return r;
}

// paired FP32 add of two bias values
__device__ __forceinline__ void addBias2(float &lo, float &hi, float2 bias) {
    asm("{\n.reg .b64 x, y;\nmov.b64 x, {%0, %1};\nmov.b64 y, {%2, %3};\nadd.rn.f32x2 x, x, y;\n"
        "mov.b64 {%0, %1}, x;\n}\n"
        : "+f"(lo), "+f"(hi)
        : "f"(bias.x), "f"(bias.y));
}

// byte offset of element (r, k) in a K-major canonical operand of width K
__host__ __device__ __forceinline__ uint32_t canonOffset(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// UMMA shared-memory descriptor, no swizzle: leading and stride byte offsets
// (K-major: LBO between the 8-element K chunks, SBO between 8-row groups;
// MN-major: LBO between 8-deep K groups, SBO between 8-element MN chunks)
__device__ __forceinline__ uint64_t ummaDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3fffu);
    d |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;  // leading byte offset
    d |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;  // stride byte offset
    d |= (uint64_t)1 << 46;                       // descriptor version (sm_100)
    return d;                                     // base offset 0, layout type 0 (no swizzle)
}
// K-major with the two K chunks of an instruction 128 B apart
__device__ __forceinline__ uint64_t ummaDesc(uint32_t addr, uint32_t sbo) { return ummaDesc(addr, 128u, sbo); }

// instruction descriptor, kind::f16: BF16 A and B (K-major), FP32 D, M x N
__device__ __forceinline__ uint32_t ummaInstr(int M, int N) {
    return (1u << 4)                       // D format: F32
           | (1u << 7) | (1u << 10)        // A, B format: BF16
           | ((uint32_t)(N >> 3) << 17)    // N / 8
           | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void umma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void ummaCommit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
                 : "memory");
}

// waits for the mbarrier phase; false after kTcSpinLimit polls
__device__ __forceinline__ bool mbarWait(uint32_t mbar, uint32_t phase) {
    for (int i = 0; i < kTcSpinLimit; i++) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// barrier of one pipeline's 128 threads (named barrier 1 + pipe)
__device__ __forceinline__ void pipeSync(int pipe) {
    asm volatile("bar.sync %0, %1;\n" ::"r"(1 + pipe), "r"(kTcPipeThreads) : "memory");
}
// pipeline barrier that also tells whether any of its threads passed true
__device__ __forceinline__ bool pipeAny(int pipe, bool v) {
    uint32_t r;
    asm volatile(
        "{\n.reg .pred p, q;\nsetp.ne.b32 p, %1, 0;\nbar.red.or.pred q, %2, %3, p;\nselp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(1 + pipe), "r"(kTcPipeThreads)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void tmemLd32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmemLd16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmemLdWait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
// the wait, with v[0..32) tied to it, so no use of them moves above it
__device__ __forceinline__ void tmemLdWaitFor(float *v) {
    asm volatile("tcgen05.wait::ld.sync.aligned;\n"
                 : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]), "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]), "+f"(v[15]), "+f"(v[16]), "+f"(v[17]), "+f"(v[18]), "+f"(v[19]), "+f"(v[20]), "+f"(v[21]), "+f"(v[22]), "+f"(v[23]), "+f"(v[24]), "+f"(v[25]), "+f"(v[26]), "+f"(v[27]), "+f"(v[28]), "+f"(v[29]), "+f"(v[30]), "+f"(v[31])
                 :
                 : "memory");
}
__device__ __forceinline__ void tcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void asyncProxyFence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// copies a row-major [rows][K] bf16 weight matrix into the canonical layout
__device__ void loadCanonical(uint16_t *dst, const uint16_t *src, int rows, int K) {
    const int chunks = K / 8;
    for (int i = threadIdx.x; i < rows * chunks; i += blockDim.x) {
        const int r = i / chunks, c = i - r * chunks;
        *reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(dst) + canonOffset(r, 8 * c, K)) =
            __ldg(reinterpret_cast<const uint4 *>(&src[r * K + 8 * c]));
    }
}

// The CTA's set-up: weights and biases into shared memory, the pipelines'
// mbarriers, and kTmemCols columns of tensor memory (warp 0 allocates).
__device__ void tcSetup(TcSmem &sm, const GuideNetView &net) {
    loadCanonical(sm.w1, net.w[0], GUIDE_HIDDEN, GUIDE_INPUTS);
    loadCanonical(sm.w2, net.w[1], GUIDE_HIDDEN, GUIDE_HIDDEN);
    loadCanonical(sm.w3, net.w[2], GUIDE_HIDDEN, GUIDE_HIDDEN);
    loadCanonical(sm.w4, net.w[3], GUIDE_OUTPUTS, GUIDE_HIDDEN);
    for (int i = threadIdx.x; i < 3 * GUIDE_HIDDEN + GUIDE_OUTPUTS; i += blockDim.x) {
        const int l = min(i / GUIDE_HIDDEN, 3);
        sm.b[i] = __ldg(&net.b[l][i - l * GUIDE_HIDDEN]);
    }
    if (threadIdx.x == 0) {
        for (int p = 0; p < kTcPipes; p++) {
            sm.failed[p] = 0;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smemU32(&sm.mbar[p])), "r"(1) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smemU32(&sm.tmemBase)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asyncProxyFence();
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
}

__device__ void tcTeardown(TcSmem &sm, int pipe, uint32_t phase) {
    if (sm.failed[pipe]) mbarWait(smemU32(&sm.mbar[pipe]), phase);  // a last bounded wait for work in flight
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(sm.tmemBase), "r"(kTmemCols)
                     : "memory");
}

// One layer of a pipeline: D (its TMEM columns) = A (its sm.a, [128][K]) x
// W^T (W [N][K]); the pipeline's first thread issues, all its threads wait.
// False if the wait expired (the pipeline then stops).
__device__ bool tcLayer(TcSmem &sm, int pipe, const uint16_t *w, int K, int N, uint32_t &phase) {
    asyncProxyFence();  // the A rows written by the pipeline's threads, visible to the tensor core
    tcFenceBefore();
    pipeSync(pipe);
    tcFenceAfter();
    const uint32_t mbar = smemU32(&sm.mbar[pipe]);
    if ((threadIdx.x & (kTcPipeThreads - 1)) == 0) {
        const uint32_t idesc = ummaInstr(kTcPipeThreads, N);
        const uint32_t aBase = smemU32(sm.a[pipe]), bBase = smemU32(w);
        const uint32_t sbo = (uint32_t)(K / 8) * 128u;
        const uint32_t tmem = sm.tmemBase + 64u * pipe;
        for (int kb = 0; kb < K / 16; kb++)
            umma(tmem, ummaDesc(aBase + kb * 256u, sbo), ummaDesc(bBase + kb * 256u, sbo), idesc, kb > 0);
        ummaCommit(mbar);
    }
    // on expiry `phase` stays that of the commit in flight, which the
    // teardown's last bounded wait then waits for
    const bool ok = mbarWait(mbar, phase);
    if (ok) phase ^= 1u;
    tcFenceAfter();
    if (!ok) atomicExch(&sm.failed[pipe], 1);
    pipeSync(pipe);
    return sm.failed[pipe] == 0;
}

// bias + ReLU of a 64-wide hidden row from TMEM, written as the next A row
__device__ void tcHiddenEpilogue(uint16_t *a, uint32_t taddr, const float *bias, int row) {
    float v[32];
#pragma unroll
    for (int half = 0; half < 2; half++) {
        tmemLd32(taddr + 32u * half, v);
        tmemLdWait();
#pragma unroll
        for (int c = 0; c < 32; c += 8) {
            uint32_t q[4];
#pragma unroll
            for (int k = 0; k < 4; k++)
                q[k] = biasReluBf16x2(v[c + 2 * k], v[c + 2 * k + 1],
                                      *reinterpret_cast<const float2 *>(&bias[32 * half + c + 2 * k]));
            *reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(a) +
                                       canonOffset(row, 32 * half + c, GUIDE_HIDDEN)) = make_uint4(q[0], q[1], q[2], q[3]);
        }
    }
}

// Forward pass of a pipeline's 128 samples (its thread r: sample r, features
// f); writes the 48 raw outputs to `o`.  False if a wait expired.
__device__ bool tcForward(TcSmem &sm, int pipe, const GuideFeatures &f, float *o, uint32_t &phase) {
    const int row = threadIdx.x & (kTcPipeThreads - 1);
    uint16_t *a = sm.a[pipe];
    // one-blob input row.  A feature v with b bins is non-zero only in bins
    // floor(v b - 1/2) and the one after (|v b - (bin + 1/2)| < 1), so the
    // row is cleared and those two bins of each of the 7 features written.
    unsigned char *aRow = reinterpret_cast<unsigned char *>(a);
#pragma unroll
    for (int c = 0; c < GUIDE_INPUTS / 8; c++)
        *reinterpret_cast<uint4 *>(aRow + canonOffset(row, 8 * c, GUIDE_INPUTS)) = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int feature = 0; feature < 7; feature++) {
        const int bins = feature < 3 ? 32 : 16;
        const int first = feature < 3 ? 32 * feature : 96 + 16 * (feature - 3);
        const float v = f.v[feature];
        const int b = (int)floorf(v * (float)bins - 0.5f);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int bin = b + k;
            if (bin >= 0 && bin < bins)
                *reinterpret_cast<uint16_t *>(aRow + canonOffset(row, first + bin, GUIDE_INPUTS)) =
                    cvtBf16(oneBlob(v, bins, bin));
        }
    }
    // this warp's 32 lanes (its quarter of the pipeline's rows) in the pipeline's 64 columns
    const uint32_t taddr = sm.tmemBase + 64u * pipe + ((uint32_t)(row & ~31) << 16);
    if (!tcLayer(sm, pipe, sm.w1, GUIDE_INPUTS, GUIDE_HIDDEN, phase)) return false;
    tcHiddenEpilogue(a, taddr, sm.b, row);
    if (!tcLayer(sm, pipe, sm.w2, GUIDE_HIDDEN, GUIDE_HIDDEN, phase)) return false;
    tcHiddenEpilogue(a, taddr, sm.b + GUIDE_HIDDEN, row);
    if (!tcLayer(sm, pipe, sm.w3, GUIDE_HIDDEN, GUIDE_HIDDEN, phase)) return false;
    tcHiddenEpilogue(a, taddr, sm.b + 2 * GUIDE_HIDDEN, row);
    if (!tcLayer(sm, pipe, sm.w4, GUIDE_HIDDEN, GUIDE_OUTPUTS, phase)) return false;
    tmemLd32(taddr, o);
    tmemLd16(taddr + 32u, o + 32);
    tmemLdWait();
    const float2 *b4 = reinterpret_cast<const float2 *>(sm.b + 3 * GUIDE_HIDDEN);
#pragma unroll
    for (int c = 0; c < GUIDE_OUTPUTS / 2; c++) addBias2(o[2 * c], o[2 * c + 1], b4[c]);
    return true;
}

// ------------------------------------------------- tcgen05 training core
// Training on the 5th-generation tensor cores.  A CTA of 128 threads takes
// tiles of 128 records, one thread per record (M = 128).  Per tile:
//
//   forward   4 layers as in inference (A = the previous layer's rows, B = W);
//             every layer's input rows stay in shared memory for the
//             backward pass, and every thread keeps its record's ReLU masks
//   loss      each thread the gradient of its record's loss with respect to
//             the 48 raw outputs (CUDA cores), as delta rows
//   backward  per layer l = 3..0: dW_l += delta_l^T . a_(l-1), contracting
//             the 128 records, accumulated in tensor memory over the CTA's
//             tiles; and delta_(l-1) = (delta_l . W_l) masked by ReLU',
//             both issued together
//
// Every operand is a [rows][features] buffer in the canonical no-swizzle
// layout with K along the features (8 x 16-byte core matrices).  Read
// K-major it is an operand whose M or N is the rows; read MN-major (UMMA
// descriptor bits 15/16, leading offset = the 8-row groups, stride offset =
// the 8-feature chunks) the same bytes are the operand whose K is the rows.
// So the record-contracted weight gradients read the delta and activation
// rows as they are (A and B MN-major, K = records), and delta . W_l reads
// the forward weights as W_l^T (B MN-major): nothing is stored transposed.
// The weight gradients' M is the layer's output width (64, or 48) padded to
// 128: the extra rows read the bytes after the delta buffer (the other delta
// buffer, then the input rows) and land in tensor-memory lanes that are
// never read.  Tensor memory: columns 0..63 the layer accumulator, then dW0
// (160), dW1, dW2, dW3 (64 each).  Bias gradients (column sums of the
// deltas) are reduced across each warp with shuffles into shared memory.  At
// the end warps 0 and 1 (lanes 0..63, the output features) read the CTA's
// weight gradient out of tensor memory into the CTA's slot of net.partials.
constexpr int kTrThreads = 128;
constexpr uint32_t kTrTmemCols = 512;
// tensor-memory column of dW_l: dW0 at 64 (160 wide), dW1 224, dW2 288, dW3 352
__device__ __forceinline__ uint32_t trColDw(int l) { return l == 0 ? 64u : 224u + 64u * (uint32_t)(l - 1); }

struct TrainSmem {
    uint16_t w0[GUIDE_HIDDEN * GUIDE_INPUTS];  // [out][in], canonical (K = in): the weight image
    uint16_t w1[GUIDE_HIDDEN * GUIDE_HIDDEN];
    uint16_t w2[GUIDE_HIDDEN * GUIDE_HIDDEN];
    uint16_t w3[GUIDE_OUTPUTS * GUIDE_HIDDEN];
    uint16_t d[2][kTrThreads * GUIDE_HIDDEN];  // delta rows [record][feature], ping-pong (delta_3 is 48 wide)
    uint16_t x[kTrThreads * GUIDE_INPUTS];     // one-blob input rows; follows the deltas (see above)
    uint16_t h[3][kTrThreads * GUIDE_HIDDEN];  // hidden activation rows, the inputs of layers 1..3
    float b[3 * GUIDE_HIDDEN + GUIDE_OUTPUTS];
    float db[3 * GUIDE_HIDDEN + GUIDE_OUTPUTS];  // the CTA's bias gradient
    float reduce[8];                             // per warp: loss sums
    unsigned long long mbar;
    uint32_t tmemBase;
    int failed;
};
static_assert(sizeof(TrainSmem) <= 232448, "training shared memory exceeds the per-CTA limit");
static_assert(GUIDE_PARAMS % 4 == 0 && (GUIDE_HIDDEN * GUIDE_INPUTS + GUIDE_HIDDEN) % 4 == 0 &&
                  (GUIDE_HIDDEN * GUIDE_HIDDEN + GUIDE_HIDDEN) % 4 == 0,
              "a CTA's gradient slot and its layers start on 16-byte boundaries");
// the weight image (GuideNetView::image) is TrainSmem's leading weight region
constexpr uint32_t kImageBytes = (uint32_t)offsetof(TrainSmem, d);
static_assert(offsetof(TrainSmem, w0) == 0 && kImageBytes % 16 == 0 &&
                  kImageBytes == sizeof(uint16_t) * GUIDE_WEIGHTS,
              "the weight image must be the contiguous weight region of the training CTA's shared memory");
// An MN-major A of M = 128 over a delta buffer of width F reads up to byte
// 15 * 16F + 2047 from its start (16 record groups of 16F bytes, 16 chunks of
// 128 bytes): at most 2 KB past the buffer, which must stay inside TrainSmem.
static_assert(offsetof(TrainSmem, x) == offsetof(TrainSmem, d) + sizeof(uint16_t) * 2 * kTrThreads * GUIDE_HIDDEN &&
                  sizeof(uint16_t) * kTrThreads * GUIDE_INPUTS >= 2048,
              "the padded delta rows of a weight gradient must read inside shared memory");

// Sum over the warp's 32 lanes of each of v[0..31]: afterwards lane l holds
// the sum of column l in v[0] (a butterfly that halves the columns a lane
// keeps at every step: 31 shuffles for 32 columns).
__device__ __forceinline__ float warpColumnSums(float v[32], int lane) {
#pragma unroll
    for (int s = 16, n = 32; s >= 1; s >>= 1, n >>= 1) {
        const bool upper = (lane & s) != 0;
#pragma unroll
        for (int k = 0; k < n / 2; k++) {
            const float send = upper ? v[k] : v[k + n / 2];
            const float keep = upper ? v[k + n / 2] : v[k];
            v[k] = keep + __shfl_xor_sync(0xffffffffu, send, s);
        }
    }
    return v[0];
}

// adds the column sums of 32 delta values per thread to db[c0..c0+32)
__device__ __forceinline__ void addBiasGrad(float *db, int c0, float v[32], int lane) {
    const float sum = warpColumnSums(v, lane);
    atomicAdd(&db[c0 + lane], sum);
}

// One operand of a training MMA: a [rows][F] canonical buffer read K-major
// (M or N = the rows, K = the F features) or MN-major (M or N = the F
// features, K = the rows); kStep: bytes per 16-deep K step.
struct TrOperand {
    uint32_t addr, lbo, sbo, kStep, mnMajor;
};
__device__ __forceinline__ TrOperand kMajor(const void *rows, int F) {
    return {smemU32(rows), 128u, (uint32_t)F * 16u, 256u, 0u};
}
__device__ __forceinline__ TrOperand mnMajor(const void *rows, int F) {
    return {smemU32(rows), (uint32_t)F * 16u, 128u, (uint32_t)F * 32u, 1u};
}

// issues D (tmem) = A . B^T over K, N columns (accumulating if asked); committed later
__device__ __forceinline__ void trMma(uint32_t tmem, TrOperand a, TrOperand b, int K, int N, bool accumulate) {
    const uint32_t idesc = ummaInstr(kTrThreads, N) | (a.mnMajor << 15) | (b.mnMajor << 16);
    for (int kb = 0; kb < K / 16; kb++)
        umma(tmem, ummaDesc(a.addr + kb * a.kStep, a.lbo, a.sbo), ummaDesc(b.addr + kb * b.kStep, b.lbo, b.sbo),
             idesc, (accumulate || kb > 0) ? 1u : 0u);
}

// makes the threads' shared-memory writes visible to the tensor core and syncs the CTA
__device__ __forceinline__ void trPublish() {
    asyncProxyFence();
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
}

// thread 0 commits the issued MMAs; everyone waits.  False if the wait expired.
__device__ bool trCommitWait(TrainSmem &sm, uint32_t &phase) {
    const uint32_t mbar = smemU32(&sm.mbar);
    if (threadIdx.x == 0) ummaCommit(mbar);
    const bool ok = mbarWait(mbar, phase);
    if (ok) phase ^= 1u;  // else the teardown waits for the commit in flight
    tcFenceAfter();
    if (!ok) atomicExch(&sm.failed, 1);
    __syncthreads();
    return sm.failed == 0;
}

// Epilogue of a forward hidden layer: bias + ReLU of the thread's row of the
// accumulator, written as the next layer's A row (kept for the backward
// pass); returns the ReLU mask (bit c: column c positive).
// The epilogues run three times per tile, and a CTA traces its code once per
// Adam step: kept out of line and not unrolled over the two column halves, so
// the second and later calls find their instructions cached (instruction
// fetch, not the tensor cores, bounds a step).
__device__ __noinline__ uint64_t trHiddenEpilogue(uint32_t taddr, const float *bias, uint16_t *rowOut, int row) {
    uint64_t mask = 0;
    float v[32];
#pragma unroll 1
    for (int half = 0; half < 2; half++) {
        tmemLd32(taddr + 32u * half, v);
        tmemLdWait();
#pragma unroll
        for (int c = 0; c < 32; c += 8) {
            uint32_t q[4];
#pragma unroll
            for (int k = 0; k < 4; k++)
                q[k] = biasReluBf16x2(v[c + 2 * k], v[c + 2 * k + 1],
                                      *reinterpret_cast<const float2 *>(&bias[32 * half + c + 2 * k]));
            *reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(rowOut) +
                                       canonOffset(row, 32 * half + c, GUIDE_HIDDEN)) = make_uint4(q[0], q[1], q[2], q[3]);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int col = 32 * half + c + 2 * k;
                mask |= (uint64_t)((q[k] & 0xffffu) != 0u) << col;
                mask |= (uint64_t)((q[k] >> 16) != 0u) << (col + 1);
            }
        }
    }
    return mask;
}

// Epilogue of a backward layer: the thread's row of delta . W masked by the
// ReLU mask, as BF16 delta rows; bias gradient into db[0..64).
__device__ __noinline__ void trDeltaEpilogue(uint32_t taddr, uint64_t mask, uint16_t *rowOut, float *db, int row,
                                             int lane) {
    float v[32];
#pragma unroll 1
    for (int half = 0; half < 2; half++) {
        tmemLd32(taddr + 32u * half, v);
        tmemLdWait();
#pragma unroll
        for (int c = 0; c < 32; c += 2) {
            const int col = 32 * half + c;
            const float a = ((mask >> col) & 1u) ? v[c] : 0.0f;
            const float b = ((mask >> (col + 1)) & 1u) ? v[c + 1] : 0.0f;
            const uint16_t lo = cvtBf16(a), hi = cvtBf16(b);
            *reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(rowOut) +
                                          canonOffset(row, col, GUIDE_HIDDEN)) = (uint32_t)lo | ((uint32_t)hi << 16);
            v[c] = fromBf16(lo);  // the bias gradient sums the rounded deltas the MMAs use
            v[c + 1] = fromBf16(hi);
        }
        addBiasGrad(db, 32 * half, v, lane);
    }
}

// The sum of a batch's targets (the loss normalises them by their mean),
// one block per Adam step of a burst: block b sums the batch drawn with seed
// batch.seed + b into sums[b].  No atomics, so nothing to clear first.
constexpr int kSumThreads = 1024;
__global__ void __launch_bounds__(kSumThreads) k_guide_sum_y(RecordBatch batch, float *sums) {
    __shared__ float part[kSumThreads / 32];
    batch.seed += blockIdx.x;
    float s = 0.0f;
#pragma unroll 8
    for (uint32_t i = threadIdx.x; i < batch.n; i += kSumThreads) s += batch.pick(i).y;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = part[threadIdx.x];
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (threadIdx.x == 0) sums[blockIdx.x] = s;
    }
}

// The gradient of the mean loss over a batch of records on the tensor cores:
// each CTA writes its gradient (weights and biases) to its slot of
// net.partials and its share of the loss to partials[GUIDE_PARTIAL_LOSS + CTA];
// the Adam (or reduce) kernel sums them.  On an expired wait the CTA sets
// ERR_GUIDE_TIMEOUT in *errors and writes a zero gradient.
__global__ void __launch_bounds__(kTrThreads, 1) k_guide_train_tc(RecordBatch batch, const float *sumY,
                                                                GuideNetView net, uint32_t *errors) {
    extern __shared__ __align__(16) unsigned char smem[];
    TrainSmem &sm = *reinterpret_cast<TrainSmem *>(smem);
    const int row = threadIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    gridDependencyWait();  // the previous Adam step's weights (launched overlapped with it)
    // set-up: the weights (forward and transposed, already in their shared-
    // memory layout) arrive by one bulk copy on the mbarrier's phase 0 while
    // the biases load, the tensor memory is allocated and the inputs encode
    if (threadIdx.x == 0) {
        sm.failed = 0;
        const uint32_t mbar = smemU32(&sm.mbar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(kImageBytes)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                         smemU32(sm.w0)),
                     "l"(net.image), "r"(kImageBytes), "r"(mbar)
                     : "memory");
    }
    for (int i = threadIdx.x; i < 3 * GUIDE_HIDDEN + GUIDE_OUTPUTS; i += blockDim.x) {
        const int l = min(i / GUIDE_HIDDEN, 3);
        sm.b[i] = __ldg(&net.b[l][i - l * GUIDE_HIDDEN]);
        sm.db[i] = 0.0f;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smemU32(&sm.tmemBase)),
                     "r"(kTrTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    trPublish();
    const uint32_t tmem = sm.tmemBase;
    const uint32_t taddr = tmem + ((uint32_t)(row & ~31) << 16);  // this warp's lanes, work columns
    const uint32_t n = batch.n;
    const float scale = 1.0f / (float)n;
    const float invMeanY = sumY[0] > 0.0f ? (float)n / sumY[0] : 0.0f;
    const uint32_t tiles = (n + kTrThreads - 1) / kTrThreads;
    float lossSum = 0.0f;
    uint32_t phase = 0;
    bool first = true, ok = true;
    {  // the weight image (phase 0); the MMA commits follow on phase 1, 0, ...
        const bool arrived = mbarWait(smemU32(&sm.mbar), phase);
        if (arrived) phase ^= 1u;  // else the teardown waits for the copy in flight
        else atomicExch(&sm.failed, 1);
        __syncthreads();
        ok = sm.failed == 0;
    }
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t r = tile * kTrThreads + row;
        GuideRecord rc = {};
        const bool valid = r < n;
        if (valid) rc = batch.pick(r);
        // inputs: one-blob rows (two non-zero bins per feature)
        unsigned char *xRow = reinterpret_cast<unsigned char *>(sm.x);
#pragma unroll
        for (int c = 0; c < GUIDE_INPUTS / 8; c++)
            *reinterpret_cast<uint4 *>(xRow + canonOffset(row, 8 * c, GUIDE_INPUTS)) = make_uint4(0u, 0u, 0u, 0u);
        if (valid) {
#pragma unroll
            for (int feature = 0; feature < 7; feature++) {
                const int bins = feature < 3 ? 32 : 16;
                const int firstCol = feature < 3 ? 32 * feature : 96 + 16 * (feature - 3);
                const float v = rc.features[feature];
                const int b = (int)floorf(v * (float)bins - 0.5f);
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int bin = b + k;
                    if (bin >= 0 && bin < bins)
                        *reinterpret_cast<uint16_t *>(xRow + canonOffset(row, firstCol + bin, GUIDE_INPUTS)) =
                            cvtBf16(oneBlob(v, bins, bin));
                }
            }
        }
        // forward: every layer's input rows stay for the backward pass
        trPublish();
        if (threadIdx.x == 0)
            trMma(tmem, kMajor(sm.x, GUIDE_INPUTS), kMajor(sm.w0, GUIDE_INPUTS), GUIDE_INPUTS, GUIDE_HIDDEN, false);
        if (!(ok = trCommitWait(sm, phase))) break;
        const uint64_t m0 = trHiddenEpilogue(taddr, sm.b, sm.h[0], row);
        trPublish();
        if (threadIdx.x == 0)
            trMma(tmem, kMajor(sm.h[0], GUIDE_HIDDEN), kMajor(sm.w1, GUIDE_HIDDEN), GUIDE_HIDDEN, GUIDE_HIDDEN, false);
        if (!(ok = trCommitWait(sm, phase))) break;
        const uint64_t m1 = trHiddenEpilogue(taddr, sm.b + GUIDE_HIDDEN, sm.h[1], row);
        trPublish();
        if (threadIdx.x == 0)
            trMma(tmem, kMajor(sm.h[1], GUIDE_HIDDEN), kMajor(sm.w2, GUIDE_HIDDEN), GUIDE_HIDDEN, GUIDE_HIDDEN, false);
        if (!(ok = trCommitWait(sm, phase))) break;
        const uint64_t m2 = trHiddenEpilogue(taddr, sm.b + 2 * GUIDE_HIDDEN, sm.h[2], row);
        trPublish();
        if (threadIdx.x == 0)
            trMma(tmem, kMajor(sm.h[2], GUIDE_HIDDEN), kMajor(sm.w3, GUIDE_HIDDEN), GUIDE_HIDDEN, GUIDE_OUTPUTS, false);
        if (!(ok = trCommitWait(sm, phase))) break;
        float o[GUIDE_OUTPUTS];
        tmemLd32(taddr, o);
        tmemLd16(taddr + 32u, o + 32);
        tmemLdWait();
        const float2 *b4 = reinterpret_cast<const float2 *>(sm.b + 3 * GUIDE_HIDDEN);
#pragma unroll
        for (int c = 0; c < GUIDE_OUTPUTS / 2; c++) addBias2(o[2 * c], o[2 * c + 1], b4[c]);
        // loss gradient of the record (zero for the padding rows of the last tile)
        uint16_t d3[GUIDE_OUTPUTS];
        if (valid) {
            const float y = fminf(rc.y * invMeanY, 100.0f);
            lossSum += lossGradient(o, make_float3(rc.dir[0], rc.dir[1], rc.dir[2]), rc.pdfBsdf, y, scale, d3);
        } else {
#pragma unroll
            for (int c = 0; c < GUIDE_OUTPUTS; c++) d3[c] = 0;
        }
        {  // delta_3 rows (48 wide) into d[0], and its bias gradient
            unsigned char *dRow = reinterpret_cast<unsigned char *>(sm.d[0]);
#pragma unroll
            for (int c = 0; c < GUIDE_OUTPUTS; c += 8)
                *reinterpret_cast<uint4 *>(dRow + canonOffset(row, c, GUIDE_OUTPUTS)) =
                    make_uint4(pack2(d3[c], d3[c + 1]), pack2(d3[c + 2], d3[c + 3]), pack2(d3[c + 4], d3[c + 5]),
                               pack2(d3[c + 6], d3[c + 7]));
            float v[32];
#pragma unroll
            for (int c = 0; c < 32; c++) v[c] = fromBf16(d3[c]);
            addBiasGrad(sm.db + 3 * GUIDE_HIDDEN, 0, v, lane);
#pragma unroll
            for (int c = 0; c < 32; c++) v[c] = c < GUIDE_OUTPUTS - 32 ? fromBf16(d3[32 + c]) : 0.0f;
            const float sum = warpColumnSums(v, lane);
            if (lane < GUIDE_OUTPUTS - 32) atomicAdd(&sm.db[3 * GUIDE_HIDDEN + 32 + lane], sum);
        }
        // backward: layer 3 (dW3, delta2), 2 (dW2, delta1), 1 (dW1, delta0), 0 (dW0); the weight
        // gradients read delta and activation rows MN-major (K = the records), delta . W_l reads
        // the forward W_l MN-major (as W_l^T)
        trPublish();
        if (threadIdx.x == 0) {
            trMma(tmem + trColDw(3), mnMajor(sm.d[0], GUIDE_OUTPUTS), mnMajor(sm.h[2], GUIDE_HIDDEN), kTrThreads,
                  GUIDE_HIDDEN, !first);
            trMma(tmem, kMajor(sm.d[0], GUIDE_OUTPUTS), mnMajor(sm.w3, GUIDE_HIDDEN), GUIDE_OUTPUTS, GUIDE_HIDDEN,
                  false);
        }
        if (!(ok = trCommitWait(sm, phase))) break;
        trDeltaEpilogue(taddr, m2, sm.d[1], sm.db + 2 * GUIDE_HIDDEN, row, lane);
        trPublish();
        if (threadIdx.x == 0) {
            trMma(tmem + trColDw(2), mnMajor(sm.d[1], GUIDE_HIDDEN), mnMajor(sm.h[1], GUIDE_HIDDEN), kTrThreads,
                  GUIDE_HIDDEN, !first);
            trMma(tmem, kMajor(sm.d[1], GUIDE_HIDDEN), mnMajor(sm.w2, GUIDE_HIDDEN), GUIDE_HIDDEN, GUIDE_HIDDEN,
                  false);
        }
        if (!(ok = trCommitWait(sm, phase))) break;
        trDeltaEpilogue(taddr, m1, sm.d[0], sm.db + GUIDE_HIDDEN, row, lane);
        trPublish();
        if (threadIdx.x == 0) {
            trMma(tmem + trColDw(1), mnMajor(sm.d[0], GUIDE_HIDDEN), mnMajor(sm.h[0], GUIDE_HIDDEN), kTrThreads,
                  GUIDE_HIDDEN, !first);
            trMma(tmem, kMajor(sm.d[0], GUIDE_HIDDEN), mnMajor(sm.w1, GUIDE_HIDDEN), GUIDE_HIDDEN, GUIDE_HIDDEN,
                  false);
        }
        if (!(ok = trCommitWait(sm, phase))) break;
        trDeltaEpilogue(taddr, m0, sm.d[1], sm.db, row, lane);
        trPublish();
        if (threadIdx.x == 0)
            trMma(tmem + trColDw(0), mnMajor(sm.d[1], GUIDE_HIDDEN), mnMajor(sm.x, GUIDE_INPUTS), kTrThreads,
                  GUIDE_INPUTS, !first);
        if (!(ok = trCommitWait(sm, phase))) break;
        first = false;
    }
    gridDependentsMayLaunch();  // the Adam step's blocks may be scheduled (they wait for this grid's gradient)
    // the CTA's gradient: weights from tensor memory (lanes = output features), biases from shared memory.
    // A warp's 32 rows x 32 columns go through shared memory (the input rows, free once the last MMA has
    // read them; rows padded to 36 floats, so neither side meets a bank conflict) and leave as four
    // 128-byte row pieces per store instruction instead of 32 scattered 16-byte pieces.
    float *part = net.partials + (size_t)blockIdx.x * GUIDE_PARAMS;
    const bool have = ok && !first;
    if (warp < 2) {
        const uint32_t lanes = (uint32_t)(warp * 32) << 16;
        constexpr int kPitch = 36;  // floats per staged row
        static_assert(2 * 32 * kPitch * sizeof(float) <= sizeof(TrainSmem::x), "gradient staging fits the input rows");
        float *stage = reinterpret_cast<float *>(sm.x) + warp * 32 * kPitch;
        // the 11 blocks of 32 columns: layer 0 (160 inputs) five, layers 1-3 two each
        auto layerOf = [](int q) { return q < 5 ? 0 : 1 + (q - 5) / 2; };
        auto colOf = [](int q) { return q < 5 ? 32 * q : 32 * ((q - 5) & 1); };
        auto load = [&](int q, float *v) {
            if (have) {
                tmemLd32(tmem + lanes + trColDw(layerOf(q)) + (uint32_t)colOf(q), v);
            } else {
#pragma unroll
                for (int c = 0; c < 32; c++) v[c] = 0.0f;
            }
        };
        auto store = [&](int q, const float *v) {
            const int l = layerOf(q), c0 = colOf(q);
            const int width = l == 0 ? GUIDE_INPUTS : GUIDE_HIDDEN, outs = l == 3 ? GUIDE_OUTPUTS : GUIDE_HIDDEN;
            float4 *mine = reinterpret_cast<float4 *>(stage + lane * kPitch);
#pragma unroll
            for (int c = 0; c < 32; c += 4) mine[c / 4] = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
            __syncwarp();
            // 16-byte pieces: every layer offset, row width and column block is a multiple of 4 floats
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int r = 4 * k + (lane >> 3), c = 4 * (lane & 7);
                const int o = warp * 32 + r;  // output feature
                if (o < outs)
                    *reinterpret_cast<float4 *>(part + net.wOffset[l] + o * width + c0 + c) =
                        *reinterpret_cast<const float4 *>(stage + r * kPitch + c);
            }
            __syncwarp();
        };
        // the next block's tensor-memory load is in flight while this one is stored
        constexpr int kBlocks = 11;
        float va[32], vb[32];
        load(0, va);
        tmemLdWaitFor(va);
#pragma unroll 1
        for (int q = 0; q < kBlocks; q += 2) {
            if (q + 1 < kBlocks) load(q + 1, vb);
            store(q, va);
            tmemLdWaitFor(vb);
            if (q + 2 < kBlocks) load(q + 2, va);
            if (q + 1 < kBlocks) store(q + 1, vb);
            tmemLdWaitFor(va);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * GUIDE_HIDDEN + GUIDE_OUTPUTS; i += blockDim.x) {
        const int l = min(i / GUIDE_HIDDEN, 3);
        part[net.bOffset[l] + i - l * GUIDE_HIDDEN] = have ? sm.db[i] : 0.0f;
    }
    for (int off = 16; off > 0; off >>= 1) lossSum += __shfl_xor_sync(0xffffffffu, lossSum, off);
    if (lane == 0) sm.reduce[warp] = lossSum;
    __syncthreads();
    if (threadIdx.x == 0)
        net.partials[GUIDE_PARTIAL_LOSS + blockIdx.x] =
            ok ? (sm.reduce[0] + sm.reduce[1] + sm.reduce[2] + sm.reduce[3]) * scale : 0.0f;
    if (!ok && threadIdx.x == 0 && errors) atomicOr(errors, ERR_GUIDE_TIMEOUT);
    // teardown: a last bounded wait for work in flight after an expired wait, then free tensor memory
    if (!ok) mbarWait(smemU32(&sm.mbar), phase);
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTrTmemCols) : "memory");
}

// ------------------------------------------------------------------ kernels
// The guide's input features of this iteration's hits (shading order
// 0..nHit-1): position on the ray, the triangle's geometric normal, the
// reversed ray direction (as the shading kernel computes them) and the
// path's depth, stored by shading-order position.  A light kernel of
// dependent gathers at full occupancy, so the inference kernel reads one
// coalesced 16-byte record per hit.
__global__ void __launch_bounds__(256) k_guide_features(Context ctx, PathPool pool, Counters *cnt, uint32_t p,
                                                        uint32_t guideDepth) {
    const uint32_t nHit = cnt->nHit;
    const PathState S = pool.s[p];
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nHit; q += gridDim.x * blockDim.x) {
        const uint32_t idx = pool.order[q];
        const uint32_t depth = __float_as_uint(S.L[idx].w) & 0xffffu;
        GuideFeatures f = {};
        if (depth < guideDepth) {  // only guided vertices need the features
            // a batch path's scene is its view's (the view in the top bits of its sample word)
            const Context &c = pool.views ? pool.views[__ldg(&S.id[idx].y) >> BATCH_SAMPLE_BITS].ctx : ctx;
            const float4 o = __ldcs(&S.rayO[idx]), dd = __ldcs(&S.rayD[idx]), h = pool.hit[idx];
            const PerInstanceData &inst = c.instances[pool.hitInst[idx]];
            const uint4 face = c.faces[inst.faceOffset + __float_as_uint(h.w)];
            const float3 Pc = xyz(c.vertices[inst.vertexOffset + face.z]);
            const float3 P0 = xyz(c.vertices[inst.vertexOffset + face.x]) - Pc;
            const float3 P1 = xyz(c.vertices[inst.vertexOffset + face.y]) - Pc;
            const float3 n = normalize(mul3(inst.normalTransform, cross(P0, P1)));
            f = guideFeatures(xyz(o) + xyz(dd) * h.x, n, -xyz(dd), pool.guideMin, pool.guideInvExtent);
        }
        pool.guideFeat[q] = packFeatures(f, depth);
    }
}

// Guide mixtures of the shading points of this iteration's hits on paths
// shallower than guideDepth, by shading-order position (the shading kernel's
// thread for hit q reads mixture q), from the features k_guide_features
// stored; tcgen05 tiles of 128 samples.  On an expired wait the CTA sets
// ERR_GUIDE_TIMEOUT in the counters and stops.
__global__ void __launch_bounds__(kTcThreads) k_guide_infer(Counters *cnt, const uint4 *features, uint32_t guideDepth,
                                                         GuideNetView net, GuideMixture *out) {
    extern __shared__ __align__(16) unsigned char smem[];
    TcSmem &sm = *reinterpret_cast<TcSmem *>(smem);
    tcSetup(sm, net);
    const int pipe = threadIdx.x / kTcPipeThreads, row = threadIdx.x & (kTcPipeThreads - 1);
    const uint32_t nHit = cnt->nHit;
    const uint32_t tiles = (nHit + kTcPipeThreads - 1) / kTcPipeThreads;
    uint32_t phase = 0;
    for (uint32_t tile = blockIdx.x * kTcPipes + pipe; tile < tiles; tile += gridDim.x * kTcPipes) {
        const uint32_t q = tile * kTcPipeThreads + row;
        uint4 packed = make_uint4(0u, 0u, 0u, 0xffff0000u);
        if (q < nHit) packed = __ldcs(&features[q]);
        const bool valid = q < nHit && (packed.w >> 16) < guideDepth;
        if (!pipeAny(pipe, valid)) continue;  // no guided vertex in this tile
        const GuideFeatures f = unpackFeatures(packed);
        float o[GUIDE_OUTPUTS];
        if (!tcForward(sm, pipe, f, o, phase)) {
            if (row == 0) atomicOr(&cnt->errors, ERR_GUIDE_TIMEOUT);
            break;
        }
        // The tile's 128 mixtures are one contiguous block of `out`: staged in
        // the pipeline's A buffer (free once the last layer's MMA has read it),
        // each row's eight 16-byte chunks rotated by the row so that 8
        // consecutive rows store to different banks, then copied out by the
        // pipeline with coalesced stores.  Rows past the guided depth are
        // written too; shading reads a mixture only at guided depths.
        union {
            GuideMixture m;
            uint4 c[8];
        } mix;
        static_assert(sizeof(GuideMixture) == 8 * sizeof(uint4), "a mixture is eight 16-byte chunks");
        mix.m = pack(decode(o));
        uint4 *stage = reinterpret_cast<uint4 *>(sm.a[pipe]);
#pragma unroll
        for (int j = 0; j < 8; j++) stage[row * 8 + (j ^ (row & 7))] = mix.c[j];
        pipeSync(pipe);
        const uint32_t first = tile * kTcPipeThreads;
        const uint32_t chunks = min((uint32_t)kTcPipeThreads, nHit - first) * 8u;
        uint4 *dst = reinterpret_cast<uint4 *>(out + first);
        for (uint32_t k = row; k < chunks; k += kTcPipeThreads) dst[k] = stage[(k & ~7u) + ((k & 7u) ^ ((k >> 3) & 7u))];
        pipeSync(pipe);  // the next tile's input rows overwrite the stage
    }
    tcTeardown(sm, pipe, phase);
}

// the training CTAs' loss shares summed into *lossOut (the first warp of block 0)
__device__ __forceinline__ void sumLoss(const GuideNetView &net, int blocks, float *lossOut) {
    if (blockIdx.x != 0 || threadIdx.x >= 32 || !lossOut) return;
    float loss = 0.0f;
    for (int b = (int)threadIdx.x; b < blocks; b += 32) loss += net.partials[GUIDE_PARTIAL_LOSS + b];
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, off);
    if (threadIdx.x == 0) *lossOut = loss;
}

// net.grad += the sum of the training blocks' gradients
__global__ void k_guide_reduce(GuideNetView net, int blocks, float *lossOut) {
    sumLoss(net, blocks, lossOut);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= GUIDE_PARAMS) return;
    float g = 0.0f;
    for (int b = 0; b < blocks; b++) g += net.partials[(size_t)b * GUIDE_PARAMS + i];
    net.grad[i] += g;
}

// Parameter i's BF16 copies: row-major and in the weight image (a bias has none).
__device__ __forceinline__ void storeBf16Weight(const GuideNetView &net, int i, float w) {
    if (net.bf16Index[i] < 0) return;
    const uint16_t q = (uint16_t)bf16Bits(w);
    net.weightsBf16[net.bf16Index[i]] = q;
    net.image[net.imageIndex[i]] = q;
}

static_assert(GUIDE_INPUTS == 5 * 32 && GUIDE_HIDDEN == 2 * 32 && GUIDE_OUTPUTS <= GUIDE_HIDDEN,
              "the gradient write-out walks 5 + 2 + 2 + 2 blocks of 32 columns");
constexpr int kAdamSplit = 8;  // a power of two, at most 32 (one warp's lanes)
// Adam step on every parameter; refreshes the bf16 weight copies and clears
// the gradient.  kAdamSplit threads per parameter (neighbouring lanes) each
// sum every kAdamSplit-th of the blocks' gradient slots, so a thread waits
// on a fraction of the loads.
__global__ void k_guide_adam(GuideNetView net, int blocks, float lr, float beta1, float beta2, float eps, float corr1,
                             float corr2, float *lossOut) {
    gridDependencyWait();  // the training blocks' gradient slots (launched overlapped with them)
    gridDependentsMayLaunch();
    sumLoss(net, blocks, lossOut);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / kAdamSplit, part = t % kAdamSplit;
    float gr = 0.0f;
    if (i < GUIDE_PARAMS)
        for (int b = part; b < blocks; b += kAdamSplit) gr += net.partials[(size_t)b * GUIDE_PARAMS + i];
    for (int off = 1; off < kAdamSplit; off <<= 1) gr += __shfl_xor_sync(0xffffffffu, gr, off);
    if (i >= GUIDE_PARAMS || part != 0) return;
    gr += net.grad[i];
    const float m = beta1 * net.adamM[i] + (1.0f - beta1) * gr;
    const float v = beta2 * net.adamV[i] + (1.0f - beta2) * gr * gr;
    net.adamM[i] = m;
    net.adamV[i] = v;
    const float w = net.master[i] - lr * (m * corr1) / (sqrtf(v * corr2) + eps);
    net.master[i] = w;
    net.grad[i] = 0.0f;
    storeBf16Weight(net, i, w);
}

// Test hook: forward pass of explicit feature vectors through the inference
// core (tcgen05), raw outputs; status[0] = 1 if a wait expired.
__global__ void __launch_bounds__(kTcThreads) k_guide_forward_test(const float *features, uint32_t n, GuideNetView net,
                                                                float *out, int *status) {
    extern __shared__ __align__(16) unsigned char smem[];
    TcSmem &sm = *reinterpret_cast<TcSmem *>(smem);
    tcSetup(sm, net);
    const int pipe = threadIdx.x / kTcPipeThreads, row = threadIdx.x & (kTcPipeThreads - 1);
    const uint32_t tiles = (n + kTcPipeThreads - 1) / kTcPipeThreads;
    uint32_t phase = 0;
    for (uint32_t tile = blockIdx.x * kTcPipes + pipe; tile < tiles; tile += gridDim.x * kTcPipes) {
        const uint32_t q = tile * kTcPipeThreads + row;
        GuideFeatures f = {};
        if (q < n)
            for (int k = 0; k < 7; k++) f.v[k] = features[7 * q + k];
        float o[GUIDE_OUTPUTS];
        if (!tcForward(sm, pipe, f, o, phase)) {
            if (row == 0) atomicExch(status, 1);
            break;
        }
        if (q < n)
            for (int c = 0; c < GUIDE_OUTPUTS; c++) out[GUIDE_OUTPUTS * q + c] = o[c];
    }
    tcTeardown(sm, pipe, phase);
}

// Uploaded parameters: clear Adam and the gradient, refresh the bf16 copies.
__global__ void k_guide_refresh(GuideNetView net) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= GUIDE_PARAMS) return;
    net.adamM[i] = 0.0f;
    net.adamV[i] = 0.0f;
    net.grad[i] = 0.0f;
    storeBf16Weight(net, i, net.master[i]);
}

// Test hook: the packed mixture of one output vector, n samples with their
// pdf and the pdf at m query directions.
__global__ void k_guide_mixture_test(const float *outputs, const float *u, int n, float *dirsPdf, const float *queries,
                                     int m, float *pdfs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n && i >= m) return;
    const GuideMixture mix = pack(decode(outputs));
    if (i < n) {
        const float3 d = guideSample(&mix, make_float3(u[3 * i], u[3 * i + 1], u[3 * i + 2]));
        dirsPdf[4 * i + 0] = d.x;
        dirsPdf[4 * i + 1] = d.y;
        dirsPdf[4 * i + 2] = d.z;
        dirsPdf[4 * i + 3] = guidePdf(&mix, d);
    }
    if (i < m) pdfs[i] = guidePdf(&mix, make_float3(queries[3 * i], queries[3 * i + 1], queries[3 * i + 2]));
}

}  // namespace
}  // namespace rmd

using namespace rmd;

size_t rmdGuideSharedBytes(bool training) { return training ? sizeof(TrainSmem) : sizeof(TcSmem); }

cudaError_t rmdGuideConfigure() {
    cudaError_t e = cudaFuncSetAttribute(k_guide_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)rmdGuideSharedBytes(true));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)rmdGuideSharedBytes(false));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_guide_forward_test, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)rmdGuideSharedBytes(false));
}

cudaError_t rmdLaunchGuideInfer(const Context &ctx, const PathPool &pool, Counters *cnt, uint32_t cur,
                                uint32_t guideDepth, const GuideNetView &net, GuideMixture *out, int blocks,
                                cudaStream_t s) {
    k_guide_features<<<pool.capacity / 256 < 1184u ? pool.capacity / 256 + 1 : 1184, 256, 0, s>>>(ctx, pool, cnt, cur,
                                                                                              guideDepth);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_guide_infer<<<blocks, kTcThreads, rmdGuideSharedBytes(false), s>>>(cnt, pool.guideFeat, guideDepth, net, out);
    return cudaGetLastError();
}

constexpr float kAdamBeta1 = 0.9f, kAdamBeta2 = 0.999f;
// Adam's bias corrections 1 / (1 - beta^step)
static void adamCorrections(int step, float &corr1, float &corr2) {
    corr1 = 1.0f / (1.0f - powf(kAdamBeta1, (float)step));
    corr2 = 1.0f / (1.0f - powf(kAdamBeta2, (float)step));
}

// Launches `kernel` allowed to start while the kernel before it in the
// stream finishes (programmatic dependent launch); the kernel waits for that
// grid before reading its results (gridDependencyWait).
template <class... Params, class... Args>
static cudaError_t launchOverlapped(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                   Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
}

cudaError_t rmdLaunchGuideTrain(const GuideRecord *rec, uint32_t total, uint32_t n, uint32_t seed, uint32_t steps,
                                const GuideNetView &net, float *scratch, int blocks, float lr, int step,
                                uint32_t *errors, cudaStream_t s) {
    // scratch[1]: the last step's mean loss (written by the Adam step);
    // scratch[kSumSlots .. 2 kSumSlots): the target sums of up to kSumSlots steps
    constexpr uint32_t kSumSlots = 32;
    if (total == 0) return cudaSuccess;
    RecordBatch batch{rec, total, std::min(n, total), seed};
    // one CTA per tile of 128 records, at most `blocks` (each CTA then takes several tiles)
    const int tiles = (int)((batch.n + kTrThreads - 1) / kTrThreads);
    blocks = std::max(1, std::min(std::min(blocks, tiles), GUIDE_TRAIN_MAX_BLOCKS));
    cudaError_t e = cudaSuccess;
    for (uint32_t k = 0; k < steps; k++) {
        float *sums = scratch + kSumSlots;
        if (k % kSumSlots == 0) {  // the batches of the next kSumSlots steps (the ring does not change meanwhile)
            RecordBatch first = batch;
            first.seed = seed + k;
            k_guide_sum_y<<<std::min(kSumSlots, steps - k), kSumThreads, 0, s>>>(first, sums);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        batch.seed = seed + k;
        // each step's two kernels overlap the tail of the one before (programmatic dependent launch)
        if ((e = launchOverlapped(k_guide_train_tc, dim3(blocks), dim3(kTrThreads), rmdGuideSharedBytes(true), s, batch,
                                  (const float *)(sums + k % kSumSlots), net, errors)) != cudaSuccess)
            return e;
        float corr1, corr2;
        adamCorrections(step + (int)k, corr1, corr2);
        if ((e = launchOverlapped(k_guide_adam, dim3((kAdamSplit * GUIDE_PARAMS + 255) / 256), dim3(256), 0, s, net,
                                  blocks, lr, kAdamBeta1, kAdamBeta2, 1e-8f, corr1, corr2, scratch + 1)) != cudaSuccess)
            return e;
    }
    return e;
}

cudaError_t rmdLaunchGuideAdam(const GuideNetView &net, int blocks, float lr, int step, float *lossOut,
                               cudaStream_t s) {
    float corr1, corr2;
    adamCorrections(step, corr1, corr2);
    k_guide_adam<<<(kAdamSplit * GUIDE_PARAMS + 255) / 256, 256, 0, s>>>(net, blocks, lr, kAdamBeta1, kAdamBeta2, 1e-8f,
                                                                         corr1, corr2, lossOut);
    return cudaGetLastError();
}

cudaError_t rmdLaunchGuideForwardTest(const float *features, uint32_t n, const GuideNetView &net, float *out,
                                      int *status, cudaStream_t s) {
    const int blocks = (int)std::min<uint32_t>(148, (n + kTcThreads - 1) / kTcThreads);
    k_guide_forward_test<<<std::max(1, blocks), kTcThreads, rmdGuideSharedBytes(false), s>>>(features, n, net, out,
                                                                                             status);
    return cudaGetLastError();
}

cudaError_t rmdLaunchGuideGradientTest(const GuideRecord *rec, uint32_t n, const GuideNetView &net, float *scratch,
                                       int blocks, cudaStream_t s) {
    // scratch[0]: target sum, [1]: mean loss, [2]: error flags
    cudaError_t e = cudaMemsetAsync(scratch, 0, 3 * sizeof(float), s);
    if (e != cudaSuccess || n == 0) return e;
    RecordBatch batch{rec, n, n, 0};
    k_guide_sum_y<<<1, kSumThreads, 0, s>>>(batch, scratch);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int tiles = (int)((n + kTrThreads - 1) / kTrThreads);
    blocks = std::max(1, std::min(std::min(blocks, tiles), GUIDE_TRAIN_MAX_BLOCKS));
    k_guide_train_tc<<<blocks, kTrThreads, rmdGuideSharedBytes(true), s>>>(batch, scratch, net,
                                                                           reinterpret_cast<uint32_t *>(scratch + 2));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_guide_reduce<<<(GUIDE_PARAMS + 255) / 256, 256, 0, s>>>(net, blocks, scratch + 1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- host side
namespace rmdhost {

void GuideNet::layout(int wOffset[4], int bOffset[4], int bf16Offset[4]) {
    const int in[4] = {GUIDE_INPUTS, GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_HIDDEN};
    const int out[4] = {GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_OUTPUTS};
    int p = 0, q = 0;
    for (int l = 0; l < 4; l++) {
        wOffset[l] = p;
        bf16Offset[l] = q;
        p += in[l] * out[l];
        q += in[l] * out[l];
        bOffset[l] = p;
        p += out[l];
    }
}

void GuideNet::release() {
    for (void *ptr : {(void *)master, (void *)adamM, (void *)adamV, (void *)grad, (void *)scratch,
                      (void *)partials, (void *)weightsBf16, (void *)bf16Index, (void *)image, (void *)imageIndex})
        if (ptr) cudaFree(ptr);
    master = adamM = adamV = grad = scratch = partials = nullptr;
    weightsBf16 = nullptr;
    bf16Index = nullptr;
    image = nullptr;
    imageIndex = nullptr;
}

cudaError_t GuideNet::allocate() {
    release();
    const size_t pb = GUIDE_PARAMS * sizeof(float);
    cudaError_t e;
    if ((e = cudaMalloc(&master, pb)) != cudaSuccess || (e = cudaMalloc(&adamM, pb)) != cudaSuccess ||
        (e = cudaMalloc(&adamV, pb)) != cudaSuccess || (e = cudaMalloc(&grad, pb)) != cudaSuccess ||
        (e = cudaMalloc(&scratch, 64 * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&partials, (size_t)GUIDE_TRAIN_MAX_BLOCKS * (pb + sizeof(float)))) != cudaSuccess ||
        (e = cudaMalloc(&weightsBf16, GUIDE_WEIGHTS * sizeof(uint16_t))) != cudaSuccess ||
        (e = cudaMalloc(&bf16Index, GUIDE_PARAMS * sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&image, kImageBytes)) != cudaSuccess ||
        (e = cudaMalloc(&imageIndex, GUIDE_PARAMS * sizeof(int))) != cudaSuccess)
        return e;
    std::vector<int> idx(GUIDE_PARAMS, -1), img(GUIDE_PARAMS, -1);
    int wOff[4], bOff[4], qOff[4];
    layout(wOff, bOff, qOff);
    const int in[4] = {GUIDE_INPUTS, GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_HIDDEN};
    const int out[4] = {GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_OUTPUTS};
    const size_t fwd[4] = {offsetof(TrainSmem, w0), offsetof(TrainSmem, w1), offsetof(TrainSmem, w2),
                           offsetof(TrainSmem, w3)};
    for (int l = 0; l < 4; l++)
        for (int o = 0; o < out[l]; o++)
            for (int k = 0; k < in[l]; k++) {
                const int p = wOff[l] + o * in[l] + k;
                idx[p] = qOff[l] + o * in[l] + k;
                img[p] = (int)((fwd[l] + canonOffset(o, k, in[l])) / sizeof(uint16_t));  // row o, K = inputs
            }
    if ((e = cudaMemcpy(bf16Index, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(imageIndex, img.data(), img.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    return rmdGuideConfigure();
}

cudaError_t GuideNet::setParams(const float *host, cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(master, host, GUIDE_PARAMS * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    k_guide_refresh<<<(GUIDE_PARAMS + 255) / 256, 256, 0, s>>>(view(make_float3(0, 0, 0), make_float3(1, 1, 1)));
    steps = 0;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

cudaError_t GuideNet::getParams(float *host, cudaStream_t s) const {
    cudaError_t e = cudaMemcpyAsync(host, master, GUIDE_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

GuideNetView GuideNet::view(float3 sceneMin, float3 sceneInvExtent) const {
    GuideNetView v;
    int qOff[4];
    layout(v.wOffset, v.bOffset, qOff);
    for (int l = 0; l < 4; l++) {
        v.w[l] = weightsBf16 + qOff[l];
        v.b[l] = master + v.bOffset[l];
    }
    v.master = master;
    v.adamM = adamM;
    v.adamV = adamV;
    v.grad = grad;
    v.partials = partials;
    v.weightsBf16 = weightsBf16;
    v.bf16Index = bf16Index;
    v.image = image;
    v.imageIndex = imageIndex;
    v.sceneMin = sceneMin;
    v.sceneInvExtent = sceneInvExtent;
    return v;
}

void GuideNet::initParams(float *params, uint32_t seed) {
    uint64_t state = 0x9E3779B97F4A7C15ull ^ seed;
    auto uniform = [&]() {  // splitmix64 -> [0, 1)
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    const int in[4] = {GUIDE_INPUTS, GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_HIDDEN};
    const int out[4] = {GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_HIDDEN, GUIDE_OUTPUTS};
    int wOff[4], bOff[4], qOff[4];
    layout(wOff, bOff, qOff);
    for (int l = 0; l < 4; l++) {
        const double a = std::sqrt(6.0 / (in[l] + out[l]));
        for (int k = 0; k < in[l] * out[l]; k++) params[wOff[l] + k] = (float)((2.0 * uniform() - 1.0) * a);
        for (int k = 0; k < out[l]; k++) params[bOff[l] + k] = 0.0f;
    }
    float *b4 = params + bOff[3];
    for (int j = 0; j < GUIDE_LOBES; j++) b4[4 * j + 2] = 1.0f;  // log kappa
    // alpha = amin + (amax - amin) sigmoid(z) = 0.2
    const double sig = (0.2 - GUIDE_ALPHA_MIN) / (GUIDE_ALPHA_MAX - GUIDE_ALPHA_MIN);
    b4[4 * GUIDE_LOBES] = (float)std::log(sig / (1.0 - sig));
}

}  // namespace rmdhost

// ---------------------------------------------------------------- test hooks
#include "../../include/raymond.h"
#include "../../include/raymond_testing.h"

namespace rmdhost {
rmd_status setLastError(rmd_status status, const char *msg);
}

namespace {
rmd_status guideFail(cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return rmdhost::setLastError(RMD_ERROR_CUDA, m.c_str());
}
struct DeviceArray {
    void *p = nullptr;
    ~DeviceArray() {
        if (p) cudaFree(p);
    }
    cudaError_t upload(const void *h, size_t n) {
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 16));
        if (e != cudaSuccess || n == 0) return e;
        return cudaMemcpy(p, h, n, cudaMemcpyHostToDevice);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 16)); }
};
}  // namespace

extern "C" int32_t rmd_guide_param_count(void) { return GUIDE_PARAMS; }

extern "C" rmd_status rmd_test_guide_forward(const float *params, const float *features, int32_t n, float *out) {
    if (!params || !features || !out || n < 0)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT, "rmd_test_guide_forward: invalid arguments");
    rmdhost::GuideNet net;
    cudaError_t e;
    if ((e = net.allocate()) != cudaSuccess) return guideFail(e, "guide allocate");
    if ((e = net.setParams(params, 0)) != cudaSuccess) return guideFail(e, "guide params");
    DeviceArray f, o, st;
    const int zero = 0;
    if ((e = f.upload(features, (size_t)n * 7 * sizeof(float))) != cudaSuccess ||
        (e = o.alloc((size_t)n * GUIDE_OUTPUTS * sizeof(float))) != cudaSuccess ||
        (e = st.upload(&zero, sizeof(int))) != cudaSuccess)
        return guideFail(e, "guide buffers");
    int status = 0;
    if ((e = rmdLaunchGuideForwardTest((const float *)f.p, (uint32_t)n,
                                       net.view(make_float3(0, 0, 0), make_float3(1, 1, 1)), (float *)o.p, (int *)st.p,
                                       0)) != cudaSuccess ||
        (e = cudaMemcpy(out, o.p, (size_t)n * GUIDE_OUTPUTS * sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(&status, st.p, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return guideFail(e, "guide forward");
    if (status) return rmdhost::setLastError(RMD_ERROR_WATCHDOG, "guide inference: a tensor-core wait expired");
    return RMD_OK;
}

extern "C" rmd_status rmd_test_guide_gradient(const float *params, const float *records, int32_t n, float *grad,
                                              float *loss) {
    if (!params || !records || !grad || n <= 0)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT, "rmd_test_guide_gradient: invalid arguments");
    static_assert(sizeof(GuideRecord) == 12 * sizeof(float), "GuideRecord is 12 floats");
    rmdhost::GuideNet net;
    cudaError_t e;
    if ((e = net.allocate()) != cudaSuccess) return guideFail(e, "guide allocate");
    if ((e = net.setParams(params, 0)) != cudaSuccess) return guideFail(e, "guide params");
    DeviceArray r;
    if ((e = r.upload(records, (size_t)n * sizeof(GuideRecord))) != cudaSuccess) return guideFail(e, "guide records");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    if ((e = rmdLaunchGuideGradientTest((const GuideRecord *)r.p, (uint32_t)n,
                                        net.view(make_float3(0, 0, 0), make_float3(1, 1, 1)), net.scratch, sms, 0)) !=
            cudaSuccess ||
        (e = cudaMemcpy(grad, net.grad, GUIDE_PARAMS * sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return guideFail(e, "guide gradient");
    float s[3];
    if ((e = cudaMemcpy(s, net.scratch, sizeof(s), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return guideFail(e, "guide loss");
    uint32_t flags;
    std::memcpy(&flags, &s[2], sizeof(flags));
    if (flags) return rmdhost::setLastError(RMD_ERROR_WATCHDOG, "guide training: a tensor-core wait expired");
    if (loss) *loss = s[1];
    return RMD_OK;
}

extern "C" rmd_status rmd_test_guide_adam(const float *params, const float *grad, const float *m, const float *v,
                                          int32_t step, float lr, float *params_out, float *m_out, float *v_out,
                                          uint16_t *bf16_out) {
    if (!params || !grad || !m || !v || step < 1 || !params_out || !m_out || !v_out || !bf16_out)
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT, "rmd_test_guide_adam: invalid arguments");
    rmdhost::GuideNet net;
    cudaError_t e;
    const size_t pb = GUIDE_PARAMS * sizeof(float);
    if ((e = net.allocate()) != cudaSuccess) return guideFail(e, "guide allocate");
    if ((e = net.setParams(params, 0)) != cudaSuccess) return guideFail(e, "guide params");
    if ((e = cudaMemcpy(net.grad, grad, pb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(net.adamM, m, pb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(net.adamV, v, pb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = rmdLaunchGuideAdam(net.view(make_float3(0, 0, 0), make_float3(1, 1, 1)), 0, lr, step, nullptr, 0)) !=
            cudaSuccess ||
        (e = cudaMemcpy(params_out, net.master, pb, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(m_out, net.adamM, pb, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(v_out, net.adamV, pb, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(bf16_out, net.weightsBf16, GUIDE_WEIGHTS * sizeof(uint16_t), cudaMemcpyDeviceToHost)) !=
            cudaSuccess)
        return guideFail(e, "guide adam");
    return RMD_OK;
}

extern "C" rmd_status rmd_test_guide_mixture(const float *outputs, const float *u, int32_t n, float *dirsPdf,
                                             const float *queries, int32_t m, float *pdfs) {
    if (!outputs || n < 0 || m < 0 || (n && (!u || !dirsPdf)) || (m && (!queries || !pdfs)))
        return rmdhost::setLastError(RMD_ERROR_INVALID_ARGUMENT, "rmd_test_guide_mixture: invalid arguments");
    DeviceArray o, du, dd, dq, dp;
    cudaError_t e;
    if ((e = o.upload(outputs, GUIDE_OUTPUTS * sizeof(float))) != cudaSuccess ||
        (e = du.upload(u, (size_t)n * 3 * sizeof(float))) != cudaSuccess ||
        (e = dd.alloc((size_t)n * 4 * sizeof(float))) != cudaSuccess ||
        (e = dq.upload(queries, (size_t)m * 3 * sizeof(float))) != cudaSuccess ||
        (e = dp.alloc((size_t)m * sizeof(float))) != cudaSuccess)
        return guideFail(e, "guide mixture buffers");
    const int total = std::max(n, m);
    k_guide_mixture_test<<<(total + 127) / 128 + 1, 128>>>((const float *)o.p, (const float *)du.p, n, (float *)dd.p,
                                                           (const float *)dq.p, m, (float *)dp.p);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (n && (e = cudaMemcpy(dirsPdf, dd.p, (size_t)n * 4 * sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess) ||
        (m && (e = cudaMemcpy(pdfs, dp.p, (size_t)m * sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess))
        return guideFail(e, "guide mixture");
    return RMD_OK;
}
