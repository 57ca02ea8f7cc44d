// Learned path-guiding proposal: a mixture of 8 von Mises-Fisher lobes per
// shading point, predicted by a small MLP from the point's position, normal
// and view direction (the network lives in guide.cu), combined with BSDF
// sampling by one-sample MIS with a learned selection probability.  No
// counterpart in the reference.
//
// Network input (160 values): one-blob encodings (quartic kernel of unit bin
// width) of the position in the scene's bounds (3 x 32 bins), and of the
// normal and the view direction as (theta / pi, phi / 2 pi) (2 x 16 bins
// each).  Output (48, 33 used): per lobe j, 4j + 0 / 1: theta / phi of the
// mean direction (through a sigmoid, scaled to [0, pi] / [0, 2 pi]),
// 4j + 2: log concentration (clamped), 4j + 3: mixture logit (softmax);
// 32: logit of the guide's selection probability.
#pragma once
#include "rt_math.cuh"

namespace rmd {

constexpr int GUIDE_LOBES = 8;
constexpr int GUIDE_INPUTS = 160;
constexpr int GUIDE_HIDDEN = 64;
constexpr int GUIDE_OUTPUTS = 48;
constexpr int GUIDE_USED_OUTPUTS = 4 * GUIDE_LOBES + 1;
// concentrations up to e^5 (lobes of about 5 degrees); selection probability
// of the guide in [0.02, 0.5], so a direction the guide misses keeps at
// least half the BSDF's sampling density
constexpr float GUIDE_LOG_KAPPA_MIN = -3.0f, GUIDE_LOG_KAPPA_MAX = 5.0f;
constexpr float GUIDE_ALPHA_MIN = 0.02f, GUIDE_ALPHA_MAX = 0.5f;

// Packed mixture of one shading point, 128 bytes: lobe j as bf16 pairs
// (mu.x, mu.y), (mu.z, kappa) (mu renormalised on use); its pdf coefficient
// weight_j / sum(weights) * C(kappa_j) in FP32; the 8 selection weights as
// bf16; the selection probability of the guide.  Sampling and pdf read the
// same rounded values, so they describe the same distribution.
struct GuideMixture {
    uint2 lobe[GUIDE_LOBES];
    float coef[GUIDE_LOBES];
    uint4 weights;
    float alpha;     // selection probability of the guide
    float invTotal;  // 1 / sum of the bf16 weights
    float pad[2];
};

RMD_HD uint32_t bf16Bits(float x) {  // round to nearest even
    const uint32_t u = __float_as_uint(x);
    return (u + 0x7fffu + ((u >> 16) & 1u)) >> 16;
}
RMD_HD float bf16Lo(uint32_t w) { return __uint_as_float(w << 16); }
RMD_HD float bf16Hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

// C(kappa) = kappa / (2 pi (1 - exp(-2 kappa))), the vMF normalisation on S2
RMD_HD float vmfNorm(float kappa) { return kappa / (2.0f * M_PI_F * -expm1f(-2.0f * kappa)); }

RMD_HD float3 lobeMu(uint2 l) { return normalize(make_float3(bf16Lo(l.x), bf16Hi(l.x), bf16Lo(l.y))); }

// pdf of the mixture (solid angle)
RMD_HD float guidePdf(const GuideMixture *m, float3 w) {
    float p = 0.0f;
#pragma unroll
    for (int j = 0; j < GUIDE_LOBES; j++) {
        const uint2 l = m->lobe[j];
        p += m->coef[j] * __expf(bf16Hi(l.y) * (dot(lobeMu(l), w) - 1.0f));
    }
    return p;
}

// direction from the mixture: lobe by u.x, then the vMF sample (Wenzel
// Jakob, "Numerically stable sampling of the von Mises Fisher distribution on
// S2", 2012) by u.y, u.z
RMD_HD float3 guideSample(const GuideMixture *m, float3 u) {
    const float target = u.x / m->invTotal;  // the stored weights sum to 1 / invTotal
    const uint4 wq = m->weights;
    float acc = 0.0f;
    int k = GUIDE_LOBES - 1;
    bool found = false;
#pragma unroll
    for (int j = 0; j < GUIDE_LOBES; j++) {
        const uint32_t w = j < 2 ? wq.x : j < 4 ? wq.y : j < 6 ? wq.z : wq.w;
        acc += (j & 1) ? bf16Hi(w) : bf16Lo(w);
        if (!found && target < acc) {
            k = j;
            found = true;
        }
    }
    const uint2 l = m->lobe[k];
    const float kappa = bf16Hi(l.y);
    const float uy = fmaxf(u.y, 1e-7f);
    const float wz = 1.0f + logf(uy + (1.0f - uy) * __expf(-2.0f * kappa)) / kappa;
    const float r = sqrtf(fmaxf(0.0f, 1.0f - wz * wz));
    const float phi = 2.0f * M_PI_F * u.z;
    return normalize(toWorld(buildOrthonormalBasis(lobeMu(l)), make_float3(r * cosf(phi), r * sinf(phi), wz)));
}

// One training sample: a path vertex's features, a direction sampled there,
// the BSDF's pdf of that direction and the radiance-weighted target
// y = f Li cos / p of the direction (luminance as the mean of RGB).
struct GuideRecord {
    float features[7];
    float dir[3];
    float pdfBsdf;
    float y;
};

// Uniform [0, 1) from a path's pixel, sample and depth: the coin of the
// training-record reservoir, kept off the PCG stream.  Mixing function:
// "lowbias32" (C. Wellons, hash-prospector).
RMD_HD float recordHash(uint32_t pixel, uint32_t sample, uint32_t depth) {
    uint32_t h = (pixel * 0x9E3779B1u) ^ ((sample + 0x7F4A7C15u) * 0x85EBCA77u) ^ (depth * 0xC2B2AE3Du);
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

// ------------------------------------------------------------ input encoding
struct GuideFeatures {
    float v[7];  // position x, y, z in [0, 1]; normal theta, phi; view theta, phi, each in [0, 1]
};

RMD_HD float2 sphericalUnit(float3 d) {
    const float theta = acosf(fminf(1.0f, fmaxf(-1.0f, d.z)));
    float phi = atan2f(d.y, d.x);
    if (phi < 0.0f) phi += 2.0f * M_PI_F;
    return make_float2(theta * (1.0f / M_PI_F), phi * (0.5f / M_PI_F));
}

// position relative to the scene bounds; the normal turned towards the viewer
RMD_HD GuideFeatures guideFeatures(float3 position, float3 normal, float3 wo, float3 sceneMin, float3 sceneInvExtent) {
    GuideFeatures f;
    const float3 p = (position - sceneMin) * sceneInvExtent;
    f.v[0] = fminf(1.0f, fmaxf(0.0f, p.x));
    f.v[1] = fminf(1.0f, fmaxf(0.0f, p.y));
    f.v[2] = fminf(1.0f, fmaxf(0.0f, p.z));
    if (dot(normal, wo) < 0.0f) normal = -normal;
    const float2 n = sphericalUnit(normal), w = sphericalUnit(wo);
    f.v[3] = n.x;
    f.v[4] = n.y;
    f.v[5] = w.x;
    f.v[6] = w.y;
    return f;
}

// features in [0, 1] as 16-bit fixed point and the path's depth (the hit's
// record between the feature and inference kernels)
RMD_HD uint4 packFeatures(const GuideFeatures &f, uint32_t depth) {
    uint32_t q[8];
#pragma unroll
    for (int k = 0; k < 7; k++) q[k] = (uint32_t)(fminf(1.0f, fmaxf(0.0f, f.v[k])) * 65535.0f + 0.5f);
    q[7] = min(depth, 0xffffu);  // the path's depth
    return make_uint4(q[0] | (q[1] << 16), q[2] | (q[3] << 16), q[4] | (q[5] << 16), q[6] | (q[7] << 16));
}
RMD_HD GuideFeatures unpackFeatures(uint4 p) {
    GuideFeatures f;
    const uint32_t w[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
    for (int k = 0; k < 7; k++) f.v[k] = (float)((w[k >> 1] >> (16 * (k & 1))) & 0xffffu) * (1.0f / 65535.0f);
    return f;
}

// one-blob value of input `col` (0..159) for the given features
RMD_HD float guideInput(const GuideFeatures &f, int col) {
    int feature, bins, bin;
    if (col < 96) {
        feature = col >> 5;
        bins = 32;
        bin = col & 31;
    } else {
        feature = 3 + ((col - 96) >> 4);
        bins = 16;
        bin = (col - 96) & 15;
    }
    const float d = f.v[feature] * (float)bins - ((float)bin + 0.5f);
    const float x = fmaxf(0.0f, 1.0f - d * d);
    return x * x;
}

}  // namespace rmd
