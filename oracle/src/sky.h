// Oracle (test infrastructure): the Nishita sky of the TEX_SKY node, restated
// on the CPU from the reference's host/sky/sky_nishita.cpp (Blender's
// single-scattering atmosphere) and SkyLoader.mm; checked against that file
// compiled from the reference (oracle/ref) by the pinning tests.
#pragma once

#include <cmath>
#include <vector>

#include "vec.h"

namespace oracle_sky {

using orc::float3;
using orc::float4;

constexpr int NW = 21;  // wavelengths 380..780 nm, sky_nishita.cpp:19-24
constexpr float kEarth = 6360e3f, kAtmosphere = 6420e3f;
constexpr float kPiF = 3.14159265358979323846f;

// sky_nishita.cpp:25-101: spectral data and the Gauss-Laguerre quadrature
static const float kIrradiance[NW] = {
    1.45756829855592995315f, 1.56596305559738380175f, 1.65148449067670455293f, 1.71496242737209314555f,
    1.75797983805020541226f, 1.78256407885924539336f, 1.79095108475838560302f, 1.78541550133410664714f,
    1.76815554864306845317f, 1.74122069647250410362f, 1.70647127164943679389f, 1.66556087452739887134f,
    1.61993437242451854274f, 1.57083597368892080581f, 1.51932335059305478886f, 1.46628494965214395407f,
    1.41245852740172450623f, 1.35844961970384092709f, 1.30474913844739281998f, 1.25174963272610817455f,
    1.19975998755420620867f};
static const float kRayleigh[NW] = {
    0.00005424820087636473f, 0.00004418549866505454f, 0.00003635151910165377f, 0.00003017929012024763f,
    0.00002526320226989157f, 0.00002130859310621843f, 0.00001809838025320633f, 0.00001547057129129042f,
    0.00001330284977336850f, 0.00001150184784075764f, 0.00000999557429990163f, 0.00000872799973630707f,
    0.00000765513700977967f, 0.00000674217203751443f, 0.00000596134125832052f, 0.00000529034598065810f,
    0.00000471115687557433f, 0.00000420910481110487f, 0.00000377218381260133f, 0.00000339051255477280f,
    0.00000305591531679811f};
static const float kOzone[NW] = {
    0.00000000325126849861f, 0.00000000585395365047f, 0.00000001977191155085f, 0.00000007309568762914f,
    0.00000020084561514287f, 0.00000040383958096161f, 0.00000063551335912363f, 0.00000096707041180970f,
    0.00000154797400424410f, 0.00000209038647223331f, 0.00000246128056164565f, 0.00000273551299461512f,
    0.00000215125863128643f, 0.00000159051840791988f, 0.00000112356197979857f, 0.00000073527551487574f,
    0.00000046450130357806f, 0.00000033096079921048f, 0.00000022512612292678f, 0.00000014879129266490f,
    0.00000016828623364192f};
static const float kCmf[NW][3] = {
    {0.00136800000f, 0.00003900000f, 0.00645000100f}, {0.01431000000f, 0.00039600000f, 0.06785001000f},
    {0.13438000000f, 0.00400000000f, 0.64560000000f}, {0.34828000000f, 0.02300000000f, 1.74706000000f},
    {0.29080000000f, 0.06000000000f, 1.66920000000f}, {0.09564000000f, 0.13902000000f, 0.81295010000f},
    {0.00490000000f, 0.32300000000f, 0.27200000000f}, {0.06327000000f, 0.71000000000f, 0.07824999000f},
    {0.29040000000f, 0.95400000000f, 0.02030000000f}, {0.59450000000f, 0.99500000000f, 0.00390000000f},
    {0.91630000000f, 0.87000000000f, 0.00165000100f}, {1.06220000000f, 0.63100000000f, 0.00080000000f},
    {0.85444990000f, 0.38100000000f, 0.00019000000f}, {0.44790000000f, 0.17500000000f, 0.00002000000f},
    {0.16490000000f, 0.06100000000f, 0.00000000000f}, {0.04677000000f, 0.01700000000f, 0.00000000000f},
    {0.01135916000f, 0.00410200000f, 0.00000000000f}, {0.00289932700f, 0.00104700000f, 0.00000000000f},
    {0.00069007860f, 0.00024920000f, 0.00000000000f}, {0.00016615050f, 0.00006000000f, 0.00000000000f},
    {0.00004150994f, 0.00001499000f, 0.00000000000f}};
static const float kNodes[8] = {0.006811185292f, 0.03614807107f, 0.09004346519f, 0.1706680068f,
                                0.2818362161f,  0.4303406404f,  0.6296271457f,  0.9145252695f};
static const float kWeights[8] = {0.01750893642f, 0.04135477391f, 0.06678839063f, 0.09507698807f,
                                  0.1283416365f,  0.1707430204f,  0.2327233347f,  0.3562490486f};

inline float3 direction(float lat, float lon) {  // :103-106
    return float3(std::cos(lat) * std::cos(lon), std::cos(lat) * std::sin(lon), std::sin(lat));
}

inline float3 toXyz(const float *spectrum) {  // :108-118, 20 nm steps
    float3 xyz(0, 0, 0);
    for (int i = 0; i < NW; i++) {
        xyz.x += kCmf[i][0] * spectrum[i];
        xyz.y += kCmf[i][1] * spectrum[i];
        xyz.z += kCmf[i][2] * spectrum[i];
    }
    return xyz * 20.0f;
}

inline float3 density(float h) {  // :120-140: Rayleigh, Mie, ozone
    float ozone = 0.0f;
    if (h >= 10000.0f && h < 25000.0f) ozone = 1.0f / 15000.0f * h - 2.0f / 3.0f;
    else if (h >= 25000 && h < 40000) ozone = -(1.0f / 15000.0f * h - 8.0f / 3.0f);
    return float3(std::exp(-h / 8e3f), std::exp(-h / 1.2e3f), ozone);
}

inline float3 exitPoint(float3 p, float3 d) {  // :168-174
    const float b = -2.0f * dot(d, -p);
    const float c = dot(p, p) - kAtmosphere * kAtmosphere;
    const float t = (-b + std::sqrt(b * b - 4.0f * c)) / 2.0f;
    return float3(p.x + d.x * t, p.y + d.y * t, p.z + d.z * t);
}

inline float3 opticalDepth(float3 p, float3 d) {  // :176-210
    const float L = length(p - exitPoint(p, d));
    const float3 seg = L * d;
    float3 depth(0, 0, 0);
    for (int i = 0; i < 8; i++) depth += density(length(p + kNodes[i] * seg) - kEarth) * kWeights[i];
    return depth * L;
}

inline float3 scatter(float3 dir, float3 sun, float3 eye, float air, float dust, float ozone) {  // :212-293
    const float L = length(eye - exitPoint(eye, dir));
    const float segLen = L / 32;
    const float3 seg = segLen * dir;
    float spectrum[NW] = {};
    const float mu = dot(dir, sun);
    const float g = 0.76f, g2 = g * g;
    const float3 phase(3.0f / (16.0f * kPiF) * (1.0f + mu * mu),
                       (3.0f * (1.0f - g2) * (1.0f + mu * mu)) /
                           (8.0f * kPiF * (2.0f + g2) * std::pow((1.0f + g2 - 2.0f * g * mu), 1.5f)),
                       0.0f);
    const float3 k(air, dust, ozone);
    float3 depth(0, 0, 0);
    float3 p = eye + 0.5f * seg;
    for (int i = 0; i < 32; i++) {
        const float3 dens = k * density(length(p) - kEarth);
        depth += segLen * dens;
        // surface_intersection: the sun below this point's horizon
        bool blocked = false;
        if (sun.z < 0) {
            const float b = -2.0f * dot(sun, -p);
            const float c = dot(p, p) - kEarth * kEarth;
            blocked = b * b - 4.0f * c >= 0.0f;
        }
        if (!blocked) {
            const float3 total = depth + k * opticalDepth(p, sun);
            for (int w = 0; w < NW; w++) {
                const float3 ext = total * float3(kRayleigh[w], 1.11f * 2e-5f, kOzone[w]);
                const float att = std::exp(-(ext.x + ext.y + ext.z));
                const float3 s = dens * float3(kRayleigh[w], 2e-5f, 0.0f);
                const float3 ps = phase * s;
                spectrum[w] += att * (ps.x + ps.y + ps.z) * kIrradiance[w] * segLen;
            }
        }
        p += seg;
    }
    return toXyz(spectrum);
}

// SKY_nishita_skymodel_precompute_texture (:295-341): RGBA float texels, XYZ in rgb, alpha 1
inline std::vector<float4> skyTexture(int W, int H, float elevation, float altitude, float air, float dust,
                                      float ozone) {
    std::vector<float4> t((size_t)W * H, float4(0, 0, 0, 1));
    const float3 eye(0, 0, kEarth + altitude), sun = direction(elevation, 0.0f);
    const float latStep = (kPiF / 2) / H, lonStep = (2 * kPiF) / W;
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; y++) {
        const float f = (float)y / H;
        const float lat = (kPiF / 2 + latStep / 2.0f) * (f * f);
        for (int x = 0; x < W / 2; x++) {
            const float3 c = scatter(direction(lat, lonStep * x - kPiF), sun, eye, air, dust, ozone);
            t[(size_t)y * W + x] = float4(c.x, c.y, c.z, 1);
            t[(size_t)y * W + (W - x - 1)] = float4(c.x, c.y, c.z, 1);
        }
    }
    return t;
}

// SKY_nishita_skymodel_precompute_sun (:344-396) and SkyLoader.generateData:
// the node's ten data values
inline void skyData(float elevation, float rotation, bool disc, float size, float intensity, float altitude, float air,
                    float dust, float out[10]) {
    const float half = size / 2.0f;
    const float solid = 2 * kPiF * (1.0f - std::cos(half));
    const float lo = elevation - half, hi = elevation + half;
    for (int k = 0; k < 2; k++) {
        const float e = k == 0 ? (lo > 0.0f ? lo : 0.0f) : (hi > 0.0f ? hi : 0.0f);
        const float3 depth = opticalDepth(float3(0, 0, kEarth + altitude), direction(e, 0.0f));
        float spectrum[NW];
        for (int w = 0; w < NW; w++)
            spectrum[w] = kIrradiance[w] * std::exp(-(kRayleigh[w] * depth.x * air + 1.11f * 2e-5f * depth.y * dust)) /
                          solid;
        const float3 c = toXyz(spectrum);
        out[3 * k] = c.x;
        out[3 * k + 1] = c.y;
        out[3 * k + 2] = c.z;
    }
    out[6] = elevation;
    out[7] = rotation;
    out[8] = disc ? size : -1.0f;
    out[9] = intensity;
}

}  // namespace oracle_sky
