// The Nishita sky model of the reference's TEX_SKY node: Blender's
// single-scattering atmosphere (raymond/host/sky/sky_nishita.cpp, which the
// reference runs on the host through SkyLoader.mm and
// MaterialBuilder.swift:329-388).  Restated for both sides of this library:
// the host derives the sun-disc parameters the generated shader code carries
// as literals, and a device kernel fills the 512 x 512 sky texture (one
// thread per texel) during scene creation instead of the host loop.
//
// The spectral tables (solar irradiance, Rayleigh and ozone coefficients, CIE
// 1931 colour matching functions at 21 wavelengths) and the 8-node
// Gauss-Laguerre quadrature are physical data and quadrature constants; they
// appear here with the reference's values, since they define the model's
// output.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define SKY_HD __host__ __device__ inline
#else
#define SKY_HD inline
#endif

namespace rmdsky {

constexpr int kSkyWavelengths = 21;
constexpr int kSkySteps = 32;          // segments of the primary ray
constexpr int kSkyQuadrature = 8;      // Gauss-Laguerre nodes of the optical depth
constexpr int kSkyTextureSize = 512;   // the reference's texture is 512 x 512 RGBA float
constexpr float kRayleighScale = 8e3f, kMieScale = 1.2e3f, kMieCoeff = 2e-5f, kMieG = 0.76f;
constexpr float kEarthRadius = 6360e3f, kAtmosphereRadius = 6420e3f;
constexpr float kPi = 3.14159265358979323846f, kHalfPi = 1.57079632679489661923f, kTwoPi = 6.28318530717958647692f;
constexpr float kStepLambda = (780 - 380) / (kSkyWavelengths - 1);

struct SkyTables {
    float irradiance[kSkyWavelengths];  // W m^-2 nm^-1 at the top of the atmosphere
    float rayleigh[kSkyWavelengths];    // m^-1
    float ozone[kSkyWavelengths];       // m^-1
    float cmf[kSkyWavelengths][3];      // CIE XYZ
    float nodes[kSkyQuadrature], weights[kSkyQuadrature];
};

SKY_HD const SkyTables &skyTables() {
    static const SkyTables t = {
        {1.45756829855592995315f, 1.56596305559738380175f, 1.65148449067670455293f, 1.71496242737209314555f,
         1.75797983805020541226f, 1.78256407885924539336f, 1.79095108475838560302f, 1.78541550133410664714f,
         1.76815554864306845317f, 1.74122069647250410362f, 1.70647127164943679389f, 1.66556087452739887134f,
         1.61993437242451854274f, 1.57083597368892080581f, 1.51932335059305478886f, 1.46628494965214395407f,
         1.41245852740172450623f, 1.35844961970384092709f, 1.30474913844739281998f, 1.25174963272610817455f,
         1.19975998755420620867f},
        {0.00005424820087636473f, 0.00004418549866505454f, 0.00003635151910165377f, 0.00003017929012024763f,
         0.00002526320226989157f, 0.00002130859310621843f, 0.00001809838025320633f, 0.00001547057129129042f,
         0.00001330284977336850f, 0.00001150184784075764f, 0.00000999557429990163f, 0.00000872799973630707f,
         0.00000765513700977967f, 0.00000674217203751443f, 0.00000596134125832052f, 0.00000529034598065810f,
         0.00000471115687557433f, 0.00000420910481110487f, 0.00000377218381260133f, 0.00000339051255477280f,
         0.00000305591531679811f},
        {0.00000000325126849861f, 0.00000000585395365047f, 0.00000001977191155085f, 0.00000007309568762914f,
         0.00000020084561514287f, 0.00000040383958096161f, 0.00000063551335912363f, 0.00000096707041180970f,
         0.00000154797400424410f, 0.00000209038647223331f, 0.00000246128056164565f, 0.00000273551299461512f,
         0.00000215125863128643f, 0.00000159051840791988f, 0.00000112356197979857f, 0.00000073527551487574f,
         0.00000046450130357806f, 0.00000033096079921048f, 0.00000022512612292678f, 0.00000014879129266490f,
         0.00000016828623364192f},
        {{0.00136800000f, 0.00003900000f, 0.00645000100f}, {0.01431000000f, 0.00039600000f, 0.06785001000f},
         {0.13438000000f, 0.00400000000f, 0.64560000000f}, {0.34828000000f, 0.02300000000f, 1.74706000000f},
         {0.29080000000f, 0.06000000000f, 1.66920000000f}, {0.09564000000f, 0.13902000000f, 0.81295010000f},
         {0.00490000000f, 0.32300000000f, 0.27200000000f}, {0.06327000000f, 0.71000000000f, 0.07824999000f},
         {0.29040000000f, 0.95400000000f, 0.02030000000f}, {0.59450000000f, 0.99500000000f, 0.00390000000f},
         {0.91630000000f, 0.87000000000f, 0.00165000100f}, {1.06220000000f, 0.63100000000f, 0.00080000000f},
         {0.85444990000f, 0.38100000000f, 0.00019000000f}, {0.44790000000f, 0.17500000000f, 0.00002000000f},
         {0.16490000000f, 0.06100000000f, 0.00000000000f}, {0.04677000000f, 0.01700000000f, 0.00000000000f},
         {0.01135916000f, 0.00410200000f, 0.00000000000f}, {0.00289932700f, 0.00104700000f, 0.00000000000f},
         {0.00069007860f, 0.00024920000f, 0.00000000000f}, {0.00016615050f, 0.00006000000f, 0.00000000000f},
         {0.00004150994f, 0.00001499000f, 0.00000000000f}},
        {0.006811185292f, 0.03614807107f, 0.09004346519f, 0.1706680068f, 0.2818362161f, 0.4303406404f, 0.6296271457f,
         0.9145252695f},
        {0.01750893642f, 0.04135477391f, 0.06678839063f, 0.09507698807f, 0.1283416365f, 0.1707430204f, 0.2327233347f,
         0.3562490486f},
    };
    return t;
}

struct V3 {
    float x, y, z;
};
SKY_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
SKY_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
SKY_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
SKY_HD V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
SKY_HD V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
SKY_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SKY_HD float len(V3 a) { return sqrtf(dot(a, a)); }

// A point on the unit sphere from latitude (elevation) and longitude.
SKY_HD V3 geographicalToDirection(float lat, float lon) {
    return v3(cosf(lat) * cosf(lon), cosf(lat) * sinf(lon), sinf(lat));
}

// Relative densities of air (Rayleigh), aerosols (Mie) and ozone at a height
// above sea level (m); ozone is a tent between 10 and 40 km peaking at 25 km.
SKY_HD V3 densities(float h) {
    float oz = 0.0f;
    if (h >= 10000.0f && h < 25000.0f) oz = 1.0f / 15000.0f * h - 2.0f / 3.0f;
    else if (h >= 25000 && h < 40000) oz = -(1.0f / 15000.0f * h - 8.0f / 3.0f);
    return v3(expf(-h / kRayleighScale), expf(-h / kMieScale), oz);
}

// Does the ray from p towards d meet the ground sphere?
SKY_HD bool hitsGround(V3 p, V3 d) {
    if (d.z >= 0) return false;
    const float b = -2.0f * dot(d, -1.0f * p);
    const float c = dot(p, p) - kEarthRadius * kEarthRadius;
    return b * b - 4.0f * c >= 0.0f;
}

// Where the ray from p (inside the atmosphere) towards d leaves it.
SKY_HD V3 atmosphereExit(V3 p, V3 d) {
    const float b = -2.0f * dot(d, -1.0f * p);
    const float c = dot(p, p) - kAtmosphereRadius * kAtmosphereRadius;
    const float t = (-b + sqrtf(b * b - 4.0f * c)) / 2.0f;
    return v3(p.x + d.x * t, p.y + d.y * t, p.z + d.z * t);
}

// Optical depth (per density type) from p to the top of the atmosphere
// along d: Gauss-Laguerre quadrature with the exponential folded into the
// weights, the nodes scaled to the ray's length inside the atmosphere.
SKY_HD V3 opticalDepth(V3 p, V3 d) {
    const SkyTables &T = skyTables();
    const float length = len(p - atmosphereExit(p, d));
    const V3 segment = length * d;
    V3 depth = v3(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < kSkyQuadrature; i++) {
        const V3 q = p + T.nodes[i] * segment;
        depth = depth + T.weights[i] * densities(len(q) - kEarthRadius);
    }
    return length * depth;
}

SKY_HD float phaseRayleigh(float mu) { return 3.0f / (16.0f * kPi) * (1.0f + mu * mu); }
SKY_HD float phaseMie(float mu) {
    const float g2 = kMieG * kMieG;
    return (3.0f * (1.0f - g2) * (1.0f + mu * mu)) /
           (8.0f * kPi * (2.0f + g2) * powf((1.0f + g2 - 2.0f * kMieG * mu), 1.5f));
}

// CIE XYZ of a spectrum sampled at the 21 wavelengths (step 20 nm)
SKY_HD V3 spectrumToXyz(const float *s) {
    const SkyTables &T = skyTables();
    V3 xyz = v3(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < kSkyWavelengths; i++) {
        xyz.x += T.cmf[i][0] * s[i];
        xyz.y += T.cmf[i][1] * s[i];
        xyz.z += T.cmf[i][2] * s[i];
    }
    return kStepLambda * xyz;
}

// Single in-scattering of sunlight along the view ray from `origin` towards
// `dir`: 32 midpoint segments; at each, the transmittance from the eye and
// towards the sun (unless the ground blocks it) times the Rayleigh and Mie
// scattering and their phase functions.  Returns CIE XYZ.
SKY_HD V3 singleScattering(V3 dir, V3 sunDir, V3 origin, float air, float dust, float ozone) {
    const SkyTables &T = skyTables();
    const float length = len(origin - atmosphereExit(origin, dir));
    const float segLength = length / kSkySteps;
    const V3 segment = segLength * dir;
    float spectrum[kSkyWavelengths];
    for (int w = 0; w < kSkyWavelengths; w++) spectrum[w] = 0.0f;
    const float mu = dot(dir, sunDir);
    const V3 phase = v3(phaseRayleigh(mu), phaseMie(mu), 0.0f);
    const V3 scale = v3(air, dust, ozone);
    V3 depth = v3(0.0f, 0.0f, 0.0f);
    V3 p = origin + 0.5f * segment;
    for (int i = 0; i < kSkySteps; i++) {
        const V3 density = scale * densities(len(p) - kEarthRadius);
        depth = depth + segLength * density;
        if (!hitsGround(p, sunDir)) {
            const V3 total = depth + scale * opticalDepth(p, sunDir);
            for (int w = 0; w < kSkyWavelengths; w++) {
                const V3 ext = total * v3(T.rayleigh[w], 1.11f * kMieCoeff, T.ozone[w]);
                const float attenuation = expf(-(ext.x + ext.y + ext.z));
                const V3 scat = density * v3(T.rayleigh[w], kMieCoeff, 0.0f);
                const V3 ps = phase * scat;
                spectrum[w] += attenuation * (ps.x + ps.y + ps.z) * T.irradiance[w] * segLength;
            }
        }
        p = p + segment;
    }
    return spectrumToXyz(spectrum);
}

// Texel (x, y) of the sky texture (width x height, x < width / 2; the other
// half mirrors it): rows sample the elevation quadratically (more rows near
// the horizon), columns the azimuth from -pi.
SKY_HD V3 skyTexel(int x, int y, int width, int height, float sunElevation, float altitude, float air, float dust,
                   float ozone) {
    const float latStep = kHalfPi / height;
    const float lonStep = kTwoPi / width;
    const float t = (float)y / height;
    const float latitude = (kHalfPi + latStep / 2.0f) * (t * t);
    const float longitude = lonStep * x - kPi;
    return singleScattering(geographicalToDirection(latitude, longitude), geographicalToDirection(sunElevation, 0.0f),
                            v3(0, 0, kEarthRadius + altitude), air, dust, ozone);
}

// The sun disc's colour at its lower and upper edge (XYZ): the irradiance
// attenuated along the line of sight, per unit solid angle of the disc.
SKY_HD void sunDisc(float sunElevation, float angularDiameter, float altitude, float air, float dust, V3 &bottom,
                    V3 &top) {
    const SkyTables &T = skyTables();
    const float half = angularDiameter / 2.0f;
    const float solidAngle = kTwoPi * (1.0f - cosf(half));
    const float lo = sunElevation - half, hi = sunElevation + half;
    for (int k = 0; k < 2; k++) {
        const float elevation = k == 0 ? (lo > 0.0f ? lo : 0.0f) : (hi > 0.0f ? hi : 0.0f);
        const V3 depth = opticalDepth(v3(0, 0, kEarthRadius + altitude), geographicalToDirection(elevation, 0.0f));
        float spectrum[kSkyWavelengths];
        for (int w = 0; w < kSkyWavelengths; w++) {
            const float tau = T.rayleigh[w] * depth.x * air + 1.11f * kMieCoeff * depth.y * dust;
            spectrum[w] = T.irradiance[w] * expf(-tau) / solidAngle;
        }
        (k == 0 ? bottom : top) = spectrumToXyz(spectrum);
    }
}

// The sky of one TEX_SKY node as MaterialBuilder.swift:329-388 resolves it.
struct SkyOptions {
    float sunElevation, sunRotation, sunSize, sunIntensity;
    float altitude, airDensity, dustDensity, ozoneDensity;
    bool sunDisc;
    float scale;  // 1, or 0.08 for a Hosek-Wilkie sky mapped onto Nishita
};

// The node's ten data values: sun disc bottom and top colours (XYZ), sun
// elevation, rotation, angular diameter (-1 without a disc), intensity
// (SkyLoader.mm:31-39).
inline void skyNodeData(const SkyOptions &o, float data[10]) {
    V3 bottom, top;
    sunDisc(o.sunElevation, o.sunSize, o.altitude, o.airDensity, o.dustDensity, bottom, top);
    data[0] = bottom.x;
    data[1] = bottom.y;
    data[2] = bottom.z;
    data[3] = top.x;
    data[4] = top.y;
    data[5] = top.z;
    data[6] = o.sunElevation;
    data[7] = o.sunRotation;
    data[8] = o.sunDisc ? o.sunSize : -1.0f;
    data[9] = o.sunIntensity;
}

}  // namespace rmdsky
