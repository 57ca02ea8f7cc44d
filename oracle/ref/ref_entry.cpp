// C entry points into the reference's own device code, built for the host
// (see Makefile).  TEST INFRASTRUCTURE ONLY: the pinning tests call these
// beside the oracle's restatement on the same inputs.
#include <metal_stdlib>
using namespace metal;

#include <bridge/PrngState.hpp>
#include "PrngState.cpp"
#include <device/utils/noise.hpp>
#include <device/bsdf/UberShader.hpp>
#include <device/nodes/nodes.hpp>

#include "materials.inc"

extern "C" {

// PrngState(a, b), then n samples (PrngState.metal:58-77)
void ref_prng_tea(uint32_t a, uint32_t b, int n, float *out) {
    PrngState p(a, b);
    for (int i = 0; i < n; i++) out[i] = p.sample();
}

// fractal_noise over float3 points (utils/noise.hpp:416-441)
void ref_fractal_noise3(const float *p, int n, float detail, float roughness, float *out) {
    for (int i = 0; i < n; i++) out[i] = fractal_noise(float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), detail, roughness);
}

int ref_num_materials() { return refmat::numMaterials(); }

// One material of pin_materials.py on shading records, evaluated and sampled
// the way handleIntersections does (intersection.metal:100-104,135-144,149-185).
// Record (28 floats): position, normal, trueNormal, generated, uv, wo, wi, rnd
// (float3 each), rayFlags, 3 unused.  Output (16 floats): emission, evaluate
// value, evaluate pdf, sampled wi, sampled weight, sampled pdf, sampled flags,
// alpha.
int ref_material_eval(int material, const float *records, int n, float *out) {
    if (material < 0 || material >= refmat::numMaterials()) return 1;
    static Context ctx;  // the pinned nodes read nothing from it
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
        sh.tu = sh.tv = float3(0);
        sh.distance = 0;
        refmat::shadeSurface(material, ctx, sh);
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

}  // extern "C"
