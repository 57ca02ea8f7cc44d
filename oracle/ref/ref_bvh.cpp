// Host BVH behind the Metal intersector stand-in of the reference's host
// build: the oracle's binned-SAH BVH and watertight test (oracle/src/bvh.h),
// wrapped in plain functions so the reference's translation unit (Metal
// vector types) and the oracle's (its own vector types) never meet.
// TEST INFRASTRUCTURE ONLY.
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../src/bvh.h"

extern "C" void *refbvh_build(const float *tris, const uint32_t *instance, const uint32_t *prim, size_t n) {
    std::vector<orc::Bvh::Tri> t(n);
    for (size_t i = 0; i < n; i++) {
        const float *v = tris + 9 * i;
        t[i].v0 = orc::float3(v[0], v[1], v[2]);
        t[i].v1 = orc::float3(v[3], v[4], v[5]);
        t[i].v2 = orc::float3(v[6], v[7], v[8]);
        t[i].instance = instance[i];
        t[i].prim = prim[i];
    }
    auto *b = new orc::Bvh();
    b->build(std::move(t));
    return b;
}

extern "C" void refbvh_destroy(void *b) { delete static_cast<orc::Bvh *>(b); }

// closest (any = 0) or any (any = 1) hit in [tmin, tmax]; returns 1 on a hit
extern "C" int refbvh_intersect(const void *b, const float *o, const float *d, float tmin, float tmax, int any,
                                float *t, uint32_t *instance, uint32_t *prim, float *b0, float *b1) {
    const orc::Bvh *bvh = static_cast<const orc::Bvh *>(b);
    const orc::float3 org(o[0], o[1], o[2]), dir(d[0], d[1], d[2]);
    if (any) {
        if (!bvh->occluded(org, dir, tmin, tmax)) return 0;
        *t = 1.0f;
        return 1;
    }
    orc::HitRecord h;
    if (!bvh->intersect(org, dir, tmin, tmax, h)) return 0;
    *t = h.t;
    *instance = h.instance;
    *prim = h.prim;
    *b0 = h.b0;
    *b1 = h.b1;
    return 1;
}
