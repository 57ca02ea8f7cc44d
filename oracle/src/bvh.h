// Oracle (test infrastructure only): CPU stand-in for Apple's closed
// `metal::raytracing::intersector<triangle_data, instancing>` used by
// raymond/device/kernels/shading/raytrace.metal:11-85 and generate.metal:165-191.
// A binned-SAH BVH over the world-space triangles of all instances, with the
// watertight ray/triangle test of Woop, Benthin and Wald (JCGT 2(1), 2013).
// Conventions kept from the reference: hits report the ray distance, the
// instance index, the primitive index within the instance's shape, and
// barycentrics stored as (weight of v0, weight of v1) (raytrace.metal:44-47);
// a miss reports distance -1 (<= 0 for intersection.metal:75, < 0 for
// shadow.metal:21).
#pragma once
#include <cstdint>
#include <vector>
#include "vec.h"

namespace orc {

struct HitRecord {
    float t = -1;
    uint32_t instance = 0;
    uint32_t prim = 0;
    float b0 = 0, b1 = 0;
};

class Bvh {
public:
    struct Tri {
        float3 v0, v1, v2;
        uint32_t instance, prim;
    };
    void build(std::vector<Tri> tris);
    // closest hit with t in [tmin, tmax]; `exhaustive` visits every box the
    // ray enters instead of culling against the best hit so far (a check of
    // the culling bound)
    bool intersect(float3 org, float3 dir, float tmin, float tmax, HitRecord &hit, bool exhaustive = false) const;
    // any hit with t in [tmin, tmax]
    bool occluded(float3 org, float3 dir, float tmin, float tmax) const;
    size_t numNodes() const { return nodes_.size(); }

private:
    struct Node {
        float bmin[3], bmax[3];
        int32_t first;  // leaf: first triangle; inner: left child (right = left + 1)
        int32_t count;  // leaf: triangle count; inner: 0
    };
    std::vector<Node> nodes_;
    std::vector<Tri> tris_;
};

// Woop/Benthin/Wald watertight test; returns t and the scaled barycentrics.
struct WatertightRay {
    int kx, ky, kz;
    float Sx, Sy, Sz;
    float3 org;
    explicit WatertightRay(float3 o, float3 d);
};
bool intersectTriangle(const WatertightRay &r, float3 v0, float3 v1, float3 v2, float tmin, float tmax, float &t,
                       float &b0, float &b1);

}  // namespace orc
