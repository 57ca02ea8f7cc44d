// Host BVH builder; the node layout is rmd::BvhNode of device/traverse.cuh.
#pragma once
#include <cstdint>
#include <vector>

namespace rmdhost {

struct GpuBvhNode {
    float c0xy[4];  // lo.x, hi.x, lo.y, hi.y of child 0
    float c1xy[4];  // of child 1
    float cz[4];    // lo.z, hi.z of child 0, lo.z, hi.z of child 1
    int link[4];    // child 0, child 1 (>= 0 inner node, < 0 leaf ~(first << 3 | count - 1))
};
static_assert(sizeof(GpuBvhNode) == 64, "BvhNode is 64 bytes");

struct GpuBvh {
    std::vector<GpuBvhNode> nodes;
    std::vector<float> tris;  // 12 floats per triangle in leaf order: v0, inst, v1, prim, v2, 0
};

// v0/v1/v2: 3 floats per triangle (world space); instance / prim per triangle.
void buildBvh(const std::vector<float> &v0, const std::vector<float> &v1, const std::vector<float> &v2,
              const std::vector<uint32_t> &instance, const std::vector<uint32_t> &prim, GpuBvh &out);

}  // namespace rmdhost
