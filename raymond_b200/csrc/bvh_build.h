// Host BVH builder; the node layout is rmd::WideNode of device/traverse.cuh.
#pragma once
#include <cstdint>
#include <vector>

namespace rmdhost {

// Compressed 8-wide node (rmd::WideNode of device/traverse.cuh), 80 bytes:
// child boxes quantised to 8 bits per plane relative to the node's origin
// and per-axis power-of-two scale (after Ylitie, Karras and Laine, "Efficient
// incoherent ray traversal on GPUs through compressed wide BVHs", HPG 2017).
struct GpuWideNode {
    float origin[3];
    uint8_t exponent[3];   // scale of axis k = 2^(exponent[k] - 127)
    uint8_t imask;         // bit c: child slot c is an inner node
    uint32_t childBase;    // first inner child node; inner children are consecutive in slot order
    uint32_t triBase;      // first triangle of the leaf children, consecutive in slot order
    uint8_t meta[8];       // leaf slot c: (unary triangle count) << 5 | offset from triBase; else 0
    uint8_t qlo[3][8];     // per axis, per slot: quantised lower bound
    uint8_t qhi[3][8];     // per axis, per slot: quantised upper bound
};
static_assert(sizeof(GpuWideNode) == 80, "WideNode is 80 bytes");

struct GpuWideBvh {
    std::vector<GpuWideNode> nodes;
    std::vector<float> tris;  // 12 floats per triangle in leaf order: v0, inst, v1, prim, v2, 0
};

// v0/v1/v2: 3 floats per triangle (world space); instance / prim per triangle.
void buildWideBvh(const std::vector<float> &v0, const std::vector<float> &v1, const std::vector<float> &v2,
                  const std::vector<uint32_t> &instance, const std::vector<uint32_t> &prim, GpuWideBvh &out);

// Surface-area cost of a wide BVH relative to its root: per node the area of
// its box (the parent's decoded slot box; 1 for the root), plus per leaf slot
// the slot's area times its triangles.  levels = the tree's depth.
double wideBvhSahCost(const GpuWideNode *nodes, size_t count, uint32_t &levels);

}  // namespace rmdhost
