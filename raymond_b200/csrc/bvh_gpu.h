// Device BVH builder (bvh_gpu.cu): the compressed 8-wide BVH of
// device/traverse.cuh built on the GPU.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace rmdhost {

struct GpuBvhResult {
    void *nodes = nullptr;   // nodeCount x 80 B (GpuWideNode), cudaMalloc'd, owned by the caller
    uint64_t nodeCount = 0;
    void *tris = nullptr;    // n x 48 B in leaf order, cudaMalloc'd, owned by the caller
    uint32_t levels = 0;     // levels of the 8-wide tree
    uint32_t clusterIterations = 0;
    std::string error;       // set when the build fails for a reason other than a CUDA error
};

// The largest triangle count the device builder takes (its scans cover
// 4096 x 4096 elements).
constexpr uint32_t kGpuBvhMaxTriangles = 1u << 24;

// Builds the BVH of n world-space triangles given as device arrays (v0, v1,
// v2: 3 floats per triangle; inst / prim: instance and primitive index per
// triangle).  Returns cudaErrorInvalidValue with `error` set when the input
// is out of range or the tree would be deeper than the traversal stack.
cudaError_t buildWideBvhGpu(const float *v0, const float *v1, const float *v2, const uint32_t *inst,
                            const uint32_t *prim, uint32_t n, cudaStream_t s, GpuBvhResult &out);

}  // namespace rmdhost
