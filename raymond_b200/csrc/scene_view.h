// Read-only view of a scene's device state for entry points outside renderer.cu.
#pragma once
#include <cuda_runtime.h>

#include "../../include/raymond.h"
#include "device/traverse.cuh"
#include "device/wavefront.cuh"

namespace rmdhost {

struct SceneView {
    rmd::Context ctx;              // device view of geometry, lights, materials, camera
    const rmd::WideNode *nodes;     // nullptr for a scene without triangles
    const float4 *tris;
    cudaKernel_t shade;            // shading megakernel of the scene's material module
    int shadeBlocks;
    cudaStream_t stream;
    int device;
    int smCount;
};

// false for a null scene
bool sceneView(const rmd_scene *scene, SceneView &out);
// records `msg` as the calling thread's rmd_last_error and returns `status`
rmd_status setLastError(rmd_status status, const char *msg);
// looks up the device address of rmd_render_noalloc's scratch array on `device` (current)
rmd_status noallocSetup(int device);

}  // namespace rmdhost
