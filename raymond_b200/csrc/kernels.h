// Launch wrappers of the static kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "device/traverse.cuh"
#include "device/wavefront.cuh"

// device-driven render loop: condition node of a CUDA-graph while loop
cudaError_t rmdLaunchLoopCondition(rmd::Counters *cnt, cudaGraphConditionalHandle handle, uint32_t itersPerBody,
                                   uint32_t maxIterations, cudaStream_t s);
cudaError_t rmdLaunchFrameInit(const rmd::PathPool &pool, rmd::Counters *cnt, uint64_t firstPath, uint64_t endPath,
                               cudaStream_t s);
cudaError_t rmdLaunchFilmRegen(const rmd::Context &ctx, const rmd::PathPool &pool, const rmd::FrameParams &fp,
                               rmd::Counters *cnt, uint32_t cur, int blocks, cudaStream_t s);
cudaError_t rmdLaunchTraceClosest(const rmd::WideNode *nodes, const float4 *tris, const rmd::PathPool &pool,
                                  rmd::Counters *cnt, uint32_t cur, int blocks, cudaStream_t s);
cudaError_t rmdLaunchTraceShadow(const rmd::WideNode *nodes, const float4 *tris, const rmd::PathPool &pool,
                                 rmd::Counters *cnt, uint32_t cur, int blocks, cudaStream_t s);
cudaError_t rmdLaunchEnvmapReduce(float *mip, int cur, cudaStream_t s);
cudaError_t rmdLaunchEnvmapNormalize(const float *sum, float *pdfs, uint32_t gridSize, cudaStream_t s);
cudaError_t rmdLaunchFilmResolve(const float4 *film, const double *film64, int fp64, float *out, uint32_t numPixels,
                                 float exposure, float divisor, uint32_t tonemapping, uint32_t channels,
                                 cudaStream_t s);
cudaError_t rmdLaunchDebugPrng(uint32_t mode, uint64_t a, uint64_t b, int n, float *out, cudaStream_t s);
// three rotated copies per triangle (the traversal kernels' layout) from n x (v0, v1, v2)
cudaError_t rmdLaunchRotateTriangles(const float4 *in, float4 *out, uint32_t n, cudaStream_t s);
cudaError_t rmdLaunchDebugTrace(const rmd::WideNode *nodes, const float4 *tris, const float *rays, int n, int any,
                                float *out, uint32_t *inst, uint32_t *errors, cudaStream_t s);
// The Nishita sky texture of a TEX_SKY node (width x height RGBA float, CIE
// XYZ in rgb): one thread per texel of the left half, mirrored to the right
cudaError_t rmdLaunchSkyTexture(float4 *texels, uint32_t width, uint32_t height, float sunElevation, float altitude,
                                float air, float dust, float ozone, cudaStream_t s);
