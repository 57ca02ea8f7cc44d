// Host interface of the path-guiding network kernels (guide.cu).  No
// counterpart in the reference.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device/wavefront.cuh"

namespace rmd {

// 160 -> 64 -> 64 -> 64 -> 48: weights and biases of the four layers
constexpr int GUIDE_PARAMS = GUIDE_HIDDEN * GUIDE_INPUTS + GUIDE_HIDDEN + 2 * (GUIDE_HIDDEN * GUIDE_HIDDEN + GUIDE_HIDDEN) +
                             GUIDE_OUTPUTS * GUIDE_HIDDEN + GUIDE_OUTPUTS;
constexpr int GUIDE_TRAIN_MAX_BLOCKS = 256;  // blocks of one training launch (each writes its gradient)
// net.partials: GUIDE_TRAIN_MAX_BLOCKS gradient slots, then one loss share per block
constexpr size_t GUIDE_PARTIAL_LOSS = (size_t)GUIDE_TRAIN_MAX_BLOCKS * GUIDE_PARAMS;
constexpr int GUIDE_WEIGHTS = GUIDE_HIDDEN * GUIDE_INPUTS + 2 * GUIDE_HIDDEN * GUIDE_HIDDEN + GUIDE_OUTPUTS * GUIDE_HIDDEN;

// Device view of the network: FP32 master parameters (row-major [out][in]
// weights then biases, layer by layer), their BF16 copies for the tensor
// cores, and the Adam state.
struct GuideNetView {
    const uint16_t *w[4];  // bf16 weights per layer, row-major [out][in]
    const float *b[4];     // fp32 biases (inside `master`)
    float *master, *adamM, *adamV, *grad;  // GUIDE_PARAMS each
    float *partials;                        // per training block: its gradient, then its loss (GUIDE_PARTIAL_LOSS)
    uint16_t *weightsBf16;                  // GUIDE_WEIGHTS
    const int *bf16Index;                   // per parameter: index into weightsBf16, or -1 (bias)
    // the BF16 weights in the training kernel's shared-memory layout (every
    // layer canonical, K = its inputs), copied into each training CTA with
    // one bulk copy; imageIndex: per parameter, its element (-1: a bias)
    uint16_t *image;
    const int *imageIndex;
    int wOffset[4], bOffset[4];             // parameter offsets of each layer's weights / biases
    float3 sceneMin, sceneInvExtent;        // position encoding frame
};

}  // namespace rmd

size_t rmdGuideSharedBytes(bool training);
cudaError_t rmdGuideConfigure();
// mixtures of this iteration's hits whose path depth is below guideDepth
cudaError_t rmdLaunchGuideInfer(const rmd::Context &ctx, const rmd::PathPool &pool, rmd::Counters *cnt, uint32_t cur,
                                uint32_t guideDepth, const rmd::GuideNetView &net, rmd::GuideMixture *out, int blocks,
                                cudaStream_t s);
// `steps` Adam steps (the first is `step`, counting from 1), each on the mean
// loss over a batch of n records drawn from the `total` stored ones (all of
// them when n >= total; step k draws with seed `seed` + k)
// (tensor cores: one CTA per 128 records, at most `blocks`); an expired
// tensor-core wait sets ERR_GUIDE_TIMEOUT in *errors
cudaError_t rmdLaunchGuideTrain(const rmd::GuideRecord *rec, uint32_t total, uint32_t n, uint32_t seed, uint32_t steps,
                                const rmd::GuideNetView &net, float *scratch, int blocks, float lr, int step,
                                uint32_t *errors, cudaStream_t s);
// Adam (beta 0.9 / 0.999, eps 1e-8, `step` from 1) on net.grad plus the first
// `blocks` per-CTA gradients; refreshes the BF16 weights, clears net.grad and
// writes the sum of the blocks' loss shares to *lossOut (when not NULL)
cudaError_t rmdLaunchGuideAdam(const rmd::GuideNetView &net, int blocks, float lr, int step, float *lossOut,
                               cudaStream_t s);
// status[0] = 1 if a tensor-core wait expired
cudaError_t rmdLaunchGuideForwardTest(const float *features, uint32_t n, const rmd::GuideNetView &net, float *out,
                                      int *status, cudaStream_t s);
// gradient only (no Adam step): net.grad += d(mean loss); scratch[1] = mean loss, scratch[2] error flags
cudaError_t rmdLaunchGuideGradientTest(const rmd::GuideRecord *rec, uint32_t n, const rmd::GuideNetView &net,
                                       float *scratch, int blocks, cudaStream_t s);

namespace rmdhost {

// Device buffers of the guiding network (FP32 master parameters, Adam
// moments, gradient, BF16 weight copy).
struct GuideNet {
    float *master = nullptr, *adamM = nullptr, *adamV = nullptr, *grad = nullptr, *scratch = nullptr;
    float *partials = nullptr;
    uint16_t *weightsBf16 = nullptr;
    int *bf16Index = nullptr;
    uint16_t *image = nullptr;
    int *imageIndex = nullptr;
    int steps = 0;
    GuideNet() = default;
    GuideNet(const GuideNet &) = delete;
    GuideNet &operator=(const GuideNet &) = delete;
    ~GuideNet() { release(); }
    void release();
    bool allocated() const { return master != nullptr; }
    cudaError_t allocate();
    // upload FP32 parameters (refreshes the BF16 copy, clears Adam and the gradient)
    cudaError_t setParams(const float *host, cudaStream_t s);
    cudaError_t getParams(float *host, cudaStream_t s) const;
    rmd::GuideNetView view(float3 sceneMin, float3 sceneInvExtent) const;
    // seeded initialisation: uniform Xavier weights, biases that start the
    // mixture broad (log kappa 1) and the guide rarely selected (alpha 0.2)
    static void initParams(float *params, uint32_t seed);
    static void layout(int wOffset[4], int bOffset[4], int bf16Offset[4]);
};

}  // namespace rmdhost
