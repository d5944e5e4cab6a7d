// Path-replay backpropagation of an image loss (see pt_adjoint.cu).
#pragma once

#include "pt_render.cuh"

namespace pt {

constexpr int kGradParams = 7;          // r, g, b, roughness, metallic, sheen, emission
constexpr int kMaxGradMaterials = 16;   // materials with gradients per call
constexpr int kAdjointBlock = 128;

int adjointBlocksPerSm();
// grad ([materialCount][kGradParams], zeroed by the caller) += d loss / d params
// for the image that pt_render draws with `spp` samples per pixel from a reset
// accumulator; dImage holds d loss / d image, `channels` (3 or 4) floats per pixel.
// record: each sample's radiance from the forward render ([sample][pixel]), or
// null to recompute it with a first replay of the path.
void launchAdjoint(const LaunchCtx* ctx, const float* dImage, int channels, int spp, int pixels, int materialCount,
    float* grad, const float4* record, int grid, cudaStream_t s);
// Preview pass of a width x height image (one centred sample per pixel, no
// accumulation) into out, with the path-replay kernel.
void launchPreview(const LaunchCtx* ctx, int width, int height, uint32_t globalSeed, int maxDepth, float4* out,
    int grid, bool inst, cudaStream_t s);

} // namespace pt
