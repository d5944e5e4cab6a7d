// Headless display output (tone map of the accumulator).
#pragma once

#include "pt_common.cuh"

namespace pt {

// RGBA8 of `pixels` accumulator entries: background for pixels without
// samples, exposure, Reinhard, 8-bit; or the adaptive-sampling overlay.
void launchTonemap(const float4* acc, const uint32_t* counts, const uint8_t* converged, int pixels,
    const pt_render_params& params, float exposure, uint8_t* out, cudaStream_t s);

// The preview image (pw x ph, one pixel per `downscale` x `downscale` block)
// upsampled to width x height and tone-mapped like the accumulator.
void launchTonemapPreview(const float4* preview, int pw, int ph, int downscale, int width, int height,
    const pt_render_params& params, float exposure, uint8_t* out, cudaStream_t s);

} // namespace pt
