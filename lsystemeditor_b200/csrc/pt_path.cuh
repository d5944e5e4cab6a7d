// Per-sample helpers shared by the wavefront pipeline and the adjoint
// (path-replay) kernel: the fallback material, the per-(pixel, sample) seed
// and the firefly clamp.
#pragma once

#include "pt_common.cuh"

namespace pt {
namespace {

// MaterialGpu{} defaults (MeshAccelScene.cpp:27-46), used for out-of-range material ids.
__constant__ pt_material kFallbackMaterial = {0.8f, 0.8f, 0.8f, 0.5f, 0.0f, 0.0f, 0.0f, 1.5f, 0.0f, 0.0f, -1.0f, 0.0f,
    0.0f, 0.0f, 1.0f, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0.0f};

// Sampling/RandCore.h:7-12 (reference) or a hash of (x, y, seed value) (extension).
__device__ __forceinline__ uint32_t pathSeed(const pt_render_params& p, uint32_t pixel, uint32_t width,
    uint32_t sampleIndex, uint32_t globalSeed)
{
    if (p.seed_mode == 1) {
        // PCG-style integer hash (O'Neill 2014 output permutation) of x, y, seed and sample index.
        auto h = [](uint32_t v) {
            const uint32_t state = v * 747796405u + 2891336453u;
            const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
            return (word >> 22u) ^ word;
        };
        const uint32_t x = pixel % width, y = pixel / width;
        return h(x ^ h(y ^ h(p.seed_value ^ h(sampleIndex))));
    }
    return pixel * 747796405u + sampleIndex + globalSeed * 2891336453u;
}

// PathTracer.cu:49-67.
__device__ __forceinline__ float3 clampFirefly(float3 c)
{
    if (!isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z)) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    c = f3(fmax2(0.0f, c.x), fmax2(0.0f, c.y), fmax2(0.0f, c.z));
    const float l = __fadd_rn(__fadd_rn(__fmul_rn(c.x, 0.2126f), __fmul_rn(c.y, 0.7152f)), __fmul_rn(c.z, 0.0722f));
    if (l <= 100.0f) {
        return c;
    }
    const float k = __fdiv_rn(100.0f, l);
    return f3(__fmul_rn(c.x, k), __fmul_rn(c.y, k), __fmul_rn(c.z, k));
}

// Spectral samples: a hero-wavelength estimate of a colour can have a
// negative sRGB channel, which is kept (zeroing it would bias the estimate);
// the non-finite and luminance rules of clampFirefly apply.
__device__ __forceinline__ float3 clampFireflySigned(float3 c)
{
    if (!isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z)) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    const float l = __fadd_rn(__fadd_rn(__fmul_rn(c.x, 0.2126f), __fmul_rn(c.y, 0.7152f)), __fmul_rn(c.z, 0.0722f));
    if (l <= 100.0f) {
        return c;
    }
    const float k = __fdiv_rn(100.0f, l);
    return f3(__fmul_rn(c.x, k), __fmul_rn(c.y, k), __fmul_rn(c.z, k));
}

} // namespace
} // namespace pt
