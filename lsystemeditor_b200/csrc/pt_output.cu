// Headless display output: the reference's display pipeline (exposure,
// Reinhard x / (1 + x), 8-bit quantisation; PathTracer.cu:421-512) written to a
// device buffer instead of a GL pixel buffer, and the physical-camera exposure
// multiplier (PhysicalCamera.cpp:392-397).
#include "pt_output.cuh"

namespace pt {

namespace {

constexpr int kDebugOverlayAdaptiveSampling = 2; // RenderParamsGpu::debugOverlayMode value (PathTracer.cu:37)

__device__ __forceinline__ unsigned char quantise(float v)
{
    // truncation of clamp(v, 0, 1) * 255, as the reference's toneMapToUchar4
    return static_cast<unsigned char>(__fmul_rn(fminf(fmaxf(v, 0.0f), 1.0f), 255.0f));
}

__device__ __forceinline__ float reinhard(float x, float exposure)
{
    const float e = __fmul_rn(x, exposure);
    return __fdiv_rn(e, __fadd_rn(1.0f, e));
}

__global__ void k_tonemap(const float4* acc, const uint32_t* counts, const uint8_t* converged, int pixels,
    pt_render_params params, float exposure, uchar4* out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < pixels; i += gridDim.x * blockDim.x) {
        if (params.debug_overlay_mode == kDebugOverlayAdaptiveSampling) {
            out[i] = converged[i] != 0 ? make_uchar4(0, quantise(0.35f), 0, 255) : make_uchar4(255, 0, 0, 255);
            continue;
        }
        float r = params.background_r, g = params.background_g, b = params.background_b;
        if (counts[i] > 0) {
            const float4 v = acc[i];
            r = v.x;
            g = v.y;
            b = v.z;
        }
        out[i] = make_uchar4(quantise(reinhard(r, exposure)), quantise(reinhard(g, exposure)),
            quantise(reinhard(b, exposure)), 255);
    }
}

// The preview shown at full resolution (pathTracerUpsamplePreviewToPbo,
// PathTracer.cu:883-920): nearest preview pixel x / downscale, clamped.
__global__ void k_tonemap_preview(const float4* preview, int pw, int ph, int downscale, int width, int height,
    pt_render_params params, float exposure, uchar4* out)
{
    const int n = width * height;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (params.debug_overlay_mode == kDebugOverlayAdaptiveSampling) {
            out[i] = make_uchar4(255, 0, 0, 255);
            continue;
        }
        const int x = i % width, y = i / width;
        const int px = min(x / downscale, pw - 1), py = min(y / downscale, ph - 1);
        const float4 v = preview[py * pw + px];
        out[i] = make_uchar4(quantise(reinhard(v.x, exposure)), quantise(reinhard(v.y, exposure)),
            quantise(reinhard(v.z, exposure)), 255);
    }
}

} // namespace

void launchTonemapPreview(const float4* preview, int pw, int ph, int downscale, int width, int height,
    const pt_render_params& params, float exposure, uint8_t* out, cudaStream_t s)
{
    const int pixels = width * height;
    if (pixels <= 0) {
        return;
    }
    const int grid = (pixels + 255) / 256 < 148 * 32 ? (pixels + 255) / 256 : 148 * 32;
    k_tonemap_preview<<<grid, 256, 0, s>>>(preview, pw, ph, downscale, width, height, params, exposure,
        reinterpret_cast<uchar4*>(out));
}

void launchTonemap(const float4* acc, const uint32_t* counts, const uint8_t* converged, int pixels,
    const pt_render_params& params, float exposure, uint8_t* out, cudaStream_t s)
{
    if (pixels <= 0) {
        return;
    }
    const int grid = (pixels + 255) / 256 < 148 * 32 ? (pixels + 255) / 256 : 148 * 32;
    k_tonemap<<<grid, 256, 0, s>>>(acc, counts, converged, pixels, params, exposure, reinterpret_cast<uchar4*>(out));
}

} // namespace pt
