// GPU harness around the REFERENCE's own CUDA render kernels: the reference
// megakernel rebuilt for sm_100a, used by the GPU parity tests as a second
// checker and by bench.py as the GPU bar.  Built into oracle/_ref/libptref_gpu.so
// by oracle/Makefile (target refgpu).  Test and benchmark infrastructure only:
// the product never loads it.
//
// What runs on the GPU is the reference's code, compiled unchanged from its
// tree (same translation units, nvcc defaults as its CMake build):
//   - PathTracerLib/src/PathTracer.cu: sampleAdaptiveKernel (:186-273),
//     clearAccumulatorKernel (:275-303), compactActiveListKernel (:372-411)
//     and their bool launch wrappers pathTracerClearAccumulator (:613-647),
//     pathTracerAdaptiveSample (:733-775), pathTracerCompactActiveList
//     (:777-823), declared in PathTracerCuda.h:12-126;
//   - PathTracerLib/src/MeshAccel/MeshAccelScene.cpp: build / allocate /
//     upload (:141-341), with MeshBvhBuilder.cpp's host median-split BVH.
//
// What this file adds (harness, not reference code):
//   - scene and environment handles over plain pointers for ctypes;
//   - the wave sequence of PathTracer::renderLoop without preview levels
//     (PathTracer.cpp:2379-2464): wave i uses globalSeed = i + 1; every 4th
//     full-resolution wave compacts the active list into the scratch list,
//     reads the 4-byte count back and swaps the lists; the loop ends when the
//     count reaches 0 or after maxWaves waves.  The reference waits for each
//     wave's completion event before the next (waitForSampleEvent); here that
//     wait is cudaEventSynchronize, without the reference's GUI-thread
//     bookkeeping, which is the most favourable host loop for the reference.
#include "Geometry/MathCore.h"
#include "MeshAccel/MeshAccelScene.h"
#include "PathTracerAdaptiveSampling.h"
#include "PathTracerCuda.h"

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

namespace {

struct RefGpuScene {
    MeshAccelScene accel;
    double buildMs = 0.0;
    double uploadMs = 0.0;
};

struct RefGpuEnv {
    float* pixels = nullptr;
    float* marginal = nullptr;
    float* row = nullptr;
    EnvironmentMapGpu* dMap = nullptr;
};

template <class T>
bool uploadArray(T** dst, const T* src, size_t count)
{
    if (cudaMalloc(dst, sizeof(T) * (count > 0 ? count : 1)) != cudaSuccess) {
        *dst = nullptr;
        return false;
    }
    return count == 0 || cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice) == cudaSuccess;
}

void freeEnv(RefGpuEnv* e)
{
    cudaFree(e->pixels);
    cudaFree(e->marginal);
    cudaFree(e->row);
    cudaFree(e->dMap);
    delete e;
}

} // namespace

extern "C" {

// Builds the reference scene on the host (median-split BVH, emissive CDF) and
// uploads it with the reference's own MeshAccelScene::allocate/upload.
//   positions 9 floats / triangle, normals 9, uvs 6; materials MaterialGpu
//   (96 B each), textures TextureDescGpu (64 B each).
// outMs (optional, 2 doubles): host build time, upload time.
void* refgpu_scene_create(
    int triCount, const float* positions, const float* normals, const float* uvs,
    const uint32_t* materialIds, int materialCount, const void* materials,
    int textureCount, const void* textures, double* outMs)
{
    if (triCount < 0 || (triCount > 0 && (positions == nullptr || normals == nullptr || uvs == nullptr ||
                                           materialIds == nullptr))) {
        return nullptr;
    }
    const auto t0 = std::chrono::steady_clock::now();
    HostMesh mesh;
    mesh.triangles.resize(static_cast<size_t>(triCount));
    for (int i = 0; i < triCount; ++i) {
        HostTriangle& t = mesh.triangles[static_cast<size_t>(i)];
        const float* p = positions + 9 * static_cast<size_t>(i);
        const float* n = normals + 9 * static_cast<size_t>(i);
        const float* q = uvs + 6 * static_cast<size_t>(i);
        t.v0 = vecMake3(p[0], p[1], p[2]);
        t.v1 = vecMake3(p[3], p[4], p[5]);
        t.v2 = vecMake3(p[6], p[7], p[8]);
        t.n0 = vecMake3(n[0], n[1], n[2]);
        t.n1 = vecMake3(n[3], n[4], n[5]);
        t.n2 = vecMake3(n[6], n[7], n[8]);
        t.uv0 = Vec2{q[0], q[1]};
        t.uv1 = Vec2{q[2], q[3]};
        t.uv2 = Vec2{q[4], q[5]};
        t.materialIndex = materialIds[i];
    }
    mesh.materials.resize(static_cast<size_t>(materialCount));
    if (materialCount > 0) {
        std::memcpy(mesh.materials.data(), materials, sizeof(MaterialGpu) * static_cast<size_t>(materialCount));
    }
    mesh.textures.resize(static_cast<size_t>(textureCount));
    if (textureCount > 0) {
        std::memcpy(mesh.textures.data(), textures, sizeof(TextureDescGpu) * static_cast<size_t>(textureCount));
    }
    RefGpuScene* s = new RefGpuScene();
    if (!s->accel.build(mesh)) {
        delete s;
        return nullptr;
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (!s->accel.allocate() || !s->accel.upload(nullptr) || cudaDeviceSynchronize() != cudaSuccess) {
        delete s;
        return nullptr;
    }
    const auto t2 = std::chrono::steady_clock::now();
    s->buildMs = std::chrono::duration<double, std::milli>(t1 - t0).count();
    s->uploadMs = std::chrono::duration<double, std::milli>(t2 - t1).count();
    if (outMs != nullptr) {
        outMs[0] = s->buildMs;
        outMs[1] = s->uploadMs;
    }
    return s;
}

void refgpu_scene_destroy(void* handle)
{
    delete static_cast<RefGpuScene*>(handle);
}

int refgpu_scene_bvh_node_count(void* handle)
{
    const MeshAccelSceneGpu* h = static_cast<RefGpuScene*>(handle)->accel.hostScene();
    return h != nullptr ? static_cast<int>(h->bvhNodeCount) : 0;
}

// Environment map on the device: RGB lat-long pixels plus the importance
// tables (marginal [height+1], row [height*(width+1)]) as the host harness
// builds them (the restatement of EnvironmentMap.cpp:76-128).
void* refgpu_env_create(int width, int height, const float* rgb, const float* marginal, const float* row)
{
    if (width <= 0 || height <= 0 || rgb == nullptr || marginal == nullptr || row == nullptr) {
        return nullptr;
    }
    RefGpuEnv* e = new RefGpuEnv();
    const size_t w = static_cast<size_t>(width), h = static_cast<size_t>(height);
    EnvironmentMapGpu view{};
    bool ok = uploadArray(&e->pixels, rgb, w * h * 3) && uploadArray(&e->marginal, marginal, h + 1) &&
        uploadArray(&e->row, row, h * (w + 1));
    if (ok) {
        view.pixels = e->pixels;
        view.marginalCdf = e->marginal;
        view.rowCdf = e->row;
        view.width = width;
        view.height = height;
        view.valid = 1;
        ok = uploadArray(&e->dMap, &view, 1);
    }
    if (!ok) {
        freeEnv(e);
        return nullptr;
    }
    return e;
}

void refgpu_env_destroy(void* handle)
{
    if (handle != nullptr) {
        freeEnv(static_cast<RefGpuEnv*>(handle));
    }
}

// Renders one frame from a cleared accumulator with the reference kernels.
//   cameraBytes: CameraGpu (80 B); paramsBytes: RenderParamsGpu (44 B).
//   maxWaves: upper bound on waves (0 = until no pixel is active).
// Outputs (host arrays of width*height entries, any may be null): acc (float4),
// counts, lumMean, m2, converged.  out (5 doubles, optional): device time of
// the wave loop in ms (CUDA events on the render stream around the loop, the
// per-wave host waits included), waves run, samples taken (sum of counts),
// wall time of the loop in ms, number of compactions.
// Returns 0, or a negative value naming the failing step.
int refgpu_render(
    void* sceneHandle, void* envHandle, const void* cameraBytes, const void* paramsBytes,
    int width, int height, int maxWaves,
    float* outAcc, uint32_t* outCounts, float* outLumMean, float* outM2, uint8_t* outConverged,
    double* out)
{
    if (sceneHandle == nullptr || cameraBytes == nullptr || paramsBytes == nullptr || width <= 0 || height <= 0) {
        return -1;
    }
    RefGpuScene* scene = static_cast<RefGpuScene*>(sceneHandle);
    const EnvironmentMapGpu* dEnv = envHandle != nullptr ? static_cast<RefGpuEnv*>(envHandle)->dMap : nullptr;
    const size_t P = static_cast<size_t>(width) * static_cast<size_t>(height);
    RenderParamsGpu params{};
    std::memcpy(&params, paramsBytes, sizeof(RenderParamsGpu));

    float4* acc = nullptr;
    uint32_t* counts = nullptr;
    float* lumMean = nullptr;
    float* m2 = nullptr;
    uint8_t* converged = nullptr;
    int* active = nullptr;
    int* scratch = nullptr;
    int* activeCount = nullptr;
    CameraGpu* dCamera = nullptr;
    RenderParamsGpu* dParams = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr, waveDone = nullptr;
    int rc = 0;
    int waves = 0;
    int compactions = 0;
    float deviceMs = 0.0f;
    double wallMs = 0.0;
    const bool allocated = cudaMalloc(&acc, sizeof(float4) * P) == cudaSuccess &&
        cudaMalloc(&counts, sizeof(uint32_t) * P) == cudaSuccess && cudaMalloc(&lumMean, sizeof(float) * P) == cudaSuccess &&
        cudaMalloc(&m2, sizeof(float) * P) == cudaSuccess && cudaMalloc(&converged, P) == cudaSuccess &&
        cudaMalloc(&active, sizeof(int) * P) == cudaSuccess && cudaMalloc(&scratch, sizeof(int) * P) == cudaSuccess &&
        cudaMalloc(&activeCount, sizeof(int)) == cudaSuccess && cudaMalloc(&dCamera, sizeof(CameraGpu)) == cudaSuccess &&
        cudaMalloc(&dParams, sizeof(RenderParamsGpu)) == cudaSuccess &&
        cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess &&
        cudaEventCreate(&start) == cudaSuccess && cudaEventCreate(&stop) == cudaSuccess &&
        cudaEventCreateWithFlags(&waveDone, cudaEventDisableTiming) == cudaSuccess;
    if (!allocated) {
        rc = -2;
    }
    if (rc == 0 &&
        (cudaMemcpy(dCamera, cameraBytes, sizeof(CameraGpu), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(dParams, &params, sizeof(RenderParamsGpu), cudaMemcpyHostToDevice) != cudaSuccess)) {
        rc = -3;
    }
    if (rc == 0 &&
        (!pathTracerClearAccumulator(acc, counts, lumMean, m2, converged, active, scratch, activeCount, width, height,
             stream) ||
         cudaStreamSynchronize(stream) != cudaSuccess)) {
        rc = -4;
    }
    if (rc == 0) {
        const MeshAccelSceneGpu* dScene = scene->accel.deviceScene();
        int activePixels = static_cast<int>(P);
        const auto w0 = std::chrono::steady_clock::now();
        cudaEventRecord(start, stream);
        for (int iter = 0; activePixels > 0 && (maxWaves <= 0 || iter < maxWaves); ++iter) {
            const unsigned int globalSeed = static_cast<unsigned int>(iter) + 1u;
            if (!pathTracerAdaptiveSample(acc, counts, lumMean, m2, converged, active, activePixels, width, height,
                    dCamera, dScene, dEnv, dParams, globalSeed, stream)) {
                rc = -5;
                break;
            }
            ++waves;
            const int fullResWave = iter + 1;
            int newCount = 0;
            const bool compact = (fullResWave % kAdaptiveCompactActiveListInterval) == 0;
            if (compact) {
                if (!pathTracerCompactActiveList(active, scratch, activeCount, converged, counts,
                        params.maxSamplesPerPixel, activePixels, width, height, false, 0, 0, 0, 0, stream) ||
                    cudaMemcpyAsync(&newCount, activeCount, sizeof(int), cudaMemcpyDeviceToHost, stream) !=
                        cudaSuccess) {
                    rc = -6;
                    break;
                }
                ++compactions;
            }
            if (cudaEventRecord(waveDone, stream) != cudaSuccess || cudaEventSynchronize(waveDone) != cudaSuccess) {
                rc = -7;
                break;
            }
            if (compact) {
                activePixels = newCount;
                std::swap(active, scratch);
            }
        }
        cudaEventRecord(stop, stream);
        if (cudaEventSynchronize(stop) != cudaSuccess) {
            rc = rc != 0 ? rc : -8;
        }
        wallMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        cudaEventElapsedTime(&deviceMs, start, stop);
    }
    double samples = 0.0;
    if (rc == 0) {
        std::vector<uint32_t> c(P);
        const bool ok = cudaMemcpy(c.data(), counts, sizeof(uint32_t) * P, cudaMemcpyDeviceToHost) == cudaSuccess &&
            (outAcc == nullptr || cudaMemcpy(outAcc, acc, sizeof(float4) * P, cudaMemcpyDeviceToHost) == cudaSuccess) &&
            (outLumMean == nullptr ||
                cudaMemcpy(outLumMean, lumMean, sizeof(float) * P, cudaMemcpyDeviceToHost) == cudaSuccess) &&
            (outM2 == nullptr || cudaMemcpy(outM2, m2, sizeof(float) * P, cudaMemcpyDeviceToHost) == cudaSuccess) &&
            (outConverged == nullptr || cudaMemcpy(outConverged, converged, P, cudaMemcpyDeviceToHost) == cudaSuccess);
        if (!ok) {
            rc = -9;
        } else {
            for (size_t i = 0; i < P; ++i) {
                samples += c[i];
            }
            if (outCounts != nullptr) {
                std::memcpy(outCounts, c.data(), sizeof(uint32_t) * P);
            }
        }
    }
    if (out != nullptr) {
        out[0] = deviceMs;
        out[1] = waves;
        out[2] = samples;
        out[3] = wallMs;
        out[4] = compactions;
    }
    cudaFree(acc);
    cudaFree(counts);
    cudaFree(lumMean);
    cudaFree(m2);
    cudaFree(converged);
    cudaFree(active);
    cudaFree(scratch);
    cudaFree(activeCount);
    cudaFree(dCamera);
    cudaFree(dParams);
    if (start != nullptr) {
        cudaEventDestroy(start);
    }
    if (stop != nullptr) {
        cudaEventDestroy(stop);
    }
    if (waveDone != nullptr) {
        cudaEventDestroy(waveDone);
    }
    if (stream != nullptr) {
        cudaStreamDestroy(stream);
    }
    return rc;
}

} // extern "C"
