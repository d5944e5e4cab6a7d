// Scene construction on the device: tube lofting and leaf quads from turtle
// output, the emissive-triangle list and its CDF, and the shading records.
#pragma once

#include "pt_common.cuh"

namespace pt {

// Tubes and leaves in device memory (see pt_tubes in include/pt_b200.h).
struct TubeSetDev {
    uint32_t tubeCount = 0;
    uint32_t sides = 0;
    uint32_t ringCount = 0;
    const uint32_t* ringStart = nullptr;  // tubeCount + 1
    const double* points = nullptr;       // 3 per ring
    const double* tangents = nullptr;     // 3 per ring
    const double* radii = nullptr;        // 1 per ring
    const uint32_t* materials = nullptr;  // per tube
    const double* cosSin = nullptr;       // 2 * (sides + 1): cos, sin of side k's angle (entry sides = entry 0)
    const double* frames = nullptr;       // 6 per ring: normal, binormal (given frames) or null
    uint32_t leafCount = 0;
    const double* leaves = nullptr;       // 10 per leaf: position, tangent, up, size
    double leafSize = 0.0;
    uint32_t leafMaterial = 0;
};

// Triangles produced by a tube set: 2 * sides per ring, plus 2 per leaf.
inline uint64_t tubeTriangles(uint32_t sides, uint32_t rings, uint32_t leaves)
{
    return 2ull * sides * rings + 2ull * leaves;
}

// Per-ring unit tangent and frame (double, 9 values per ring) in `frames`.
void launchRingFrames(const TubeSetDev& t, double* frames, cudaStream_t s);
// Writes the triangles of the tube set (tubes first, tube-major, then leaves)
// at triangle offset 0 of the output arrays (9 / 9 / 6 floats, 1 id per triangle).
void launchLoft(const TubeSetDev& t, const double* frames, float* positions, float* normals, float* uvs,
    uint32_t* materialIds, cudaStream_t s);

// Emissive weights (area x luminance x emission) per triangle in original order
// and their inclusive prefix sum over the emissive triangles only, summed in
// triangle order in single precision (MeshAccelScene.cpp:62-95).
void launchEmissiveWeights(const float* positions, const uint32_t* materialIds, uint32_t n,
    const pt_material* materials, uint32_t materialCount, float* weights, uint8_t* flags, cudaStream_t s);
size_t emissiveSelectTempBytes(uint32_t n);
// Stable compaction of the flagged triangle indices into `idx`; count into *dCount.
cudaError_t emissiveSelect(void* temp, size_t tempBytes, const uint8_t* flags, uint32_t n, uint32_t* idx,
    uint32_t* dCount, cudaStream_t s);
// cdf[0] = 0, cdf[k + 1] = sum of weights[idx[0..k]]; out[0] = count, out[1] = bits of the total.
// Per-triangle area density of emissive NEE's point sampling (0 for non-emitters;
// out must be zeroed first).
void launchEmitterPdf(const float* positions, const uint32_t* idx, const float* cdf, uint32_t count, float* out,
    cudaStream_t s);
void launchEmissiveCdf(const float* weights, const uint32_t* idx, const uint32_t* dCount, float* cdf, uint32_t* out,
    cudaStream_t s);

// Shading records from per-triangle normals / uvs / material ids.
void launchBuildShade(const float* normals, const float* uvs, const uint32_t* materialIds, uint32_t n, TriShade* out,
    cudaStream_t s);
// Inverse of launchBuildShade (for export): normals, uvs and material ids.
void launchUnpackShade(const TriShade* shade, uint32_t n, float* normals, float* uvs, uint32_t* materialIds,
    cudaStream_t s);

// Environment-map importance tables on the device (EnvironmentMap.cpp:76-128,
// same single-precision sums in the same order): row CDFs [H][W + 1] and the
// marginal [H + 1] from the RGB pixels and the per-row sin(theta) (computed on
// the host with the reference's expression).  rowW: H floats of scratch.
void launchEnvTables(const float* rgb, int width, int height, const float* sinTheta, float* marginal, float* row,
    float* rowW, cudaStream_t s);

} // namespace pt
