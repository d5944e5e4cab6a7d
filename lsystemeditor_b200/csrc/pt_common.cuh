// Shared device-side types and math for the sm_100a path tracer.
//
// Floating-point policy.  Everything that decides WHICH triangle a ray hits
// (direction normalisation, reciprocal direction, Moller-Trumbore, hit-normal
// and uv interpolation) is written with explicitly rounded intrinsics
// (__fmul_rn / __fadd_rn / __fsub_rn / __fdiv_rn / __fsqrt_rn) so that the
// compiler cannot fuse it into FMAs; it then rounds exactly like the reference
// code compiled without contraction, which is what makes closest-hit ids
// bit-exact.  Shading code may use FMA.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pt_b200.h"

namespace pt {

constexpr float kPi = 3.14159265f;
constexpr float kInvPi = 1.0f / 3.14159265f;
constexpr float kMinPdf = 1.0e-8f;
constexpr float kRayTMax = 1.0e6f;
constexpr float kShadowBias = 1.0e-4f;

// ---------------------------------------------------------------------------
// Exactly-rounded vector helpers (no contraction).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }

__device__ __forceinline__ float xdot(float3 a, float3 b)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float3 xsub(float3 a, float3 b)
{
    return f3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
__device__ __forceinline__ float3 xadd(float3 a, float3 b)
{
    return f3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z));
}
__device__ __forceinline__ float3 xscl(float3 a, float s)
{
    return f3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s));
}
// a.y*b.z - a.z*b.y etc. with separate roundings.
__device__ __forceinline__ float3 xcross(float3 a, float3 b)
{
    return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
        __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
// Normalisation as in the reference's vecNormalize3: zero length -> (0, 0, -1).
__device__ __forceinline__ float3 xnormalize(float3 v)
{
    const float l = __fsqrt_rn(xdot(v, v));
    if (l <= 0.0f) {
        return f3(0.0f, 0.0f, -1.0f);
    }
    const float inv = __fdiv_rn(1.0f, l);
    return xscl(v, inv);
}

// ---------------------------------------------------------------------------
// Ordinary helpers for shading code.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 scl3(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float fmax2(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float fmin2(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 v)
{
    const float l = sqrtf(dot3(v, v));
    if (l <= 0.0f) {
        return f3(0.0f, 0.0f, -1.0f);
    }
    const float inv = 1.0f / l;
    return scl3(v, inv);
}
__device__ __forceinline__ float lum709(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// ---------------------------------------------------------------------------
// Device scene.
// ---------------------------------------------------------------------------

// Compressed 8-wide BVH node, 80 bytes = five 16-byte words (quantised child
// boxes after Ylitie, Karras & Laine, "Efficient Incoherent Ray Traversal on
// GPUs Through Compressed Wide BVHs", HPG 2017):
//   w0: origin p.xyz (float), exponents ex|ey<<8|ez<<16, internal-child mask <<24
//   w1: child node base, triangle base, meta[0..3], meta[4..7]
//   w2: qlo.x[0..7], qlo.y[0..7]      w3: qlo.z[0..7], qhi.x[0..7]
//   w4: qhi.y[0..7], qhi.z[0..7]
// meta per slot: 0 = empty; internal child in slot s = 0x20 | (24 + s);
// leaf with k (1..3) triangles at offset o (0..23) = ((1<<k)-1) << 5 | o.
struct alignas(16) CwNode {
    uint4 w[5];
};
static_assert(sizeof(CwNode) == 80, "compressed node is 80 bytes");

// Per-triangle record for intersection, in BVH leaf order: three float4
// holding v0, v1, v2; v0.w carries the original triangle index.
struct alignas(16) TriVerts {
    float4 v0, v1, v2;
};

// Per-triangle shading record in original order (64 bytes):
//   a = n0.xyz, uv0.x   b = n1.xyz, uv0.y   c = n2.xyz, uv1.x   d = uv1.y, uv2.x, uv2.y, material
struct alignas(16) TriShade {
    float4 a, b, c, d;
};

// Instanced scenes (no reference counterpart; the reference flattens its
// instances into one mesh, MeshSceneContent.h:16-20): an instance places one
// object (a bottom-level BVH) with an affine transform.
struct alignas(16) DevInstance {
    float4 w2o[3]; // world -> object rows (linear part, translation in w)
    float4 o2w[3]; // object -> world rows
    uint4 meta;    // x = object index
};

struct DevBlas {
    const CwNode* nodes;
    const TriVerts* tris;  // leaf order, v0.w = the object's own triangle index
    uint32_t triBase;      // first shading record of the object in the scene's shade array
    uint32_t nodeCount;
};

struct DevScene {
    const CwNode* nodes = nullptr;
    const TriVerts* tris = nullptr;      // leaf order
    const TriShade* shade = nullptr;     // original order
    const float4* origVerts = nullptr;   // original order, 9 floats per triangle (emissive sampling)
    const pt_material* materials = nullptr;
    const pt_texture* textures = nullptr;
    const uint32_t* emissiveIdx = nullptr;
    const float* emissiveCdf = nullptr;
    // per original triangle: the probability density (per unit area) with which
    // emissive NEE picks a point of it, 0 for non-emitters (emitter MIS mode)
    const float* emitPdfArea = nullptr;
    // spectral mode: spectrum coefficients (c0, c1, c2, scale) of each
    // material's base colour [2 m] and scatter radii [2 m + 1], and of each
    // albedo texture's colours [2 t] (constant / grid colour 1), [2 t + 1] (grid colour 2)
    const float4* matSpec = nullptr;
    const float4* texSpec = nullptr;
    // instanced scene (instanceCount > 0): a top-level BVH over the instances'
    // world boxes (its leaf records hold the instance index in v0.w), the
    // instances and their objects; nodes / tris above are then unused and the
    // shading records of all objects are concatenated in `shade`
    const CwNode* tlasNodes = nullptr;
    const TriVerts* tlasLeaves = nullptr;
    const DevInstance* instances = nullptr;
    const DevBlas* blases = nullptr;
    uint32_t instanceCount = 0;
    uint32_t nodeCount = 0;
    uint32_t triCount = 0;
    uint32_t materialCount = 0;
    uint32_t textureCount = 0;
    uint32_t emissiveCount = 0;
};

struct DevEnv {
    const float* pixels = nullptr; // RGB lat-long
    const float* marginal = nullptr;
    const float* row = nullptr;
    const float4* spec = nullptr;  // spectral mode: per-texel radiance spectrum coefficients
    int width = 0;
    int height = 0;
    int valid = 0;
};

} // namespace pt
