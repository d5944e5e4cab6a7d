// GPU BVH build interface (see pt_bvh.cu).
#pragma once

#include "pt_common.cuh"

#include <cstddef>
#include <cstdint>

namespace pt {

// Grow-only pool of device scratch buffers addressed by slot; reused across
// builds so that a scene rebuild does not re-allocate.
struct DeviceArena {
    static constexpr int kSlots = 24;
    void* ptr[kSlots] = {};
    size_t bytes[kSlots] = {};
    bool failed = false;

    void* getBytes(int slot, size_t n)
    {
        if (n == 0) {
            n = 16;
        }
        if (bytes[slot] < n) {
            if (ptr[slot] != nullptr) {
                cudaFree(ptr[slot]);
                ptr[slot] = nullptr;
                bytes[slot] = 0;
            }
            if (cudaMalloc(&ptr[slot], n) != cudaSuccess) {
                ptr[slot] = nullptr;
                failed = true;
                return nullptr;
            }
            bytes[slot] = n;
        }
        return ptr[slot];
    }
    template <class T> T* get(int slot, size_t count) { return static_cast<T*>(getBytes(slot, count * sizeof(T))); }
    bool ok() const { return !failed; }
    void release()
    {
        for (int i = 0; i < kSlots; ++i) {
            if (ptr[i] != nullptr) {
                cudaFree(ptr[i]);
            }
            ptr[i] = nullptr;
            bytes[i] = 0;
        }
        failed = false;
    }
    size_t totalBytes() const
    {
        size_t t = 0;
        for (int i = 0; i < kSlots; ++i) {
            t += bytes[i];
        }
        return t;
    }
};

// Tuning knobs (compile-time; the defaults are the measured best).
#ifndef PT_BVH_LEAF_SIZE
#define PT_BVH_LEAF_SIZE 3
#endif
#ifndef PT_BVH_TREELET_PASSES
#define PT_BVH_TREELET_PASSES 1
#endif
#ifndef PT_BVH_COST_NODE
#define PT_BVH_COST_NODE 1.2f
#endif
struct BvhBuildOptions {
    int maxLeafSize = PT_BVH_LEAF_SIZE;          // triangles per compressed-node leaf (1..3)
    int treeletPasses = PT_BVH_TREELET_PASSES;   // treelet SAH reordering passes (0 = plain LBVH)
    int treeletMinLeaves = 16;                   // subtrees smaller than this are left as built
    float costTriangle = 1.0f;                   // SAH cost of one triangle test
    float costNode = PT_BVH_COST_NODE;           // SAH cost of one node visit
};

struct BvhBuffers {
    CwNode* nodes = nullptr;
    TriVerts* tris = nullptr;
    uint32_t nodeCount = 0;
    uint32_t triCount = 0;
    int levels = 0;
    size_t nodeCapacity = 0; // allocated entries, kept across builds
    size_t triCapacity = 0;
    DeviceArena scratch;

    // Output arrays for at least `n` nodes and `t` triangles; arrays that are
    // large enough are reused, so a rebuild of a scene that does not grow
    // neither frees nor allocates (cudaFree waits for the whole device).
    bool reserve(size_t n, size_t t)
    {
        if (n > nodeCapacity) {
            if (nodes != nullptr) {
                cudaFree(nodes);
            }
            nodes = nullptr;
            nodeCapacity = 0;
            if (cudaMalloc(&nodes, n * sizeof(CwNode)) != cudaSuccess) {
                nodes = nullptr;
                return false;
            }
            nodeCapacity = n;
        }
        if (t > triCapacity) {
            if (tris != nullptr) {
                cudaFree(tris);
            }
            tris = nullptr;
            triCapacity = 0;
            if (cudaMalloc(&tris, t * sizeof(TriVerts)) != cudaSuccess) {
                tris = nullptr;
                return false;
            }
            triCapacity = t;
        }
        return true;
    }
    void release()
    {
        if (nodes != nullptr) {
            cudaFree(nodes);
        }
        if (tris != nullptr) {
            cudaFree(tris);
        }
        nodes = nullptr;
        tris = nullptr;
        nodeCapacity = triCapacity = 0;
        nodeCount = triCount = 0;
        levels = 0;
    }
};

// Caller-provided scratch for buildBvhInto (n = triangle count):
//   triLo, triHi: n float4; cbounds: 8; keys, vals, keysSorted, valsSorted: n;
//   child: n int2; parent: 2n int; nodeLo, nodeHi: 2n float4; visits: n; frontier: n; frontierCount: 1;
//   subCost: 2n; taskA, taskB: n + 1 int2; counters: 4; sortTemp: sortTempBytes.
struct BvhScratch {
    float4* triLo;
    float4* triHi;
    unsigned int* cbounds;
    uint32_t* keys;
    uint32_t* vals;
    uint32_t* keysSorted;
    uint32_t* valsSorted;
    int2* child;
    int* parent;
    float4* nodeLo;
    float4* nodeHi;
    int* visits;
    float* subCost;
    int* frontier;               // n: nodes where treelet work starts
    unsigned int* frontierCount; // 1
    int2* taskA;
    int2* taskB;
    unsigned int* counters;
    void* sortTemp;
    size_t sortTempBytes;
};

// Radix-sort scratch bytes for n keys (a size query; nothing is launched).
size_t bvhSortTempBytes(uint32_t n);

// Stable LSD radix sort of n (key, value) pairs on the low `bits` bits of the
// keys (pt_sort.cu); keys/vals are left unchanged, the sorted pairs go to
// keysOut/valsOut.  temp needs radixSortTempBytes(n) bytes.
size_t radixSortTempBytes(uint32_t n);
cudaError_t radixSortPairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keysOut, uint32_t* valsOut, uint32_t n,
    int bits, void* temp, size_t tempBytes, cudaStream_t s);

// The build of buildBvh into caller-provided buffers (outNodes: n + 1 nodes,
// outTris: n records); performs no device allocation.
int buildBvhInto(const float* dPositions, uint32_t n, const BvhScratch& scratch, CwNode* outNodes, TriVerts* outTris,
    uint32_t* outNodeCount, cudaStream_t stream, const BvhBuildOptions& opt, char* err, size_t errLen);

// Builds the compressed 8-wide BVH over n triangles whose positions
// (9 floats per triangle) are already in device memory. Synchronises the
// stream once per collapse level. Returns a pt_status code.
int buildBvh(const float* dPositions, uint32_t n, BvhBuffers& out, cudaStream_t stream, const BvhBuildOptions& opt,
    char* err, size_t errLen);

} // namespace pt
