// GPU acceleration-structure build: LBVH -> compressed 8-wide BVH.
//
// Replaces the reference's host-side median-split builder
// (PathTracerLib/src/MeshAccel/MeshBvhBuilder.cpp:52-142, O(N log^2 N) on one
// core) with a fully parallel build:
//   1. per-triangle bounds + centroid, centroid bounds       (k_prepare)
//   2. 30-bit Morton codes of the centroids                   (k_morton)
//   3. radix sort of (code, index) pairs                      (CUB onesweep)
//   4. binary radix tree, Karras 2012 "Maximizing Parallelism in the
//      Construction of BVHs, Octrees, and k-d Trees"         (k_karras)
//   5. bottom-up bounds + leaf counts                         (k_refit)
//   6. treelet reordering of the binary tree for SAH cost,
//      after Karras & Aila 2013 "Fast Parallel Construction of
//      High-Quality Bounding Volume Hierarchies"             (k_treelet)
//   7. top-down collapse to 8-wide nodes with quantised child boxes and
//      octant-ordered child slots, Ylitie, Karras & Laine 2017 (k_collapse)
//
// Closest-hit results do not depend on the tree shape (any BVH whose boxes
// contain their triangles returns the same nearest hit), so the product
// builds whatever tree traverses fastest.
#include "pt_bvh.cuh"


#include <cfloat>
#include <cmath>
#include <cstdio>

namespace pt {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ unsigned int floatToOrdered(float f)
{
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float orderedToFloat(unsigned int u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ float3 loadVertex(const float* pos, uint32_t tri, int k)
{
    const float* p = pos + 9ull * tri + 3 * k;
    return make_float3(p[0], p[1], p[2]);
}

// (1) triangle bounds, centroids and the centroid bounding box.
__global__ void k_prepare(const float* __restrict__ pos, uint32_t n, float4* __restrict__ triLo,
    float4* __restrict__ triHi, unsigned int* __restrict__ cbounds)
{
    float3 cmin = make_float3(FLT_MAX, FLT_MAX, FLT_MAX);
    float3 cmax = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float3 a = loadVertex(pos, i, 0), b = loadVertex(pos, i, 1), c = loadVertex(pos, i, 2);
        const float3 lo = make_float3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
        const float3 hi = make_float3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
        triLo[i] = make_float4(lo.x, lo.y, lo.z, 0.0f);
        triHi[i] = make_float4(hi.x, hi.y, hi.z, 0.0f);
        const float3 ce = make_float3((lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f);
        cmin = make_float3(fminf(cmin.x, ce.x), fminf(cmin.y, ce.y), fminf(cmin.z, ce.z));
        cmax = make_float3(fmaxf(cmax.x, ce.x), fmaxf(cmax.y, ce.y), fmaxf(cmax.z, ce.z));
    }
    // warp reduce, then one atomic per warp
    for (int off = 16; off > 0; off >>= 1) {
        cmin.x = fminf(cmin.x, __shfl_xor_sync(0xffffffffu, cmin.x, off));
        cmin.y = fminf(cmin.y, __shfl_xor_sync(0xffffffffu, cmin.y, off));
        cmin.z = fminf(cmin.z, __shfl_xor_sync(0xffffffffu, cmin.z, off));
        cmax.x = fmaxf(cmax.x, __shfl_xor_sync(0xffffffffu, cmax.x, off));
        cmax.y = fmaxf(cmax.y, __shfl_xor_sync(0xffffffffu, cmax.y, off));
        cmax.z = fmaxf(cmax.z, __shfl_xor_sync(0xffffffffu, cmax.z, off));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&cbounds[0], floatToOrdered(cmin.x));
        atomicMin(&cbounds[1], floatToOrdered(cmin.y));
        atomicMin(&cbounds[2], floatToOrdered(cmin.z));
        atomicMax(&cbounds[3], floatToOrdered(cmax.x));
        atomicMax(&cbounds[4], floatToOrdered(cmax.y));
        atomicMax(&cbounds[5], floatToOrdered(cmax.z));
    }
}

__device__ __forceinline__ uint32_t expandBits10(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// (2) Morton codes of the box centroids in the centroid bounds.
__global__ void k_morton(const float4* __restrict__ triLo, const float4* __restrict__ triHi, uint32_t n,
    const unsigned int* __restrict__ cbounds, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
    const float3 lo = make_float3(orderedToFloat(cbounds[0]), orderedToFloat(cbounds[1]), orderedToFloat(cbounds[2]));
    const float3 hi = make_float3(orderedToFloat(cbounds[3]), orderedToFloat(cbounds[4]), orderedToFloat(cbounds[5]));
    const float3 ext = make_float3(hi.x - lo.x, hi.y - lo.y, hi.z - lo.z);
    const float3 inv = make_float3(ext.x > 0.0f ? 1.0f / ext.x : 0.0f, ext.y > 0.0f ? 1.0f / ext.y : 0.0f,
        ext.z > 0.0f ? 1.0f / ext.z : 0.0f);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = triLo[i], b = triHi[i];
        const float cx = ((a.x + b.x) * 0.5f - lo.x) * inv.x;
        const float cy = ((a.y + b.y) * 0.5f - lo.y) * inv.y;
        const float cz = ((a.z + b.z) * 0.5f - lo.z) * inv.z;
        const uint32_t x = min(max(__float2int_rd(cx * 1024.0f), 0), 1023);
        const uint32_t y = min(max(__float2int_rd(cy * 1024.0f), 0), 1023);
        const uint32_t z = min(max(__float2int_rd(cz * 1024.0f), 0), 1023);
        keys[i] = (expandBits10(x) << 2) | (expandBits10(y) << 1) | expandBits10(z);
        vals[i] = i;
    }
}

// Common-prefix length of sorted keys i, j with the position as tie-breaker.
__device__ __forceinline__ int delta(const uint32_t* __restrict__ k, int n, int i, int j)
{
    if (j < 0 || j >= n) {
        return -1;
    }
    const uint32_t a = k[i], b = k[j];
    if (a != b) {
        return __clz(a ^ b);
    }
    return 32 + __clz(static_cast<uint32_t>(i) ^ static_cast<uint32_t>(j));
}

// (4) Karras radix tree. Internal nodes 0..n-2, leaf j is node n-1+j.
__global__ void k_karras(const uint32_t* __restrict__ keys, int n, int2* __restrict__ child, int* __restrict__ parent)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = delta(keys, n, i, i - d);
        int lmax = 2;
        while (delta(keys, n, i, i + lmax * d) > dmin) {
            lmax <<= 1;
        }
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1) {
            if (delta(keys, n, i, i + (l + t) * d) > dmin) {
                l += t;
            }
        }
        const int j = i + l * d;
        const int dnode = delta(keys, n, i, j);
        int s = 0;
        int t = l;
        do {
            t = (t + 1) >> 1;
            if (delta(keys, n, i, i + (s + t) * d) > dnode) {
                s += t;
            }
        } while (t > 1);
        const int gamma = i + s * d + min(d, 0);
        const int left = (min(i, j) == gamma) ? (n - 1 + gamma) : gamma;
        const int right = (max(i, j) == gamma + 1) ? (n - 1 + gamma + 1) : gamma + 1;
        child[i] = make_int2(left, right);
        parent[left] = i;
        parent[right] = i;
    }
}

// (5) Bottom-up bounds. Node bounds: lo.xyz + leaf count (w, int bits), hi.xyz + area (w).
__global__ void k_refit(const uint32_t* __restrict__ sortedIdx, const float4* __restrict__ triLo,
    const float4* __restrict__ triHi, int n, const int2* __restrict__ child, const int* __restrict__ parent,
    float4* nodeLo, float4* nodeHi, int* visits)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        int node = n - 1 + j;
        const uint32_t tri = sortedIdx[j];
        float4 lo = triLo[tri], hi = triHi[tri];
        lo.w = __int_as_float(1);
        hi.w = 2.0f * ((hi.x - lo.x) * (hi.y - lo.y) + (hi.y - lo.y) * (hi.z - lo.z) + (hi.z - lo.z) * (hi.x - lo.x));
        nodeLo[node] = lo;
        nodeHi[node] = hi;
        if (n == 1) {
            continue;
        }
        __threadfence();
        int p = parent[node];
        while (p >= 0) {
            if (atomicAdd(&visits[p], 1) == 0) {
                break; // the sibling's thread finishes this node
            }
            __threadfence();
            const int2 c = child[p];
            const float4 al = __ldcg(&nodeLo[c.x]), ah = __ldcg(&nodeHi[c.x]);
            const float4 bl = __ldcg(&nodeLo[c.y]), bh = __ldcg(&nodeHi[c.y]);
            float4 ml = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z),
                __int_as_float(__float_as_int(al.w) + __float_as_int(bl.w)));
            float4 mh = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
            mh.w = 2.0f * ((mh.x - ml.x) * (mh.y - ml.y) + (mh.y - ml.y) * (mh.z - ml.z) + (mh.z - ml.z) * (mh.x - ml.x));
            __stcg(&nodeLo[p], ml);
            __stcg(&nodeHi[p], mh);
            __threadfence();
            p = parent[p];
        }
    }
}

__device__ __forceinline__ float boxArea(float3 lo, float3 hi)
{
    const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// (6) Treelet restructuring (Karras & Aila 2013): every node whose subtree
// holds at least `minLeaves` triangles forms a treelet of up to 7 leaves by
// repeatedly opening its largest-area leaf; the optimal binary topology over
// those leaves is found by dynamic programming over leaf subsets with the SAH
// cost, and the treelet is rewritten in place. Processed bottom-up, one
// treelet per warp, with visit counters like k_refit so that a node is
// optimised only after both subtrees are final.
constexpr int kTreeletLeaves = 7;
constexpr int kSubsets = 1 << kTreeletLeaves;

struct TreeletScratch {
    float area[kSubsets];
    float cost[kSubsets];
    uint8_t split[kSubsets];
    float4 lo[kSubsets];
    float4 hi[kSubsets];
};

__device__ __forceinline__ bool isLeafNode(int node, int n) { return node >= n - 1; }

__device__ void treeletOptimize(int root, int n, int2* child, int* parent, float4* nodeLo, float4* nodeHi,
    float* subtreeCost, TreeletScratch& s, float costNode)
{
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    __shared__ int sLeaves[kBlock / 32][kTreeletLeaves];
    __shared__ int sInternals[kBlock / 32][kTreeletLeaves - 1];
    __shared__ int sLeafCount[kBlock / 32];
    // --- form the treelet: open the largest-area treelet leaf until 7 leaves ---
    if (lane == 0) {
        int leaves[kTreeletLeaves];
        int internals[kTreeletLeaves - 1];
        int nl = 2, ni = 1;
        internals[0] = root;
        const int2 c = __ldcg(&child[root]);
        leaves[0] = c.x;
        leaves[1] = c.y;
        while (nl < kTreeletLeaves) {
            int best = -1;
            float bestArea = -1.0f;
            for (int k = 0; k < nl; ++k) {
                if (!isLeafNode(leaves[k], n)) {
                    const float a = __ldcg(&nodeHi[leaves[k]]).w;
                    if (a > bestArea) {
                        bestArea = a;
                        best = k;
                    }
                }
            }
            if (best < 0) {
                break;
            }
            const int opened = leaves[best];
            internals[ni++] = opened;
            const int2 cc = __ldcg(&child[opened]);
            leaves[best] = cc.x;
            leaves[nl++] = cc.y;
        }
        for (int k = 0; k < nl; ++k) {
            sLeaves[w][k] = leaves[k];
        }
        for (int k = 0; k < ni; ++k) {
            sInternals[w][k] = internals[k];
        }
        sLeafCount[w] = nl;
    }
    __syncwarp();
    const int nl = sLeafCount[w];
    if (nl < 3) {
        return;
    }
    const int subsets = 1 << nl;
    // --- bounds, triangle counts and areas of every leaf subset ---
    for (int m = lane + 1; m < subsets; m += 32) {
        float3 lo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), hi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
        int tris = 0;
        for (int k = 0; k < nl; ++k) {
            if (m & (1 << k)) {
                const float4 a = __ldcg(&nodeLo[sLeaves[w][k]]), b = __ldcg(&nodeHi[sLeaves[w][k]]);
                lo = make_float3(fminf(lo.x, a.x), fminf(lo.y, a.y), fminf(lo.z, a.z));
                hi = make_float3(fmaxf(hi.x, b.x), fmaxf(hi.y, b.y), fmaxf(hi.z, b.z));
                tris += __float_as_int(a.w);
            }
        }
        s.lo[m] = make_float4(lo.x, lo.y, lo.z, __int_as_float(tris));
        s.hi[m] = make_float4(hi.x, hi.y, hi.z, 0.0f);
        s.area[m] = boxArea(lo, hi);
        if (__popc(m) == 1) {
            // a treelet leaf keeps its (already optimised) subtree
            s.cost[m] = __ldcg(&subtreeCost[sLeaves[w][__ffs(m) - 1]]);
            s.split[m] = 0;
        }
    }
    __syncwarp();
    // --- SAH-optimal topology by dynamic programming over subsets of growing size ---
    for (int size = 2; size <= nl; ++size) {
        for (int m = lane + 1; m < subsets; m += 32) {
            if (__popc(m) != size) {
                continue;
            }
            float best = FLT_MAX;
            int bestP = 0;
            const int low = m & -m;
            for (int p = (m - 1) & m; p > 0; p = (p - 1) & m) {
                if ((p & low) == 0) {
                    continue; // each partition once
                }
                const float c = s.cost[p] + s.cost[m ^ p];
                if (c < best) {
                    best = c;
                    bestP = p;
                }
            }
            s.cost[m] = costNode * s.area[m] + best;
            s.split[m] = static_cast<uint8_t>(bestP);
        }
        __syncwarp();
    }
    // --- rewrite the treelet in place, reusing its internal node ids ---
    if (lane == 0) {
        int stackM[kTreeletLeaves];
        int stackNode[kTreeletLeaves];
        int sp = 0;
        int nextInternal = 1;
        stackM[sp] = subsets - 1;
        stackNode[sp] = root;
        ++sp;
        while (sp > 0) {
            --sp;
            const int m = stackM[sp];
            const int node = stackNode[sp];
            const int parts[2] = {static_cast<int>(s.split[m]), m ^ static_cast<int>(s.split[m])};
            int kids[2];
            for (int h = 0; h < 2; ++h) {
                if (__popc(parts[h]) == 1) {
                    kids[h] = sLeaves[w][__ffs(parts[h]) - 1];
                } else {
                    kids[h] = sInternals[w][nextInternal++];
                    stackM[sp] = parts[h];
                    stackNode[sp] = kids[h];
                    ++sp;
                }
                parent[kids[h]] = node;
            }
            child[node] = make_int2(kids[0], kids[1]);
            float4 hi = s.hi[m];
            hi.w = s.area[m];
            __stcg(&nodeLo[node], s.lo[m]);
            __stcg(&nodeHi[node], hi);
            __stcg(&subtreeCost[node], s.cost[m]);
        }
    }
    __threadfence();
    __syncwarp();
}

// One warp per leaf climbs towards the root; the warp that reaches a node
// second (both subtrees final) optimises the treelet rooted there.
// Bottom-up pass of the subtrees too small for treelets, one thread per leaf
// (as the refit): the SAH cost of every subtree with fewer than minLeaves
// triangles, and the list of the nodes where treelet work starts (at least
// minLeaves triangles, both children finished here).  The second thread to
// reach a node goes on; the first stops.
__global__ void k_treelet_leaves(int n, const int2* child, const int* parent, const float4* nodeLo,
    const float4* nodeHi, int* visits, float* subtreeCost, int minLeaves, float costTri, float costNode,
    int* frontier, unsigned int* frontierCount)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int leaf = n - 1 + j;
        __stcg(&subtreeCost[leaf], costTri * __ldcg(&nodeHi[leaf]).w);
        __threadfence();
        int p = __ldcg(&parent[leaf]);
        while (p >= 0) {
            if (atomicAdd(&visits[p], 1) == 0) {
                break;
            }
            __threadfence();
            if (__float_as_int(__ldcg(&nodeLo[p]).w) >= minLeaves) {
                frontier[atomicAdd(frontierCount, 1u)] = p;
                break;
            }
            const int2 c = __ldcg(&child[p]);
            __stcg(&subtreeCost[p],
                costNode * __ldcg(&nodeHi[p]).w + __ldcg(&subtreeCost[c.x]) + __ldcg(&subtreeCost[c.y]));
            __threadfence();
            p = __ldcg(&parent[p]);
        }
    }
}

// Treelet reordering (Karras & Aila 2013), one warp per node of the frontier
// list and then up the tree: a node is optimised by the second warp to reach it
// (its first arrival may have come from k_treelet_leaves, for a small child).
// Every node from the frontier up has at least minLeaves triangles.
__global__ void k_treelet(int n, int2* child, int* parent, float4* nodeLo, float4* nodeHi, int* visits,
    float* subtreeCost, float costNode, const int* frontier, const unsigned int* frontierCount)
{
    __shared__ TreeletScratch scratch[kBlock / 32];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    TreeletScratch& s = scratch[threadIdx.x >> 5];
    const int count = static_cast<int>(*frontierCount);
    for (int f = warp; f < count; f += warps) {
        int p = frontier[f];
        for (;;) {
            treeletOptimize(p, n, child, parent, nodeLo, nodeHi, subtreeCost, s, costNode);
            __threadfence();
            p = __shfl_sync(0xffffffffu, lane == 0 ? __ldcg(&parent[p]) : 0, 0);
            if (p < 0) {
                break;
            }
            int arrived = 0;
            if (lane == 0) {
                arrived = atomicAdd(&visits[p], 1);
            }
            arrived = __shfl_sync(0xffffffffu, arrived, 0);
            if (arrived == 0) {
                break;
            }
            __threadfence();
        }
    }
}

// The treelet passes of a build: per pass, the small subtrees bottom-up (one
// thread per leaf), then the treelets from the frontier up (one warp per
// frontier node, a grid of resident warps).
static cudaError_t runTreelets(int N, int2* child, int* parent, float4* nodeLo, float4* nodeHi, int* visits,
    float* subCost, int* frontier, unsigned int* frontierCount, const BvhBuildOptions& opt, cudaStream_t stream)
{
    for (int pass = 0; pass < opt.treeletPasses; ++pass) {
        cudaError_t e = cudaMemsetAsync(visits, 0, sizeof(int) * (N - 1), stream);
        if (e == cudaSuccess) {
            e = cudaMemsetAsync(frontierCount, 0, sizeof(unsigned int), stream);
        }
        if (e != cudaSuccess) {
            return e;
        }
        k_treelet_leaves<<<(N + kBlock - 1) / kBlock, kBlock, 0, stream>>>(N, child, parent, nodeLo, nodeHi, visits, subCost,
            opt.treeletMinLeaves, opt.costTriangle, opt.costNode, frontier, frontierCount);
        int dev = 0, sms = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_treelet<<<sms * 4, kBlock, 0, stream>>>(N, child, parent, nodeLo, nodeHi, visits, subCost, opt.costNode,
            frontier, frontierCount);
    }
    return cudaGetLastError();
}

// (7) Collapse to 8-wide compressed nodes. One thread per task (binary node ->
// compressed node slot). Emits the next level's tasks.
struct CollapseArgs {
    int n;
    const int2* child;
    const float4* nodeLo;
    const float4* nodeHi;
    const uint32_t* sortedIdx;
    const float* pos;
    CwNode* cw;
    TriVerts* tris;
    unsigned int* counters; // [0] next node, [1] next triangle
    int maxLeafSize;
};

// Smallest exponent e with extent <= 255 * 2^e (extent computed exactly in double).
__device__ __forceinline__ int quantExp(double extent)
{
    if (!(extent > 0.0)) {
        return -126;
    }
    int e;
    frexp(extent / 255.0, &e); // extent/255 in [2^(e-1), 2^e)
    e -= 1;
    while (ldexp(255.0, e) < extent) {
        ++e;
    }
    return max(e, -126);
}

__global__ void k_collapse(CollapseArgs a, const int2* __restrict__ tasks, int taskCount, int2* __restrict__ nextTasks,
    unsigned int* __restrict__ nextCount)
{
    for (int ti = blockIdx.x * blockDim.x + threadIdx.x; ti < taskCount; ti += gridDim.x * blockDim.x) {
        const int bnode = tasks[ti].x;
        const int cwIndex = tasks[ti].y;
        int cand[8];
        int nc = 0;
        if (isLeafNode(bnode, a.n)) {
            cand[nc++] = bnode;
        } else {
            const int2 c = a.child[bnode];
            cand[nc++] = c.x;
            cand[nc++] = c.y;
        }
        // Open the largest-area candidate until 8 slots are used: first those
        // that are too big for a leaf, then the remaining internal ones.
        while (nc < 8) {
            int best = -1;
            float bestArea = -1.0f;
            bool bestBig = false;
            for (int k = 0; k < nc; ++k) {
                if (isLeafNode(cand[k], a.n)) {
                    continue;
                }
                const bool big = __float_as_int(a.nodeLo[cand[k]].w) > a.maxLeafSize;
                const float ar = a.nodeHi[cand[k]].w;
                if ((big && !bestBig) || (big == bestBig && ar > bestArea)) {
                    best = k;
                    bestArea = ar;
                    bestBig = big;
                }
            }
            if (best < 0) {
                break;
            }
            const int2 c = a.child[cand[best]];
            cand[best] = c.x;
            cand[nc++] = c.y;
        }
        // Node bounds.
        const float4 nl4 = a.nodeLo[bnode], nh4 = a.nodeHi[bnode];
        const float3 lo = make_float3(nl4.x, nl4.y, nl4.z);
        const float3 hi = make_float3(nh4.x, nh4.y, nh4.z);
        const int ex = quantExp(static_cast<double>(hi.x) - lo.x), ey = quantExp(static_cast<double>(hi.y) - lo.y),
                  ez = quantExp(static_cast<double>(hi.z) - lo.z);
        const double sx = ldexp(1.0, ex), sy = ldexp(1.0, ey), sz = ldexp(1.0, ez);
        // Octant-ordered slot assignment: slot s receives the child that is nearest
        // for rays whose direction signs are s (bit 2 = -x, bit 1 = -y, bit 0 = -z).
        const float3 nc3 = make_float3((lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f);
        float cost[8][8];
        for (int k = 0; k < nc; ++k) {
            const float4 cl = a.nodeLo[cand[k]], ch = a.nodeHi[cand[k]];
            const float3 d = make_float3((cl.x + ch.x) * 0.5f - nc3.x, (cl.y + ch.y) * 0.5f - nc3.y,
                (cl.z + ch.z) * 0.5f - nc3.z);
            for (int s = 0; s < 8; ++s) {
                const float dx = (s & 4) ? -d.x : d.x;
                const float dy = (s & 2) ? -d.y : d.y;
                const float dz = (s & 1) ? -d.z : d.z;
                cost[k][s] = dx + dy + dz;
            }
        }
        int slotOf[8];
        int bySlot[8];
        for (int s = 0; s < 8; ++s) {
            bySlot[s] = -1;
        }
        for (int k = 0; k < nc; ++k) {
            slotOf[k] = -1;
        }
        for (int round = 0; round < nc; ++round) {
            float best = FLT_MAX;
            int bk = -1, bs = -1;
            for (int k = 0; k < nc; ++k) {
                if (slotOf[k] >= 0) {
                    continue;
                }
                for (int s = 0; s < 8; ++s) {
                    if (bySlot[s] >= 0) {
                        continue;
                    }
                    if (cost[k][s] < best || bk < 0) {
                        best = cost[k][s];
                        bk = k;
                        bs = s;
                    }
                }
            }
            slotOf[bk] = bs;
            bySlot[bs] = bk;
        }
        // Count internal children and leaf triangles.
        int internals = 0, triTotal = 0;
        for (int k = 0; k < nc; ++k) {
            const int cnt = __float_as_int(a.nodeLo[cand[k]].w);
            if (cnt > a.maxLeafSize) {
                ++internals;
            } else {
                triTotal += cnt;
            }
        }
        const unsigned int childBase = internals ? atomicAdd(&a.counters[0], static_cast<unsigned>(internals)) : 0u;
        const unsigned int triBase = triTotal ? atomicAdd(&a.counters[1], static_cast<unsigned>(triTotal)) : 0u;
        unsigned int taskBase = internals ? atomicAdd(nextCount, static_cast<unsigned>(internals)) : 0u;

        uint8_t meta[8], qlo[3][8], qhi[3][8];
        unsigned int imask = 0;
        int rank = 0, triOff = 0;
        for (int s = 0; s < 8; ++s) {
            meta[s] = 0;
            qlo[0][s] = qlo[1][s] = qlo[2][s] = 0;
            qhi[0][s] = qhi[1][s] = qhi[2][s] = 0;
            const int k = bySlot[s];
            if (k < 0) {
                continue;
            }
            const int c = cand[k];
            const float4 cl = a.nodeLo[c], ch = a.nodeHi[c];
            const float clv[3] = {cl.x, cl.y, cl.z};
            const float chv[3] = {ch.x, ch.y, ch.z};
            const float pv[3] = {lo.x, lo.y, lo.z};
            const double sv[3] = {sx, sy, sz};
            for (int ax = 0; ax < 3; ++ax) {
                const double ql = floor((static_cast<double>(clv[ax]) - static_cast<double>(pv[ax])) / sv[ax]);
                const double qh = ceil((static_cast<double>(chv[ax]) - static_cast<double>(pv[ax])) / sv[ax]);
                qlo[ax][s] = static_cast<uint8_t>(fmin(fmax(ql, 0.0), 255.0));
                qhi[ax][s] = static_cast<uint8_t>(fmin(fmax(qh, 0.0), 255.0));
            }
            const int cnt = __float_as_int(cl.w);
            if (cnt > a.maxLeafSize) {
                meta[s] = static_cast<uint8_t>(0x20 | (24 + s));
                imask |= 1u << s;
                nextTasks[taskBase + rank] = make_int2(c, static_cast<int>(childBase) + rank);
                ++rank;
            } else {
                meta[s] = static_cast<uint8_t>((((1 << cnt) - 1) << 5) | triOff);
                // gather the subtree's triangles (at most maxLeafSize leaves)
                int st[8];
                int sp = 0;
                st[sp++] = c;
                while (sp > 0) {
                    const int x = st[--sp];
                    if (isLeafNode(x, a.n)) {
                        const uint32_t tri = a.sortedIdx[x - (a.n - 1)];
                        const float3 v0 = loadVertex(a.pos, tri, 0), v1 = loadVertex(a.pos, tri, 1),
                                     v2 = loadVertex(a.pos, tri, 2);
                        TriVerts tv;
                        tv.v0 = make_float4(v0.x, v0.y, v0.z, __uint_as_float(tri));
                        tv.v1 = make_float4(v1.x, v1.y, v1.z, 0.0f);
                        tv.v2 = make_float4(v2.x, v2.y, v2.z, 0.0f);
                        a.tris[triBase + triOff] = tv;
                        ++triOff;
                    } else {
                        const int2 cc = a.child[x];
                        st[sp++] = cc.y;
                        st[sp++] = cc.x;
                    }
                }
            }
        }
        CwNode node;
        node.w[0] = make_uint4(__float_as_uint(lo.x), __float_as_uint(lo.y), __float_as_uint(lo.z),
            static_cast<unsigned>(ex + 127) | (static_cast<unsigned>(ey + 127) << 8) |
                (static_cast<unsigned>(ez + 127) << 16) | (imask << 24));
        auto pack4 = [](const uint8_t* b) {
            return static_cast<unsigned>(b[0]) | (static_cast<unsigned>(b[1]) << 8) |
                (static_cast<unsigned>(b[2]) << 16) | (static_cast<unsigned>(b[3]) << 24);
        };
        node.w[1] = make_uint4(childBase, triBase, pack4(meta), pack4(meta + 4));
        node.w[2] = make_uint4(pack4(qlo[0]), pack4(qlo[0] + 4), pack4(qlo[1]), pack4(qlo[1] + 4));
        node.w[3] = make_uint4(pack4(qlo[2]), pack4(qlo[2] + 4), pack4(qhi[0]), pack4(qhi[0] + 4));
        node.w[4] = make_uint4(pack4(qhi[1]), pack4(qhi[1] + 4), pack4(qhi[2]), pack4(qhi[2] + 4));
        a.cw[cwIndex] = node;
    }
}

inline int gridFor(long long n, int block = kBlock)
{
    long long g = (n + block - 1) / block;
    if (g < 1) {
        g = 1;
    }
    if (g > 148 * 32) {
        g = 148 * 32;
    }
    return static_cast<int>(g);
}

} // namespace

#define PT_TRY(call)                                                                                              \
    do {                                                                                                          \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess) {                                                                                  \
            std::snprintf(err, errLen, "%s failed: %s", #call, cudaGetErrorString(e_));                          \
            return e_ == cudaErrorMemoryAllocation ? PT_ERR_OUT_OF_MEMORY : PT_ERR_CUDA;                          \
        }                                                                                                         \
    } while (0)

int buildBvh(const float* dPositions, uint32_t n, BvhBuffers& out, cudaStream_t stream, const BvhBuildOptions& opt,
    char* err, size_t errLen)
{
    out.nodeCount = out.triCount = 0;
    out.levels = 0;
    if (n == 0) {
        return PT_OK;
    }
    const int N = static_cast<int>(n);
    const int nodesBin = 2 * N - 1;
    DeviceArena& ar = out.scratch;
    float4* triLo = ar.get<float4>(0, n);
    float4* triHi = ar.get<float4>(1, n);
    unsigned int* cbounds = ar.get<unsigned int>(2, 8);
    uint32_t* keys = ar.get<uint32_t>(3, n);
    uint32_t* vals = ar.get<uint32_t>(4, n);
    uint32_t* keysSorted = ar.get<uint32_t>(5, n);
    uint32_t* valsSorted = ar.get<uint32_t>(6, n);
    int2* child = ar.get<int2>(7, static_cast<size_t>(N > 1 ? N - 1 : 1));
    int* parent = ar.get<int>(8, static_cast<size_t>(nodesBin));
    float4* nodeLo = ar.get<float4>(9, static_cast<size_t>(nodesBin));
    float4* nodeHi = ar.get<float4>(10, static_cast<size_t>(nodesBin));
    int* visits = ar.get<int>(11, static_cast<size_t>(N > 1 ? N - 1 : 1));
    float* subCost = ar.get<float>(12, static_cast<size_t>(nodesBin));
    if (!ar.ok()) {
        std::snprintf(err, errLen, "BVH scratch allocation failed (%u triangles)", n);
        return PT_ERR_OUT_OF_MEMORY;
    }

    // bounds sentinel: min slots get 0xFFFFFFFF, max slots 0
    const unsigned int init[8] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u, 0u, 0u};
    PT_TRY(cudaMemcpyAsync(cbounds, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    k_prepare<<<gridFor(n), kBlock, 0, stream>>>(dPositions, n, triLo, triHi, cbounds);
    k_morton<<<gridFor(n), kBlock, 0, stream>>>(triLo, triHi, n, cbounds, keys, vals);
    const size_t tempBytes = radixSortTempBytes(n);
    void* temp = ar.getBytes(13, tempBytes);
    if (!ar.ok()) {
        std::snprintf(err, errLen, "radix sort scratch allocation failed");
        return PT_ERR_OUT_OF_MEMORY;
    }
    PT_TRY(radixSortPairs(keys, vals, keysSorted, valsSorted, n, 30, temp, tempBytes, stream));
    PT_TRY(cudaMemsetAsync(parent, 0xff, sizeof(int) * nodesBin, stream));
    if (N > 1) {
        k_karras<<<gridFor(N - 1), kBlock, 0, stream>>>(keysSorted, N, child, parent);
        PT_TRY(cudaMemsetAsync(visits, 0, sizeof(int) * (N - 1), stream));
    }
    k_refit<<<gridFor(N), kBlock, 0, stream>>>(valsSorted, triLo, triHi, N, child, parent, nodeLo, nodeHi, visits);
    if (N > 1 && opt.treeletPasses > 0) {
        int* frontier = ar.get<int>(17, static_cast<size_t>(N - 1));
        unsigned int* frontierCount = ar.get<unsigned int>(18, 1);
        if (!ar.ok()) {
            std::snprintf(err, errLen, "treelet scratch allocation failed");
            return PT_ERR_OUT_OF_MEMORY;
        }
        PT_TRY(runTreelets(N, child, parent, nodeLo, nodeHi, visits, subCost, frontier, frontierCount, opt, stream));
    }
    PT_TRY(cudaGetLastError());

    // Collapse. Upper bounds: nodes <= n (every compressed node has >= 2 children or is the root),
    // triangles == n.
    const size_t maxNodes = static_cast<size_t>(n) + 1;
    if (!out.reserve(maxNodes, static_cast<size_t>(n))) {
        std::snprintf(err, errLen, "BVH output allocation failed (%u triangles)", n);
        out.release();
        return PT_ERR_OUT_OF_MEMORY;
    }
    int2* taskA = ar.get<int2>(14, maxNodes);
    int2* taskB = ar.get<int2>(15, maxNodes);
    unsigned int* counters = ar.get<unsigned int>(16, 4);
    if (!ar.ok()) {
        std::snprintf(err, errLen, "collapse scratch allocation failed");
        return PT_ERR_OUT_OF_MEMORY;
    }
    // counters: [0] next node (root = 0 already taken), [1] next triangle, [2] next task count
    const unsigned int cinit[4] = {1u, 0u, 0u, 0u};
    PT_TRY(cudaMemcpyAsync(counters, cinit, sizeof(cinit), cudaMemcpyHostToDevice, stream));
    const int rootBin = N > 1 ? 0 : 0; // internal root 0, or the single leaf node 0 (= n - 1) when n == 1
    const int2 rootTask = make_int2(N > 1 ? rootBin : 0, 0);
    PT_TRY(cudaMemcpyAsync(taskA, &rootTask, sizeof(int2), cudaMemcpyHostToDevice, stream));
    CollapseArgs ca{N, child, nodeLo, nodeHi, valsSorted, dPositions, out.nodes, out.tris, counters, opt.maxLeafSize};
    int taskCount = 1;
    int levels = 0;
    while (taskCount > 0) {
        PT_TRY(cudaMemsetAsync(counters + 2, 0, sizeof(unsigned int), stream));
        k_collapse<<<gridFor(taskCount, 64), 64, 0, stream>>>(ca, taskA, taskCount, taskB, counters + 2);
        unsigned int next = 0;
        PT_TRY(cudaMemcpyAsync(&next, counters + 2, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream));
        PT_TRY(cudaStreamSynchronize(stream));
        taskCount = static_cast<int>(next);
        int2* t = taskA;
        taskA = taskB;
        taskB = t;
        if (++levels > 256) {
            std::snprintf(err, errLen, "BVH collapse did not terminate");
            return PT_ERR_INTERNAL;
        }
    }
    unsigned int finalCounts[2] = {0, 0};
    PT_TRY(cudaMemcpyAsync(finalCounts, counters, sizeof(finalCounts), cudaMemcpyDeviceToHost, stream));
    PT_TRY(cudaStreamSynchronize(stream));
    out.nodeCount = finalCounts[0];
    out.triCount = finalCounts[1];
    out.levels = levels;
    if (out.triCount != n) {
        std::snprintf(err, errLen, "BVH collapse placed %u of %u triangles", out.triCount, n);
        return PT_ERR_INTERNAL;
    }
    return PT_OK;
}

} // namespace pt

namespace pt {

size_t bvhSortTempBytes(uint32_t n)
{
    return radixSortTempBytes(n);
}

// Same build as buildBvh, into caller-provided buffers: nothing is allocated.
int buildBvhInto(const float* dPositions, uint32_t n, const BvhScratch& sc, CwNode* outNodes, TriVerts* outTris,
    uint32_t* outNodeCount, cudaStream_t stream, const BvhBuildOptions& opt, char* err, size_t errLen)
{
    if (n == 0) {
        *outNodeCount = 0;
        return PT_OK;
    }
    const int N = static_cast<int>(n);
    const int nodesBin = 2 * N - 1;
    const unsigned int init[8] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u, 0u, 0u};
    PT_TRY(cudaMemcpyAsync(sc.cbounds, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    k_prepare<<<gridFor(n), kBlock, 0, stream>>>(dPositions, n, sc.triLo, sc.triHi, sc.cbounds);
    k_morton<<<gridFor(n), kBlock, 0, stream>>>(sc.triLo, sc.triHi, n, sc.cbounds, sc.keys, sc.vals);
    const size_t tempBytes = radixSortTempBytes(n);
    if (tempBytes > sc.sortTempBytes) {
        std::snprintf(err, errLen, "radix sort needs %zu scratch bytes, %zu reserved", tempBytes, sc.sortTempBytes);
        return PT_ERR_INVALID_ARGUMENT;
    }
    PT_TRY(radixSortPairs(sc.keys, sc.vals, sc.keysSorted, sc.valsSorted, n, 30, sc.sortTemp, tempBytes, stream));
    PT_TRY(cudaMemsetAsync(sc.parent, 0xff, sizeof(int) * nodesBin, stream));
    if (N > 1) {
        k_karras<<<gridFor(N - 1), kBlock, 0, stream>>>(sc.keysSorted, N, sc.child, sc.parent);
        PT_TRY(cudaMemsetAsync(sc.visits, 0, sizeof(int) * (N - 1), stream));
    }
    k_refit<<<gridFor(N), kBlock, 0, stream>>>(sc.valsSorted, sc.triLo, sc.triHi, N, sc.child, sc.parent, sc.nodeLo,
        sc.nodeHi, sc.visits);
    if (N > 1 && opt.treeletPasses > 0) {
        PT_TRY(runTreelets(N, sc.child, sc.parent, sc.nodeLo, sc.nodeHi, sc.visits, sc.subCost, sc.frontier,
            sc.frontierCount, opt, stream));
    }
    PT_TRY(cudaGetLastError());
    const unsigned int cinit[4] = {1u, 0u, 0u, 0u};
    PT_TRY(cudaMemcpyAsync(sc.counters, cinit, sizeof(cinit), cudaMemcpyHostToDevice, stream));
    const int2 rootTask = make_int2(0, 0);
    PT_TRY(cudaMemcpyAsync(sc.taskA, &rootTask, sizeof(int2), cudaMemcpyHostToDevice, stream));
    CollapseArgs ca{N, sc.child, sc.nodeLo, sc.nodeHi, sc.valsSorted, dPositions, outNodes, outTris, sc.counters,
        opt.maxLeafSize};
    int2* taskA = sc.taskA;
    int2* taskB = sc.taskB;
    int taskCount = 1;
    int levels = 0;
    while (taskCount > 0) {
        PT_TRY(cudaMemsetAsync(sc.counters + 2, 0, sizeof(unsigned int), stream));
        k_collapse<<<gridFor(taskCount, 64), 64, 0, stream>>>(ca, taskA, taskCount, taskB, sc.counters + 2);
        unsigned int next = 0;
        PT_TRY(cudaMemcpyAsync(&next, sc.counters + 2, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream));
        PT_TRY(cudaStreamSynchronize(stream));
        taskCount = static_cast<int>(next);
        int2* t = taskA;
        taskA = taskB;
        taskB = t;
        if (++levels > 256) {
            std::snprintf(err, errLen, "BVH collapse did not terminate");
            return PT_ERR_INTERNAL;
        }
    }
    unsigned int finalCounts[2] = {0, 0};
    PT_TRY(cudaMemcpyAsync(finalCounts, sc.counters, sizeof(finalCounts), cudaMemcpyDeviceToHost, stream));
    PT_TRY(cudaStreamSynchronize(stream));
    if (finalCounts[1] != n) {
        std::snprintf(err, errLen, "BVH collapse placed %u of %u triangles", finalCounts[1], n);
        return PT_ERR_INTERNAL;
    }
    *outNodeCount = finalCounts[0];
    return PT_OK;
}

} // namespace pt
