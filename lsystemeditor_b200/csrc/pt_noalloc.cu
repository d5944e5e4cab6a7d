// pt_trace_soup_noalloc: closest-hit queries against a small triangle soup
// that never allocates device memory.
//
// Who needs it: callers that must not allocate device memory -- hosts whose
// own allocator owns the whole device and hands out every byte (an allocation
// behind its back can fail or break its accounting), and interactive
// callbacks such as a viewport's surface pick, for which cudaMalloc/cudaFree
// would cost an implicit device synchronisation on every call.  They pass
// device buffers for the triangles, rays and results; every temporary of the
// BVH build and the traversal lives in one file-scope device array
// (kScratchBytes, room for PT_NOALLOC_MAX_TRIANGLES triangles).  The array is
// reserved on a device when this module is first loaded there (with CUDA's
// lazy module loading, at the latest at the first call) and stays reserved
// until the process exits.
//
// Set-up: the first call in a CUDA context (per device, and again if that
// device's context is destroyed and created anew, e.g. after cudaDeviceReset,
// or if the caller makes another context of the device current) looks up the
// array's device address with cudaGetSymbolAddress while that context is
// current, and keeps it keyed by the context's unique id; make that first call
// before any stream capture in the context.
//
// Blocking: the BVH build waits for `stream` between its levels, so a call
// returns to the host only once the build is done (the traversal is left
// enqueued on `stream`).
//
// Sharing: all calls in a context use the same array, which keeps the previous
// call's contents; everything that must start at zero or at a sentinel (the
// bounds reduction, parent links, visit counters, work counters, the root
// task) is written by the call itself before use.  Calls whose GPU work
// overlaps (several streams or host threads at once) race on the array and
// must be serialised by the caller.
#include "pt_bvh.cuh"
#include "pt_render.cuh"


#include <cuda.h> // CUcontext / CUresult types; the two driver calls are fetched through the runtime

#include <cstdio>
#include <cstring>
#include <mutex>

namespace pt {
namespace {

constexpr uint32_t kMaxTriangles = PT_NOALLOC_MAX_TRIANGLES;
constexpr size_t kScratchBytes = size_t(8) << 20; // 8 MiB per device

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch per device.  In host code `g_scratch` names a
// host-side stand-in, so the address is looked up with cudaGetSymbolAddress
// while the device's context is current.  A module global has a different
// address in every context it is loaded into, so the cached address is keyed
// by the unique id of the context it was looked up in (cuCtxGetId) and looked
// up again when the current context's id differs.
constexpr int kMaxDevices = 64;
struct ScratchSlot {
    unsigned long long context = 0; // cuCtxGetId of the context `address` belongs to (0 = none yet)
    void* address = nullptr;
};
ScratchSlot g_scratchSlot[kMaxDevices];
std::mutex g_setupMutex;

typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);
PfnCtxGetCurrent g_ctxGetCurrent = nullptr;
PfnCtxGetId g_ctxGetId = nullptr;

// Id of the calling thread's current context (0 if none is current); the
// caller holds g_setupMutex.
int currentContextId(unsigned long long* id, char* err, size_t errLen)
{
    if (g_ctxGetCurrent == nullptr || g_ctxGetId == nullptr) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa = cudaDriverEntryPointSymbolNotFound, qb = qa;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || a == nullptr || b == nullptr) {
            std::snprintf(err, errLen, "driver entry points cuCtxGetCurrent/cuCtxGetId unavailable");
            return PT_ERR_CUDA;
        }
        g_ctxGetCurrent = reinterpret_cast<PfnCtxGetCurrent>(a);
        g_ctxGetId = reinterpret_cast<PfnCtxGetId>(b);
    }
    CUcontext ctx = nullptr;
    if (g_ctxGetCurrent(&ctx) != CUDA_SUCCESS) {
        std::snprintf(err, errLen, "cuCtxGetCurrent failed");
        return PT_ERR_CUDA;
    }
    *id = 0;
    if (ctx != nullptr && g_ctxGetId(ctx, id) != CUDA_SUCCESS) {
        std::snprintf(err, errLen, "cuCtxGetId failed");
        return PT_ERR_CUDA;
    }
    return PT_OK;
}

int scratchFor(int device, void** out, char* err, size_t errLen)
{
    if (device < 0 || device >= kMaxDevices) {
        std::snprintf(err, errLen, "device %d out of range", device);
        return PT_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_setupMutex);
    unsigned long long ctx = 0;
    int st = currentContextId(&ctx, err, errLen);
    if (st != PT_OK) {
        return st;
    }
    ScratchSlot& slot = g_scratchSlot[device];
    if (ctx == 0 || slot.context != ctx || slot.address == nullptr) {
        // set-up in this context (the runtime makes the device's primary
        // context current first if no context is current yet)
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || p == nullptr) {
            std::snprintf(err, errLen, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
            return PT_ERR_CUDA;
        }
        st = currentContextId(&ctx, err, errLen);
        if (st != PT_OK) {
            return st;
        }
        if (ctx == 0) {
            std::snprintf(err, errLen, "no CUDA context is current after the symbol lookup");
            return PT_ERR_CUDA;
        }
        slot.context = ctx;
        slot.address = p;
    }
    *out = slot.address;
    return PT_OK;
}

// Bump allocator over the scratch array (256-byte aligned pieces).
struct Carve {
    unsigned char* base;
    size_t used = 0;
    size_t cap;
    bool ok = true;
    template <class T> T* take(size_t count)
    {
        const size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
        if (used + bytes > cap) {
            ok = false;
            return nullptr;
        }
        T* p = reinterpret_cast<T*>(base + used);
        used += bytes;
        return p;
    }
};

// Shading records of the soup.  Without vertex normals every vertex gets the
// triangle's geometric normal (v1 - v0) x (v2 - v0), so the reported normal is
// the face normal flipped to face the ray.
__global__ void k_soup_shade(const float* pos, const float* nrm, const float* uv, uint32_t n, TriShade* out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        TriShade s;
        if (nrm != nullptr) {
            const float* a = nrm + 9ull * i;
            s.a = make_float4(a[0], a[1], a[2], 0.0f);
            s.b = make_float4(a[3], a[4], a[5], 0.0f);
            s.c = make_float4(a[6], a[7], a[8], 0.0f);
        } else {
            // rounded products (no contraction): the same bits as a float32 host cross product
            const float* p = pos + 9ull * i;
            const float e1x = p[3] - p[0], e1y = p[4] - p[1], e1z = p[5] - p[2];
            const float e2x = p[6] - p[0], e2y = p[7] - p[1], e2z = p[8] - p[2];
            const float4 g = make_float4(__fsub_rn(__fmul_rn(e1y, e2z), __fmul_rn(e1z, e2y)),
                __fsub_rn(__fmul_rn(e1z, e2x), __fmul_rn(e1x, e2z)),
                __fsub_rn(__fmul_rn(e1x, e2y), __fmul_rn(e1y, e2x)), 0.0f);
            s.a = s.b = s.c = g;
        }
        float t[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (uv != nullptr) {
            for (int k = 0; k < 6; ++k) {
                t[k] = uv[6ull * i + k];
            }
        }
        s.a.w = t[0];
        s.b.w = t[1];
        s.c.w = t[2];
        s.d = make_float4(t[3], t[4], t[5], 0.0f);
        out[i] = s;
    }
}

void setError(char* dst, size_t cap, const char* src)
{
    if (dst != nullptr && cap > 0) {
        std::snprintf(dst, cap, "%s", src);
    }
}

} // namespace
} // namespace pt

using namespace pt;

extern "C" int pt_trace_soup_noalloc(uint32_t triangle_count, const float* positions, const float* normals,
    const float* uvs, int n, const float* origins, const float* dirs, const float* tmin, const float* tmax, uint8_t* hit,
    float* t, uint32_t* tri, float* normal, float* uv, void* stream, char* error_message, size_t error_capacity)
{
    char err[256] = {0};
    if (triangle_count > kMaxTriangles) {
        std::snprintf(err, sizeof(err), "pt_trace_soup_noalloc: %u triangles exceed the maximum of %u", triangle_count,
            kMaxTriangles);
        setError(error_message, error_capacity, err);
        return PT_ERR_INVALID_ARGUMENT;
    }
    if (n < 0 || (triangle_count > 0 && positions == nullptr) ||
        (n > 0 && (origins == nullptr || dirs == nullptr || tmin == nullptr || tmax == nullptr || hit == nullptr))) {
        setError(error_message, error_capacity, "pt_trace_soup_noalloc: null or negative argument");
        return PT_ERR_INVALID_ARGUMENT;
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        setError(error_message, error_capacity, "pt_trace_soup_noalloc: no current CUDA device");
        return PT_ERR_CUDA;
    }
    void* base = nullptr;
    int st = scratchFor(device, &base, err, sizeof(err));
    if (st != PT_OK) {
        setError(error_message, error_capacity, err);
        return st;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t N = triangle_count;
    const size_t Nn = N > 0 ? N : 1;
    Carve cv{static_cast<unsigned char*>(base), 0, kScratchBytes};
    BvhScratch sc{};
    sc.triLo = cv.take<float4>(Nn);
    sc.triHi = cv.take<float4>(Nn);
    sc.cbounds = cv.take<unsigned int>(8);
    sc.keys = cv.take<uint32_t>(Nn);
    sc.vals = cv.take<uint32_t>(Nn);
    sc.keysSorted = cv.take<uint32_t>(Nn);
    sc.valsSorted = cv.take<uint32_t>(Nn);
    sc.child = cv.take<int2>(Nn);
    sc.parent = cv.take<int>(2 * Nn);
    sc.nodeLo = cv.take<float4>(2 * Nn);
    sc.nodeHi = cv.take<float4>(2 * Nn);
    sc.visits = cv.take<int>(Nn);
    sc.subCost = cv.take<float>(2 * Nn);
    sc.frontier = cv.take<int>(Nn);
    sc.frontierCount = cv.take<unsigned int>(1);
    sc.taskA = cv.take<int2>(Nn + 1);
    sc.taskB = cv.take<int2>(Nn + 1);
    sc.counters = cv.take<unsigned int>(4);
    CwNode* nodes = cv.take<CwNode>(Nn + 1);
    TriVerts* tris = cv.take<TriVerts>(Nn);
    TriShade* shade = cv.take<TriShade>(Nn);
    sc.sortTempBytes = bvhSortTempBytes(static_cast<uint32_t>(Nn));
    sc.sortTemp = cv.take<unsigned char>(sc.sortTempBytes);
    if (!cv.ok) {
        std::snprintf(err, sizeof(err), "pt_trace_soup_noalloc: scratch of %zu bytes too small for %u triangles",
            kScratchBytes, N);
        setError(error_message, error_capacity, err);
        return PT_ERR_INVALID_ARGUMENT;
    }
    uint32_t nodeCount = 0;
    BvhBuildOptions opt;
    st = buildBvhInto(positions, N, sc, nodes, tris, &nodeCount, s, opt, err, sizeof(err));
    if (st != PT_OK) {
        setError(error_message, error_capacity, err);
        return st;
    }
    if (N > 0) {
        const int grid = static_cast<int>((N + 255) / 256);
        k_soup_shade<<<grid, 256, 0, s>>>(positions, normals, uvs, N, shade);
    }
    if (n > 0) {
        DevScene scene;
        scene.nodes = nodes;
        scene.tris = tris;
        scene.shade = shade;
        scene.nodeCount = N > 0 ? nodeCount : 0u;
        scene.triCount = N;
        launchTraceRays(scene, n, origins, dirs, tmin, tmax, hit, t, tri, normal, uv, s);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::snprintf(err, sizeof(err), "pt_trace_soup_noalloc: launch failed: %s", cudaGetErrorString(e));
        setError(error_message, error_capacity, err);
        return PT_ERR_CUDA;
    }
    return PT_OK;
}
