// Wavefront render pipeline: device buffers and launchers (see pt_render.cu).
#pragma once

#include "pt_common.cuh"

#ifndef PT_PATH_GENERATIONS
// Jobs of a batch run in generations of the slot count, each drained before
// the next, instead of refilling each finished path's slot with the next job:
// the launches of a generation hold paths of the same depth (camera rays
// together, then first bounces, ...).  Same images; plain-large 1106 -> 1068
// ms per frame, a 1920x1080 forest view 10.59 -> 10.47 s, the 64-tree batch
// 20.71 -> 18.37 s; and 1068 -> 1035 ms once finished paths stopped claiming
// jobs from the batch's counter.
#define PT_PATH_GENERATIONS 1
#endif

namespace pt {

// Structure-of-arrays path state, capacity `capacity` paths.
struct PathSoA {
    uint32_t* pixel = nullptr;   // pixel index
    uint32_t* outIdx = nullptr;  // slot * activeCount + listIndex into the sample buffer
    uint4* rngA = nullptr;       // XORWOW d, v0, v1, v2
    uint2* rngB = nullptr;       // XORWOW v3, v4
    float4* orig = nullptr;      // ray origin, tMin
    float4* dir = nullptr;       // ray direction (as produced, not renormalised), pdf of the sampled direction
    float4* thr = nullptr;       // throughput, medium IOR
    float4* rad = nullptr;       // radiance, depth (int bits)
    float4* hit = nullptr;       // t, u, v, triangle (uint bits, 0xFFFFFFFF = miss)
    uint32_t* hitInst = nullptr; // instance of the hit (instanced scenes only)
    float4* neeEnv = nullptr;    // pending environment-NEE contribution
    float4* neeEmis = nullptr;   // pending emissive-NEE contribution
    uint8_t* visEnv = nullptr;   // 1 = that contribution is unoccluded
    uint8_t* visEmis = nullptr;
    uint16_t* scene = nullptr;   // scene of the path (written only when more than one scene is rendered)
    // spectral mode (NW wavelengths per path): the path's hero draw, and NW / 4
    // float4 per path of throughput, radiance and pending NEE contributions,
    // word j of path i at [j * capacity + i] (the RGB fields above then carry
    // only the medium IOR in thr.w and the depth in rad.w)
    float* hero = nullptr;
    float4* thrS = nullptr;
    float4* radS = nullptr;
    float4* neeEnvS = nullptr;
    float4* neeEmisS = nullptr;
    int capacity = 0;
};

// Current batch of (pixel, sample) jobs (device memory; written by the host at
// batch start, nextJob advanced by the kernels that recycle path slots).
struct BatchInfo {
    unsigned long long jobs;     // activeCount x waves in this batch
    unsigned long long nextJob;  // first job not yet handed to a path slot
    int activeCount;
    uint32_t waveBase;
    int slotCount;               // path slots in use in this batch
};

struct QueueSet {
    uint32_t* extend[2] = {nullptr, nullptr}; // path indices, ping-pong
    // slot-ordered mode (non-null): the shade kernels mark the paths of the next
    // bounce here and k_next_queue lists them in slot order
    uint8_t* nextFlag = nullptr;
    uint32_t* finish = nullptr;               // paths that ended with shadow rays in flight
    uint32_t* missQueue = nullptr;            // paths whose last ray left the scene
    uint32_t* hitQueue = nullptr;             // paths whose last ray hit a triangle
    uint32_t* shadowPath = nullptr;           // path index | kind << 31
    float4* shadowOrig = nullptr;
    float4* shadowDir = nullptr;
    // counters: [0],[1] extend ping-pong, [2] shadow, [3] finish,
    // [4 + 2p] misses / [5 + 2p] hits of bounce parity p, [8 + p] extend and
    // [10 + p] shadow work-fetch counters
    unsigned int* counts = nullptr;
    unsigned long long* rays = nullptr;       // [0] closest-hit rays, [1] shadow rays
    unsigned long long* visits = nullptr;     // [0..1] extend nodes/tris, [2..3] shadow nodes/tris
    unsigned int* overflow = nullptr;         // traversal stack overflows
    BatchInfo* batch = nullptr;
};

struct AccumState {
    float4* acc = nullptr;
    uint32_t* counts = nullptr;
    float* lumMean = nullptr;
    float* m2 = nullptr;
    uint8_t* converged = nullptr;
    int* active[2] = {nullptr, nullptr};
    int* activeCount = nullptr; // [0] current, [1] next
    float4* samples = nullptr;  // per-batch sample buffer
    size_t sampleCapacity = 0;
};

// One scene of a batch: its camera, image size and first pixel in the batch's
// concatenated pixel range.
struct SceneView {
    pt_camera cam;
    int width;
    int height;
    uint32_t pixelBase;
    uint32_t pad;
};

// Distant light (no reference counterpart): a cone of directions around
// `dir` of constant radiance, sampled together
// with the environment: the sky's next-event sample picks the light with
// probability `select`, else the environment, and is weighted against BSDF
// sampling by the mixture's density.
struct DevSun {
    float3 dir, t, b;   // unit direction towards the light and a frame around it
    float omc;          // 1 - cos(half-angle), from double precision
    float sin2;         // sin^2(half-angle)
    float pdf;          // 1 / (2 pi omc): uniform over the cone
    float select;
    float3 rgb;         // RGB radiance
    float temperature;  // spectral mode: > 0 -> scale * Planck(lambda, temperature)
    float scale;
    float4 coef;        // spectral mode, temperature <= 0: spectrum of rgb
    int enabled;
};

struct LaunchCtx {
    DevScene scene;           // scene 0
    DevEnv env;
    pt_camera cam;            // scene 0
    pt_render_params params;
    int width;                // scene 0
    int height;
    // batch of several scenes (sceneCount > 1): per-scene geometry and views;
    // pixels are numbered scene after scene
    int sceneCount;
    const DevScene* scenes;
    const SceneView* views;
    // per batch: first active-list entry of each scene (sceneCount + 1) and
    // first job of each scene (sceneCount + 1); jobs are taken scene by scene
    uint32_t* sceneActiveStart;
    unsigned long long* sceneJobStart;
    int maxDepth;     // effective (0 -> 256, <0 -> 32)
    int rrMinDepth;   // effective
    PathSoA paths;
    QueueSet q;
    AccumState acc;
    int activeSel;    // which active[] list is current
    // optional record of every sample's radiance before the firefly clamp,
    // [sample index][pixel], for samples 0 .. recordSpp - 1 (the adjoint's input)
    float4* record;
    int recordSpp;
    // preview passes rendered before the full-resolution waves: wave w draws with
    // global seed seedOffset + w + 1 (the reference counts its preview passes as
    // iterations, PathTracer.cpp:2379)
    int seedOffset;
    // spectral mode: wavelengths per path (0 = RGB, the reference's integrator),
    // the sRGB response table (401 entries, 1 nm apart from 380 nm) and the
    // spectrum coefficients of the background colour times the environment intensity
    int spectral;
    const float4* specResp;
    float4 specBackground;
    DevSun sun;
};

// Launchers. The LaunchCtx lives in DEVICE memory (one per renderer) and is
// passed by pointer: a large by-value kernel parameter whose members are
// taken by reference would be copied to local memory by every thread.
// `grid` is a persistent-style grid; kernels loop over device-side counts.
// `nw` (generate, shade-miss, shade, finalize): wavelengths per path, 0 = RGB.
void launchGenerate(const LaunchCtx* d, int count, int extendSel, int nw, cudaStream_t s,
    unsigned long long jobOffset = 0);
// inst: compile-time instanced-scene traversal (any scene of the context instanced).
// Closest-hit stage.  lane: per-lane ray replacement (k_extend_lane + k_route;
// flat scenes, no visit counting), else one warp-fetch k_extend.
void launchExtend(const LaunchCtx* d, int sel, bool identity, int iter, int grid, bool count, bool inst, bool lane,
    cudaStream_t s);
// Kernels one launchExtend call launches (closest hit, and the routing pass after it).
int extendKernels(bool count, bool inst, bool lane);
// Resident blocks per SM of the per-lane closest-hit kernel and of the miss shader.
int extendLaneOccupancy();
int shadeMissOccupancy();
int shadowLaneOccupancy();
int extendLaneInstOccupancy();
int shadowLaneInstOccupancy();
// Resident blocks per SM of the hit shader for nw wavelengths (0 = RGB).
int shadeOccupancy(int nw);
// Slot-ordered mode: the next bounce's extend queue from the marked slots.
void launchNextQueue(const LaunchCtx* d, int sel, int grid, cudaStream_t s);
void launchShadeMiss(const LaunchCtx* d, int iter, int sel, int grid, int nw, cudaStream_t s);
void launchShade(const LaunchCtx* d, int sel, int iter, int grid, int nw, cudaStream_t s);
// Shadow stage.  lane: per-lane ray replacement (k_shadow_lane; flat scenes,
// no visit counting), else one warp per 32 queued rays (k_shadow).
void launchShadow(const LaunchCtx* d, int iter, int grid, bool count, bool inst, bool lane, cudaStream_t s);
void launchFinalize(const LaunchCtx* d, int sel, int grid, int nw, cudaStream_t s);
void launchAccumulate(const LaunchCtx* d, int activeCount, int batch, cudaStream_t s);
// Stable compaction of the active list (pixels neither converged nor at the
// sample cap), so that the list stays sorted by pixel and thereby by scene.
size_t compactTempBytes(int n);
cudaError_t launchCompactStable(const int* in, int* out, int* outCount, int n, const uint8_t* converged,
    const uint32_t* counts, int maxSpp, void* temp, size_t tempBytes, cudaStream_t s);
// Batches of several scenes: the per-scene active ranges and job offsets of
// the current batch (B waves).
void launchSceneJobs(const LaunchCtx* d, int sceneCount, int waves, cudaStream_t s);
void launchResetAccum(const LaunchCtx* d, int pixels, cudaStream_t s);
void launchTraceRays(const DevScene& S, int n, const float* o, const float* d, const float* tmin, const float* tmax,
    uint8_t* hit, float* t, uint32_t* tri, float* normal, float* uv, cudaStream_t s, unsigned int* overflow = nullptr);
// Resident blocks per SM of the stage kernels (occupancy calculator).
void stageOccupancy(int& extendBlocks, int& shadeBlocks, int& shadowBlocks);
void launchRngTape(int width, int height, int firstWave, int waves, int stride, int seedOffset, float* out,
    cudaStream_t s);
// Region render: the pixels of [minX, maxX] x [minY, maxY] become the active
// list (their accumulators cleared when `clear`).
void launchRegion(const LaunchCtx* c, int width, int minX, int minY, int maxX, int maxY, bool clear, cudaStream_t s);

} // namespace pt
