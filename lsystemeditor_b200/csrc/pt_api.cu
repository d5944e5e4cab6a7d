// C ABI (include/pt_b200.h) and the host-side renderer object.
//
// The renderer owns every device buffer, one CUDA stream and its events, like
// the reference's PathTracer (PathTracerLib/src/PathTracer.cpp:40-122), but
// runs synchronously: pt_render replaces the worker thread's render loop
// (PathTracer.cpp:2220-2543) with a loop over batches of waves.
#include "pt_bvh.cuh"
#include "pt_render.cuh"
#include "pt_adjoint.cuh"
#include "pt_output.cuh"
#include "pt_scene.cuh"
#include "pt_spectral.cuh"

namespace pt {
// pt_l2probe.cu
int measureL2ReadBandwidth(size_t bytes, int reps, int smCount, cudaStream_t s, double& gbPerS);
} // namespace pt

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace pt;

namespace {

template <class T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    bool ensure(size_t count)
    {
        if (count <= n && p != nullptr) {
            return true;
        }
        release();
        if (count == 0) {
            count = 1;
        }
        if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
            p = nullptr;
            n = 0;
            return false;
        }
        n = count;
        return true;
    }
    void release()
    {
        if (p != nullptr) {
            cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
};

// One scene: geometry on the device, its image size, camera and first pixel
// in the renderer's concatenated pixel range.  A plain renderer has one
// scene; a batch has several that render together.
struct SceneSlot {
    DevBuf<float> positions;      // 9 floats per triangle, original order
    DevBuf<TriShade> shade;
    DevBuf<pt_material> materials;
    DevBuf<pt_texture> textures;
    DevBuf<uint32_t> emissiveIdx;
    DevBuf<float> emissiveCdf;
    DevBuf<float> emitPdf; // per triangle, emitter MIS mode
    // spectral mode: host copies of the banks and their spectrum coefficients
    std::vector<pt_material> hostMats;
    std::vector<pt_texture> hostTex;
    DevBuf<float4> matSpec, texSpec;
    bool specValid = false;
    BvhBuffers bvh;
    // instanced scene: one BVH per object, the top-level BVH over the instances
    std::vector<BvhBuffers> objBvh;
    BvhBuffers tlas;
    DevBuf<float> tlasBoxes;
    DevBuf<DevInstance> instances;
    DevBuf<DevBlas> blases;
    uint32_t instanceCount = 0;
    int shareFrom = -1;           // batch view of another slot's geometry (-1: own geometry)
    uint32_t triCount = 0;
    uint32_t materialCount = 0;
    uint32_t textureCount = 0;
    uint32_t emissiveCount = 0;
    bool hasScene = false;
    int width = 0;
    int height = 0;
    uint32_t pixelBase = 0;
    pt_camera camera{};

    void releaseInstances()
    {
        for (BvhBuffers& b : objBvh) {
            b.release();
            b.scratch.release();
        }
        objBvh.clear();
        tlas.release();
        tlas.scratch.release();
        tlasBoxes.release();
        instances.release();
        blases.release();
        instanceCount = 0;
    }

    // Forgets the slot's scene but keeps its device arrays for the next one
    // (they are reused where large enough: a batch reconfigured with scenes of
    // the same sizes allocates nothing).
    void clearScene()
    {
        hostMats.clear();
        hostTex.clear();
        specValid = false;
        releaseInstances();
        bvh.nodeCount = bvh.triCount = 0;
        bvh.levels = 0;
        shareFrom = -1;
        triCount = materialCount = textureCount = emissiveCount = 0;
        hasScene = false;
    }

    void release()
    {
        positions.release();
        shade.release();
        materials.release();
        textures.release();
        emissiveIdx.release();
        emissiveCdf.release();
        emitPdf.release();
        matSpec.release();
        texSpec.release();
        specValid = false;
        releaseInstances();
        bvh.release();
        bvh.scratch.release();
        hasScene = false;
    }
};

} // namespace

struct pt_renderer {
    int device = 0;
    cudaStream_t stream = nullptr;      // stream all work is issued on
    cudaStream_t ownStream = nullptr;   // the renderer's own stream
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string lastError = "";
    int smCount = 148;

    // scenes (scenes[0] is the one the single-scene calls address)
    std::vector<SceneSlot> scenes = std::vector<SceneSlot>(1);
    DevBuf<DevScene> dScenes;             // device copies for batches
    DevBuf<SceneView> dViews;
    DevBuf<float> stage;          // upload staging (normals / uvs)
    DevBuf<uint32_t> stageIds;
    // scene-build scratch: emissive selection, tube loft inputs
    DevBuf<float> eWeights;
    DevBuf<uint8_t> eFlags;
    DevBuf<uint32_t> eIdx;
    DevBuf<float> eCdf;
    DevBuf<uint32_t> eOut;
    DevBuf<unsigned char> eTemp;
    DevBuf<uint32_t> tRingStart, tMaterials;
    DevBuf<double> tPoints, tTangents, tRadii, tCosSin, tLeaves, tFrames;
    DevBuf<double> tGivenFrames; // given ring frames (pt_tubes.frames)
    BvhBuildOptions bvhOptions;

    // environment
    DevBuf<float> envPixels, envMarginal, envRow;
    DevBuf<float> envScratch;             // sin(theta) per row and row totals of the table build
    int envW = 0, envH = 0;
    bool envValid = false;

    // spectral mode (hero wavelengths)
    std::vector<float> specRespHost;      // sRGB response table, 401 x 4
    DevBuf<float4> specResp;
    DevBuf<float4> envSpec;               // per-texel coefficients of the environment map
    bool envSpecValid = false;
    std::map<std::array<uint32_t, 3>, spectral::Coef> specCache; // colour bits -> coefficients
    float4 specBackground{};
    int specCapacity = 0;
    DevSun sun{};                         // distant light (enabled = 0: none)
    DevBuf<float> pHero;
    DevBuf<float4> pThrS, pRadS, pNeeEnvS, pNeeEmisS;

    // accumulation over the concatenated pixels of all scenes
    int width = 0, height = 0;            // scene 0
    size_t pixelCount = 0;
    DevBuf<float4> acc;
    DevBuf<uint32_t> counts;
    DevBuf<float> lumMean, m2;
    DevBuf<uint8_t> converged;
    DevBuf<int> active0, active1, activeCount;
    DevBuf<float4> samples;
    DevBuf<uint8_t> displayBuf;           // RGBA8 output of pt_tonemap
    DevBuf<float> adjImage;               // dLoss/dImage of pt_backward
    // preview passes (PathTracerPreviewLevels.h): level i at 1 / 2^(levels - i)
    int previewLevels = 0;
    int previewDone = -1;                 // finest preview level rendered since the last reset
    DevBuf<float4> previewBuf;            // all levels, coarsest first
    // region render (PathTracer.h:134-140)
    bool regionEnabled = false;
    int regionMinX = 0, regionMinY = 0, regionMaxX = 0, regionMaxY = 0;
    DevBuf<float4> record;                // per-sample radiance of the last fixed-spp render
    int recordSpp = 0;                    // samples per pixel kept (0 = off)
    bool recordValid = false;             // record matches the current scene, camera and params
    DevBuf<float> adjGrad;                // its parameter gradient
    DevBuf<unsigned char> compactTemp;    // scratch of the active-list compaction
    DevBuf<uint32_t> sceneActiveStart;    // batches: per-scene active ranges
    DevBuf<unsigned long long> sceneJobStart;
    int activeSel = 0;
    int hostActive = 0;
    int64_t wavesDone = 0;
    int64_t samplesDone = 0;

    // paths
    int capacity = 0;
    DevBuf<uint32_t> pPixel, pOut;
    DevBuf<uint4> pRngA;
    DevBuf<uint2> pRngB;
    DevBuf<float4> pOrig, pDir, pThr, pRad, pHit, pNeeEnv, pNeeEmis;
    DevBuf<uint32_t> pHitInst;
    DevBuf<uint8_t> pVisEnv, pVisEmis;
    DevBuf<uint16_t> pScene;
    DevBuf<uint8_t> pNextFlag;            // slot-ordered mode: paths marked for the next bounce
    DevBuf<uint32_t> qExt0, qExt1, qFinish, qShadowPath, qMiss, qHit;
    DevBuf<float4> qShadowO, qShadowD;
    DevBuf<unsigned int> qCounts;
    DevBuf<unsigned long long> qRays;     // [0] extend, [1] shadow
    DevBuf<unsigned long long> qVisits;   // [0..1] extend nodes/tris, [2..3] shadow nodes/tris
    DevBuf<unsigned int> qOverflow;
    int gridExtend = 0, gridShade = 0, gridShadow = 0;
    int gridExtendLane = 0;          // grid of the per-lane closest-hit kernel
    int gridShadowLane = 0;          // grid of the per-lane shadow kernel
    int gridExtendLaneInst = 0;      // grids of the per-lane kernels of instanced scenes
    int gridShadowLaneInst = 0;
    int gridShadeMiss = 0;           // grid of the miss shader (its own occupancy)
    bool extendLane = false;         // per-lane ray replacement in this render's closest-hit stage
    int extendMode = PT_EXTEND_MODE_AUTO;
    // CUDA graphs of four bounce iterations (the first block of a batch, later
    // blocks) and the launch configuration they were captured for
    cudaGraphExec_t bounceGraph[2] = {nullptr, nullptr};
    unsigned long long bounceKey[6] = {0, 0, 0, 0, 0, 0};
    bool useGraphs = true;
    int capacityWanted = 1 << 24;     // paths in flight per launch (one chunk for most frames)
    int blocksPerSmOverride = 0;

    DevBuf<LaunchCtx> dctx;               // device copy of the launch context
    LaunchCtx hostCtx{};                  // its host staging (lives until the copy has run)
    std::vector<DevScene> hostScenes;     // host staging of dScenes / dViews
    std::vector<SceneView> hostViews;
    DevBuf<BatchInfo> dbatch;             // current batch of jobs
    BatchInfo hbatch{};                   // host staging of dbatch
    double lastStopRate = 1.0;            // fraction of active pixels that stopped per 4 waves

    // profiling
    int profileFlags = 0;
    pt_profile profile{};
    std::vector<cudaEvent_t> eventPool;
    std::vector<std::pair<int, int>> eventMarks; // (stage, first event index)

    pt_render_params params{};

    pt_stats stats{};
    int64_t launches = 0;
};

namespace {

int fail(pt_renderer* r, int code, const char* fmt, ...)
{
    if (r != nullptr) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        r->lastError = buf;
    }
    return code;
}

int cudaFail(pt_renderer* r, cudaError_t e, const char* what)
{
    return fail(r, e == cudaErrorMemoryAllocation ? PT_ERR_OUT_OF_MEMORY : PT_ERR_CUDA, "%s: %s", what,
        cudaGetErrorString(e));
}

#define PT_CHECK(r, call)                                                                                         \
    do {                                                                                                          \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess) {                                                                                  \
            return cudaFail((r), e_, #call);                                                                      \
        }                                                                                                         \
    } while (0)

pt_camera defaultCamera()
{
    pt_camera c{};
    c.orientation[0] = 1.0f;
    c.fov_y = 0.7f;
    c.aspect = 1.0f;
    c.near_plane = 0.1f;
    c.far_plane = 1000.0f;
    return c;
}

pt_material defaultMaterial()
{
    // MeshAccelScene.cpp:27-46 / MaterialGpu{} defaults.
    pt_material m{};
    m.r = m.g = m.b = 0.8f;
    m.roughness = 0.5f;
    m.ior = 1.5f;
    m.diffuse_roughness = -1.0f;
    m.specular = 1.0f;
    return m;
}

uint32_t sceneNodeCount(const SceneSlot& sl)
{
    uint32_t n = sl.instanceCount > 0 ? sl.tlas.nodeCount : sl.bvh.nodeCount;
    for (const BvhBuffers& b : sl.objBvh) {
        n += b.nodeCount;
    }
    return n;
}

DevScene deviceScene(const SceneSlot* r)
{
    DevScene s;
    s.nodes = r->bvh.nodes;
    s.tris = r->bvh.tris;
    s.shade = r->shade.p;
    s.origVerts = reinterpret_cast<const float4*>(r->positions.p);
    s.materials = r->materials.p;
    s.textures = r->textureCount ? r->textures.p : nullptr;
    s.emissiveIdx = r->emissiveIdx.p;
    s.emissiveCdf = r->emissiveCdf.p;
    s.emitPdfArea = r->emissiveCount > 0 ? r->emitPdf.p : nullptr;
    s.matSpec = r->specValid ? r->matSpec.p : nullptr;
    s.texSpec = r->specValid ? r->texSpec.p : nullptr;
    if (r->instanceCount > 0) {
        s.tlasNodes = r->tlas.nodes;
        s.tlasLeaves = r->tlas.tris;
        s.instances = r->instances.p;
        s.blases = r->blases.p;
        s.instanceCount = r->hasScene ? r->instanceCount : 0u;
    }
    s.nodeCount = r->hasScene ? r->bvh.nodeCount : 0u;
    s.triCount = r->triCount;
    s.materialCount = r->materialCount;
    s.textureCount = r->textureCount;
    s.emissiveCount = r->emissiveCount;
    return s;
}

int ensurePaths(pt_renderer* r, int capacity)
{
    if (r->capacity >= capacity) {
        return PT_OK;
    }
    const size_t Q = static_cast<size_t>(capacity);
    bool ok = r->pPixel.ensure(Q) && r->pOut.ensure(Q) && r->pRngA.ensure(Q) && r->pRngB.ensure(Q) &&
        r->pOrig.ensure(Q) && r->pDir.ensure(Q) && r->pThr.ensure(Q) && r->pRad.ensure(Q) && r->pHit.ensure(Q) && r->pHitInst.ensure(Q) &&
        r->pNeeEnv.ensure(Q) && r->pNeeEmis.ensure(Q) && r->pVisEnv.ensure(Q) && r->pVisEmis.ensure(Q) && r->pScene.ensure(Q) &&
        r->qExt0.ensure(Q) && r->qExt1.ensure(Q) && r->qFinish.ensure(Q) && r->qShadowPath.ensure(2 * Q) &&
        r->qMiss.ensure(Q) && r->qHit.ensure(Q) &&
        r->qShadowO.ensure(2 * Q) && r->qShadowD.ensure(2 * Q) && r->qCounts.ensure(16) && r->qRays.ensure(2) &&
        r->qVisits.ensure(4) && r->qOverflow.ensure(1) && r->dbatch.ensure(1) && r->pNextFlag.ensure(Q);
    if (!ok) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "path state allocation failed for %d paths", capacity);
    }
    if (cudaMemset(r->pNextFlag.p, 0, Q) != cudaSuccess) {
        return fail(r, PT_ERR_CUDA, "path state initialisation failed");
    }
    r->capacity = capacity;
    return PT_OK;
}

#ifndef PT_SLOT_ORDER
#define PT_SLOT_ORDER 1
#endif

// Slot-ordered next queue (k_next_queue): with the per-lane closest-hit kernel,
// whose queue order does not matter to it, the shade kernels read consecutive
// slots' path state.
bool slotOrdered(const pt_renderer* r) { return PT_SLOT_ORDER && r->extendLane; }

LaunchCtx makeCtx(pt_renderer* r)
{
    LaunchCtx c{};
    c.scene = deviceScene(&r->scenes[0]);
    c.env.pixels = r->envPixels.p;
    c.env.marginal = r->envMarginal.p;
    c.env.row = r->envRow.p;
    c.env.width = r->envW;
    c.env.height = r->envH;
    c.env.valid = r->envValid ? 1 : 0;
    c.env.spec = r->envSpecValid ? r->envSpec.p : nullptr;
    c.cam = r->scenes[0].camera;
    c.params = r->params;
    c.width = r->width;
    c.height = r->height;
    c.sceneCount = static_cast<int>(r->scenes.size());
    c.scenes = r->dScenes.p;
    c.views = r->dViews.p;
    c.sceneActiveStart = r->sceneActiveStart.p;
    c.sceneJobStart = r->sceneJobStart.p;
    c.maxDepth = r->params.max_path_depth > 0 ? r->params.max_path_depth : (r->params.max_path_depth == 0 ? 256 : 32);
    c.rrMinDepth = r->params.russian_roulette_min_depth >= 0 ? r->params.russian_roulette_min_depth : 3;
    c.paths.pixel = r->pPixel.p;
    c.paths.outIdx = r->pOut.p;
    c.paths.rngA = r->pRngA.p;
    c.paths.rngB = r->pRngB.p;
    c.paths.orig = r->pOrig.p;
    c.paths.dir = r->pDir.p;
    c.paths.thr = r->pThr.p;
    c.paths.rad = r->pRad.p;
    c.paths.hit = r->pHit.p;
    c.paths.hitInst = r->pHitInst.p;
    c.paths.neeEnv = r->pNeeEnv.p;
    c.paths.neeEmis = r->pNeeEmis.p;
    c.paths.visEnv = r->pVisEnv.p;
    c.paths.visEmis = r->pVisEmis.p;
    c.paths.scene = r->pScene.p;
    c.paths.hero = r->pHero.p;
    c.paths.thrS = r->pThrS.p;
    c.paths.radS = r->pRadS.p;
    c.paths.neeEnvS = r->pNeeEnvS.p;
    c.paths.neeEmisS = r->pNeeEmisS.p;
    c.paths.capacity = r->capacity;
    c.q.extend[0] = r->qExt0.p;
    c.q.extend[1] = r->qExt1.p;
    c.q.nextFlag = slotOrdered(r) ? r->pNextFlag.p : nullptr;
    c.q.finish = r->qFinish.p;
    c.q.missQueue = r->qMiss.p;
    c.q.hitQueue = r->qHit.p;
    c.q.shadowPath = r->qShadowPath.p;
    c.q.shadowOrig = r->qShadowO.p;
    c.q.shadowDir = r->qShadowD.p;
    c.q.counts = r->qCounts.p;
    c.q.rays = r->qRays.p;
    c.q.batch = r->dbatch.p;
    c.q.visits = r->qVisits.p;
    c.q.overflow = r->qOverflow.p;
    c.acc.acc = r->acc.p;
    c.acc.counts = r->counts.p;
    c.acc.lumMean = r->lumMean.p;
    c.acc.m2 = r->m2.p;
    c.acc.converged = r->converged.p;
    c.acc.active[0] = r->active0.p;
    c.acc.active[1] = r->active1.p;
    c.acc.activeCount = r->activeCount.p;
    c.acc.samples = r->samples.p;
    c.acc.sampleCapacity = r->samples.n;
    c.activeSel = r->activeSel;
    const bool rec = r->recordSpp > 0 && r->scenes.size() == 1 && r->record.p != nullptr;
    c.record = rec ? r->record.p : nullptr;
    c.recordSpp = rec ? r->recordSpp : 0;
    c.seedOffset = r->previewLevels;
    c.spectral = r->params.spectral_wavelengths;
    c.specResp = r->specResp.p;
    c.specBackground = r->specBackground;
    c.sun = r->sun;
    if (c.sun.enabled) {
        // a black sky leaves every next-event sample to the light
        const float k = r->params.environment_intensity;
        const bool skyLit = r->envValid || r->params.background_r * k != 0.0f || r->params.background_g * k != 0.0f ||
            r->params.background_b * k != 0.0f;
        c.sun.select = skyLit ? 0.5f : 1.0f;
    }
    return c;
}

// Uploads the current launch context; returns its device address (nullptr on failure).
const LaunchCtx* uploadCtx(pt_renderer* r)
{
    if (!r->dctx.ensure(1)) {
        return nullptr;
    }
    if (r->scenes.size() > 1) {
        const size_t n = r->scenes.size();
        if (!r->dScenes.ensure(n) || !r->dViews.ensure(n) || !r->sceneActiveStart.ensure(n + 1) ||
            !r->sceneJobStart.ensure(n + 1)) {
            return nullptr;
        }
        r->hostScenes.resize(n);
        r->hostViews.resize(n);
        for (size_t k = 0; k < n; ++k) {
            const SceneSlot& sl = r->scenes[k];
            r->hostScenes[k] = deviceScene(sl.shareFrom >= 0 ? &r->scenes[static_cast<size_t>(sl.shareFrom)] : &sl);
            SceneView v{};
            v.cam = sl.camera;
            v.width = sl.width;
            v.height = sl.height;
            v.pixelBase = sl.pixelBase;
            r->hostViews[k] = v;
        }
        if (cudaMemcpyAsync(r->dScenes.p, r->hostScenes.data(), n * sizeof(DevScene), cudaMemcpyHostToDevice,
                r->stream) != cudaSuccess ||
            cudaMemcpyAsync(r->dViews.p, r->hostViews.data(), n * sizeof(SceneView), cudaMemcpyHostToDevice,
                r->stream) != cudaSuccess) {
            return nullptr;
        }
    }
    r->hostCtx = makeCtx(r);
    if (cudaMemcpyAsync(r->dctx.p, &r->hostCtx, sizeof(LaunchCtx), cudaMemcpyHostToDevice, r->stream) != cudaSuccess) {
        return nullptr;
    }
    return r->dctx.p;
}

int resetAccum(pt_renderer* r)
{
    if (r->width <= 0) {
        return PT_OK;
    }
    r->activeSel = 0;
    const LaunchCtx* dc = uploadCtx(r);
    if (dc == nullptr) {
        return fail(r, PT_ERR_CUDA, "launch context upload failed");
    }
    launchResetAccum(dc, static_cast<int>(r->pixelCount), r->stream);
    PT_CHECK(r, cudaGetLastError());
    r->hostActive = static_cast<int>(r->pixelCount);
    r->previewDone = -1;
    if (r->regionEnabled && r->scenes.size() == 1) {
        // only the region's pixels take samples
        launchRegion(dc, r->width, r->regionMinX, r->regionMinY, r->regionMaxX, r->regionMaxY, false, r->stream);
        PT_CHECK(r, cudaGetLastError());
        r->hostActive = (r->regionMaxX - r->regionMinX + 1) * (r->regionMaxY - r->regionMinY + 1);
    }
    r->lastStopRate = 1.0;
    r->wavesDone = 0;
    r->samplesDone = 0;
    r->recordValid = false;
    return PT_OK;
}

enum Stage { kGenerate = 0, kExtend, kShade, kShadow, kFinalize, kAccumulate, kCompact, kStageCount };
// (the miss-shading kernel is accounted to kShade)

// Stage timing: a pair of events around each launch when profiling is on.
struct StageTimer {
    pt_renderer* r;
    int idx = -1;
    int stage;
    StageTimer(pt_renderer* rr, int st) : r(rr), stage(st)
    {
        if (!(r->profileFlags & PT_PROFILE_STAGE_TIMES)) {
            return;
        }
        const size_t need = r->eventMarks.size() * 2 + 2;
        while (r->eventPool.size() < need) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) {
                return;
            }
            r->eventPool.push_back(e);
        }
        idx = static_cast<int>(r->eventMarks.size()) * 2;
        cudaEventRecord(r->eventPool[idx], r->stream);
    }
    ~StageTimer()
    {
        if (idx >= 0) {
            cudaEventRecord(r->eventPool[idx + 1], r->stream);
            r->eventMarks.emplace_back(stage, idx);
        }
    }
};

void collectStageTimes(pt_renderer* r)
{
    double* ms[kStageCount] = {&r->profile.ms_generate, &r->profile.ms_extend, &r->profile.ms_shade,
        &r->profile.ms_shadow, &r->profile.ms_finalize, &r->profile.ms_accumulate, &r->profile.ms_compact};
    for (const auto& m : r->eventMarks) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, r->eventPool[m.second], r->eventPool[m.second + 1]) == cudaSuccess) {
            *ms[m.first] += t;
        }
    }
    r->eventMarks.clear();
}

// Number of waves folded into one batch (see the render loop comment).
// Results do not depend on it; a pixel that converges inside a batch leaves
// the rest of the batch's samples unused, so the batch grows when few pixels
// stopped during the previous one.
#ifndef PT_SAMPLE_BUFFER_BYTES
// (8 GiB: on the 64-tree batch, 31 M pixels, a 1 GiB buffer held batches to 2
// waves, so every pass put ~16 scenes' paths in flight and drained often; at
// 8 GiB the render took 20.9 s instead of 22.0 s, extend and shadow 7% and 11%
// faster; renders of up to 1 M pixels are unaffected)
#define PT_SAMPLE_BUFFER_BYTES (8ll << 30)
#endif
int chooseBatch(const pt_renderer* r, int remaining)
{
    const pt_render_params& p = r->params;
    int64_t B;
    if (p.samples_per_launch > 0) {
        B = p.samples_per_launch;
    } else if (r->wavesDone < p.min_samples) {
        B = p.min_samples - r->wavesDone; // nothing can converge before min_samples
    } else {
        B = r->lastStopRate > 0.02 ? 4 : (r->lastStopRate > 0.005 ? 16 : 64);
    }
    if (p.max_samples_per_pixel > 0) {
        B = std::min<int64_t>(B, p.max_samples_per_pixel - r->wavesDone);
    }
    if (remaining > 0) {
        B = std::min<int64_t>(B, remaining);
    }
    // cap the sample buffer (one float4 per active pixel and wave of the batch)
    const int64_t cap = std::max<int64_t>(1, static_cast<int64_t>(PT_SAMPLE_BUFFER_BYTES) / (16 * std::max(1, r->hostActive)));
    B = std::min<int64_t>(B, std::min<int64_t>(cap, 1024));
    return static_cast<int>(std::max<int64_t>(B, 1));
}

} // namespace

namespace {

// Image sizes of scenes 0..n-1 (n = scenes.size()): pixel ranges laid out
// scene after scene, accumulators sized for all of them, accumulation reset.
int configureLayout(pt_renderer* r, const int* widths, const int* heights)
{
    const size_t n = r->scenes.size();
    size_t total = 0;
    for (size_t k = 0; k < n; ++k) {
        if (widths[k] <= 0 || heights[k] <= 0) {
            return fail(r, PT_ERR_INVALID_ARGUMENT, "bad image size %dx%d for scene %zu", widths[k], heights[k], k);
        }
        total += static_cast<size_t>(widths[k]) * heights[k];
    }
    if (total > (size_t(1) << 30)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "%zu pixels in total exceed 2^30", total);
    }
    if (!(r->acc.ensure(total) && r->counts.ensure(total) && r->lumMean.ensure(total) && r->m2.ensure(total) &&
            r->converged.ensure(total) && r->active0.ensure(total) && r->active1.ensure(total) &&
            r->activeCount.ensure(4))) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "accumulator allocation failed for %zu pixels", total);
    }
    size_t base = 0;
    for (size_t k = 0; k < n; ++k) {
        SceneSlot& sl = r->scenes[k];
        sl.width = widths[k];
        sl.height = heights[k];
        sl.pixelBase = static_cast<uint32_t>(base);
        base += static_cast<size_t>(widths[k]) * heights[k];
    }
    r->pixelCount = total;
    r->width = r->scenes[0].width;
    r->height = r->scenes[0].height;
    int st = resetAccum(r);
    if (st != PT_OK) {
        return st;
    }
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    return PT_OK;
}

// Material and texture banks of a scene; MeshAccelScene::build adds one
// default material when none is given.
int uploadBank(pt_renderer* r, SceneSlot& sl, const pt_mesh* mesh)
{
    cudaStream_t s = r->stream;
    std::vector<pt_material> mats(mesh->materials, mesh->materials + mesh->material_count);
    if (mats.empty()) {
        mats.push_back(defaultMaterial());
    }
    sl.materialCount = static_cast<uint32_t>(mats.size());
    sl.hostMats = mats;
    sl.specValid = false;
    if (!sl.materials.ensure(mats.size())) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "material upload failed");
    }
    // (a copy from pageable memory has read the source when the call returns)
    PT_CHECK(r, cudaMemcpyAsync(sl.materials.p, mats.data(), mats.size() * sizeof(pt_material), cudaMemcpyHostToDevice, s));
    sl.textureCount = mesh->texture_count;
    if (mesh->texture_count > 0) {
        if (!sl.textures.ensure(mesh->texture_count)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "texture upload failed");
        }
        PT_CHECK(r, cudaMemcpyAsync(sl.textures.p, mesh->textures, mesh->texture_count * sizeof(pt_texture),
            cudaMemcpyHostToDevice, s));
        sl.hostTex.assign(mesh->textures, mesh->textures + mesh->texture_count);
    }
    return PT_OK;
}

// --- spectral mode ---------------------------------------------------------------

const std::vector<float>& responseTable(pt_renderer* r)
{
    if (r->specRespHost.empty()) {
        r->specRespHost.resize(4 * spectral::kRespCount);
        spectral::buildResponseTable(r->specRespHost.data());
    }
    return r->specRespHost;
}

// Radiance-mode coefficients of an RGB colour (cached by the colour's bits).
spectral::Coef colourCoef(pt_renderer* r, float cr, float cg, float cb)
{
    std::array<uint32_t, 3> key;
    std::memcpy(&key[0], &cr, 4);
    std::memcpy(&key[1], &cg, 4);
    std::memcpy(&key[2], &cb, 4);
    auto it = r->specCache.find(key);
    if (it != r->specCache.end()) {
        return it->second;
    }
    const spectral::Coef c = spectral::upliftSolve(responseTable(r).data(), cr, cg, cb, true);
    r->specCache.emplace(key, c);
    return c;
}

float4 coefToFloat4(const spectral::Coef& c) { return make_float4(c.c0, c.c1, c.c2, c.scale); }

// The distant light's device record: frame, cone constants (double precision),
// and its radiance: RGB as given, or a blackbody of the given temperature whose
// sRGB (through the response table) has the given Rec. 709 luminance.
int setDistantLight(pt_renderer* r, const pt_distant_light* l)
{
    r->sun = DevSun{};
    if (l == nullptr || l->enabled == 0) {
        return PT_OK;
    }
    const double dx = l->direction[0], dy = l->direction[1], dz = l->direction[2];
    const double len = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (!(len > 0.0) || !std::isfinite(len) || !(l->half_angle > 0.0f) || !(l->half_angle < 1.5f)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_distant_light: bad direction or half-angle");
    }
    const double d[3] = {dx / len, dy / len, dz / len};
    // frame: the same construction as the BSDF's basis()
    const double up[3] = {std::fabs(d[1]) < 0.999 ? 0.0 : 1.0, std::fabs(d[1]) < 0.999 ? 1.0 : 0.0, 0.0};
    double t[3] = {up[1] * d[2] - up[2] * d[1], up[2] * d[0] - up[0] * d[2], up[0] * d[1] - up[1] * d[0]};
    const double tl = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    for (double& x : t) {
        x /= tl;
    }
    const double b[3] = {d[1] * t[2] - d[2] * t[1], d[2] * t[0] - d[0] * t[2], d[0] * t[1] - d[1] * t[0]};
    DevSun& S = r->sun;
    S.dir = make_float3(static_cast<float>(d[0]), static_cast<float>(d[1]), static_cast<float>(d[2]));
    S.t = make_float3(static_cast<float>(t[0]), static_cast<float>(t[1]), static_cast<float>(t[2]));
    S.b = make_float3(static_cast<float>(b[0]), static_cast<float>(b[1]), static_cast<float>(b[2]));
    const double ha = l->half_angle;
    const double omc = 2.0 * std::sin(0.5 * ha) * std::sin(0.5 * ha);
    S.omc = static_cast<float>(omc);
    S.sin2 = static_cast<float>(std::sin(ha) * std::sin(ha));
    S.pdf = static_cast<float>(1.0 / (2.0 * 3.14159265358979323846 * omc));
    S.temperature = l->temperature_k;
    if (l->temperature_k > 0.0f) {
        const std::vector<float>& resp = responseTable(r);
        double rgb[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < spectral::kRespCount; ++i) {
            const double lu = (380.0 + i) * 1.0e-3;
            const double B = 1.0 / (lu * lu * lu * lu * lu * std::expm1(14387.769 / (lu * l->temperature_k)));
            const double w = (i == 0 || i == spectral::kRespCount - 1) ? 0.5 : 1.0;
            for (int c = 0; c < 3; ++c) {
                rgb[c] += w * B * resp[4 * i + c];
            }
        }
        const double K = 0.2126 * rgb[0] + 0.7152 * rgb[1] + 0.0722 * rgb[2];
        if (!(K > 0.0)) {
            return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_distant_light: temperature %g K gives no light",
                static_cast<double>(l->temperature_k));
        }
        const double scale = l->luminance / K;
        S.scale = static_cast<float>(scale);
        S.rgb = make_float3(static_cast<float>(rgb[0] * scale), static_cast<float>(rgb[1] * scale),
            static_cast<float>(rgb[2] * scale));
    } else {
        S.rgb = make_float3(l->radiance[0], l->radiance[1], l->radiance[2]);
        S.coef = coefToFloat4(colourCoef(r, l->radiance[0], l->radiance[1], l->radiance[2]));
    }
    S.select = 1.0f;
    S.enabled = 1;
    return PT_OK;
}

// Response table, the scenes' and environment's spectrum coefficients and the
// spectral path state, for a render with nw wavelengths per path.
int prepareSpectral(pt_renderer* r, int nw)
{
    cudaStream_t s = r->stream;
    const std::vector<float>& resp = responseTable(r);
    if (r->specResp.p == nullptr || r->specResp.n < static_cast<size_t>(spectral::kRespCount)) {
        if (!r->specResp.ensure(spectral::kRespCount)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "spectral response table allocation failed");
        }
        PT_CHECK(r, cudaMemcpy(r->specResp.p, resp.data(), resp.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    for (SceneSlot& sl : r->scenes) {
        if (sl.specValid || sl.shareFrom >= 0) {
            continue;
        }
        std::vector<float4> mc(2 * std::max<size_t>(sl.hostMats.size(), 1));
        for (size_t m = 0; m < sl.hostMats.size(); ++m) {
            const pt_material& q = sl.hostMats[m];
            mc[2 * m] = coefToFloat4(colourCoef(r, q.r, q.g, q.b));
            mc[2 * m + 1] = coefToFloat4(colourCoef(r, q.scatter_radius_r, q.scatter_radius_g, q.scatter_radius_b));
        }
        const size_t nt = std::min<size_t>(sl.textureCount, sl.hostTex.size());
        std::vector<float4> tc(2 * std::max<size_t>(nt, 1), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
        for (size_t t = 0; t < nt; ++t) {
            const pt_texture& q = sl.hostTex[t];
            if (q.kind == 1) {
                tc[2 * t] = coefToFloat4(colourCoef(r, q.p0[0], q.p0[1], q.p0[2]));
            } else if (q.kind == 2) {
                tc[2 * t] = coefToFloat4(colourCoef(r, q.p1[0], q.p1[1], q.p1[2]));
                tc[2 * t + 1] = coefToFloat4(colourCoef(r, q.p2[0], q.p2[1], q.p2[2]));
            }
        }
        if (!sl.matSpec.ensure(mc.size()) || !sl.texSpec.ensure(tc.size())) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "spectral material tables allocation failed");
        }
        // (synchronous copies: the host vectors go out of scope)
        PT_CHECK(r, cudaMemcpy(sl.matSpec.p, mc.data(), mc.size() * sizeof(float4), cudaMemcpyHostToDevice));
        PT_CHECK(r, cudaMemcpy(sl.texSpec.p, tc.data(), tc.size() * sizeof(float4), cudaMemcpyHostToDevice));
        sl.specValid = true;
    }
    if (r->envValid && !r->envSpecValid) {
        const size_t texels = static_cast<size_t>(r->envW) * r->envH;
        if (!r->envSpec.ensure(texels)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "spectral environment table allocation failed");
        }
        spectral::launchUpliftTexels(r->envPixels.p, texels, reinterpret_cast<const float*>(r->specResp.p),
            r->envSpec.p, s);
        PT_CHECK(r, cudaGetLastError());
        r->envSpecValid = true;
    }
    const float k = r->params.environment_intensity;
    r->specBackground =
        coefToFloat4(colourCoef(r, r->params.background_r * k, r->params.background_g * k, r->params.background_b * k));
    if (r->specCapacity < r->capacity) {
        const size_t Q = static_cast<size_t>(r->capacity);
        const size_t words = static_cast<size_t>(spectral::kMaxWavelengths / 4) * Q;
        if (!r->pHero.ensure(Q) || !r->pThrS.ensure(words) || !r->pRadS.ensure(words) || !r->pNeeEnvS.ensure(words) ||
            !r->pNeeEmisS.ensure(words)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "spectral path state allocation failed for %d paths", r->capacity);
        }
        r->specCapacity = r->capacity;
    }
    (void)nw;
    return PT_OK;
}

// Preview level i of n (PathTracerPreviewLevels.h:17-49): downscale 2^(n - i),
// size max(1, axis / downscale).
void previewDims(int width, int height, int levels, int level, int& w, int& h, int& ds)
{
    ds = 1 << (levels - level);
    w = width / ds >= 1 ? width / ds : 1;
    h = height / ds >= 1 ? height / ds : 1;
}

size_t previewOffset(int width, int height, int levels, int level)
{
    size_t off = 0;
    for (int i = 0; i < level; ++i) {
        int w, h, ds;
        previewDims(width, height, levels, i, w, h, ds);
        off += static_cast<size_t>(w) * h;
    }
    return off;
}

// kPreviewMaxPathDepth (PathTracerPreviewLevels.h:13)
constexpr int kPreviewDepth = 4;

int renderPreviews(pt_renderer* r)
{
    const size_t total = previewOffset(r->width, r->height, r->previewLevels, r->previewLevels);
    if (!r->previewBuf.ensure(total)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "preview buffers allocation failed");
    }
    const LaunchCtx* c = uploadCtx(r);
    if (c == nullptr) {
        return fail(r, PT_ERR_CUDA, "launch context upload failed");
    }
    const int grid = r->smCount * adjointBlocksPerSm();
    for (int lv = r->previewDone + 1; lv < r->previewLevels; ++lv) {
        int w, h, ds;
        previewDims(r->width, r->height, r->previewLevels, lv, w, h, ds);
        launchPreview(c, w, h, static_cast<uint32_t>(lv + 1), kPreviewDepth,
            r->previewBuf.p + previewOffset(r->width, r->height, r->previewLevels, lv), grid,
            r->scenes[0].instanceCount > 0, r->stream);
        PT_CHECK(r, cudaGetLastError());
        r->launches += 1;
        r->previewDone = lv;
    }
    return PT_OK;
}

// Emissive triangles (MeshAccelScene.cpp:62-95), selected and summed on the
// device from sl.positions, the material ids in the staging buffer and the
// scene's material bank.
int buildEmissive(pt_renderer* r, SceneSlot& sl, uint32_t n)
{
    cudaStream_t s = r->stream;
    const size_t tempBytes = emissiveSelectTempBytes(n);
    if (!r->eWeights.ensure(n) || !r->eFlags.ensure(n) || !r->eIdx.ensure(n) || !r->eCdf.ensure(n + 1ull) ||
        !r->eOut.ensure(4) || !r->eTemp.ensure(tempBytes)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "emissive scratch allocation failed for %u triangles", n);
    }
    launchEmissiveWeights(sl.positions.p, r->stageIds.p, n, sl.materials.p, sl.materialCount, r->eWeights.p,
        r->eFlags.p, s);
    PT_CHECK(r, emissiveSelect(r->eTemp.p, tempBytes, r->eFlags.p, n, r->eIdx.p, r->eOut.p + 2, s));
    launchEmissiveCdf(r->eWeights.p, r->eIdx.p, r->eOut.p + 2, r->eCdf.p, r->eOut.p, s);
    PT_CHECK(r, cudaGetLastError());
    uint32_t out[2] = {0, 0};
    PT_CHECK(r, cudaMemcpyAsync(out, r->eOut.p, sizeof(out), cudaMemcpyDeviceToHost, s));
    PT_CHECK(r, cudaStreamSynchronize(s));
    float total;
    std::memcpy(&total, &out[1], sizeof(float));
    const uint32_t count = total <= 0.0f ? 0u : out[0];
    sl.emissiveCount = count;
    if (!sl.emissiveIdx.ensure(std::max<uint32_t>(1u, count)) || !sl.emissiveCdf.ensure(count + 1ull)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "emissive list allocation failed");
    }
    if (count > 0) {
        PT_CHECK(r, cudaMemcpyAsync(sl.emissiveIdx.p, r->eIdx.p, count * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(sl.emissiveCdf.p, r->eCdf.p, (count + 1ull) * sizeof(float), cudaMemcpyDeviceToDevice, s));
        if (!sl.emitPdf.ensure(n)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "emitter density allocation failed for %u triangles", n);
        }
        PT_CHECK(r, cudaMemsetAsync(sl.emitPdf.p, 0, n * sizeof(float), s));
        launchEmitterPdf(sl.positions.p, sl.emissiveIdx.p, sl.emissiveCdf.p, count, sl.emitPdf.p, s);
        PT_CHECK(r, cudaGetLastError());
    } else {
        PT_CHECK(r, cudaMemsetAsync(sl.emissiveCdf.p, 0, sizeof(float), s));
    }
    return PT_OK;
}

// With the triangles of a scene in sl.positions (9 floats each) and their
// normals, uvs and material ids in the staging buffers: shading records, the
// emissive list and CDF, and the BVH, all on the device.
int finishScene(pt_renderer* r, SceneSlot& sl, uint32_t n)
{
    cudaStream_t s = r->stream;
    sl.triCount = n;
    if (n == 0) {
        sl.emissiveCount = 0;
        if (!sl.emissiveIdx.ensure(1) || !sl.emissiveCdf.ensure(1)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "emissive list allocation failed");
        }
        PT_CHECK(r, cudaMemsetAsync(sl.emissiveCdf.p, 0, sizeof(float), s));
        sl.bvh.release();
        return PT_OK;
    }
    if (!sl.shade.ensure(n)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "shading records allocation failed for %u triangles", n);
    }
    launchBuildShade(r->stage.p, r->stage.p + 9ull * n, r->stageIds.p, n, sl.shade.p, s);
    PT_CHECK(r, cudaGetLastError());
    {
        const int st = buildEmissive(r, sl, n);
        if (st != PT_OK) {
            return st;
        }
    }
    char err[256] = {0};
    const int st = buildBvh(sl.positions.p, n, sl.bvh, s, r->bvhOptions, err, sizeof(err));
    if (st != PT_OK) {
        return fail(r, st, "BVH build: %s", err);
    }
    return PT_OK;
}

// Uploads a mesh into a scene slot and builds its BVH (MeshAccelScene::build +
// upload, MeshAccelScene.cpp:141-341).
int setSceneMesh(pt_renderer* r, SceneSlot& sl, const pt_mesh* mesh)
{
    const uint32_t n = mesh->triangle_count;
    if (n > 0 && (mesh->positions == nullptr || mesh->normals == nullptr || mesh->uvs == nullptr ||
                     mesh->material_ids == nullptr)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_mesh: missing per-triangle arrays");
    }
    if ((mesh->material_count > 0 && mesh->materials == nullptr) || (mesh->texture_count > 0 && mesh->textures == nullptr)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_mesh: missing material or texture bank");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    cudaStream_t s = r->stream;
    PT_CHECK(r, cudaEventRecord(r->ev0, s));
    sl.hasScene = false;
    sl.shareFrom = -1;
    sl.releaseInstances();
    sl.triCount = n;
    {
        const int st = uploadBank(r, sl, mesh);
        if (st != PT_OK) {
            return st;
        }
    }
    if (n > 0) {
        if (!sl.positions.ensure(9ull * n) || !r->stage.ensure(15ull * n) || !r->stageIds.ensure(n)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "mesh upload failed for %u triangles", n);
        }
        PT_CHECK(r, cudaMemcpyAsync(sl.positions.p, mesh->positions, 9ull * n * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stage.p, mesh->normals, 9ull * n * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stage.p + 9ull * n, mesh->uvs, 6ull * n * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stageIds.p, mesh->material_ids, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    }
    {
        const int st = finishScene(r, sl, n);
        if (st != PT_OK) {
            return st;
        }
    }
    PT_CHECK(r, cudaEventRecord(r->ev1, s));
    PT_CHECK(r, cudaEventSynchronize(r->ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r->ev0, r->ev1);
    r->stats.build_ms = ms;
    sl.hasScene = true;
    uint32_t nodes = 0;
    for (const SceneSlot& x : r->scenes) {
        nodes += x.hasScene ? sceneNodeCount(x) : 0u;
    }
    r->stats.bvh_nodes = static_cast<int32_t>(nodes);
    return resetAccum(r);
}

// Instanced scene (no reference counterpart: the reference flattens its
// ProceduralInstance list into one mesh).  Objects are uploaded one after the
// other (positions and shading records concatenated, each object's shading
// records at its triBase), each gets its own BVH, and the instances' world
// boxes (the object's vertex bounds through the transform) get a top-level BVH
// built by the same builder from one box-shaped record per instance
// (v0 = lo, v1 = hi, v2 = lo).
int setSceneInstances(pt_renderer* r, SceneSlot& sl, uint32_t objectCount, const pt_mesh* objects,
    uint32_t instanceCount, const pt_instance* inst)
{
    if (objectCount == 0 || objects == nullptr || instanceCount == 0 || inst == nullptr) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_instances: no objects or no instances");
    }
    uint64_t total = 0;
    std::vector<uint32_t> triBase(objectCount);
    std::vector<double> objLo(3 * objectCount, 0.0), objHi(3 * objectCount, 0.0);
    for (uint32_t o = 0; o < objectCount; ++o) {
        const pt_mesh& m = objects[o];
        if (m.triangle_count > 0 && (m.positions == nullptr || m.normals == nullptr || m.uvs == nullptr ||
                                        m.material_ids == nullptr)) {
            return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_instances: object %u misses per-triangle arrays", o);
        }
        triBase[o] = static_cast<uint32_t>(total);
        total += m.triangle_count;
        for (int a = 0; a < 3; ++a) {
            objLo[3 * o + a] = 1e300;
            objHi[3 * o + a] = -1e300;
        }
        for (size_t k = 0; k < 3ull * m.triangle_count; ++k) {
            for (int a = 0; a < 3; ++a) {
                const double v = m.positions[3 * k + a];
                objLo[3 * o + a] = std::min(objLo[3 * o + a], v);
                objHi[3 * o + a] = std::max(objHi[3 * o + a], v);
            }
        }
    }
    if (total == 0 || total > 0x7FFFFFFFull) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_instances: %llu object triangles",
            static_cast<unsigned long long>(total));
    }
    // instance records and world boxes
    std::vector<DevInstance> dinst(instanceCount);
    std::vector<float> boxes(9ull * instanceCount);
    for (uint32_t i = 0; i < instanceCount; ++i) {
        const pt_instance& I = inst[i];
        if (I.object >= objectCount) {
            return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_instances: instance %u names object %u of %u", i, I.object,
                objectCount);
        }
        double M[3][4];
        for (int a = 0; a < 3; ++a) {
            for (int b = 0; b < 4; ++b) {
                M[a][b] = I.object_to_world[4 * a + b];
            }
        }
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
            M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) + M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        if (!(std::fabs(det) > 1e-12) || !std::isfinite(det)) {
            return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_instances: instance %u has a singular transform", i);
        }
        double Inv[3][3];
        Inv[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
        Inv[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
        Inv[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
        Inv[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
        Inv[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
        Inv[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
        Inv[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det;
        Inv[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
        Inv[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
        DevInstance& D = dinst[i];
        for (int a = 0; a < 3; ++a) {
            const double tw = -(Inv[a][0] * M[0][3] + Inv[a][1] * M[1][3] + Inv[a][2] * M[2][3]);
            D.w2o[a] = make_float4(static_cast<float>(Inv[a][0]), static_cast<float>(Inv[a][1]),
                static_cast<float>(Inv[a][2]), static_cast<float>(tw));
            D.o2w[a] = make_float4(static_cast<float>(M[a][0]), static_cast<float>(M[a][1]), static_cast<float>(M[a][2]),
                static_cast<float>(M[a][3]));
        }
        D.meta = make_uint4(I.object, 0u, 0u, 0u);
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int c = 0; c < 8; ++c) {
            const double p[3] = {(c & 1) ? objHi[3 * I.object] : objLo[3 * I.object],
                (c & 2) ? objHi[3 * I.object + 1] : objLo[3 * I.object + 1],
                (c & 4) ? objHi[3 * I.object + 2] : objLo[3 * I.object + 2]};
            for (int a = 0; a < 3; ++a) {
                const double w = M[a][0] * p[0] + M[a][1] * p[1] + M[a][2] * p[2] + M[a][3];
                lo[a] = std::min(lo[a], w);
                hi[a] = std::max(hi[a], w);
            }
        }
        for (int a = 0; a < 3; ++a) {
            // widened by a relative margin so that float rounding of the object
            // space ray cannot step outside
            const double pad = 1e-5 * (hi[a] - lo[a]) + 1e-6 * std::max(std::fabs(lo[a]), std::fabs(hi[a])) + 1e-7;
            boxes[9 * i + a] = static_cast<float>(lo[a] - pad);
            boxes[9 * i + 3 + a] = static_cast<float>(hi[a] + pad);
            boxes[9 * i + 6 + a] = static_cast<float>(lo[a] - pad);
        }
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    cudaStream_t s = r->stream;
    PT_CHECK(r, cudaEventRecord(r->ev0, s));
    sl.hasScene = false;
    sl.shareFrom = -1;
    sl.releaseInstances();
    sl.bvh.release();
    int st = uploadBank(r, sl, &objects[0]);
    if (st != PT_OK) {
        return st;
    }
    const uint32_t n = static_cast<uint32_t>(total);
    sl.triCount = n;
    if (!sl.positions.ensure(9ull * n) || !sl.shade.ensure(n) || !r->stage.ensure(15ull * n) || !r->stageIds.ensure(n)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "pt_set_instances: allocation failed for %u object triangles", n);
    }
    for (uint32_t o = 0; o < objectCount; ++o) {
        const pt_mesh& m = objects[o];
        const size_t e = m.triangle_count, b = triBase[o];
        if (e == 0) {
            continue;
        }
        PT_CHECK(r, cudaMemcpyAsync(sl.positions.p + 9 * b, m.positions, 9 * e * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stage.p + 9 * b, m.normals, 9 * e * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stage.p + 9ull * n + 6 * b, m.uvs, 6 * e * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stageIds.p + b, m.material_ids, e * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    }
    launchBuildShade(r->stage.p, r->stage.p + 9ull * n, r->stageIds.p, n, sl.shade.p, s);
    PT_CHECK(r, cudaGetLastError());
    // emitters inside objects are reached by BSDF sampling only
    sl.emissiveCount = 0;
    if (!sl.emissiveIdx.ensure(1) || !sl.emissiveCdf.ensure(1)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "emissive list allocation failed");
    }
    PT_CHECK(r, cudaMemsetAsync(sl.emissiveCdf.p, 0, sizeof(float), s));
    sl.objBvh.resize(objectCount);
    std::vector<DevBlas> dblas(objectCount);
    char err[256] = {0};
    for (uint32_t o = 0; o < objectCount; ++o) {
        const uint32_t e = objects[o].triangle_count;
        dblas[o] = DevBlas{nullptr, nullptr, triBase[o], 0u};
        if (e == 0) {
            continue;
        }
        st = buildBvh(sl.positions.p + 9ull * triBase[o], e, sl.objBvh[o], s, r->bvhOptions, err, sizeof(err));
        if (st != PT_OK) {
            return fail(r, st, "object %u BVH build: %s", o, err);
        }
        dblas[o].nodes = sl.objBvh[o].nodes;
        dblas[o].tris = sl.objBvh[o].tris;
        dblas[o].nodeCount = sl.objBvh[o].nodeCount;
    }
    if (!sl.tlasBoxes.ensure(9ull * instanceCount) || !sl.instances.ensure(instanceCount) ||
        !sl.blases.ensure(objectCount)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "instance tables allocation failed");
    }
    // (synchronous copies: the host vectors go out of scope)
    PT_CHECK(r, cudaMemcpy(sl.tlasBoxes.p, boxes.data(), boxes.size() * sizeof(float), cudaMemcpyHostToDevice));
    PT_CHECK(r, cudaMemcpy(sl.instances.p, dinst.data(), dinst.size() * sizeof(DevInstance), cudaMemcpyHostToDevice));
    PT_CHECK(r, cudaMemcpy(sl.blases.p, dblas.data(), dblas.size() * sizeof(DevBlas), cudaMemcpyHostToDevice));
    // one instance per top-level leaf: every instance box is tested before its object is entered
    BvhBuildOptions topOptions = r->bvhOptions;
    topOptions.maxLeafSize = 1;
    st = buildBvh(sl.tlasBoxes.p, instanceCount, sl.tlas, s, topOptions, err, sizeof(err));
    if (st != PT_OK) {
        return fail(r, st, "top-level BVH build: %s", err);
    }
    sl.instanceCount = instanceCount;
    PT_CHECK(r, cudaEventRecord(r->ev1, s));
    PT_CHECK(r, cudaEventSynchronize(r->ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r->ev0, r->ev1);
    r->stats.build_ms = ms;
    sl.hasScene = true;
    uint32_t nodes = 0;
    for (const SceneSlot& x : r->scenes) {
        nodes += x.hasScene ? sceneNodeCount(x) : 0u;
    }
    r->stats.bvh_nodes = static_cast<int32_t>(nodes);
    return resetAccum(r);
}

void releaseBounceGraphs(pt_renderer* r)
{
    for (cudaGraphExec_t& g : r->bounceGraph) {
        if (g != nullptr) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    }
}

#ifndef PT_EXTEND_LANE_MIN_NODES
#define PT_EXTEND_LANE_MIN_NODES 32768
#endif

// Grid of the closest-hit stage: the per-lane kernel has its own occupancy.
int extendGrid(const pt_renderer* r, bool count, bool inst)
{
    if (r->extendLane && !count) {
        return inst ? r->gridExtendLaneInst : r->gridExtendLane;
    }
    return r->gridExtend;
}
// Grid of the hit shader: RGB and spectral forms differ in registers, and a
// grid above one form's occupancy leaves a partial second wave of blocks.
int shadeGrid(const pt_renderer* r, int nw)
{
    const int occ = shadeOccupancy(nw);
    return r->smCount * (r->blocksPerSmOverride > 0 ? std::min(r->blocksPerSmOverride, occ) : occ);
}
int shadowGrid(const pt_renderer* r, bool count, bool inst)
{
    if (r->extendLane && !count) {
        return inst ? r->gridShadowLaneInst : r->gridShadowLane;
    }
    return r->gridShadow;
}

// The graphs of four bounce iterations for this launch configuration
// (captured on first use; false: run without graphs, e.g. when the caller's
// stream is itself being captured).
bool ensureBounceGraphs(pt_renderer* r, const LaunchCtx* c, bool inst, int nw)
{
    const unsigned long long key[6] = {reinterpret_cast<unsigned long long>(c), static_cast<unsigned long long>(r->gridExtend),
        static_cast<unsigned long long>(r->gridShade) | (static_cast<unsigned long long>(r->gridExtendLaneInst) << 16) |
            (static_cast<unsigned long long>(r->gridShadowLaneInst) << 32),
        static_cast<unsigned long long>(r->gridShadow),
        static_cast<unsigned long long>(inst ? 1 : 0) | (static_cast<unsigned long long>(nw) << 1) |
            (static_cast<unsigned long long>(r->extendLane ? 1 : 0) << 8) |
            (static_cast<unsigned long long>(r->gridExtendLane) << 9) |
            (static_cast<unsigned long long>(r->gridShadowLane) << 22) |
            (static_cast<unsigned long long>(r->gridShadeMiss) << 36),
        reinterpret_cast<unsigned long long>(r->stream)};
    if (r->bounceGraph[0] != nullptr && std::equal(key, key + 6, r->bounceKey)) {
        return true;
    }
    releaseBounceGraphs(r);
    cudaStream_t s = r->stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        return false;
    }
    for (int g = 0; g < 2; ++g) {
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            releaseBounceGraphs(r);
            r->useGraphs = false;
            return false;
        }
        int sel = 0;
        for (int it = 0; it < 4; ++it) {
            launchExtend(c, sel, g == 0 && it == 0, it, extendGrid(r, false, inst), false, inst, r->extendLane, s);
            launchShadeMiss(c, it, sel, r->gridShadeMiss, nw, s);
            launchShade(c, sel, it, shadeGrid(r, nw), nw, s);
            launchShadow(c, it, shadowGrid(r, false, inst), false, inst, r->extendLane, s);
            launchFinalize(c, sel, r->gridShadow, nw, s);
            if (slotOrdered(r)) {
                launchNextQueue(c, sel, r->gridShadow, s);
            }
            sel ^= 1;
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (e != cudaSuccess || graph == nullptr ||
            cudaGraphInstantiate(&r->bounceGraph[g], graph, 0) != cudaSuccess) {
            if (graph != nullptr) {
                cudaGraphDestroy(graph);
            }
            cudaGetLastError();
            releaseBounceGraphs(r);
            r->useGraphs = false;
            return false;
        }
        cudaGraphDestroy(graph);
    }
    std::copy(key, key + 6, r->bounceKey);
    return true;
}

} // namespace


extern "C" {

int pt_create(pt_renderer** out, int device)
{
    if (out == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    pt_renderer* r = new pt_renderer();
    if (device < 0) {
        if (cudaGetDevice(&r->device) != cudaSuccess) {
            delete r;
            return PT_ERR_CUDA;
        }
    } else {
        r->device = device;
    }
    if (cudaSetDevice(r->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&r->ownStream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess) {
        delete r;
        return PT_ERR_CUDA;
    }
    r->stream = r->ownStream;
    cudaDeviceGetAttribute(&r->smCount, cudaDevAttrMultiProcessorCount, r->device);
    pt_default_params(&r->params);
    r->scenes[0].camera = defaultCamera();
    int be = 1, bs = 1, bsh = 1;
    stageOccupancy(be, bs, bsh);
    r->gridExtend = r->smCount * std::max(be, 1);
    r->gridShade = r->smCount * std::max(bs, 1);
    r->gridShadow = r->smCount * std::max(bsh, 1);
    r->gridExtendLane = r->smCount * extendLaneOccupancy();
    r->gridShadowLane = r->smCount * shadowLaneOccupancy();
    r->gridExtendLaneInst = r->smCount * extendLaneInstOccupancy();
    r->gridShadowLaneInst = r->smCount * shadowLaneInstOccupancy();
    r->gridShadeMiss = r->smCount * shadeMissOccupancy();
    *out = r;
    return PT_OK;
}

int pt_destroy(pt_renderer* r)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    cudaSetDevice(r->device);
    if (r->stream) {
        cudaStreamSynchronize(r->stream);
    }
    for (SceneSlot& sl : r->scenes) {
        sl.release();
    }
    r->dScenes.release();
    r->dViews.release();
    r->stage.release();
    r->stageIds.release();
    r->eWeights.release();
    r->eFlags.release();
    r->eIdx.release();
    r->eCdf.release();
    r->eOut.release();
    r->eTemp.release();
    r->tRingStart.release();
    r->tMaterials.release();
    r->tPoints.release();
    r->tTangents.release();
    r->tRadii.release();
    r->tCosSin.release();
    r->tLeaves.release();
    r->tFrames.release();
    r->tGivenFrames.release();
    r->envPixels.release();
    r->envMarginal.release();
    r->envRow.release();
    r->envScratch.release();
    r->specResp.release();
    r->envSpec.release();
    r->pHero.release();
    r->pThrS.release();
    r->pRadS.release();
    r->pNeeEnvS.release();
    r->pNeeEmisS.release();
    r->acc.release();
    r->counts.release();
    r->lumMean.release();
    r->m2.release();
    r->converged.release();
    r->active0.release();
    r->active1.release();
    r->activeCount.release();
    r->samples.release();
    r->displayBuf.release();
    r->adjImage.release();
    r->record.release();
    r->previewBuf.release();
    r->adjGrad.release();
    r->compactTemp.release();
    r->sceneActiveStart.release();
    r->sceneJobStart.release();
    r->pPixel.release();
    r->pOut.release();
    r->pRngA.release();
    r->pRngB.release();
    r->pOrig.release();
    r->pDir.release();
    r->pThr.release();
    r->pRad.release();
    r->pHit.release();
    r->pHitInst.release();
    r->pNeeEnv.release();
    r->pNeeEmis.release();
    r->pVisEnv.release();
    r->pVisEmis.release();
    r->pScene.release();
    r->pNextFlag.release();
    r->qExt0.release();
    r->qExt1.release();
    r->qFinish.release();
    r->qMiss.release();
    r->qHit.release();
    r->qShadowPath.release();
    r->qShadowO.release();
    r->qShadowD.release();
    r->qCounts.release();
    r->qRays.release();
    r->qVisits.release();
    r->qOverflow.release();
    r->dctx.release();
    r->dbatch.release();
    releaseBounceGraphs(r);
    for (cudaEvent_t e : r->eventPool) {
        cudaEventDestroy(e);
    }
    if (r->ev0) {
        cudaEventDestroy(r->ev0);
    }
    if (r->ev1) {
        cudaEventDestroy(r->ev1);
    }
    if (r->ownStream) {
        cudaStreamDestroy(r->ownStream);
    }
    delete r;
    return PT_OK;
}

const char* pt_last_error(const pt_renderer* r)
{
    return r == nullptr ? "null renderer" : r->lastError.c_str();
}

void pt_default_params(pt_render_params* out)
{
    if (out == nullptr) {
        return;
    }
    std::memset(out, 0, sizeof(*out));
    out->background_r = out->background_g = out->background_b = 10.0f / 255.0f;
    out->environment_intensity = 1.0f;
    out->max_path_depth = 32;
    out->russian_roulette_min_depth = 3;
    out->min_samples = 16;
    out->max_samples_per_pixel = 1024;
    out->relative_error_threshold = 0.02f;
}

int pt_configure(pt_renderer* r, int width, int height)
{
    if (r == nullptr || width <= 0 || height <= 0 || static_cast<int64_t>(width) * height > (int64_t(1) << 30)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_configure: bad size %dx%d", width, height);
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    // back to a single scene: drop the geometry of any further batch scenes
    for (size_t k = 1; k < r->scenes.size(); ++k) {
        r->scenes[k].release();
    }
    r->scenes.resize(1);
    return configureLayout(r, &width, &height);
}

int pt_set_mesh(pt_renderer* r, const pt_mesh* mesh)
{
    if (r == nullptr || mesh == nullptr) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_mesh: null argument");
    }
    return setSceneMesh(r, r->scenes[0], mesh);
}

int pt_set_camera(pt_renderer* r, const pt_camera* camera)
{
    if (r == nullptr || camera == nullptr) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_camera: null argument");
    }
    r->scenes[0].camera = *camera;
    return resetAccum(r);
}

int pt_get_camera(const pt_renderer* r, pt_camera* out)
{
    if (r == nullptr || out == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    *out = r->scenes[0].camera;
    return PT_OK;
}

int pt_set_params(pt_renderer* r, const pt_render_params* params)
{
    if (r == nullptr || params == nullptr) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_params: null argument");
    }
    if (params->emitter_mis != 0 && params->emitter_mis != 1) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_params: emitter_mis must be 0 or 1 (got %d)", params->emitter_mis);
    }
    if (params->spectral_wavelengths != 0 && params->spectral_wavelengths != 4 && params->spectral_wavelengths != 8) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_params: spectral_wavelengths must be 0, 4 or 8 (got %d)",
            params->spectral_wavelengths);
    }
    r->params = *params;
    // The ranges the reference's setters clamp to (PathTracer.cpp:126-190):
    // max spp in [0, 1e6] (0 = no cap), min spp in [1, 1e4], relative error in
    // [0.001, 1] (a NaN becomes the lower bound); the RR depth is not negative.
    pt_render_params& p = r->params;
    p.max_samples_per_pixel = std::min(std::max(p.max_samples_per_pixel, 0), 1000000);
    p.min_samples = std::min(std::max(p.min_samples, 1), 10000);
    if (!(p.relative_error_threshold >= 0.001f)) {
        p.relative_error_threshold = 0.001f;
    }
    p.relative_error_threshold = std::min(p.relative_error_threshold, 1.0f);
    p.russian_roulette_min_depth = std::max(p.russian_roulette_min_depth, 0);
    return resetAccum(r);
}

int pt_get_params(const pt_renderer* r, pt_render_params* out)
{
    if (r == nullptr || out == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    *out = r->params;
    return PT_OK;
}

int pt_set_environment(pt_renderer* r, int width, int height, const float* rgb)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    if (rgb == nullptr) {
        r->envValid = false;
        return resetAccum(r);
    }
    if (width <= 0 || height <= 0) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_environment: bad size %dx%d", width, height);
    }
    // importance tables (EnvironmentMap.cpp:76-128) built on the device with the
    // reference's sequential single-precision sums; only sin(theta) per row is
    // evaluated here, with the reference's host expression
    const size_t W = static_cast<size_t>(width), H = static_cast<size_t>(height);
    std::vector<float> sinTheta(H);
    for (size_t y = 0; y < H; ++y) {
        const float v = (static_cast<float>(y) + 0.5f) / static_cast<float>(height);
        sinTheta[y] = std::sin(v * 3.14159265f);
    }
    if (!r->envPixels.ensure(W * H * 3) || !r->envMarginal.ensure(H + 1) || !r->envRow.ensure(H * (W + 1)) ||
        !r->envScratch.ensure(2 * H)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "environment upload failed");
    }
    PT_CHECK(r, cudaMemcpyAsync(r->envPixels.p, rgb, W * H * 3 * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    PT_CHECK(r, cudaMemcpyAsync(r->envScratch.p, sinTheta.data(), H * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    launchEnvTables(r->envPixels.p, width, height, r->envScratch.p, r->envMarginal.p, r->envRow.p, r->envScratch.p + H,
        r->stream);
    PT_CHECK(r, cudaGetLastError());
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    r->envW = width;
    r->envH = height;
    r->envValid = true;
    r->envSpecValid = false;
    return resetAccum(r);
}

int pt_reset(pt_renderer* r)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    return resetAccum(r);
}

// Render loop.  Each iteration folds B waves into one launch sequence: the
// active pixels x B samples are generated (in chunks of the path capacity),
// traced bounce by bounce, then folded per pixel in sample order and the
// active list compacted.  Wave w of the reference uses globalSeed = w + 1 and
// sampleIndex = counts[pixel] (PathTracer.cpp:2379, RandCore.h:7-12); an
// active pixel has counts == w, so slot s of a batch starting at wave W uses
// exactly the reference's seed for wave W + s.  Pixels that converge inside a
// batch ignore the batch's remaining samples, which is what the reference's
// per-wave convergence skip does.
int pt_render(pt_renderer* r, int waves)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    if (r->width <= 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_render before pt_configure");
    }
    for (size_t k = 0; k < r->scenes.size(); ++k) {
        const SceneSlot& sl = r->scenes[k];
        const bool has = sl.shareFrom >= 0 ? r->scenes[static_cast<size_t>(sl.shareFrom)].hasScene : sl.hasScene;
        if (!has) {
            return fail(r, PT_ERR_NO_SCENE, "pt_render before the mesh of scene %zu was set", k);
        }
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    cudaStream_t s = r->stream;
    {
        // path state for min(cap, pixels x first batch) paths
        const int B0 = chooseBatch(r, waves > 0 ? waves : 0);
        const long long jobs0 = static_cast<long long>(std::max(r->hostActive, 1)) * B0;
        const int want = static_cast<int>(std::min<long long>(r->capacityWanted, std::max<long long>(jobs0, 1 << 16)));
        int st = ensurePaths(r, want);
        if (st != PT_OK) {
            return st;
        }
    }
    bool inst = false;
    uint32_t maxNodes = 0;
    for (const SceneSlot& sl : r->scenes) {
        inst = inst || sl.instanceCount > 0;
        maxNodes = std::max(maxNodes, sl.bvh.nodeCount);
        for (const BvhBuffers& b : sl.objBvh) {
            maxNodes = std::max(maxNodes, b.nodeCount); // an instanced scene's objects
        }
    }
    // Per-lane ray replacement pays where traversals are long (large trees, and
    // instanced scenes of large objects: the two-level traversal); on small
    // scenes the extra routing launch costs more than it saves.
    r->extendLane = r->extendMode == PT_EXTEND_MODE_LANE ||
        (r->extendMode == PT_EXTEND_MODE_AUTO && maxNodes >= static_cast<uint32_t>(PT_EXTEND_LANE_MIN_NODES));
    const int nw = r->params.spectral_wavelengths;
    if (nw > 0) {
        const int st = prepareSpectral(r, nw);
        if (st != PT_OK) {
            return st;
        }
    }
    if (r->previewLevels > 0 && r->wavesDone == 0 && r->previewDone < r->previewLevels - 1 && r->scenes.size() == 1) {
        // the preview passes come first (PathTracer.cpp:2382-2396); iteration i
        // renders level i with global seed i + 1
        const int st = renderPreviews(r);
        if (st != PT_OK) {
            return st;
        }
    }
    const bool countVisits = (r->profileFlags & PT_PROFILE_COUNT_VISITS) != 0;
    r->profile = pt_profile{};
    r->eventMarks.clear();
    PT_CHECK(r, cudaMemsetAsync(r->qRays.p, 0, 2 * sizeof(unsigned long long), s));
    PT_CHECK(r, cudaMemsetAsync(r->qVisits.p, 0, 4 * sizeof(unsigned long long), s));
    PT_CHECK(r, cudaMemsetAsync(r->qOverflow.p, 0, sizeof(unsigned int), s));
    PT_CHECK(r, cudaEventRecord(r->ev0, s));
    int remaining = waves;
    int64_t launches = 0;
    const int maxDepthEff = r->params.max_path_depth > 0 ? r->params.max_path_depth : (r->params.max_path_depth == 0 ? 256 : 32);
    while ((waves <= 0 || remaining > 0) && r->hostActive > 0) {
        const int active = r->hostActive;
        const int B = chooseBatch(r, waves > 0 ? remaining : 0);
        const size_t need = static_cast<size_t>(active) * B;
        if (!r->samples.ensure(need)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "sample buffer allocation failed (%zu samples)", need);
        }
        const long long jobs = static_cast<long long>(active) * B;
        const int slots = static_cast<int>(std::min<long long>(std::min(r->capacity, r->capacityWanted), jobs));
        r->hbatch.jobs = static_cast<unsigned long long>(jobs);
        // generations: no slot takes a second job; each generation of `slots`
        // jobs drains before the next one starts
        r->hbatch.nextJob = static_cast<unsigned long long>(PT_PATH_GENERATIONS ? jobs : slots);
        r->hbatch.activeCount = active;
        r->hbatch.waveBase = static_cast<uint32_t>(r->wavesDone);
        r->hbatch.slotCount = slots;
        if (slotOrdered(r)) {
            // (marks are cleared by k_next_queue; this also clears those of a render that failed)
            PT_CHECK(r, cudaMemsetAsync(r->pNextFlag.p, 0, static_cast<size_t>(slots), s));
        }
        PT_CHECK(r, cudaMemcpyAsync(r->dbatch.p, &r->hbatch, sizeof(BatchInfo), cudaMemcpyHostToDevice, s));
        const LaunchCtx* c = uploadCtx(r);
        if (c == nullptr) {
            return fail(r, PT_ERR_CUDA, "launch context upload failed");
        }
        if (r->scenes.size() > 1) {
            launchSceneJobs(c, static_cast<int>(r->scenes.size()), B, s);
            ++launches;
        }
        for (long long jobOffset = 0; jobOffset < jobs; jobOffset += slots) {
            const int genCount = static_cast<int>(std::min<long long>(slots, jobs - jobOffset));
            {
                StageTimer tm(r, kGenerate);
                launchGenerate(c, genCount, 0, nw, s, static_cast<unsigned long long>(jobOffset));
            }
            ++launches;
            // Every live path advances one bounce per iteration and a finished path's
            // slot takes the next job, so iterations <= bounce-steps / slots + drain.
            const long long maxIters =
                (jobs * (maxDepthEff + 1) + slots - 1) / std::max(slots, 1) + maxDepthEff + 8;
            int sel = 0;
            const bool graphs = r->useGraphs && r->profileFlags == 0 && ensureBounceGraphs(r, c, inst, nw);
            for (long long it = 0; graphs; it += 4) {
                // the same four iterations as below, replayed from a graph: sel is 0
                // again after four, and the kernels use only the parity of `iter`
                if (it > maxIters) {
                    return fail(r, PT_ERR_INTERNAL, "path queue did not drain after %lld iterations", it);
                }
                PT_CHECK(r, cudaGraphLaunch(r->bounceGraph[it == 0 ? 0 : 1], s));
                launches += 4 * (4 + extendKernels(false, inst, r->extendLane) + (slotOrdered(r) ? 1 : 0));
                r->profile.launches_extend += 4;
                r->profile.launches_shadow += 4;
                unsigned int live = 0;
                PT_CHECK(r, cudaMemcpyAsync(&live, r->qCounts.p, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
                PT_CHECK(r, cudaStreamSynchronize(s));
                if (live == 0) {
                    break;
                }
            }
            for (long long it = 0; !graphs; ++it) {
                if (it > maxIters) {
                    return fail(r, PT_ERR_INTERNAL, "path queue did not drain after %lld iterations", it);
                }
                const int iter = static_cast<int>(it & 0x7fffffff);
                {
                    StageTimer tm(r, kExtend);
                    launchExtend(c, sel, it == 0, iter, extendGrid(r, countVisits, inst), countVisits, inst, r->extendLane, s);
                }
                {
                    StageTimer tm(r, kShade);
                    launchShadeMiss(c, iter, sel, r->gridShadeMiss, nw, s);
                    launchShade(c, sel, iter, shadeGrid(r, nw), nw, s);
                }
                {
                    StageTimer tm(r, kShadow);
                    launchShadow(c, iter, shadowGrid(r, countVisits, inst), countVisits, inst, r->extendLane, s);
                }
                {
                    StageTimer tm(r, kFinalize);
                    launchFinalize(c, sel, r->gridShadow, nw, s);
                    if (slotOrdered(r)) {
                        launchNextQueue(c, sel, r->gridShadow, s);
                    }
                }
                launches += 4 + extendKernels(countVisits, inst, r->extendLane) + (slotOrdered(r) ? 1 : 0);
                r->profile.launches_extend += 1;
                r->profile.launches_shadow += 1;
                sel ^= 1;
                if ((it & 3) == 3) {
                    unsigned int live = 0;
                    PT_CHECK(r, cudaMemcpyAsync(&live, r->qCounts.p + sel, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
                    PT_CHECK(r, cudaStreamSynchronize(s));
                    if (live == 0) {
                        break;
                    }
                }
            }
            if (!PT_PATH_GENERATIONS) {
                break; // one pass: finished paths' slots took the batch's later jobs
            }
        }
        PT_CHECK(r, cudaGetLastError());
        {
            StageTimer tm(r, kAccumulate);
            launchAccumulate(c, active, B, s);
        }
        PT_CHECK(r, cudaMemsetAsync(r->activeCount.p + 1, 0, sizeof(int), s));
        {
            StageTimer tm(r, kCompact);
            const size_t tb = compactTempBytes(active);
            if (!r->compactTemp.ensure(tb)) {
                return fail(r, PT_ERR_OUT_OF_MEMORY, "compaction scratch allocation failed");
            }
            int* lists[2] = {r->active0.p, r->active1.p};
            PT_CHECK(r, launchCompactStable(lists[r->activeSel], lists[r->activeSel ^ 1], r->activeCount.p + 1, active,
                r->converged.p, r->counts.p, r->params.max_samples_per_pixel, r->compactTemp.p, tb, s));
        }
        launches += 2;
        int next = 0;
        PT_CHECK(r, cudaMemcpyAsync(&next, r->activeCount.p + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        PT_CHECK(r, cudaStreamSynchronize(s));
        PT_CHECK(r, cudaGetLastError());
        r->lastStopRate = static_cast<double>(active - next) / active / std::max(1.0, B / 4.0);
        r->activeSel ^= 1;
        r->hostActive = next;
        r->wavesDone += B;
        r->samplesDone += jobs;
        if (waves > 0) {
            remaining -= B;
        }
    }
    // the record holds samples 0 .. recordSpp - 1 of every pixel when each pixel
    // was rendered to exactly that many samples
    r->recordValid = r->recordSpp > 0 && r->scenes.size() == 1 && r->record.p != nullptr &&
        r->wavesDone >= r->recordSpp && r->params.min_samples == r->recordSpp &&
        r->params.max_samples_per_pixel == r->recordSpp;
    PT_CHECK(r, cudaEventRecord(r->ev1, s));
    PT_CHECK(r, cudaEventSynchronize(r->ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r->ev0, r->ev1);
    unsigned long long rays[2] = {0, 0};
    unsigned long long visits[4] = {0, 0, 0, 0};
    unsigned int overflow = 0;
    PT_CHECK(r, cudaMemcpy(rays, r->qRays.p, sizeof(rays), cudaMemcpyDeviceToHost));
    PT_CHECK(r, cudaMemcpy(visits, r->qVisits.p, sizeof(visits), cudaMemcpyDeviceToHost));
    PT_CHECK(r, cudaMemcpy(&overflow, r->qOverflow.p, sizeof(overflow), cudaMemcpyDeviceToHost));
    collectStageTimes(r);
    r->profile.rays_extend = static_cast<int64_t>(rays[0]);
    r->profile.rays_shadow = static_cast<int64_t>(rays[1]);
    r->profile.nodes_extend = static_cast<int64_t>(visits[0]);
    r->profile.tris_extend = static_cast<int64_t>(visits[1]);
    r->profile.nodes_shadow = static_cast<int64_t>(visits[2]);
    r->profile.tris_shadow = static_cast<int64_t>(visits[3]);
    r->stats.render_ms = ms;
    r->stats.rays += static_cast<int64_t>(rays[0] + rays[1]);
    r->stats.stack_overflows += static_cast<int32_t>(overflow);
    r->launches += launches;
    return PT_OK;
}

int pt_readback(pt_renderer* r, float* rgba, uint32_t* counts, uint8_t* converged)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    if (r->width <= 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_readback before pt_configure");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    const size_t P = static_cast<size_t>(r->width) * r->height;
    if (rgba) {
        PT_CHECK(r, cudaMemcpyAsync(rgba, r->acc.p, P * sizeof(float4), cudaMemcpyDeviceToHost, r->stream));
    }
    if (counts) {
        PT_CHECK(r, cudaMemcpyAsync(counts, r->counts.p, P * sizeof(uint32_t), cudaMemcpyDeviceToHost, r->stream));
    }
    if (converged) {
        PT_CHECK(r, cudaMemcpyAsync(converged, r->converged.p, P, cudaMemcpyDeviceToHost, r->stream));
    }
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    return PT_OK;
}

int pt_device_buffers(pt_renderer* r, void** rgba, void** counts, void** converged)
{
    if (r == nullptr || r->width <= 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_device_buffers before pt_configure");
    }
    if (rgba) {
        *rgba = r->acc.p;
    }
    if (counts) {
        *counts = r->counts.p;
    }
    if (converged) {
        *converged = r->converged.p;
    }
    return PT_OK;
}

int pt_get_stats(const pt_renderer* r, pt_stats* out)
{
    if (r == nullptr || out == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    *out = r->stats;
    out->waves = r->wavesDone;
    out->active_pixels = r->hostActive;
    out->samples = r->samplesDone;
    out->launches = r->launches;
    out->budget_exhausted = r->hostActive <= 0 ? 1 : 0;
    return PT_OK;
}

int pt_trace_rays_device(pt_renderer* r, int n, const float* origins, const float* dirs, const float* tmin,
    const float* tmax, uint8_t* hit, float* t, uint32_t* tri, float* normal, float* uv, void* stream)
{
    if (r == nullptr || n < 0 || (n > 0 && (origins == nullptr || dirs == nullptr || tmin == nullptr || tmax == nullptr ||
                                              hit == nullptr))) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_trace_rays: bad arguments");
    }
    if (!r->scenes[0].hasScene) {
        return fail(r, PT_ERR_NO_SCENE, "pt_trace_rays before pt_set_mesh");
    }
    if (n == 0) {
        return PT_OK;
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : r->stream;
    launchTraceRays(deviceScene(&r->scenes[0]), n, origins, dirs, tmin, tmax, hit, t, tri, normal, uv, s);
    PT_CHECK(r, cudaGetLastError());
    return PT_OK;
}

int pt_trace_rays(pt_renderer* r, int n, const float* origins, const float* dirs, const float* tmin, const float* tmax,
    uint8_t* hit, float* t, uint32_t* tri, float* normal, float* uv)
{
    if (r == nullptr || n < 0 || (n > 0 && (origins == nullptr || dirs == nullptr || tmin == nullptr || tmax == nullptr ||
                                              hit == nullptr))) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_trace_rays: bad arguments");
    }
    if (!r->scenes[0].hasScene) {
        return fail(r, PT_ERR_NO_SCENE, "pt_trace_rays before pt_set_mesh");
    }
    if (n == 0) {
        return PT_OK;
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    const size_t N = static_cast<size_t>(n);
    // one staging allocation: inputs 8 floats, outputs 1 byte + 7 words per ray
    const size_t bytes = N * (8 * sizeof(float) + 7 * sizeof(float) + 16);
    void* buf = nullptr;
    PT_CHECK(r, cudaMallocAsync(&buf, bytes + 16, r->stream));
    // traversal stack overflows of this query (pt_stats.stack_overflows)
    unsigned int* dOverflow = reinterpret_cast<unsigned int*>(static_cast<char*>(buf) + ((bytes + 15) & ~size_t(15)));
    float* dO = static_cast<float*>(buf);
    float* dD = dO + 3 * N;
    float* dTmin = dD + 3 * N;
    float* dTmax = dTmin + N;
    float* dT = dTmax + N;
    uint32_t* dTri = reinterpret_cast<uint32_t*>(dT + N);
    float* dN = reinterpret_cast<float*>(dTri + N);
    float* dUv = dN + 3 * N;
    uint8_t* dHit = reinterpret_cast<uint8_t*>(dUv + 2 * N);
    cudaStream_t s = r->stream;
    int rc = PT_OK;
    unsigned int overflow = 0;
    cudaError_t e = cudaMemsetAsync(dOverflow, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dO, origins, 3 * N * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dD, dirs, 3 * N * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dTmin, tmin, N * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dTmax, tmax, N * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        launchTraceRays(deviceScene(&r->scenes[0]), n, dO, dD, dTmin, dTmax, dHit, dT, dTri, dN, dUv, s, dOverflow);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&overflow, dOverflow, sizeof(overflow), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hit, dHit, N, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && t) e = cudaMemcpyAsync(t, dT, N * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && tri) e = cudaMemcpyAsync(tri, dTri, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && normal) e = cudaMemcpyAsync(normal, dN, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && uv) e = cudaMemcpyAsync(uv, dUv, 2 * N * sizeof(float), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(buf, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (e == cudaSuccess) {
        e = e2;
    }
    if (e != cudaSuccess) {
        rc = cudaFail(r, e, "pt_trace_rays");
    } else {
        r->stats.stack_overflows += static_cast<int32_t>(overflow);
    }
    return rc;
}

int pt_set_stream(pt_renderer* r, void* stream)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    r->stream = stream ? static_cast<cudaStream_t>(stream) : r->ownStream;
    return PT_OK;
}

int pt_set_profiling(pt_renderer* r, int flags)
{
    if (r == nullptr || (flags & ~(PT_PROFILE_STAGE_TIMES | PT_PROFILE_COUNT_VISITS)) != 0) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_profiling: unknown flags %d", flags);
    }
    r->profileFlags = flags;
    return PT_OK;
}

int pt_get_profile(const pt_renderer* r, pt_profile* out)
{
    if (r == nullptr || out == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    *out = r->profile;
    return PT_OK;
}

int pt_set_extend_mode(pt_renderer* r, int mode)
{
    if (r == nullptr || mode < PT_EXTEND_MODE_AUTO || mode > PT_EXTEND_MODE_LANE) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_extend_mode: mode must be 0 (auto), 1 (warp) or 2 (lane)");
    }
    r->extendMode = mode;
    return PT_OK;
}

int pt_set_tuning(pt_renderer* r, int path_capacity, int blocks_per_sm)
{
    if (r == nullptr || path_capacity < 0 || blocks_per_sm < 0 || path_capacity > (1 << 26)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_tuning: bad arguments");
    }
    r->capacityWanted = path_capacity > 0 ? path_capacity : (1 << 24);
    r->blocksPerSmOverride = blocks_per_sm;
    if (blocks_per_sm > 0) {
        r->gridExtend = r->gridShade = r->gridShadow = r->smCount * blocks_per_sm;
        r->gridExtendLane = r->smCount * std::min(blocks_per_sm, extendLaneOccupancy());
        r->gridShadowLane = r->smCount * std::min(blocks_per_sm, shadowLaneOccupancy());
        r->gridExtendLaneInst = r->smCount * std::min(blocks_per_sm, extendLaneInstOccupancy());
        r->gridShadowLaneInst = r->smCount * std::min(blocks_per_sm, shadowLaneInstOccupancy());
        r->gridShadeMiss = r->smCount * std::min(blocks_per_sm, shadeMissOccupancy());
    } else {
        int be = 1, bs = 1, bsh = 1;
        stageOccupancy(be, bs, bsh);
        r->gridExtend = r->smCount * std::max(be, 1);
        r->gridShade = r->smCount * std::max(bs, 1);
        r->gridShadow = r->smCount * std::max(bsh, 1);
        r->gridExtendLane = r->smCount * extendLaneOccupancy();
        r->gridShadowLane = r->smCount * shadowLaneOccupancy();
    r->gridExtendLaneInst = r->smCount * extendLaneInstOccupancy();
    r->gridShadowLaneInst = r->smCount * shadowLaneInstOccupancy();
        r->gridShadeMiss = r->smCount * shadeMissOccupancy();
    }
    return PT_OK;
}

int pt_measure_l2(pt_renderer* r, uint64_t bytes, int reps, double* gb_per_s)
{
    if (r == nullptr || gb_per_s == nullptr || bytes < 16 || reps <= 0) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_measure_l2: bad arguments");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    const int st = measureL2ReadBandwidth(static_cast<size_t>(bytes), reps, r->smCount, r->stream, *gb_per_s);
    if (st != PT_OK) {
        return fail(r, st, "pt_measure_l2: the measurement failed");
    }
    return PT_OK;
}

int pt_set_bvh_options(pt_renderer* r, int treelet_passes)
{
    if (r == nullptr || treelet_passes < 0 || treelet_passes > 8) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_bvh_options: treelet_passes must be in 0..8");
    }
    r->bvhOptions.treeletPasses = treelet_passes;
    return PT_OK;
}

// SAH cost of a scene's binary BVH as built (Karras hierarchy after the
// treelet passes, one triangle per leaf): (C_node * sum of the internal nodes'
// areas + C_tri * sum of the leaves' areas) / root area, with the builder's
// costs.  Internal nodes are 0 .. n-2 (root 0), leaves n-1 .. 2n-2; the
// refit stores each node's surface area in nodeHi.w.
int pt_bvh_sah_cost(pt_renderer* r, int scene, double* cost)
{
    if (r == nullptr || cost == nullptr || scene < 0 || scene >= static_cast<int>(r->scenes.size())) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_bvh_sah_cost: bad arguments");
    }
    const SceneSlot& sl = r->scenes[static_cast<size_t>(scene)];
    const uint32_t n = sl.bvh.triCount;
    if (n == 0 || sl.bvh.nodes == nullptr) {
        return fail(r, PT_ERR_NO_SCENE, "pt_bvh_sah_cost: scene %d has no flat BVH", scene);
    }
    if (n == 1) {
        *cost = r->bvhOptions.costTriangle;
        return PT_OK;
    }
    const size_t nodes = 2ull * n - 1;
    const float4* nodeHi = static_cast<const float4*>(sl.bvh.scratch.ptr[10]);
    if (nodeHi == nullptr || sl.bvh.scratch.bytes[10] < nodes * sizeof(float4)) {
        return fail(r, PT_ERR_INTERNAL, "pt_bvh_sah_cost: the build's node bounds are not available");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    std::vector<float4> hi(nodes);
    PT_CHECK(r, cudaMemcpyAsync(hi.data(), nodeHi, nodes * sizeof(float4), cudaMemcpyDeviceToHost, r->stream));
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    double inner = 0.0, leaves = 0.0;
    for (size_t i = 0; i < nodes; ++i) {
        (i + 1 < n ? inner : leaves) += hi[i].w;
    }
    const double root = hi[0].w;
    if (!(root > 0.0)) {
        return fail(r, PT_ERR_INTERNAL, "pt_bvh_sah_cost: degenerate root box");
    }
    *cost = (r->bvhOptions.costNode * inner + r->bvhOptions.costTriangle * leaves) / root;
    return PT_OK;
}

int pt_autotune(pt_renderer* r, int waves, pt_tuning* out)
{
    if (r == nullptr || waves <= 0 || out == nullptr) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_autotune: bad arguments");
    }
    if (r->width <= 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_autotune before pt_configure");
    }
    *out = pt_tuning{};
    struct Knobs {
        int capacity, blocks, perLaunch;
    };
    Knobs cur{r->capacityWanted, r->blocksPerSmOverride, r->params.samples_per_launch};
    int trials = 0;
    auto trial = [&](const Knobs& k, double& ms) -> int {
        int st = pt_set_tuning(r, k.capacity, k.blocks);
        if (st != PT_OK) {
            return st;
        }
        r->params.samples_per_launch = k.perLaunch;
        st = resetAccum(r);
        if (st != PT_OK) {
            return st;
        }
        st = pt_render(r, waves);
        ms = r->stats.render_ms;
        ++trials;
        return st;
    };
    double ms = 0.0;
    int st = trial(cur, ms); // warm-up: allocations, graphs
    if (st == PT_OK) {
        st = trial(cur, ms);
    }
    if (st != PT_OK) {
        return st;
    }
    out->ms_default = ms;
    Knobs best = cur;
    double bestMs = ms;
    const int capacities[4] = {1 << 21, 1 << 22, 1 << 23, 1 << 24};
    const int blocks[4] = {0, 2, 3, 4};
    const int perLaunch[4] = {0, 4, 16, 64};
    for (int knob = 0; knob < 3; ++knob) {
        const Knobs base = best;
        for (int i = 0; i < 4; ++i) {
            Knobs k = base;
            if (knob == 0) {
                k.capacity = capacities[i];
            } else if (knob == 1) {
                k.blocks = blocks[i];
            } else {
                k.perLaunch = perLaunch[i];
            }
            if (k.capacity == base.capacity && k.blocks == base.blocks && k.perLaunch == base.perLaunch) {
                continue;
            }
            st = trial(k, ms);
            if (st != PT_OK) {
                return st;
            }
            // (a knob moves only for a gain above the probes' run-to-run noise:
            // a few waves are a short sample of the full render)
            if (ms < 0.99 * bestMs) {
                bestMs = ms;
                best = k;
            }
        }
    }
    st = pt_set_tuning(r, best.capacity, best.blocks);
    if (st != PT_OK) {
        return st;
    }
    r->params.samples_per_launch = best.perLaunch;
    out->path_capacity = best.capacity;
    out->blocks_per_sm = best.blocks;
    out->samples_per_launch = best.perLaunch;
    out->trials = trials;
    out->ms_best = bestMs;
    return resetAccum(r);
}

int pt_rng_tape(pt_renderer* r, int first_wave, int waves, int stride, float* out)
{
    if (r == nullptr || out == nullptr || waves <= 0 || stride <= 0 || first_wave < 0) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_rng_tape: bad arguments");
    }
    if (r->width <= 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_rng_tape before pt_configure");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    const size_t total = static_cast<size_t>(r->width) * r->height * waves * stride;
    float* d = nullptr;
    PT_CHECK(r, cudaMallocAsync(reinterpret_cast<void**>(&d), total * sizeof(float), r->stream));
    launchRngTape(r->width, r->height, first_wave, waves, stride, r->previewLevels, d, r->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(out, d, total * sizeof(float), cudaMemcpyDeviceToHost, r->stream);
    }
    cudaFreeAsync(d, r->stream);
    const cudaError_t e2 = cudaStreamSynchronize(r->stream);
    if (e == cudaSuccess) {
        e = e2;
    }
    if (e != cudaSuccess) {
        return cudaFail(r, e, "pt_rng_tape");
    }
    return PT_OK;
}

// ---------------------------------------------------------------------------
// Batched form: several scenes in one render (no reference counterpart)
// ---------------------------------------------------------------------------
int pt_batch_configure(pt_renderer* r, int scene_count, const int* widths, const int* heights)
{
    if (r == nullptr || scene_count < 1 || scene_count > 65535 || widths == nullptr || heights == nullptr) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_configure: bad arguments");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    // slots beyond the new count are freed; the others keep their device
    // arrays for the new scenes (freeing waits for the device, and a batch
    // rebuilt with the same scenes would allocate it all again)
    const size_t n = static_cast<size_t>(scene_count);
    for (size_t k = n; k < r->scenes.size(); ++k) {
        r->scenes[k].release();
    }
    r->scenes.resize(n);
    for (SceneSlot& sl : r->scenes) {
        sl.clearScene();
        sl.camera = defaultCamera();
    }
    return configureLayout(r, widths, heights);
}

int pt_batch_share_scene(pt_renderer* r, int scene, int source)
{
    if (r == nullptr || scene < 0 || source < 0 || scene == source || static_cast<size_t>(scene) >= r->scenes.size() ||
        static_cast<size_t>(source) >= r->scenes.size() || r->scenes[static_cast<size_t>(source)].shareFrom >= 0) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_share_scene: bad scene %d or source %d", scene, source);
    }
    SceneSlot& sl = r->scenes[static_cast<size_t>(scene)];
    for (const SceneSlot& x : r->scenes) {
        if (x.shareFrom == scene) {
            return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_share_scene: scene %d is itself shared", scene);
        }
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    const int w = sl.width, h = sl.height;
    const uint32_t base = sl.pixelBase;
    const pt_camera cam = sl.camera;
    sl.release();
    sl.width = w;
    sl.height = h;
    sl.pixelBase = base;
    sl.camera = cam;
    sl.shareFrom = source;
    return resetAccum(r);
}

int pt_batch_set_mesh(pt_renderer* r, int scene, const pt_mesh* mesh)
{
    if (r == nullptr || mesh == nullptr || scene < 0 || static_cast<size_t>(scene) >= r->scenes.size()) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_mesh: bad scene %d or null mesh", scene);
    }
    return setSceneMesh(r, r->scenes[static_cast<size_t>(scene)], mesh);
}

int pt_batch_set_camera(pt_renderer* r, int scene, const pt_camera* camera)
{
    if (r == nullptr || camera == nullptr || scene < 0 || static_cast<size_t>(scene) >= r->scenes.size()) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_camera: bad scene %d or null camera", scene);
    }
    r->scenes[static_cast<size_t>(scene)].camera = *camera;
    return resetAccum(r);
}

int pt_batch_readback(pt_renderer* r, int scene, float* rgba, uint32_t* counts, uint8_t* converged)
{
    if (r == nullptr || scene < 0 || static_cast<size_t>(scene) >= r->scenes.size()) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_readback: bad scene %d", scene);
    }
    if (r->pixelCount == 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_batch_readback before pt_batch_configure");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    const SceneSlot& sl = r->scenes[static_cast<size_t>(scene)];
    const size_t P = static_cast<size_t>(sl.width) * sl.height;
    const size_t o = sl.pixelBase;
    if (rgba) {
        PT_CHECK(r, cudaMemcpyAsync(rgba, r->acc.p + o, P * sizeof(float4), cudaMemcpyDeviceToHost, r->stream));
    }
    if (counts) {
        PT_CHECK(r, cudaMemcpyAsync(counts, r->counts.p + o, P * sizeof(uint32_t), cudaMemcpyDeviceToHost, r->stream));
    }
    if (converged) {
        PT_CHECK(r, cudaMemcpyAsync(converged, r->converged.p + o, P, cudaMemcpyDeviceToHost, r->stream));
    }
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    return PT_OK;
}

int pt_batch_set_tubes(pt_renderer* r, int scene, const pt_tubes* tubes, const pt_mesh* extra)
{
    if (r == nullptr || tubes == nullptr || extra == nullptr || scene < 0 ||
        static_cast<size_t>(scene) >= r->scenes.size()) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_tubes: bad scene %d or null argument", scene);
    }
    const uint32_t T = tubes->tube_count, S = tubes->sides, Lc = tubes->leaf_count;
    if (T > 0 && (S < 3 || tubes->ring_start == nullptr || tubes->points == nullptr || tubes->tangents == nullptr ||
                     tubes->radii == nullptr || tubes->materials == nullptr)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_tubes: missing tube arrays or sides < 3");
    }
    if (Lc > 0 && tubes->leaves == nullptr) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_tubes: missing leaf array");
    }
    const uint32_t rings = T > 0 ? tubes->ring_start[T] : 0u;
    if (T > 0) {
        if (tubes->ring_start[0] != 0u) {
            return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_tubes: ring_start[0] must be 0");
        }
        for (uint32_t t = 0; t < T; ++t) {
            if (tubes->ring_start[t + 1] <= tubes->ring_start[t]) {
                return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_tubes: tube %u has no ring", t);
            }
        }
    }
    const uint64_t gen = tubeTriangles(S, rings, Lc);
    const uint64_t total = gen + extra->triangle_count;
    if (total > 0xFFFFFFFFull / 2) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_tubes: %llu triangles are too many",
            static_cast<unsigned long long>(total));
    }
    const uint32_t n = static_cast<uint32_t>(total);
    const pt_mesh* m = extra;
    if (m->triangle_count > 0 && (m->positions == nullptr || m->normals == nullptr || m->uvs == nullptr ||
                                     m->material_ids == nullptr)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_batch_set_tubes: missing extra triangle arrays");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    cudaStream_t s = r->stream;
    SceneSlot& sl = r->scenes[static_cast<size_t>(scene)];
    PT_CHECK(r, cudaEventRecord(r->ev0, s));
    sl.hasScene = false;
    sl.shareFrom = -1;
    sl.releaseInstances();
    int st = uploadBank(r, sl, extra);
    if (st != PT_OK) {
        return st;
    }
    if (n > 0 && (!sl.positions.ensure(9ull * n) || !r->stage.ensure(15ull * n) || !r->stageIds.ensure(n))) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "mesh allocation failed for %u triangles", n);
    }
    if (gen > 0) {
        std::vector<double> cs;
        const double* csp = tubes->cos_sin;
        if (csp == nullptr && S > 0) {
            // the reference's angles (Loft.cpp:25): k * 6.283185307f / sides in single
            // precision, cosine and sine rounded to single precision; entry S = entry 0
            cs.resize(2ull * (S + 1));
            for (uint32_t k = 0; k <= S; ++k) {
                const uint32_t kk = k == S ? 0u : k;
                const float ang = (static_cast<float>(kk) * 6.283185307f) / static_cast<float>(S);
                cs[2 * k] = static_cast<double>(static_cast<float>(std::cos(static_cast<double>(ang))));
                cs[2 * k + 1] = static_cast<double>(static_cast<float>(std::sin(static_cast<double>(ang))));
            }
            csp = cs.data();
        }
        const size_t R = rings;
        if (!r->tRingStart.ensure(T + 1ull) || !r->tMaterials.ensure(std::max<uint32_t>(T, 1)) ||
            !r->tPoints.ensure(3 * R + 1) || !r->tTangents.ensure(3 * R + 1) || !r->tRadii.ensure(R + 1) ||
            !r->tCosSin.ensure(2ull * (S + 1)) || !r->tLeaves.ensure(10ull * Lc + 1) || !r->tFrames.ensure(9 * R + 1) ||
            (tubes->frames != nullptr && !r->tGivenFrames.ensure(6 * R + 1))) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "tube upload failed (%u rings, %u leaves)", rings, Lc);
        }
        if (T > 0) {
            PT_CHECK(r, cudaMemcpyAsync(r->tRingStart.p, tubes->ring_start, (T + 1ull) * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
            PT_CHECK(r, cudaMemcpyAsync(r->tMaterials.p, tubes->materials, T * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
            PT_CHECK(r, cudaMemcpyAsync(r->tPoints.p, tubes->points, 3 * R * sizeof(double), cudaMemcpyHostToDevice, s));
            PT_CHECK(r, cudaMemcpyAsync(r->tTangents.p, tubes->tangents, 3 * R * sizeof(double), cudaMemcpyHostToDevice, s));
            PT_CHECK(r, cudaMemcpyAsync(r->tRadii.p, tubes->radii, R * sizeof(double), cudaMemcpyHostToDevice, s));
            PT_CHECK(r, cudaMemcpyAsync(r->tCosSin.p, csp, 2ull * (S + 1) * sizeof(double), cudaMemcpyHostToDevice, s));
            if (tubes->frames != nullptr) {
                PT_CHECK(r, cudaMemcpyAsync(r->tGivenFrames.p, tubes->frames, 6 * R * sizeof(double),
                    cudaMemcpyHostToDevice, s));
            }
        }
        if (Lc > 0) {
            PT_CHECK(r, cudaMemcpyAsync(r->tLeaves.p, tubes->leaves, 10ull * Lc * sizeof(double), cudaMemcpyHostToDevice, s));
        }
        TubeSetDev d;
        d.tubeCount = T;
        d.sides = S;
        d.ringCount = rings;
        d.ringStart = r->tRingStart.p;
        d.points = r->tPoints.p;
        d.tangents = r->tTangents.p;
        d.radii = r->tRadii.p;
        d.materials = r->tMaterials.p;
        d.cosSin = r->tCosSin.p;
        d.frames = (tubes->frames != nullptr && T > 0) ? r->tGivenFrames.p : nullptr;
        d.leafCount = Lc;
        d.leaves = r->tLeaves.p;
        d.leafSize = tubes->leaf_size;
        d.leafMaterial = tubes->leaf_material;
        launchRingFrames(d, r->tFrames.p, s);
        launchLoft(d, r->tFrames.p, sl.positions.p, r->stage.p, r->stage.p + 9ull * n, r->stageIds.p, s);
        PT_CHECK(r, cudaGetLastError());
    }
    if (m->triangle_count > 0) {
        const size_t e = m->triangle_count;
        PT_CHECK(r, cudaMemcpyAsync(sl.positions.p + 9 * gen, m->positions, 9 * e * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stage.p + 9 * gen, m->normals, 9 * e * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stage.p + 9ull * n + 6 * gen, m->uvs, 6 * e * sizeof(float), cudaMemcpyHostToDevice, s));
        PT_CHECK(r, cudaMemcpyAsync(r->stageIds.p + gen, m->material_ids, e * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    }
    st = finishScene(r, sl, n);
    if (st != PT_OK) {
        return st;
    }
    PT_CHECK(r, cudaEventRecord(r->ev1, s));
    PT_CHECK(r, cudaEventSynchronize(r->ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r->ev0, r->ev1);
    r->stats.build_ms = ms;
    sl.hasScene = true;
    uint32_t nodes = 0;
    for (const SceneSlot& x : r->scenes) {
        nodes += x.hasScene ? sceneNodeCount(x) : 0u;
    }
    r->stats.bvh_nodes = static_cast<int32_t>(nodes);
    return resetAccum(r);
}

int pt_export_mesh(pt_renderer* r, int scene, uint32_t* triangle_count, float* positions, float* normals,
    float* uvs, uint32_t* material_ids)
{
    if (r == nullptr || scene < 0 || static_cast<size_t>(scene) >= r->scenes.size()) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_export_mesh: bad scene %d", scene);
    }
    const SceneSlot& sl = r->scenes[static_cast<size_t>(scene)];
    if (!sl.hasScene) {
        return fail(r, PT_ERR_NO_SCENE, "pt_export_mesh: scene %d has no mesh", scene);
    }
    if (sl.instanceCount > 0) {
        return fail(r, PT_ERR_UNSUPPORTED, "pt_export_mesh: scene %d is instanced", scene);
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    cudaStream_t s = r->stream;
    const uint32_t n = sl.triCount;
    if (triangle_count != nullptr) {
        *triangle_count = n;
    }
    if (n == 0) {
        return PT_OK;
    }
    if (positions != nullptr) {
        PT_CHECK(r, cudaMemcpyAsync(positions, sl.positions.p, 9ull * n * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    if (normals != nullptr || uvs != nullptr || material_ids != nullptr) {
        if (!r->stage.ensure(15ull * n) || !r->stageIds.ensure(n)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "export staging allocation failed");
        }
        launchUnpackShade(sl.shade.p, n, r->stage.p, r->stage.p + 9ull * n, r->stageIds.p, s);
        PT_CHECK(r, cudaGetLastError());
        if (normals != nullptr) {
            PT_CHECK(r, cudaMemcpyAsync(normals, r->stage.p, 9ull * n * sizeof(float), cudaMemcpyDeviceToHost, s));
        }
        if (uvs != nullptr) {
            PT_CHECK(r, cudaMemcpyAsync(uvs, r->stage.p + 9ull * n, 6ull * n * sizeof(float), cudaMemcpyDeviceToHost, s));
        }
        if (material_ids != nullptr) {
            PT_CHECK(r, cudaMemcpyAsync(material_ids, r->stageIds.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        }
    }
    PT_CHECK(r, cudaStreamSynchronize(s));
    return PT_OK;
}

float pt_exposure_multiplier(float f_stop, float shutter_seconds, float iso)
{
    const float f = f_stop < 0.1f ? 0.1f : f_stop;
    const float i = iso < 1.0f ? 1.0f : iso;
    return shutter_seconds * (i / 100.0f) / (f * f);
}

int pt_tonemap(pt_renderer* r, int scene, float exposure, uint8_t* rgba8)
{
    if (r == nullptr || rgba8 == nullptr || scene < 0 || static_cast<size_t>(scene) >= r->scenes.size()) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_tonemap: bad scene %d or null output", scene);
    }
    if (r->pixelCount == 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_tonemap before pt_configure");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    const SceneSlot& sl = r->scenes[static_cast<size_t>(scene)];
    const size_t P = static_cast<size_t>(sl.width) * sl.height;
    if (!r->displayBuf.ensure(4 * P)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "display buffer allocation failed");
    }
    if (scene == 0 && r->scenes.size() == 1 && r->previewLevels > 0 && r->wavesDone == 0 && r->previewDone >= 0) {
        // no full-resolution wave yet: the finest preview, upsampled (PathTracer.cpp:1546-1552)
        int w, h, ds;
        previewDims(r->width, r->height, r->previewLevels, r->previewDone, w, h, ds);
        launchTonemapPreview(r->previewBuf.p + previewOffset(r->width, r->height, r->previewLevels, r->previewDone),
            w, h, ds, r->width, r->height, r->params, exposure, r->displayBuf.p, r->stream);
    } else {
        launchTonemap(r->acc.p + sl.pixelBase, r->counts.p + sl.pixelBase, r->converged.p + sl.pixelBase,
            static_cast<int>(P), r->params, exposure, r->displayBuf.p, r->stream);
    }
    PT_CHECK(r, cudaGetLastError());
    PT_CHECK(r, cudaMemcpyAsync(rgba8, r->displayBuf.p, 4 * P, cudaMemcpyDeviceToHost, r->stream));
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    return PT_OK;
}

// ---------------------------------------------------------------------------
// Differentiation (no reference counterpart)
// ---------------------------------------------------------------------------
int pt_set_materials(pt_renderer* r, int scene, uint32_t material_count, const pt_material* materials)
{
    if (r == nullptr || (material_count > 0 && materials == nullptr) || scene < 0 ||
        static_cast<size_t>(scene) >= r->scenes.size()) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_materials: bad arguments");
    }
    SceneSlot& sl = r->scenes[static_cast<size_t>(scene)];
    if (!sl.hasScene) {
        return fail(r, PT_ERR_NO_SCENE, "pt_set_materials: scene %d has no mesh", scene);
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    // new material bank, texture bank kept (uploadBank re-reads textures only when given)
    pt_mesh bank{};
    bank.material_count = material_count;
    bank.materials = materials;
    const uint32_t texCount = sl.textureCount;
    int st = uploadBank(r, sl, &bank);
    sl.textureCount = texCount;
    if (st != PT_OK) {
        return st;
    }
    // the emissive list depends on the materials: rebuild it, with the material
    // ids taken from the shading records (instanced scenes have none)
    const uint32_t n = sl.instanceCount > 0 ? 0u : sl.triCount;
    if (n > 0) {
        if (!r->stage.ensure(15ull * n) || !r->stageIds.ensure(n)) {
            return fail(r, PT_ERR_OUT_OF_MEMORY, "staging allocation failed");
        }
        launchUnpackShade(sl.shade.p, n, r->stage.p, r->stage.p + 9ull * n, r->stageIds.p, r->stream);
        PT_CHECK(r, cudaGetLastError());
        st = buildEmissive(r, sl, n);
        if (st != PT_OK) {
            return st;
        }
    }
    return resetAccum(r);
}

int pt_record_samples(pt_renderer* r, int spp)
{
    if (r == nullptr || spp < 0) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_record_samples: bad arguments");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    if (spp == 0) {
        r->record.release();
        r->recordSpp = 0;
        r->recordValid = false;
        return PT_OK;
    }
    if (r->scenes.size() != 1 || r->pixelCount == 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_record_samples needs a configured single-scene renderer");
    }
    if (!r->record.ensure(static_cast<size_t>(spp) * r->pixelCount)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "pt_record_samples: %d x %zu samples do not fit", spp, r->pixelCount);
    }
    r->recordSpp = spp;
    return resetAccum(r);
}

int pt_backward(pt_renderer* r, const float* d_image, int channels, int spp, float* grad, uint32_t grad_materials,
    double* device_ms)
{
    if (r == nullptr || d_image == nullptr || grad == nullptr || spp <= 0 || (channels != 3 && channels != 4)) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_backward: bad arguments");
    }
    if (r->scenes.size() != 1 || r->pixelCount == 0) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_backward needs a configured single-scene renderer");
    }
    if (r->params.spectral_wavelengths != 0) {
        return fail(r, PT_ERR_UNSUPPORTED, "pt_backward: the adjoint differentiates the RGB integrator only");
    }
    if (r->params.emitter_mis != 0) {
        return fail(r, PT_ERR_UNSUPPORTED, "pt_backward: the adjoint replays the reference estimator (emitter_mis 0)");
    }
    if (r->scenes[0].instanceCount > 0 || r->sun.enabled) {
        return fail(r, PT_ERR_UNSUPPORTED, "pt_backward: instanced scenes and the distant light are not differentiated");
    }
    const SceneSlot& sl = r->scenes[0];
    if (!sl.hasScene) {
        return fail(r, PT_ERR_NO_SCENE, "pt_backward before pt_set_mesh");
    }
    if (sl.materialCount > static_cast<uint32_t>(kMaxGradMaterials)) {
        return fail(r, PT_ERR_UNSUPPORTED, "pt_backward: %u materials, at most %d have gradients", sl.materialCount,
            kMaxGradMaterials);
    }
    const uint32_t M = std::min<uint32_t>(sl.materialCount, grad_materials);
    PT_CHECK(r, cudaSetDevice(r->device));
    cudaStream_t s = r->stream;
    const size_t P = r->pixelCount;
    if (!r->adjImage.ensure(P * channels) || !r->adjGrad.ensure(static_cast<size_t>(kMaxGradMaterials) * kGradParams)) {
        return fail(r, PT_ERR_OUT_OF_MEMORY, "pt_backward: allocation failed");
    }
    PT_CHECK(r, cudaMemcpyAsync(r->adjImage.p, d_image, P * channels * sizeof(float), cudaMemcpyHostToDevice, s));
    PT_CHECK(r, cudaMemsetAsync(r->adjGrad.p, 0, sizeof(float) * kMaxGradMaterials * kGradParams, s));
    const LaunchCtx* c = uploadCtx(r);
    if (c == nullptr) {
        return fail(r, PT_ERR_CUDA, "launch context upload failed");
    }
    const int grid = r->smCount * adjointBlocksPerSm();
    const float4* rec = (r->recordValid && r->recordSpp == spp) ? r->record.p : nullptr;
    PT_CHECK(r, cudaEventRecord(r->ev0, s));
    launchAdjoint(c, r->adjImage.p, channels, spp, static_cast<int>(P), static_cast<int>(sl.materialCount),
        r->adjGrad.p, rec, grid, s);
    PT_CHECK(r, cudaGetLastError());
    PT_CHECK(r, cudaEventRecord(r->ev1, s));
    std::vector<float> g(static_cast<size_t>(kMaxGradMaterials) * kGradParams);
    PT_CHECK(r, cudaMemcpyAsync(g.data(), r->adjGrad.p, g.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
    PT_CHECK(r, cudaStreamSynchronize(s));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r->ev0, r->ev1);
    if (device_ms != nullptr) {
        *device_ms = ms;
    }
    std::memset(grad, 0, sizeof(float) * grad_materials * kGradParams);
    std::memcpy(grad, g.data(), sizeof(float) * M * kGradParams);
    r->launches += 1;
    return PT_OK;
}

// ---------------------------------------------------------------------------
// Preview passes and region render (PathTracer.h:89-92, 134-140)
// ---------------------------------------------------------------------------
int pt_set_instances(pt_renderer* r, int scene, uint32_t object_count, const pt_mesh* objects,
    uint32_t instance_count, const pt_instance* instances)
{
    if (r == nullptr || scene < 0 || static_cast<size_t>(scene) >= r->scenes.size()) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_set_instances: bad scene %d", scene);
    }
    return setSceneInstances(r, r->scenes[static_cast<size_t>(scene)], object_count, objects, instance_count,
        instances);
}

int pt_set_distant_light(pt_renderer* r, const pt_distant_light* light)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    const int st = setDistantLight(r, light);
    if (st != PT_OK) {
        r->sun = DevSun{};
        return st;
    }
    return resetAccum(r);
}

// Spectral mode helpers (host only; no device work).
int pt_spectral_response(float* rgb, float* cie, float* xyz_to_rgb)
{
    if (rgb != nullptr) {
        std::vector<float> t(4 * spectral::kRespCount);
        spectral::buildResponseTable(t.data());
        for (int i = 0; i < spectral::kRespCount; ++i) {
            rgb[3 * i] = t[4 * i];
            rgb[3 * i + 1] = t[4 * i + 1];
            rgb[3 * i + 2] = t[4 * i + 2];
        }
    }
    spectral::spectralSourceTables(cie, xyz_to_rgb);
    return PT_OK;
}

int pt_spectral_uplift(uint32_t count, const float* rgb, float* coef)
{
    if (count > 0 && (rgb == nullptr || coef == nullptr)) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    std::vector<float> t(4 * spectral::kRespCount);
    spectral::buildResponseTable(t.data());
    for (uint32_t i = 0; i < count; ++i) {
        const spectral::Coef c = spectral::upliftSolve(t.data(), rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2], true);
        coef[4 * i] = c.c0;
        coef[4 * i + 1] = c.c1;
        coef[4 * i + 2] = c.c2;
        coef[4 * i + 3] = c.scale;
    }
    return PT_OK;
}

int pt_set_preview_levels(pt_renderer* r, int levels)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    // clampPreviewStepsPerLevel (PathTracer.cpp:181-190)
    r->previewLevels = levels < 0 ? 0 : (levels > 128 ? 128 : levels);
    PT_CHECK(r, cudaSetDevice(r->device));
    return resetAccum(r);
}

int pt_render_previews(pt_renderer* r)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    if (r->width <= 0 || r->scenes.size() != 1 || !r->scenes[0].hasScene) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_render_previews needs a configured single scene with a mesh");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    if (r->previewLevels > 0 && r->wavesDone == 0 && r->previewDone < r->previewLevels - 1) {
        const int st = renderPreviews(r);
        if (st != PT_OK) {
            return st;
        }
    }
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    return PT_OK;
}

int pt_preview_readback(pt_renderer* r, int level, float* rgba, int* width, int* height)
{
    if (r == nullptr || level < 0 || level >= r->previewLevels) {
        return fail(r, PT_ERR_INVALID_ARGUMENT, "pt_preview_readback: bad level %d", level);
    }
    if (level > r->previewDone) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_preview_readback: level %d not rendered since the last reset", level);
    }
    int w, h, ds;
    previewDims(r->width, r->height, r->previewLevels, level, w, h, ds);
    if (width != nullptr) {
        *width = w;
    }
    if (height != nullptr) {
        *height = h;
    }
    if (rgba != nullptr) {
        PT_CHECK(r, cudaSetDevice(r->device));
        PT_CHECK(r, cudaMemcpyAsync(rgba, r->previewBuf.p + previewOffset(r->width, r->height, r->previewLevels, level),
            static_cast<size_t>(w) * h * sizeof(float4), cudaMemcpyDeviceToHost, r->stream));
        PT_CHECK(r, cudaStreamSynchronize(r->stream));
    }
    return PT_OK;
}

int pt_set_region(pt_renderer* r, int enabled, int min_x, int min_y, int max_x, int max_y)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    if (enabled && (r->scenes.size() != 1 || r->width <= 0)) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_set_region needs a configured single-scene renderer");
    }
    // PathTracer::setRenderRegion (PathTracer.cpp:1447-1463): ordered and clamped to the image
    const int mx = std::max(0, r->width - 1), my = std::max(0, r->height - 1);
    r->regionMinX = std::max(0, std::min(min_x, max_x));
    r->regionMaxX = std::min(mx, std::max(min_x, max_x));
    r->regionMinY = std::max(0, std::min(min_y, max_y));
    r->regionMaxY = std::min(my, std::max(min_y, max_y));
    r->regionEnabled = enabled != 0;
    return pt_reset_region(r);
}

int pt_reset_region(pt_renderer* r)
{
    if (r == nullptr) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    if (!r->regionEnabled) {
        return resetAccum(r);
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    // PathTracer::resetRegionAccumulation: only the region is cleared, the rest
    // of the image keeps its samples
    r->activeSel = 0;
    const LaunchCtx* dc = uploadCtx(r);
    if (dc == nullptr) {
        return fail(r, PT_ERR_CUDA, "launch context upload failed");
    }
    launchRegion(dc, r->width, r->regionMinX, r->regionMinY, r->regionMaxX, r->regionMaxY, true, r->stream);
    PT_CHECK(r, cudaGetLastError());
    r->hostActive = (r->regionMaxX - r->regionMinX + 1) * (r->regionMaxY - r->regionMinY + 1);
    r->lastStopRate = 1.0;
    r->wavesDone = 0;
    r->samplesDone = 0;
    r->recordValid = false;
    r->previewDone = -1;
    return PT_OK;
}

int pt_environment_tables(pt_renderer* r, float* marginal, float* row)
{
    if (r == nullptr || !r->envValid) {
        return fail(r, PT_ERR_NOT_CONFIGURED, "pt_environment_tables: no environment map");
    }
    PT_CHECK(r, cudaSetDevice(r->device));
    const size_t W = static_cast<size_t>(r->envW), H = static_cast<size_t>(r->envH);
    if (marginal != nullptr) {
        PT_CHECK(r, cudaMemcpyAsync(marginal, r->envMarginal.p, (H + 1) * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
    }
    if (row != nullptr) {
        PT_CHECK(r, cudaMemcpyAsync(row, r->envRow.p, H * (W + 1) * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
    }
    PT_CHECK(r, cudaStreamSynchronize(r->stream));
    return PT_OK;
}

} // extern "C"
