// Parity harness around the REFERENCE's own hot-path code, compiled for the
// host from the sources where they lie (see oracle/Makefile).  Built into
// oracle/_ref/libptref.so.  Test infrastructure only: the product never loads it.
//
// What runs here is the reference's code, unmodified:
//   - meshAccelTraceRay / meshAccelRayTriangle / meshAccelRayAabb
//       (PathTracerLib/src/MeshAccel/MeshAccelIntersectCore.h:12-221)
//   - MeshAccelScene::build -> meshAccelBuildBvh + emissive CDF
//       (PathTracerLib/src/MeshAccel/MeshAccelScene.cpp:141-194,
//        PathTracerLib/src/MeshAccel/MeshBvhBuilder.cpp:52-142)
//   - tracePathRand and everything below it: Principled BSDF, NEE, MIS, RR
//       (PathTracerLib/src/PathIntegratorRandCore.h:206-363)
//   - cameraPrimaryRaySampled (PathTracerLib/src/CameraDevice.cuh:88-139)
//   - isAdaptivePixelConverged (PathTracerLib/src/PathTracerAdaptiveSampling.h:16-40)
//   - buildImportanceTables for environment maps is restated below because
//     EnvironmentMap.cpp needs stb_image/Qt (EnvironmentMap.cpp:76-128).
//
// What this file adds (harness, not reference code):
//   - a tape-replaying curand stand-in (ref_shim/curand_kernel.h),
//   - the per-pixel loop of sampleAdaptiveKernel / tracePixelRadiance, which
//     live in a .cu translation unit with __global__ code and cannot be
//     included on the host (restated from PathTracer.cu:49-105, 186-273),
//   - extern "C" entry points with plain pointers for ctypes.

#include "PathIntegratorRandCore.h"
#include "CameraDevice.cuh"
#include "MeshAccel/MeshAccelScene.h"
#include "PathTracerAdaptiveSampling.h"

#include <omp.h>

#include <cstdint>
#include <cstring>
#include <vector>

// ---------------------------------------------------------------------------
// Tape-replaying curand stand-in.
// ---------------------------------------------------------------------------
namespace {

struct TapeCursor {
    const float* row = nullptr;
    int length = 0;
    unsigned int expectSeed = 0;
    bool checkSeed = false;
    // PCG32 fallback when no tape row is registered (timing / statistics runs).
    bool usePcg = false;
    uint64_t pcgState = 0;
    uint64_t pcgInc = 0;
};

thread_local TapeCursor gCursor;
thread_local int gTapeErrors = 0;
thread_local int gConsumed = 0;

// PCG32 (O'Neill 2014, "PCG: A Family of Simple Fast Space-Efficient
// Statistically Good Algorithms for Random Number Generation"), XSH-RR variant.
inline uint32_t pcg32Next(uint64_t& state, uint64_t inc)
{
    const uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    const uint32_t xorshifted = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = static_cast<uint32_t>(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
}

inline void pcg32Seed(uint64_t& state, uint64_t& inc, uint64_t seed, uint64_t stream)
{
    state = 0u;
    inc = (stream << 1u) | 1u;
    pcg32Next(state, inc);
    state += seed;
    pcg32Next(state, inc);
}

} // namespace

void curand_init(unsigned long long seed, unsigned long long, unsigned long long, curandState* state)
{
    state->row = gCursor.row;
    state->cursor = 0;
    state->length = gCursor.length;
    state->seed = static_cast<unsigned int>(seed);
    gConsumed = 0;
    if (gCursor.checkSeed && static_cast<unsigned int>(seed) != gCursor.expectSeed) {
        ++gTapeErrors;
    }
    if (gCursor.usePcg) {
        pcg32Seed(gCursor.pcgState, gCursor.pcgInc, seed, 0x9e3779b97f4a7c15ULL);
    }
}

float curand_uniform(curandState* state)
{
    ++gConsumed;
    if (gCursor.usePcg) {
        // (0, 1] like curand_uniform's documented range.
        const uint32_t bits = pcg32Next(gCursor.pcgState, gCursor.pcgInc);
        return (static_cast<float>(bits >> 8) + 1.0f) * (1.0f / 16777216.0f);
    }
    if (state->row == nullptr || state->cursor >= state->length) {
        ++gTapeErrors;
        return 0.5f;
    }
    return state->row[state->cursor++];
}

// Spectral model hook required by SpectralCore.h on the host; the integrator
// never evaluates it (it runs at a fixed 550 nm with wavelength-independent IOR).
Rgb2SpecGpu spectralHostModel()
{
    return Rgb2SpecGpu{};
}

// ---------------------------------------------------------------------------
// Scene handle.
// ---------------------------------------------------------------------------
namespace {

struct RefScene {
    MeshAccelScene accel;
    MeshAccelSceneGpu view{};
};

struct RefEnv {
    std::vector<float> pixels;
    std::vector<float> marginal;
    std::vector<float> row;
    EnvironmentMapGpu view{};
};

// PathTracer.cu:49-67 (clampSampleFirefly), harness restatement.
Vec3 refClampFirefly(Vec3 radiance)
{
    if (!std::isfinite(radiance.x) || !std::isfinite(radiance.y) || !std::isfinite(radiance.z)) {
        return vecMake3(0.0f, 0.0f, 0.0f);
    }
    radiance = vecMake3(vecMax2(0.0f, radiance.x), vecMax2(0.0f, radiance.y), vecMax2(0.0f, radiance.z));
    const float lum = radiance.x * 0.2126f + radiance.y * 0.7152f + radiance.z * 0.0722f;
    if (lum <= 100.0f) {
        return radiance;
    }
    const float s = 100.0f / lum;
    return vecMake3(radiance.x * s, radiance.y * s, radiance.z * s);
}

// PathTracer.cu:69-105 (tracePixelRadiance), harness restatement.
Vec3 refTracePixel(
    int idx, int x, int y, int width, int height, bool jitter, int sampleIndex,
    const CameraGpu* camera, const MeshAccelSceneGpu* scene, const EnvironmentMapGpu* env,
    const RenderParamsGpu* params, unsigned int globalSeed)
{
    curandState rng{};
    randInitState(&rng, idx, sampleIndex, globalSeed);
    const float jitterU = jitter ? rand01(&rng) : 0.5f;
    const float jitterV = jitter ? rand01(&rng) : 0.5f;
    const float u = (static_cast<float>(x) + jitterU) / static_cast<float>(width);
    const float v = (static_cast<float>(y) + jitterV) / static_cast<float>(height);
    float3 ro{};
    float3 rd{};
    const float lensU1 = rand01(&rng);
    const float lensU2 = rand01(&rng);
    cameraPrimaryRaySampled(camera, u, v, lensU1, lensU2, ro, rd);
    return refClampFirefly(tracePathRand(
        vecMake3(ro.x, ro.y, ro.z), vecMake3(rd.x, rd.y, rd.z), scene, params, env, &rng));
}

} // namespace

extern "C" {

// The reference's spectral helpers (Spectral/SpectralCore.h:42-139,
// Spectral/Rgb2Spec.h:58-66; not called by its RGB integrator): per
// wavelength x-bar, y-bar, z-bar and D65 (4 floats).
void ref_spectral_cie(const float* lambdas, int n, float* out)
{
    for (int i = 0; i < n; ++i) {
        out[4 * i] = SpectralDetail::cieXAtWavelength(lambdas[i]);
        out[4 * i + 1] = SpectralDetail::cieYAtWavelength(lambdas[i]);
        out[4 * i + 2] = SpectralDetail::cieZAtWavelength(lambdas[i]);
        out[4 * i + 3] = SpectralDetail::d65IlluminantAtWavelength(lambdas[i]);
    }
}

// spectralLinearSrgbFromXyz of n XYZ triples.
void ref_spectral_xyz_to_srgb(const float* xyz, int n, float* rgb)
{
    for (int i = 0; i < n; ++i) {
        SpectralDetail::spectralLinearSrgbFromXyz(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], rgb[3 * i], rgb[3 * i + 1],
            rgb[3 * i + 2]);
    }
}

// rgb2specEvalCoefficients of n coefficient triples at n wavelengths.
void ref_spectral_sigmoid(const float* coef, const float* lambdas, int n, float* out)
{
    for (int i = 0; i < n; ++i) {
        out[i] = rgb2specEvalCoefficients(coef + 3 * i, lambdas[i]);
    }
}

int ref_sizeof_material() { return static_cast<int>(sizeof(MaterialGpu)); }
int ref_sizeof_texture() { return static_cast<int>(sizeof(TextureDescGpu)); }
int ref_sizeof_camera() { return static_cast<int>(sizeof(CameraGpu)); }
int ref_sizeof_params() { return static_cast<int>(sizeof(RenderParamsGpu)); }
int ref_sizeof_triangle() { return static_cast<int>(sizeof(TriangleGpu)); }
int ref_sizeof_bvh_node() { return static_cast<int>(sizeof(MeshBvhNode)); }

// Builds the reference acceleration scene from flat SoA arrays.
//   positions: 9 floats / triangle (v0, v1, v2)
//   normals:   9 floats / triangle (n0, n1, n2)
//   uvs:       6 floats / triangle (uv0, uv1, uv2)
//   materials: MaterialGpu records (96 B each), textures: TextureDescGpu (64 B)
void* ref_scene_create(
    int triCount, const float* positions, const float* normals, const float* uvs,
    const uint32_t* materialIds, int materialCount, const void* materials,
    int textureCount, const void* textures)
{
    HostMesh mesh;
    mesh.triangles.resize(static_cast<size_t>(triCount));
    for (int i = 0; i < triCount; ++i) {
        HostTriangle& t = mesh.triangles[static_cast<size_t>(i)];
        const float* p = positions + 9 * i;
        const float* n = normals + 9 * i;
        const float* q = uvs + 6 * i;
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
    RefScene* scene = new RefScene();
    if (!scene->accel.build(mesh)) {
        delete scene;
        return nullptr;
    }
    scene->view = *scene->accel.hostScene();
    return scene;
}

void ref_scene_destroy(void* handle)
{
    delete static_cast<RefScene*>(handle);
}

int ref_scene_bvh_node_count(void* handle)
{
    return static_cast<int>(static_cast<RefScene*>(handle)->view.bvhNodeCount);
}

// Emissive list + CDF as the reference builds them (MeshAccelScene.cpp:62-95).
int ref_scene_emissive(void* handle, uint32_t* outIndices, float* outCdf)
{
    const RefScene* s = static_cast<RefScene*>(handle);
    const auto& idx = s->accel.emissiveTriangleIndicesHost();
    const auto& cdf = s->accel.emissiveTriangleCdfHost();
    if (outIndices != nullptr) {
        std::memcpy(outIndices, idx.data(), idx.size() * sizeof(uint32_t));
    }
    if (outCdf != nullptr) {
        std::memcpy(outCdf, cdf.data(), cdf.size() * sizeof(float));
    }
    return static_cast<int>(idx.size());
}

// Closest-hit queries through the reference traversal.
void ref_trace_rays(
    void* handle, int n, const float* origins, const float* dirs, const float* tmin, const float* tmax,
    uint8_t* outHit, float* outT, uint32_t* outTri, float* outNormal, float* outUv)
{
    const MeshAccelSceneGpu* scene = &static_cast<RefScene*>(handle)->view;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const MeshHit h = meshAccelTraceRay(
            vecMake3(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]),
            vecMake3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]), scene, tmin[i], tmax[i]);
        outHit[i] = h.hit ? 1 : 0;
        outT[i] = h.t;
        outTri[i] = h.triangleIndex;
        outNormal[3 * i] = h.normal.x;
        outNormal[3 * i + 1] = h.normal.y;
        outNormal[3 * i + 2] = h.normal.z;
        outUv[2 * i] = h.uv.x;
        outUv[2 * i + 1] = h.uv.y;
    }
}

// Environment map (lat-long RGB float) with importance tables, restated from
// EnvironmentMap.cpp:76-128 because that file cannot be built without stb/Qt.
void* ref_env_create(int width, int height, const float* rgb)
{
    RefEnv* e = new RefEnv();
    e->pixels.assign(rgb, rgb + static_cast<size_t>(width) * height * 3);
    e->marginal.assign(static_cast<size_t>(height) + 1, 0.0f);
    e->row.assign(static_cast<size_t>(height) * (width + 1), 0.0f);
    std::vector<float> rowWeights(static_cast<size_t>(height), 0.0f);
    for (int y = 0; y < height; ++y) {
        const float v = (static_cast<float>(y) + 0.5f) / static_cast<float>(height);
        const float sinTheta = std::sin(v * 3.14159265f);
        float rowSum = 0.0f;
        const size_t off = static_cast<size_t>(y) * (width + 1);
        for (int x = 0; x < width; ++x) {
            const size_t i = (static_cast<size_t>(y) * width + x) * 3;
            const float lum = std::max(e->pixels[i], std::max(e->pixels[i + 1], e->pixels[i + 2]));
            rowSum += std::max(lum, 1.0e-6f) * sinTheta;
            e->row[off + x + 1] = rowSum;
        }
        if (rowSum > 0.0f) {
            for (int x = 0; x < width; ++x) {
                e->row[off + x + 1] /= rowSum;
            }
        }
        rowWeights[static_cast<size_t>(y)] = rowSum;
    }
    float total = 0.0f;
    for (int y = 0; y < height; ++y) {
        total += rowWeights[static_cast<size_t>(y)];
        e->marginal[static_cast<size_t>(y) + 1] = total;
    }
    if (total > 0.0f) {
        for (int y = 0; y < height; ++y) {
            e->marginal[static_cast<size_t>(y) + 1] /= total;
        }
    }
    e->view.pixels = e->pixels.data();
    e->view.marginalCdf = e->marginal.data();
    e->view.rowCdf = e->row.data();
    e->view.width = width;
    e->view.height = height;
    e->view.valid = 1;
    return e;
}

void ref_env_destroy(void* handle)
{
    delete static_cast<RefEnv*>(handle);
}

void ref_env_tables(void* handle, float* marginal, float* row)
{
    const RefEnv* e = static_cast<RefEnv*>(handle);
    std::memcpy(marginal, e->marginal.data(), e->marginal.size() * sizeof(float));
    std::memcpy(row, e->row.data(), e->row.size() * sizeof(float));
}

// Runs `waves` full-resolution adaptive waves the way PathTracer::renderLoop
// drives sampleAdaptiveKernel with no preview levels (PathTracer.cpp:2379-2421):
// wave w uses globalSeed = seedBase + w and, per active pixel,
// sampleIndex = counts[idx].  Pixels stop at maxSamplesPerPixel or when the
// relative-std-dev test passes on a multiple of 4 samples (PathTracer.cu:186-273).
//
// tape: if non-null, uniforms for (wave w, pixel p) start at
//       tape[((size_t)w * pixelCount + p) * tapeStride]; otherwise PCG32 streams
//       keyed by the reference seed are used.
// pixelList/pixelListCount: optional subset of pixels (bounded CPU samples);
//       null means every pixel.
// State buffers are in/out so that a caller can continue a render.
// Returns the number of tape underruns / seed mismatches (0 = clean).
int ref_render(
    void* sceneHandle, void* envHandle, const void* cameraBytes, const void* paramsBytes,
    int width, int height, int waves, unsigned int seedBase,
    const float* tape, int tapeStride,
    const int* pixelList, int pixelListCount,
    float* acc, uint32_t* counts, float* lumMean, float* m2, uint8_t* converged,
    int threads)
{
    const MeshAccelSceneGpu* scene = sceneHandle ? &static_cast<RefScene*>(sceneHandle)->view : nullptr;
    const EnvironmentMapGpu* env = envHandle ? &static_cast<RefEnv*>(envHandle)->view : nullptr;
    CameraGpu camera{};
    std::memcpy(&camera, cameraBytes, sizeof(CameraGpu));
    RenderParamsGpu params{};
    std::memcpy(&params, paramsBytes, sizeof(RenderParamsGpu));

    const int pixelCount = width * height;
    const int listCount = pixelList ? pixelListCount : pixelCount;
    int errors = 0;
    if (threads > 0) {
        omp_set_num_threads(threads);
    }

#pragma omp parallel reduction(+ : errors)
    {
        gTapeErrors = 0;
#pragma omp for schedule(dynamic, 64)
        for (int li = 0; li < listCount; ++li) {
            const int idx = pixelList ? pixelList[li] : li;
            const int x = idx % width;
            const int y = idx / width;
            for (int w = 0; w < waves; ++w) {
                if (converged[idx] != 0) {
                    break;
                }
                const unsigned int globalSeed = seedBase + static_cast<unsigned int>(w);
                const int sampleIndex = static_cast<int>(counts[idx]);
                if (tape != nullptr) {
                    gCursor.row = tape + (static_cast<size_t>(w) * pixelCount + idx) * static_cast<size_t>(tapeStride);
                    gCursor.length = tapeStride;
                    gCursor.usePcg = false;
                } else {
                    gCursor.row = nullptr;
                    gCursor.length = 0;
                    gCursor.usePcg = true;
                }
                const Vec3 s = refTracePixel(
                    idx, x, y, width, height, true, sampleIndex, &camera, scene, env, &params, globalSeed);
                const float sampleLum = s.x * 0.2126f + s.y * 0.7152f + s.z * 0.0722f;
                const uint32_t n = counts[idx];
                const float prevMean = lumMean[idx];
                const float delta = sampleLum - prevMean;
                const float newMean = prevMean + delta / static_cast<float>(n + 1);
                m2[idx] = m2[idx] + delta * (sampleLum - newMean);
                lumMean[idx] = newMean;
                float* a = acc + 4 * static_cast<size_t>(idx);
                const float invN = 1.0f / static_cast<float>(n + 1);
                a[0] = (a[0] * static_cast<float>(n) + s.x) * invN;
                a[1] = (a[1] * static_cast<float>(n) + s.y) * invN;
                a[2] = (a[2] * static_cast<float>(n) + s.z) * invN;
                a[3] = 1.0f;
                const uint32_t newCount = n + 1;
                counts[idx] = newCount;
                if (params.maxSamplesPerPixel > 0 && newCount >= static_cast<uint32_t>(params.maxSamplesPerPixel)) {
                    converged[idx] = 1;
                    continue;
                }
                if ((newCount % static_cast<uint32_t>(kAdaptiveConvergenceCheckInterval)) != 0) {
                    continue;
                }
                if (isAdaptivePixelConverged(newCount, newMean, m2[idx], params.minSamples,
                        params.relativeErrorThreshold)) {
                    converged[idx] = 1;
                }
            }
        }
        errors += gTapeErrors;
    }
    return errors;
}

// One path sample for one (pixel, sample) with an explicit tape row; writes the
// clamped radiance and returns the number of uniforms consumed (draw-order
// checks), or -1 if the row ran out.
int ref_trace_pixel(
    void* sceneHandle, void* envHandle, const void* cameraBytes, const void* paramsBytes,
    int width, int height, int idx, int sampleIndex, unsigned int globalSeed,
    const float* tapeRow, int tapeLength, float* outRgb)
{
    const MeshAccelSceneGpu* scene = sceneHandle ? &static_cast<RefScene*>(sceneHandle)->view : nullptr;
    const EnvironmentMapGpu* env = envHandle ? &static_cast<RefEnv*>(envHandle)->view : nullptr;
    CameraGpu camera{};
    std::memcpy(&camera, cameraBytes, sizeof(CameraGpu));
    RenderParamsGpu params{};
    std::memcpy(&params, paramsBytes, sizeof(RenderParamsGpu));
    gCursor.row = tapeRow;
    gCursor.length = tapeLength;
    gCursor.usePcg = false;
    gTapeErrors = 0;
    const Vec3 s = refTracePixel(idx, idx % width, idx / width, width, height, true, sampleIndex,
        &camera, scene, env, &params, globalSeed);
    outRgb[0] = s.x;
    outRgb[1] = s.y;
    outRgb[2] = s.z;
    return gTapeErrors != 0 ? -1 : gConsumed;
}

// Principled BSDF entry points for known-answer and property checks
// (Brdf/BrdfDispatch.h:11-76).  ctxBytes layout: normal[3], wo[3], etaMedium,
// wavelengthNm, debugFlags(int) followed by a MaterialGpu record.
void ref_brdf_eval(const float* normal, const float* wo, const void* material, float etaMedium,
    int debugFlags, const float* wi, float* outRgb)
{
    BrdfContext ctx{};
    ctx.normal = vecMake3(normal[0], normal[1], normal[2]);
    ctx.wo = vecMake3(wo[0], wo[1], wo[2]);
    std::memcpy(&ctx.material, material, sizeof(MaterialGpu));
    ctx.etaMedium = etaMedium;
    ctx.debugFlags = debugFlags;
    const Vec3 f = brdfEval(ctx, vecMake3(wi[0], wi[1], wi[2]));
    outRgb[0] = f.x;
    outRgb[1] = f.y;
    outRgb[2] = f.z;
}

float ref_brdf_pdf(const float* normal, const float* wo, const void* material, float etaMedium,
    int debugFlags, const float* wi)
{
    BrdfContext ctx{};
    ctx.normal = vecMake3(normal[0], normal[1], normal[2]);
    ctx.wo = vecMake3(wo[0], wo[1], wo[2]);
    std::memcpy(&ctx.material, material, sizeof(MaterialGpu));
    ctx.etaMedium = etaMedium;
    ctx.debugFlags = debugFlags;
    return brdfPdf(ctx, vecMake3(wi[0], wi[1], wi[2]));
}

// out: dir[3], pdf, nextMediumEta, exitOffset[3]; flags: valid | transmitted<<1 |
// subsurface<<2; returns subsurfaceInternalSteps.
int ref_brdf_sample(const float* normal, const float* wo, const void* material, float etaMedium,
    int debugFlags, float u1, float u2, float* outDir, float* outPdf, float* outNextEta,
    float* outExitOffset, int* outFlags)
{
    BrdfContext ctx{};
    ctx.normal = vecMake3(normal[0], normal[1], normal[2]);
    ctx.wo = vecMake3(wo[0], wo[1], wo[2]);
    std::memcpy(&ctx.material, material, sizeof(MaterialGpu));
    ctx.etaMedium = etaMedium;
    ctx.debugFlags = debugFlags;
    const BrdfSampleResult r = brdfSample(ctx, u1, u2);
    outDir[0] = r.direction.x;
    outDir[1] = r.direction.y;
    outDir[2] = r.direction.z;
    *outPdf = r.pdf;
    *outNextEta = r.nextMediumEta;
    outExitOffset[0] = r.subsurfaceExitOffset.x;
    outExitOffset[1] = r.subsurfaceExitOffset.y;
    outExitOffset[2] = r.subsurfaceExitOffset.z;
    *outFlags = (r.valid ? 1 : 0) | (r.transmitted ? 2 : 0) | (r.subsurfaceScatter ? 4 : 0);
    return r.subsurfaceInternalSteps;
}

// Throughput update after a BSDF sample (BrdfDispatch.h:42-76).
void ref_brdf_apply_throughput(const float* throughput, const float* normal, const float* wo,
    const void* material, float etaMedium, float u1, float u2, float* outThroughput)
{
    BrdfContext ctx{};
    ctx.normal = vecMake3(normal[0], normal[1], normal[2]);
    ctx.wo = vecMake3(wo[0], wo[1], wo[2]);
    std::memcpy(&ctx.material, material, sizeof(MaterialGpu));
    ctx.etaMedium = etaMedium;
    const BrdfSampleResult r = brdfSample(ctx, u1, u2);
    const Vec3 f = brdfEval(ctx, r.direction);
    const Vec3 t = brdfApplyThroughput(vecMake3(throughput[0], throughput[1], throughput[2]), ctx, r, f);
    outThroughput[0] = t.x;
    outThroughput[1] = t.y;
    outThroughput[2] = t.z;
}

// Camera primary ray (CameraDevice.cuh:88-139).
void ref_camera_ray(const void* cameraBytes, float u, float v, float lensU1, float lensU2,
    float* outOrigin, float* outDir)
{
    CameraGpu camera{};
    std::memcpy(&camera, cameraBytes, sizeof(CameraGpu));
    float3 ro{};
    float3 rd{};
    cameraPrimaryRaySampled(&camera, u, v, lensU1, lensU2, ro, rd);
    outOrigin[0] = ro.x;
    outOrigin[1] = ro.y;
    outOrigin[2] = ro.z;
    outDir[0] = rd.x;
    outDir[1] = rd.y;
    outDir[2] = rd.z;
}

// Environment / background light sampling (LightSamplingCore.h:94-185).
void ref_env_sample(void* envHandle, const void* paramsBytes, float u1, float u2, float* outDir, float* outPdf)
{
    const EnvironmentMapGpu* env = envHandle ? &static_cast<RefEnv*>(envHandle)->view : nullptr;
    RenderParamsGpu params{};
    std::memcpy(&params, paramsBytes, sizeof(RenderParamsGpu));
    float pdf = 0.0f;
    const Vec3 d = lightSampleEnvironmentOrBackground(env, &params, u1, u2, pdf);
    outDir[0] = d.x;
    outDir[1] = d.y;
    outDir[2] = d.z;
    *outPdf = pdf;
}

float ref_env_pdf(void* envHandle, const void* paramsBytes, const float* dir)
{
    const EnvironmentMapGpu* env = envHandle ? &static_cast<RefEnv*>(envHandle)->view : nullptr;
    RenderParamsGpu params{};
    std::memcpy(&params, paramsBytes, sizeof(RenderParamsGpu));
    return lightPdfEnvironmentOrBackground(env, &params, vecMake3(dir[0], dir[1], dir[2]));
}

void ref_env_eval(void* envHandle, const void* paramsBytes, const float* dir, float* outRgb)
{
    const EnvironmentMapGpu* env = envHandle ? &static_cast<RefEnv*>(envHandle)->view : nullptr;
    RenderParamsGpu params{};
    std::memcpy(&params, paramsBytes, sizeof(RenderParamsGpu));
    const Vec3 c = lightEvalEnvironmentOrBackground(env, &params, vecMake3(dir[0], dir[1], dir[2]));
    outRgb[0] = c.x;
    outRgb[1] = c.y;
    outRgb[2] = c.z;
}

// Emissive triangle sampling (LightSamplingCore.h:257-313).
int ref_sample_emissive(void* sceneHandle, float uTri, float u1, float u2, float* outPos, float* outNormal,
    float* outRadiance, float* outPdf)
{
    const MeshAccelSceneGpu* scene = &static_cast<RefScene*>(sceneHandle)->view;
    Vec3 p{};
    Vec3 n{};
    Vec3 L{};
    float pdf = 0.0f;
    const bool ok = lightSampleEmissiveTriangle(scene, uTri, u1, u2, p, n, L, pdf);
    outPos[0] = p.x;
    outPos[1] = p.y;
    outPos[2] = p.z;
    outNormal[0] = n.x;
    outNormal[1] = n.y;
    outNormal[2] = n.z;
    outRadiance[0] = L.x;
    outRadiance[1] = L.y;
    outRadiance[2] = L.z;
    *outPdf = pdf;
    return ok ? 1 : 0;
}

// PrincipledBrdf::sampleTransmit alone (PrincipledBrdf.h:476-551).
int ref_brdf_sample_transmit(const float* normal, const float* wo, const void* material, float etaMedium,
    int debugFlags, float u1, float u2, float* outDir, float* outPdf, float* outNextEta, int* outFlags)
{
    BrdfContext ctx{};
    ctx.normal = vecMake3(normal[0], normal[1], normal[2]);
    ctx.wo = vecMake3(wo[0], wo[1], wo[2]);
    std::memcpy(&ctx.material, material, sizeof(MaterialGpu));
    ctx.etaMedium = etaMedium;
    ctx.debugFlags = debugFlags;
    const BrdfSampleResult r = PrincipledBrdf{}.sampleTransmit(ctx, u1, u2);
    outDir[0] = r.direction.x;
    outDir[1] = r.direction.y;
    outDir[2] = r.direction.z;
    *outPdf = r.pdf;
    *outNextEta = r.nextMediumEta;
    *outFlags = (r.valid ? 1 : 0) | (r.transmitted ? 2 : 0) | (r.subsurfaceScatter ? 4 : 0);
    return r.subsurfaceInternalSteps;
}

// Lobe weights (PrincipledBrdf.h:75-100): diffuse, specular, transmit, subsurface.
void ref_lobe_weights(const void* material, float* out)
{
    BrdfContext ctx{};
    std::memcpy(&ctx.material, material, sizeof(MaterialGpu));
    const PrincipledDetail::LobeWeights w = PrincipledDetail::computeLobeWeights(ctx);
    out[0] = w.diffuse;
    out[1] = w.specular;
    out[2] = w.transmit;
    out[3] = w.subsurface;
}

// Texture bank resolve (Texture/ProceduralTexture.h:138-207); writes the 15
// MaterialGpu float fields of the resolved material.
void ref_resolve_material(const void* material, float u, float v, const void* textures, int textureCount, float* out)
{
    MaterialGpu m{};
    std::memcpy(&m, material, sizeof(MaterialGpu));
    const TextureEvalContext ctx{Vec2{u, v}, u};
    const MaterialGpu r = materialFromResolved(resolveMaterial(m, ctx,
        textureCount > 0 ? static_cast<const TextureDescGpu*>(textures) : nullptr, static_cast<uint32_t>(textureCount)));
    std::memcpy(out, &r, 15 * sizeof(float));
}

// Adaptive convergence predicate (PathTracerAdaptiveSampling.h:16-40).
int ref_is_converged(uint32_t count, float lumMean, float m2, int minSamples, float threshold)
{
    return isAdaptivePixelConverged(count, lumMean, m2, minSamples, threshold) ? 1 : 0;
}

int ref_max_threads()
{
    return omp_get_max_threads();
}

} // extern "C"
