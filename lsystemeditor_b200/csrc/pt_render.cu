// Wavefront path-tracing pipeline for sm_100a.
//
// The reference runs one megakernel thread per pixel and sample
// (sampleAdaptiveKernel, PathTracerLib/src/PathTracer.cu:186-273, body
// tracePathRand, PathIntegratorRandCore.h:206-363).  Here the same estimator
// is split into stages over structure-of-arrays path state:
//
//   generate   camera ray per (pixel, sample): curand_init with the reference
//              seed, jitter + lens draws (PathTracer.cu:69-96)
//   extend     closest hit for every live path            (pt_trace.cuh);
//              large flat scenes: per-lane ray replacement (k_extend_lane)
//              + k_route, which splits the queue into miss and hit queues
//   shade      pending NEE resolve, miss/env MIS, emission, environment and
//              emissive NEE (shadow rays queued), BSDF sample, throughput,
//              subsurface tier B, Russian roulette, continuation ray
//   shadow     any-hit occlusion for the queued shadow rays
//   finalize   paths that ended with shadow rays in flight
//   next_queue (with k_extend_lane) the next bounce's extend queue in slot
//              order, from the slots the shade kernels marked
//   accumulate per pixel, the batch's samples in sample order: running mean,
//              Welford luminance variance, convergence every 4 samples
//              (PathTracer.cu:232-272)
//   compact    active-pixel list without converged pixels
//
// Radiance is added in exactly the reference's order: emission, env NEE,
// emissive NEE (resolved after the shadow stage), then at the next bounce the
// miss term.  Random numbers are drawn in the reference's order from the same
// per-(pixel, sample) XORWOW stream, so a path takes the same decisions as the
// reference's; the state lives in registers within a stage and in the SoA
// between stages.
#include "pt_render.cuh"

#include "pt_bsdf.cuh"
#include "pt_path.cuh"
#include "pt_spectral.cuh"
#include "pt_trace.cuh"

#include <atomic>
#include <cooperative_groups.h>
#include "pt_select.cuh"
#include <curand_kernel.h>

namespace cg = cooperative_groups;

namespace pt {

namespace {

__device__ __forceinline__ uint32_t warpPush(unsigned int* counter)
{
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned int base = 0;
    if (g.thread_rank() == 0) {
        base = atomicAdd(counter, g.size());
    }
    base = g.shfl(base, 0);
    return base + g.thread_rank();
}

// Warp-granular work distribution: each warp takes the next 32 queue entries
// from a per-launch counter, so warps that drew cheap rays keep working
// instead of idling while others finish (no static grid-stride split).
__device__ __forceinline__ unsigned int warpFetch(unsigned int* counter)
{
    unsigned int base = 0;
    if ((threadIdx.x & 31) == 0) {
        base = atomicAdd(counter, 32u);
    }
    return __shfl_sync(0xffffffffu, base, 0) + (threadIdx.x & 31);
}

__device__ __forceinline__ void rngLoad(const PathSoA& P, uint32_t i, curandStateXORWOW& s)
{
    const uint4 a = P.rngA[i];
    const uint2 b = P.rngB[i];
    s.d = a.x;
    s.v[0] = a.y;
    s.v[1] = a.z;
    s.v[2] = a.w;
    s.v[3] = b.x;
    s.v[4] = b.y;
    s.boxmuller_flag = 0;
    s.boxmuller_flag_double = 0;
    s.boxmuller_extra = 0.0f;
    s.boxmuller_extra_double = 0.0;
}

__device__ __forceinline__ void rngStore(const PathSoA& P, uint32_t i, const curandStateXORWOW& s)
{
    P.rngA[i] = make_uint4(s.d, s.v[0], s.v[1], s.v[2]);
    P.rngB[i] = make_uint2(s.v[3], s.v[4]);
}

// Geometry of path i's scene.
__device__ __forceinline__ const DevScene& sceneOf(const LaunchCtx& c, uint32_t i)
{
    return c.sceneCount > 1 ? c.scenes[c.paths.scene[i]] : c.scene;
}

// --- per-path colour: RGB (NW = 0, the reference's integrator) or the
// radiance at NW hero wavelengths (spectral mode) -----------------------------
template <int NW> struct Col {
    float v[NW];
};
template <> struct Col<0> {
    float3 c;
};

template <int NW> __device__ __forceinline__ Col<NW> czero()
{
    Col<NW> r;
    if constexpr (NW == 0) {
        r.c = f3(0.0f, 0.0f, 0.0f);
    } else {
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            r.v[k] = 0.0f;
        }
    }
    return r;
}
template <int NW> __device__ __forceinline__ Col<NW> cadd(const Col<NW>& a, const Col<NW>& b)
{
    Col<NW> r;
    if constexpr (NW == 0) {
        r.c = add3(a.c, b.c);
    } else {
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            r.v[k] = a.v[k] + b.v[k];
        }
    }
    return r;
}
template <int NW> __device__ __forceinline__ Col<NW> cmul(const Col<NW>& a, const Col<NW>& b)
{
    Col<NW> r;
    if constexpr (NW == 0) {
        r.c = mul3(a.c, b.c);
    } else {
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            r.v[k] = a.v[k] * b.v[k];
        }
    }
    return r;
}
template <int NW> __device__ __forceinline__ Col<NW> cscl(const Col<NW>& a, float s)
{
    Col<NW> r;
    if constexpr (NW == 0) {
        r.c = scl3(a.c, s);
    } else {
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            r.v[k] = a.v[k] * s;
        }
    }
    return r;
}
template <int NW> __device__ __forceinline__ bool cnonzero(const Col<NW>& a)
{
    if constexpr (NW == 0) {
        return a.c.x != 0.0f || a.c.y != 0.0f || a.c.z != 0.0f;
    } else {
        bool nz = false;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            nz = nz || a.v[k] != 0.0f;
        }
        return nz;
    }
}

// Wavelengths of a path (spectral mode): the hero draw, wavelength k derived
// on use (a few instructions, cheaper than keeping NW registers live).
template <int NW> struct Waves {
    float u;
    __device__ __forceinline__ float lam(int k) const { return spectral::heroLambda(u, k, NW); }
};
template <int NW> __device__ __forceinline__ Waves<NW> pathWaves(const LaunchCtx& c, uint32_t i)
{
    Waves<NW> w;
    if constexpr (NW > 0) {
        w.u = c.paths.hero[i];
    } else {
        w.u = 0.0f;
    }
    return w;
}

// The spectrum of coefficient record q at the path's wavelengths.  A grey
// record (c = 0) is the constant scale / 2 and a zero scale is 0, exactly what
// evalCoef gives for them, without its square root and division.
template <int NW> __device__ __forceinline__ Col<NW> coefCol(float4 q, const Waves<NW>& w)
{
    Col<NW> r;
    if (q.x == 0.0f && q.y == 0.0f && q.z == 0.0f) {
        const float v = __fmul_rn(0.5f, q.w);
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            r.v[k] = v;
        }
    } else {
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            r.v[k] = spectral::evalCoef(q, w.lam(k));
        }
    }
    return r;
}

// Colour of a float4 path field (xyz in RGB mode; the spectral words otherwise).
template <int NW> __device__ __forceinline__ Col<NW> loadCol(float4 rgb, const float4* spec, int cap, uint32_t i)
{
    Col<NW> r;
    if constexpr (NW == 0) {
        r.c = f3(rgb.x, rgb.y, rgb.z);
    } else {
        (void)rgb;
#pragma unroll
        for (int j = 0; j < NW / 4; ++j) {
            const float4 q = spec[static_cast<size_t>(j) * cap + i];
            r.v[4 * j] = q.x;
            r.v[4 * j + 1] = q.y;
            r.v[4 * j + 2] = q.z;
            r.v[4 * j + 3] = q.w;
        }
    }
    return r;
}
// Stores a colour with `w` in the RGB field's fourth word (the RGB field
// keeps only w in spectral mode).
template <int NW> __device__ __forceinline__ void storeCol(float4* rgb, float4* spec, int cap, uint32_t i, const Col<NW>& v,
    float w)
{
    if constexpr (NW == 0) {
        rgb[i] = make_float4(v.c.x, v.c.y, v.c.z, w);
    } else {
        if (rgb != nullptr) {
            rgb[i] = make_float4(0.0f, 0.0f, 0.0f, w);
        }
#pragma unroll
        for (int j = 0; j < NW / 4; ++j) {
            spec[static_cast<size_t>(j) * cap + i] =
                make_float4(v.v[4 * j], v.v[4 * j + 1], v.v[4 * j + 2], v.v[4 * j + 3]);
        }
    }
}
template <int NW> __device__ __forceinline__ Col<NW> pendingEnv(const LaunchCtx& c, uint32_t i)
{
    if constexpr (NW == 0) {
        return loadCol<0>(c.paths.neeEnv[i], nullptr, 0, i);
    } else {
        return loadCol<NW>(make_float4(0.0f, 0.0f, 0.0f, 0.0f), c.paths.neeEnvS, c.paths.capacity, i);
    }
}
template <int NW> __device__ __forceinline__ Col<NW> pendingEmis(const LaunchCtx& c, uint32_t i)
{
    if constexpr (NW == 0) {
        return loadCol<0>(c.paths.neeEmis[i], nullptr, 0, i);
    } else {
        return loadCol<NW>(make_float4(0.0f, 0.0f, 0.0f, 0.0f), c.paths.neeEmisS, c.paths.capacity, i);
    }
}

// Environment / background radiance in direction d (LightSamplingCore.h:56-77).
template <int NW> __device__ __forceinline__ Col<NW> envCol(const LaunchCtx& c, float3 d, const Waves<NW>& w)
{
    Col<NW> r;
    if constexpr (NW == 0) {
        r.c = envEval(c.env, c.params, d);
    } else {
        float4 q = c.specBackground;
        if (c.env.valid) {
            float u, v;
            dirToLatLong(d, u, v);
            const int x = min(max(static_cast<int>(u * static_cast<float>(c.env.width)), 0), c.env.width - 1);
            const int y = min(max(static_cast<int>(v * static_cast<float>(c.env.height)), 0), c.env.height - 1);
            q = c.env.spec[static_cast<size_t>(y) * c.env.width + x];
        }
        r = coefCol<NW>(q, w);
    }
    return r;
}

// --- distant light ---------------------------------------------------------------
// Is direction d (any length) inside the light's cone?  Tested through the
// sine (|d x dir|^2 <= sin^2 * |d|^2), which keeps its precision for the small
// half-angles of a sun.
__device__ __forceinline__ bool inSun(const DevSun& s, float3 d)
{
    const float3 x = cross3(d, s.dir);
    return dot3(d, s.dir) > 0.0f && dot3(x, x) <= s.sin2 * dot3(d, d);
}
// Uniform direction in the cone (u1 -> 1 - cos theta over [0, omc], u2 -> phi).
__device__ __forceinline__ float3 sunSample(const DevSun& s, float u1, float u2)
{
    const float h = u1 * s.omc;
    const float ct = 1.0f - h;
    const float st = sqrtf(fmax2(0.0f, h * (2.0f - h)));
    float sp, cp;
    sincosf(2.0f * kPi * u2, &sp, &cp);
    return normalize3(add3(add3(scl3(s.t, st * cp), scl3(s.b, st * sp)), scl3(s.dir, ct)));
}
// Density of the sky's next-event sample (the light with probability select,
// else the environment) in direction d.
__device__ __forceinline__ float skyPdf(const LaunchCtx& c, float3 d)
{
    const float ls = inSun(c.sun, d) ? c.sun.pdf : 0.0f;
    return c.sun.select * ls + (1.0f - c.sun.select) * envPdf(c.env, d);
}
// Relative blackbody spectral radiance (Planck's law, lambda in micrometres).
__device__ __forceinline__ float planckRel(float lambdaNm, float temperature)
{
    const float lu = lambdaNm * 1.0e-3f;
    const float l2 = lu * lu;
    return 1.0f / (l2 * l2 * lu * expm1f(14387.769f / (lu * temperature)));
}
template <int NW> __device__ __forceinline__ Col<NW> sunCol(const LaunchCtx& c, const Waves<NW>& w)
{
    Col<NW> r;
    if constexpr (NW == 0) {
        (void)w;
        r.c = c.sun.rgb;
    } else if (c.sun.temperature > 0.0f) {
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            r.v[k] = c.sun.scale * planckRel(w.lam(k), c.sun.temperature);
        }
    } else {
        r = coefCol<NW>(c.sun.coef, w);
    }
    return r;
}
// Sky radiance (environment plus the light where d is inside its cone).
template <int NW> __device__ __forceinline__ Col<NW> skyCol(const LaunchCtx& c, float3 d, const Waves<NW>& w)
{
    Col<NW> L = envCol<NW>(c, d, w);
    if (c.sun.enabled && inSun(c.sun, d)) {
        L = cadd(L, sunCol<NW>(c, w));
    }
    return L;
}

// Spectrum coefficients of the base colour and scatter radii of the material
// at a hit, following resolveMaterial's albedo-texture rules.
__device__ __forceinline__ void matCoefs(const DevScene& S, uint32_t mi, const pt_material& src, float u, float v,
    float4& base, float4& scatter)
{
    if (S.matSpec == nullptr || S.materials == nullptr || mi >= S.materialCount) {
        base = make_float4(0.0f, 0.0f, 0.0f, 1.6f); // the fallback material's grey 0.8
        scatter = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
        base = S.matSpec[2 * mi];
        scatter = S.matSpec[2 * mi + 1];
    }
    const uint32_t ti = src.albedo_tex;
    if (ti != 0u && S.textures != nullptr && ti < S.textureCount) {
        const pt_texture& t = S.textures[ti];
        if (t.kind == 1) {
            base = S.texSpec[2 * ti];
        } else if (t.kind == 2) {
            const float fx = fractf(u * t.p0[0]);
            const float fy = fractf(v * t.p0[1]);
            base = S.texSpec[2 * ti + ((fx < t.p0[2] || fy < t.p0[2]) ? 1 : 0)];
        } else {
            base = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
}

// BSDF value (RGB), or at each wavelength.  The spectral value at lambda is
// the RGB BSDF of the material with every colour channel set to the colour's
// spectrum at lambda.  All lobes but a scattering subsurface lobe are affine in
// the base colour, f(rho) = f(0) + rho (f(1) - f(0)), so one RGB evaluation
// with base (0, 1, 1) gives every wavelength: in spectral mode the shade
// kernel keeps the material's base at (0, 1, 1) (sampling and pdfs do not read
// it).  With a scattering subsurface lobe (radius per wavelength) each
// wavelength is evaluated on its own, cx's colour fields modified in place and
// restored.
template <int NW>
__device__ __forceinline__ Col<NW> evalCol(Ctx& cx, float3 wi, const Col<NW>& rho, float4 scatter, const Waves<NW>& w)
{
    Col<NW> f;
    if constexpr (NW == 0) {
        (void)rho;
        (void)scatter;
        (void)w;
        f.c = bsdfEval(cx, wi);
    } else {
        if (cx.w.subsurface != 0.0f && maxScatter(cx.m) > kMinRadius) {
            const float sr = cx.m.scatterR, sg = cx.m.scatterG, sb = cx.m.scatterB;
#pragma unroll 1
            for (int k = 0; k < NW; ++k) {
                cx.m.r = cx.m.g = cx.m.b = rho.v[k];
                const float rk = spectral::evalCoef(scatter, w.lam(k));
                cx.m.scatterR = cx.m.scatterG = cx.m.scatterB = rk;
                f.v[k] = bsdfEval(cx, wi).x;
            }
            cx.m.r = 0.0f;
            cx.m.g = cx.m.b = 1.0f;
            cx.m.scatterR = sr;
            cx.m.scatterG = sg;
            cx.m.scatterB = sb;
        } else {
            const float3 e = bsdfEval(cx, wi);
            const float b = e.y - e.x;
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                f.v[k] = e.x + b * rho.v[k];
            }
        }
    }
    return f;
}

template <int NW>
__device__ __forceinline__ Col<NW> throughCol(const Col<NW>& T, const Ctx& cx, const BsdfSample& smp, const Col<NW>& f,
    const Col<NW>& rho)
{
    Col<NW> r;
    if constexpr (NW == 0) {
        (void)rho;
        r.c = applyThroughput(T.c, cx, smp, f.c);
    } else {
        float k;
        bool tint;
        if (!throughputFactor(cx, smp, k, tint)) {
            return czero<NW>();
        }
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            float sc = f.v[j] * k;
            if (tint) {
                sc = sc * rho.v[j];
            }
            r.v[j] = T.v[j] * sc;
        }
    }
    return r;
}

// Russian-roulette weight of a throughput: Rec. 709 luminance (RGB), the mean
// over the wavelengths (spectral).
template <int NW> __device__ __forceinline__ float pathWeight(const Col<NW>& T)
{
    if constexpr (NW == 0) {
        return lum709(T.c);
    } else {
        float s = 0.0f;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            s += T.v[k];
        }
        return s * (1.0f / static_cast<float>(NW));
    }
}

template <int NW>
__device__ __forceinline__ void writeSample(const LaunchCtx& c, uint32_t i, const Col<NW>& Lc, const Waves<NW>& w)
{
    float3 L;
    if constexpr (NW == 0) {
        (void)w;
        L = Lc.c;
    } else {
        // hero-wavelength estimate of linear sRGB: each wavelength is uniform
        // over the range, so sum_k L_k resp(lambda_k) (range / NW); a zero
        // spectrum (a path that left a black scene) gives exactly 0
        L = f3(0.0f, 0.0f, 0.0f);
        if (cnonzero(Lc)) {
            float3 a = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                a = add3(a, scl3(spectral::responseAt(c.specResp, w.lam(k)), Lc.v[k]));
            }
            L = scl3(a, spectral::kLambdaRange / static_cast<float>(NW));
        }
    }
    const uint32_t o = c.paths.outIdx[i];
    const float3 s = NW == 0 ? clampFirefly(L) : clampFireflySigned(L);
    c.acc.samples[o] = make_float4(s.x, s.y, s.z, 1.0f);
    if (c.record != nullptr) {
        // sample index = samples the pixel had at batch start + the job's slot
        const uint32_t pixel = c.paths.pixel[i];
        const uint32_t k = c.acc.counts[pixel] + o / static_cast<uint32_t>(c.q.batch->activeCount);
        if (k < static_cast<uint32_t>(c.recordSpp)) {
            c.record[static_cast<size_t>(k) * static_cast<size_t>(c.width) * static_cast<size_t>(c.height) + pixel] =
                make_float4(L.x, L.y, L.z, 0.0f);
        }
    }
}

// Camera path for job j of the current batch (PathTracer.cu:69-96): job
// j = slot * activeCount + listIndex draws sample `counts[pixel] + slot` of
// pixel active[listIndex] with the reference seed for wave waveBase + slot.
template <int NW> __device__ __forceinline__ void initPath(const LaunchCtx& c, uint32_t i, unsigned long long j)
{
    const BatchInfo& bt = *c.q.batch;
    const int activeCount = bt.activeCount;
    const int* active = c.acc.active[c.activeSel];
    int li;
    uint32_t slot;
    uint32_t local;
    const pt_camera* cam = &c.cam;
    uint32_t width = static_cast<uint32_t>(c.width), height = static_cast<uint32_t>(c.height);
    uint32_t pixel;
    if (c.sceneCount > 1) {
        // scene-major job order: all of a scene's jobs before the next scene's,
        // so that the paths in flight share few scenes' geometry
        int lo = 0, hi = c.sceneCount - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (c.sceneJobStart[mid] <= j) {
                lo = mid;
            } else {
                hi = mid - 1;
            }
        }
        const uint32_t a0 = c.sceneActiveStart[lo];
        const uint32_t n = c.sceneActiveStart[lo + 1] - a0;
        const unsigned long long q = j - c.sceneJobStart[lo];
        slot = static_cast<uint32_t>(q / n);
        li = static_cast<int>(a0 + static_cast<uint32_t>(q % n));
        pixel = static_cast<uint32_t>(active[li]);
        const SceneView& sv = c.views[lo];
        // seeds and film coordinates use the pixel's index within its own
        // image, so a scene renders the same in a batch as alone
        local = pixel - sv.pixelBase;
        cam = &sv.cam;
        width = static_cast<uint32_t>(sv.width);
        height = static_cast<uint32_t>(sv.height);
        c.paths.scene[i] = static_cast<uint16_t>(lo);
    } else {
        li = static_cast<int>(j % static_cast<unsigned long long>(activeCount));
        slot = static_cast<uint32_t>(j / static_cast<unsigned long long>(activeCount));
        pixel = static_cast<uint32_t>(active[li]);
        local = pixel;
    }
    const uint32_t sampleIndex = c.acc.counts[pixel] + slot;
    const uint32_t globalSeed = bt.waveBase + slot + 1u + static_cast<uint32_t>(c.seedOffset);
    curandStateXORWOW st;
    const uint32_t seed = pathSeed(c.params, local, width, sampleIndex, globalSeed);
    curand_init(seed, 0ull, 0ull, &st);
    const uint32_t x = local % width, y = local / width;
    const float ju = curand_uniform(&st);
    const float jv = curand_uniform(&st);
    const float u = (static_cast<float>(x) + ju) / static_cast<float>(width);
    const float v = (static_cast<float>(y) + jv) / static_cast<float>(height);
    const float l1 = curand_uniform(&st);
    const float l2 = curand_uniform(&st);
    float3 ro, rd;
    cameraRay(*cam, u, v, l1, l2, ro, rd);
    c.paths.pixel[i] = pixel;
    c.paths.outIdx[i] = slot * static_cast<uint32_t>(activeCount) + static_cast<uint32_t>(li);
    rngStore(c.paths, i, st);
    c.paths.orig[i] = make_float4(ro.x, ro.y, ro.z, 0.0f);
    c.paths.dir[i] = make_float4(rd.x, rd.y, rd.z, 0.0f);
    c.paths.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    c.paths.rad[i] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(0));
    if constexpr (NW > 0) {
        // (the spectral throughput and radiance of a path at depth 0 are 1 and
        // 0: they are not stored, the shade kernels know them)
        c.paths.hero[i] = spectral::heroU(seed);
    }
    c.paths.visEnv[i] = 0;
    c.paths.visEmis[i] = 0;
}

// Path i joins the next bounce's extend queue: marked for k_next_queue in
// slot-ordered mode, else pushed (one atomic per warp).
__device__ __forceinline__ void queueNext(const LaunchCtx& c, uint32_t i, unsigned int* nextCount, uint32_t* nextQueue)
{
    if (c.q.nextFlag != nullptr) {
        c.q.nextFlag[i] = 1;
    } else {
        const uint32_t s = warpPush(nextCount);
        nextQueue[s] = i;
    }
}

// A terminated path's slot takes the batch's next job, if any, and joins the
// next extend queue: launches stay full until the batch drains.
template <int NW>
__device__ __forceinline__ void recyclePath(const LaunchCtx& c, uint32_t i, unsigned int* nextCount, uint32_t* nextQueue)
{
#if PT_PATH_GENERATIONS
    // (generations: a finished path's slot stays empty until the next
    // generation; the batch's job counter is not touched per path)
    (void)c;
    (void)i;
    (void)nextCount;
    (void)nextQueue;
    return;
#endif
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) {
        base = atomicAdd(&c.q.batch->nextJob, static_cast<unsigned long long>(g.size()));
    }
    base = g.shfl(base, 0);
    const unsigned long long j = base + g.thread_rank();
    if (j < c.q.batch->jobs) {
        initPath<NW>(c, i, j);
        queueNext(c, i, nextCount, nextQueue);
    }
}

// Jobs jobOffset .. jobOffset + count - 1 of a batch into slots 0..count-1
// (extend queue = identity).
template <int NW>
__global__ void __launch_bounds__(256) k_generate(const LaunchCtx* __restrict__ cp, int count, int extendSel,
    unsigned long long jobOffset)
{
    const LaunchCtx& c = *cp;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.q.counts[extendSel] = static_cast<unsigned int>(count);
        c.q.counts[extendSel ^ 1] = 0u;
        c.q.counts[2] = 0u;
        c.q.counts[3] = 0u;
        c.q.counts[4] = 0u;
        c.q.counts[5] = 0u;
        c.q.counts[8] = 0u;  // fetch counters of the first extend and shadow stages
        c.q.counts[10] = 0u;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        initPath<NW>(c, static_cast<uint32_t>(i), jobOffset + static_cast<unsigned long long>(i));
    }
}

// Closest hit for every queued path; each path is then routed to the miss or
// the hit queue of this bounce so that the two shade kernels run coherent work.
// Counters: [4 + 2p] misses and [5 + 2p] hits of bounce parity p; this kernel
// zeroes the other parity's pair for the next bounce.
template <bool Count, bool Inst>
#ifndef PT_EXTEND_MIN_BLOCKS
#define PT_EXTEND_MIN_BLOCKS 4
#endif
#ifndef PT_SHADE_MIN_BLOCKS
// (RGB shade at 4 blocks per SM, 64 registers: 8% less time per frame than at
// 3 blocks and 80 registers on the 972k-triangle tree, 10% on the 64-tree
// batch; the stage waits on dependent path-state and material loads, and the
// fourth block hides more of that latency than the spills cost)
#define PT_SHADE_MIN_BLOCKS 4
#endif
#ifndef PT_SHADE_SPEC_MIN_BLOCKS
// (spectral shade at 4 blocks per SM, 64 registers: 531 -> 474 ms per frame on
// the 972k-triangle tree with 8 wavelengths, each form on a grid of its own
// occupancy)
#define PT_SHADE_SPEC_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(256, PT_EXTEND_MIN_BLOCKS) k_extend(const LaunchCtx* __restrict__ cp, int sel, bool identity, int iter)
{
    const LaunchCtx& c = *cp;
    extern __shared__ uint2 smemStack[];
    const unsigned int count = c.q.counts[sel];
    const int par = iter & 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&c.q.rays[0], static_cast<unsigned long long>(count));
        // output counters of the shade stage that follows, and next bounce's routing counters
        c.q.counts[sel ^ 1] = 0u;
        c.q.counts[2] = 0u;
        c.q.counts[3] = 0u;
        c.q.counts[4 + 2 * (par ^ 1)] = 0u;
        c.q.counts[5 + 2 * (par ^ 1)] = 0u;
        c.q.counts[8 + (par ^ 1)] = 0u; // next extend's fetch counter
    }
    const uint32_t* queue = c.q.extend[sel];
    unsigned int* fetch = &c.q.counts[8 + par];
    for (;;) {
        const unsigned int k = warpFetch(fetch);
        if (__shfl_sync(0xffffffffu, k, 0) >= count) {
            break;
        }
        if (k >= count) {
            continue;
        }
        const uint32_t i = identity ? k : queue[k];
        const float4 o4 = c.paths.orig[i];
        const float4 d4 = c.paths.dir[i];
        const float3 dn = xnormalize(f3(d4.x, d4.y, d4.z));
        HitRec h;
        const DevScene& S = sceneOf(c, i);
        const bool hit = traceRay<false, Count, Inst>(S, f3(o4.x, o4.y, o4.z), dn, o4.w, kRayTMax, h, c.q.overflow,
            c.q.visits, smemStack + threadIdx.x, blockDim.x);
        if (hit) {
            c.paths.hit[i] = make_float4(h.t, h.u, h.v, __uint_as_float(h.tri));
            if (Inst && S.instanceCount > 0) {
                c.paths.hitInst[i] = h.inst;
            }
            const uint32_t s = warpPush(&c.q.counts[5 + 2 * par]);
            c.q.hitQueue[s] = i;
        } else {
            const uint32_t s = warpPush(&c.q.counts[4 + 2 * par]);
            c.q.missQueue[s] = i;
        }
    }
}

#ifndef PT_EXTEND_LANE_THREADS
#define PT_EXTEND_LANE_THREADS 256
#endif
#ifndef PT_EXTEND_LANE_MIN_BLOCKS
#define PT_EXTEND_LANE_MIN_BLOCKS 3
#endif
#ifndef PT_SHADOW_LANE_MIN_BLOCKS
#define PT_SHADOW_LANE_MIN_BLOCKS 4
#endif
#ifndef PT_EXTEND_LANE_SYNC
#define PT_EXTEND_LANE_SYNC false
#endif
#ifndef PT_SHADOW_LANE_SYNC
#define PT_SHADOW_LANE_SYNC false
#endif
#ifndef PT_SHADOW_LANE
#define PT_SHADOW_LANE 1
#endif

// A ray of the per-lane traversal: its scene, origin, normalised direction and
// the parametric interval it is tested on.
struct LaneRay {
    const DevScene* S;
    float3 o;
    float3 dn;
    float tMin;
    float tMax;
};

// Per-lane ray replacement (Aila & Laine 2009, "dynamic fetch") over a queue of
// `count` rays of flat scenes: a lane whose ray is finished takes the next
// queue entry at once, while the other lanes of its warp go on traversing, so
// a warp is not held by its longest ray.  One loop iteration is one step of
// traceRay's traversal (a node's children, then the triangles of that node),
// with the same postponing, stacks and tie rule, so the results are
// traceRay's.  Two loop forms:
//   Sync = false: a lane fetches as soon as it is idle (the idle lanes of the
//     moment share one atomic) and the lanes of a warp are not reconverged, so
//     the scheduler can issue from the lanes that fetch while the others wait
//     on node loads.  This form is the faster of the two on the 972k-triangle
//     tree (closest hit) and on the 64-tree batch (shadow rays).
//   Sync = true: every iteration is warp-synchronous (one ballot fetch for the
//     idle lanes at the top, a full-warp vote to leave), so the lanes of a
//     warp step together.
//   load(k, ray) -> bool: reads queue entry k into `ray`; false when the entry
//     was decided without the wide traversal (and its result written).
//   finish(k, hit, t, u, v, tri): the result of entry k (tri = original
//     triangle index; for AnyHit, hit means occluded and t, u, v, tri are unset).
// Rays finish in no particular order.
template <bool AnyHit, bool Sync, class Load, class Finish>
__device__ __forceinline__ void laneTraversal(unsigned int count, unsigned int* fetch, uint2* sstack, int sstride,
    unsigned int* overflowCounter, Load load, Finish finish)
{
    uint2 stack[kTraversalStack];
    bool active = false;
    unsigned int k = 0;
    LaneRay r{nullptr, f3(0.0f, 0.0f, 0.0f), f3(0.0f, 0.0f, 0.0f), 0.0f, 0.0f};
    float3 idir = r.o;
    uint32_t octinv = 0;
    uint2 ngroup = make_uint2(0u, 0u), tgroup = make_uint2(0u, 0u);
    int sp = 0;
    float closest = kRayTMax;
    uint32_t best = 0xFFFFFFFFu;
    float bu = 0.0f, bv = 0.0f;
    bool overflow = false;

    auto push = [&](uint2 g) -> bool {
        if (sp < kSharedStack) {
            sstack[sp * sstride] = g;
        } else if (sp < kSharedStack + kTraversalStack) {
            stack[sp - kSharedStack] = g;
        } else {
            return false;
        }
        ++sp;
        return true;
    };
    auto done = [&](bool hit) {
        finish(k, hit, closest, bu, bv, hit && !AnyHit ? leafId(r.S->tris, best) : 0xFFFFFFFFu);
        if (overflow && overflowCounter != nullptr && !(AnyHit && hit)) {
            atomicAdd(overflowCounter, 1u); // rays whose stack overflowed, as traceRay counts them (an occluded any-hit ray is not counted)
        }
        overflow = false;
        active = false;
    };
    auto begin = [&]() {
        idir = f3(__frcp_rn(r.dn.x), __frcp_rn(r.dn.y), __frcp_rn(r.dn.z));
        const uint32_t oct = (r.dn.x < 0.0f ? 4u : 0u) | (r.dn.y < 0.0f ? 2u : 0u) | (r.dn.z < 0.0f ? 1u : 0u);
        octinv = 7u - oct;
        ngroup = make_uint2(0u, 0x80000000u | (1u << oct));
        tgroup = make_uint2(0u, 0u);
        sp = 0;
        closest = r.tMax;
        best = 0xFFFFFFFFu;
        bu = bv = 0.0f;
        active = true;
    };
    const unsigned int lane = threadIdx.x & 31u;
    bool drained = false;
    for (;;) {
        if constexpr (Sync) {
            const bool want = !active && !drained;
            const unsigned int wantMask = __ballot_sync(0xFFFFFFFFu, want);
            if (wantMask != 0u) {
                const int leader = __ffs(wantMask) - 1;
                unsigned int base = 0;
                if (static_cast<int>(lane) == leader) {
                    base = atomicAdd(fetch, static_cast<unsigned int>(__popc(wantMask)));
                }
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (want) {
                    k = base + __popc(wantMask & ((1u << lane) - 1u));
                    if (k >= count) {
                        drained = true; // the queue is drained
                    } else if (load(k, r)) {
                        begin();
                    }
                    // (an entry decided by load leaves the lane idle: it fetches again)
                }
            }
            if (!__any_sync(0xFFFFFFFFu, active || !drained)) {
                break;
            }
        } else if (!active) {
            // the lanes without a ray take the next queue entries together (one atomic)
            cg::coalesced_group g = cg::coalesced_threads();
            unsigned int base = 0;
            if (g.thread_rank() == 0) {
                base = atomicAdd(fetch, g.size());
            }
            k = g.shfl(base, 0) + g.thread_rank();
            if (k >= count) {
                break; // the queue is drained
            }
            if (!load(k, r)) {
                continue; // decided without the wide traversal
            }
            begin();
        }
        if (active) {
            // one traversal step (traceRay's loop body)
            if (ngroup.y > 0x00FFFFFFu) {
                const uint32_t bit = 31u - __clz(ngroup.y);
                ngroup.y &= ~(1u << bit);
                const uint32_t slot = (bit - 24u) ^ octinv;
                const uint32_t child = ngroup.x + __popc(ngroup.y & 0xffu & ((1u << slot) - 1u));
                if (ngroup.y > 0x00FFFFFFu && !push(ngroup)) {
                    overflow = true;
                }
                uint32_t childBase, triBase, imask;
                const uint32_t hits =
                    intersectChildren(r.S->nodes, child, r.o, idir, octinv, r.tMin, closest, childBase, triBase, imask);
                ngroup = make_uint2(childBase, (hits & 0xFF000000u) | imask);
                tgroup = make_uint2(triBase, hits & 0x00FFFFFFu);
            } else {
                tgroup = ngroup;
                ngroup = make_uint2(0u, 0u);
            }
            bool occluded = false;
            while (tgroup.y != 0u) {
                if (ngroup.y > 0x00FFFFFFu && __popc(__activemask()) < kPostponeLanes && push(tgroup)) {
                    break;
                }
                const int kt = __ffs(tgroup.y) - 1;
                tgroup.y &= tgroup.y - 1u;
                const TriVerts tv = r.S->tris[tgroup.x + kt];
                float t, u, v;
                if (intersectTriExact(r.o, r.dn, f3(tv.v0.x, tv.v0.y, tv.v0.z), f3(tv.v1.x, tv.v1.y, tv.v1.z),
                        f3(tv.v2.x, tv.v2.y, tv.v2.z), r.tMin, closest, t, u, v)) {
                    if (AnyHit) {
                        if (t < r.tMax) {
                            occluded = true; // traceRay's any-hit: the first hit below tMax ends the ray
                            break;
                        }
                    } else if (t < closest || best == 0xFFFFFFFFu ||
                               leafId(r.S->tris, tgroup.x + kt) > leafId(r.S->tris, best)) {
                        closest = t; // (traceRay's tie rule: the higher original triangle index)
                        best = tgroup.x + kt;
                        bu = u;
                        bv = v;
                    }
                }
            }
            if (occluded) {
                done(true);
            } else if (ngroup.y <= 0x00FFFFFFu) {
                if (sp == 0) {
                    // the ray is finished
                    done(!AnyHit && best != 0xFFFFFFFFu && closest < r.tMax);
                } else {
                    --sp;
                    ngroup = sp < kSharedStack ? sstack[sp * sstride] : stack[sp - kSharedStack];
                }
            }
        }
    }
}

// Per-lane ray replacement over the two-level BVH of an instanced scene: the
// free-running loop of laneTraversal around traceInstanced's step (top-level
// leaves are instances; on reaching one the ray goes to the object's space on
// the same stack above the top level's entries, and comes back when those are
// used up), with traceInstanced's postponing, overflow and tie rule, so the
// results are traceInstanced's.  finish(k, hit, t, u, v, tri, inst): tri is
// the shading-record index (object base + object triangle), inst the instance.
template <bool AnyHit, class Load, class Finish>
__device__ __forceinline__ void laneTraversalInst(unsigned int count, unsigned int* fetch, uint2* sstack, int sstride,
    unsigned int* overflowCounter, Load load, Finish finish)
{
    uint2 stack[kTraversalStack];
    bool active = false;
    unsigned int k = 0;
    LaneRay r{nullptr, f3(0.0f, 0.0f, 0.0f), f3(0.0f, 0.0f, 0.0f), 0.0f, 0.0f};
    float3 ro = r.o, rd = r.o, idir = r.o;
    uint32_t oct = 0, octinv = 7;
    const CwNode* nodes = nullptr;
    const TriVerts* leaves = nullptr;
    int level = 0, base = 0;
    uint32_t curInst = 0, curTriBase = 0;
    uint2 ngroup = make_uint2(0u, 0u), tgroup = make_uint2(0u, 0u);
    int sp = 0;
    float closest = kRayTMax;
    unsigned long long bestKey = ~0ull;
    uint32_t bestTri = 0xFFFFFFFFu, bestInst = 0xFFFFFFFFu;
    float bu = 0.0f, bv = 0.0f;
    bool overflow = false;

    auto setRay = [&](float3 a, float3 d) {
        ro = a;
        const float dx = fabsf(d.x) < 1.0e-20f ? copysignf(1.0e-20f, d.x) : d.x;
        const float dy = fabsf(d.y) < 1.0e-20f ? copysignf(1.0e-20f, d.y) : d.y;
        const float dz = fabsf(d.z) < 1.0e-20f ? copysignf(1.0e-20f, d.z) : d.z;
        idir = f3(__frcp_rn(dx), __frcp_rn(dy), __frcp_rn(dz));
        oct = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
        octinv = 7u - oct;
    };
    auto push = [&](uint2 g) -> bool {
        if (sp < kSharedStack) {
            sstack[sp * sstride] = g;
        } else if (sp < kSharedStack + kTraversalStack) {
            stack[sp - kSharedStack] = g;
        } else {
            return false;
        }
        ++sp;
        return true;
    };
    auto done = [&](bool hit) {
        finish(k, hit, closest, bu, bv, bestTri, bestInst);
        if (overflow && overflowCounter != nullptr && !(AnyHit && hit)) {
            atomicAdd(overflowCounter, 1u); // rays whose stack overflowed, as traceInstanced counts them
        }
        overflow = false;
        active = false;
    };
    for (;;) {
        if (!active) {
            // the lanes without a ray take the next queue entries together (one atomic)
            cg::coalesced_group g = cg::coalesced_threads();
            unsigned int b = 0;
            if (g.thread_rank() == 0) {
                b = atomicAdd(fetch, g.size());
            }
            k = g.shfl(b, 0) + g.thread_rank();
            if (k >= count) {
                break; // the queue is drained
            }
            if (!load(k, r)) {
                continue; // decided without the wide traversal
            }
            setRay(r.o, r.dn);
            rd = r.dn;
            nodes = r.S->tlasNodes;
            leaves = r.S->tlasLeaves;
            level = 0;
            base = 0;
            curInst = 0;
            curTriBase = 0;
            ngroup = make_uint2(0u, 0x80000000u | (1u << oct));
            tgroup = make_uint2(0u, 0u);
            sp = 0;
            closest = r.tMax;
            bestKey = ~0ull;
            bestTri = bestInst = 0xFFFFFFFFu;
            bu = bv = 0.0f;
            active = true;
        }
        // one step of traceInstanced's loop
        if (ngroup.y > 0x00FFFFFFu) {
            const uint32_t bit = 31u - __clz(ngroup.y);
            ngroup.y &= ~(1u << bit);
            const uint32_t slot = (bit - 24u) ^ octinv;
            const uint32_t child = ngroup.x + __popc(ngroup.y & 0xffu & ((1u << slot) - 1u));
            if (ngroup.y > 0x00FFFFFFu && !push(ngroup)) {
                overflow = true;
            }
            uint32_t childBase, triBase, imask;
            const uint32_t hits = intersectChildren(nodes, child, ro, idir, octinv, r.tMin, closest, childBase, triBase,
                imask);
            ngroup = make_uint2(childBase, (hits & 0xFF000000u) | imask);
            tgroup = make_uint2(triBase, hits & 0x00FFFFFFu);
        } else {
            tgroup = ngroup;
            ngroup = make_uint2(0u, 0u);
        }
        bool occluded = false;
        while (tgroup.y != 0u) {
            if (level == 0) {
                // an instance: descend into its object
                const int kt = __ffs(tgroup.y) - 1;
                tgroup.y &= tgroup.y - 1u;
                const uint32_t inst = __float_as_uint(__ldg(&leaves[tgroup.x + kt].v0.w));
                bool saved = true;
                if (ngroup.y > 0x00FFFFFFu) {
                    saved = push(ngroup);
                }
                if (saved && tgroup.y != 0u) {
                    saved = push(tgroup);
                }
                if (!saved) {
                    overflow = true; // the rest of this top-level group is dropped
                }
                const DevInstance& I = r.S->instances[inst];
                const DevBlas B = r.S->blases[I.meta.x];
                curInst = inst;
                curTriBase = B.triBase;
                nodes = B.nodes;
                leaves = B.tris;
                rd = xformVector(I.w2o, r.dn);
                setRay(xformPoint(I.w2o, r.o), rd);
                level = 1;
                base = sp;
                ngroup = make_uint2(0u, B.nodeCount > 0 ? (0x80000000u | (1u << oct)) : 0u);
                tgroup = make_uint2(0u, 0u);
                break;
            }
            if (ngroup.y > 0x00FFFFFFu && __popc(__activemask()) < kPostponeLanes && push(tgroup)) {
                break;
            }
            const int kt = __ffs(tgroup.y) - 1;
            tgroup.y &= tgroup.y - 1u;
            const TriVerts tv = leaves[tgroup.x + kt];
            float t, u, v;
            if (intersectTriExact(ro, rd, f3(tv.v0.x, tv.v0.y, tv.v0.z), f3(tv.v1.x, tv.v1.y, tv.v1.z),
                    f3(tv.v2.x, tv.v2.y, tv.v2.z), r.tMin, closest, t, u, v)) {
                const unsigned long long key = (static_cast<unsigned long long>(curInst) << 32) |
                    static_cast<unsigned long long>(__float_as_uint(tv.v0.w));
                if (AnyHit) {
                    if (t < r.tMax) {
                        occluded = true; // the first hit below tMax ends the ray
                        break;
                    }
                } else if (t < closest || key > bestKey || bestKey == ~0ull) {
                    closest = t;
                    bestKey = key;
                    bestTri = curTriBase + __float_as_uint(tv.v0.w);
                    bestInst = curInst;
                    bu = u;
                    bv = v;
                }
            }
        }
        if (occluded) {
            done(true);
            continue;
        }
        if (ngroup.y <= 0x00FFFFFFu) {
            if (level == 1 && sp == base) {
                // the object is done: back to the top level in world space
                level = 0;
                nodes = r.S->tlasNodes;
                leaves = r.S->tlasLeaves;
                rd = r.dn;
                setRay(r.o, r.dn);
            }
            if (sp == 0) {
                // the ray is finished
                done(!AnyHit && bestTri != 0xFFFFFFFFu && closest < r.tMax);
            } else {
                --sp;
                ngroup = sp < kSharedStack ? sstack[sp * sstride] : stack[sp - kSharedStack];
            }
        }
    }
}

// Closest hit of every queued path by the per-lane traversal.  The result of
// queue entry k goes back into entry k (path index, bit 31 set for a miss) and
// k_route splits the queue into the miss and hit queues in queue order
// afterwards.  Flat scenes only (no instances, no visit counting).
__global__ void __launch_bounds__(PT_EXTEND_LANE_THREADS, PT_EXTEND_LANE_MIN_BLOCKS)
    k_extend_lane(const LaunchCtx* __restrict__ cp, int sel, bool identity, int iter)
{
    const LaunchCtx& c = *cp;
    extern __shared__ uint2 smemStack[];
    const unsigned int count = c.q.counts[sel];
    const int par = iter & 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&c.q.rays[0], static_cast<unsigned long long>(count));
        c.q.counts[sel ^ 1] = 0u;
        c.q.counts[2] = 0u;
        c.q.counts[3] = 0u;
        c.q.counts[4 + 2 * (par ^ 1)] = 0u;
        c.q.counts[5 + 2 * (par ^ 1)] = 0u;
        c.q.counts[8 + (par ^ 1)] = 0u;
    }
    uint32_t* queue = c.q.extend[sel];
    uint32_t i = 0;
    laneTraversal<false, PT_EXTEND_LANE_SYNC>(count, &c.q.counts[8 + par], smemStack + threadIdx.x, static_cast<int>(blockDim.x),
        c.q.overflow,
        [&](unsigned int k, LaneRay& r) -> bool {
            i = identity ? k : queue[k];
            r.S = &sceneOf(c, i);
            const float4 o4 = c.paths.orig[i];
            const float4 d4 = c.paths.dir[i];
            r.o = f3(o4.x, o4.y, o4.z);
            r.tMin = o4.w;
            r.tMax = kRayTMax;
            r.dn = xnormalize(f3(d4.x, d4.y, d4.z));
            if (r.S->nodeCount != 0 && !isDegenerateDir(r.dn)) {
                return true;
            }
            // empty scene, or quirk Q1: decided here without the wide traversal
            HitRec h;
            bool hit = false;
            h.tri = 0xFFFFFFFFu;
            if (r.S->nodeCount != 0) {
                hit = traceQ1(*r.S, r.o, r.dn, r.tMin, kRayTMax, false, h, c.q.overflow);
            }
            if (hit) {
                c.paths.hit[i] = make_float4(h.t, h.u, h.v, __uint_as_float(h.tri));
            }
            queue[k] = hit ? i : (i | 0x80000000u);
            return false;
        },
        [&](unsigned int k, bool hit, float t, float u, float v, uint32_t tri) {
            if (hit) {
                c.paths.hit[i] = make_float4(t, u, v, __uint_as_float(tri));
            }
            queue[k] = hit ? i : (i | 0x80000000u);
        });
}

// Occlusion of every queued shadow ray by the per-lane traversal (any hit
// below the ray's tMax); unoccluded rays mark their path's pending NEE
// contribution visible.  Flat scenes only (no instances, no visit counting).
__global__ void __launch_bounds__(PT_EXTEND_LANE_THREADS, PT_SHADOW_LANE_MIN_BLOCKS)
    k_shadow_lane(const LaunchCtx* __restrict__ cp, int iter)
{
    const LaunchCtx& c = *cp;
    extern __shared__ uint2 smemStack[];
    const unsigned int count = c.q.counts[2];
    const int par = iter & 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&c.q.rays[1], static_cast<unsigned long long>(count));
        c.q.counts[10 + (par ^ 1)] = 0u; // next shadow stage's fetch counter
    }
    uint32_t e = 0;
    laneTraversal<true, PT_SHADOW_LANE_SYNC>(count, &c.q.counts[10 + par], smemStack + threadIdx.x, static_cast<int>(blockDim.x),
        c.q.overflow,
        [&](unsigned int k, LaneRay& r) -> bool {
            e = c.q.shadowPath[k];
            r.S = &sceneOf(c, e & 0x7FFFFFFFu);
            const float4 o4 = c.q.shadowOrig[k];
            const float4 d4 = c.q.shadowDir[k];
            r.o = f3(o4.x, o4.y, o4.z);
            r.dn = xnormalize(f3(d4.x, d4.y, d4.z));
            r.tMin = kShadowBias;
            r.tMax = d4.w > 0.0f ? d4.w : kRayTMax; // emitter MIS rays end short of the light
            bool occluded = false;
            if (r.S->nodeCount != 0) {
                if (!isDegenerateDir(r.dn)) {
                    return true;
                }
                HitRec h;
                occluded = traceQ1(*r.S, r.o, r.dn, r.tMin, r.tMax, true, h, c.q.overflow);
            }
            if (!occluded) {
                const uint32_t i = e & 0x7FFFFFFFu;
                if (e & 0x80000000u) {
                    c.paths.visEmis[i] = 1;
                } else {
                    c.paths.visEnv[i] = 1;
                }
            }
            return false;
        },
        [&](unsigned int, bool occluded, float, float, float, uint32_t) {
            if (!occluded) {
                const uint32_t i = e & 0x7FFFFFFFu;
                if (e & 0x80000000u) {
                    c.paths.visEmis[i] = 1;
                } else {
                    c.paths.visEnv[i] = 1;
                }
            }
        });
}

// Closest hit of every queued path of an instanced scene by the two-level
// per-lane traversal; results and routing as k_extend_lane.
__global__ void __launch_bounds__(PT_EXTEND_LANE_THREADS, PT_EXTEND_LANE_MIN_BLOCKS)
    k_extend_lane_inst(const LaunchCtx* __restrict__ cp, int sel, bool identity, int iter)
{
    const LaunchCtx& c = *cp;
    extern __shared__ uint2 smemStack[];
    const unsigned int count = c.q.counts[sel];
    const int par = iter & 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&c.q.rays[0], static_cast<unsigned long long>(count));
        c.q.counts[sel ^ 1] = 0u;
        c.q.counts[2] = 0u;
        c.q.counts[3] = 0u;
        c.q.counts[4 + 2 * (par ^ 1)] = 0u;
        c.q.counts[5 + 2 * (par ^ 1)] = 0u;
        c.q.counts[8 + (par ^ 1)] = 0u;
    }
    uint32_t* queue = c.q.extend[sel];
    uint32_t i = 0;
    laneTraversalInst<false>(count, &c.q.counts[8 + par], smemStack + threadIdx.x, static_cast<int>(blockDim.x),
        c.q.overflow,
        [&](unsigned int k, LaneRay& r) -> bool {
            i = identity ? k : queue[k];
            r.S = &sceneOf(c, i);
            const float4 o4 = c.paths.orig[i];
            const float4 d4 = c.paths.dir[i];
            r.o = f3(o4.x, o4.y, o4.z);
            r.tMin = o4.w;
            r.tMax = kRayTMax;
            r.dn = xnormalize(f3(d4.x, d4.y, d4.z));
            return true;
        },
        [&](unsigned int k, bool hit, float t, float u, float v, uint32_t tri, uint32_t inst) {
            if (hit) {
                c.paths.hit[i] = make_float4(t, u, v, __uint_as_float(tri));
                c.paths.hitInst[i] = inst;
            }
            queue[k] = hit ? i : (i | 0x80000000u);
        });
}

// Occlusion of every queued shadow ray of an instanced scene by the two-level
// per-lane traversal; results as k_shadow_lane.
__global__ void __launch_bounds__(PT_EXTEND_LANE_THREADS, PT_SHADOW_LANE_MIN_BLOCKS)
    k_shadow_lane_inst(const LaunchCtx* __restrict__ cp, int iter)
{
    const LaunchCtx& c = *cp;
    extern __shared__ uint2 smemStack[];
    const unsigned int count = c.q.counts[2];
    const int par = iter & 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&c.q.rays[1], static_cast<unsigned long long>(count));
        c.q.counts[10 + (par ^ 1)] = 0u; // next shadow stage's fetch counter
    }
    uint32_t e = 0;
    laneTraversalInst<true>(count, &c.q.counts[10 + par], smemStack + threadIdx.x, static_cast<int>(blockDim.x),
        c.q.overflow,
        [&](unsigned int k, LaneRay& r) -> bool {
            e = c.q.shadowPath[k];
            r.S = &sceneOf(c, e & 0x7FFFFFFFu);
            const float4 o4 = c.q.shadowOrig[k];
            const float4 d4 = c.q.shadowDir[k];
            r.o = f3(o4.x, o4.y, o4.z);
            r.dn = xnormalize(f3(d4.x, d4.y, d4.z));
            r.tMin = kShadowBias;
            r.tMax = d4.w > 0.0f ? d4.w : kRayTMax; // emitter MIS rays end short of the light
            return true;
        },
        [&](unsigned int, bool occluded, float, float, float, uint32_t, uint32_t) {
            if (!occluded) {
                const uint32_t i = e & 0x7FFFFFFFu;
                if (e & 0x80000000u) {
                    c.paths.visEmis[i] = 1;
                } else {
                    c.paths.visEnv[i] = 1;
                }
            }
        });
}

// Splits the queue that k_extend_lane marked into the miss and hit queues of
// this bounce, in queue order.  A block takes a tile of 8 x 256 consecutive
// entries, counts its hits and misses per warp and row (ballots), reserves
// both output ranges with one atomic each, and writes every entry to its rank
// within the tile: two atomics per 2048 entries instead of two per warp.
constexpr int kRouteRows = 8;
// (blocks of 256 threads = 8 warps; warp 0 scans the 64 (row, warp) counts, two per lane)
static_assert(kRouteRows * 8 == 64, "the tile scan covers exactly 64 (row, warp) counts");
__global__ void __launch_bounds__(256) k_route(const LaunchCtx* __restrict__ cp, int sel, int iter)
{
    const LaunchCtx& c = *cp;
    const unsigned int count = c.q.counts[sel];
    const int par = iter & 1;
    const uint32_t* queue = c.q.extend[sel];
    __shared__ unsigned int sHit[kRouteRows * 8], sMiss[kRouteRows * 8]; // exclusive offsets per (row, warp)
    __shared__ unsigned int sBase[2];
    const unsigned int lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned int below = (1u << lane) - 1u;
    const unsigned int tile = 256u * kRouteRows;
    for (unsigned int t0 = blockIdx.x * tile; t0 < count; t0 += gridDim.x * tile) {
        uint32_t e[kRouteRows];
        unsigned int hitMask[kRouteRows], missMask[kRouteRows];
#pragma unroll
        for (int r = 0; r < kRouteRows; ++r) {
            const unsigned int k = t0 + static_cast<unsigned int>(r) * 256u + threadIdx.x;
            const bool valid = k < count;
            e[r] = valid ? queue[k] : 0u;
            const bool miss = valid && (e[r] & 0x80000000u) != 0u;
            hitMask[r] = __ballot_sync(0xffffffffu, valid && !miss);
            missMask[r] = __ballot_sync(0xffffffffu, miss);
            if (lane == 0) {
                sHit[r * 8 + warp] = __popc(hitMask[r]);
                sMiss[r * 8 + warp] = __popc(missMask[r]);
            }
        }
        __syncthreads();
        if (warp == 0) {
            // exclusive scan of the 64 (row, warp) counts in queue order, two per lane
            const unsigned int h0 = sHit[2 * lane], h1 = sHit[2 * lane + 1];
            const unsigned int m0 = sMiss[2 * lane], m1 = sMiss[2 * lane + 1];
            unsigned int h = h0 + h1, m = m0 + m1;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned int ho = __shfl_up_sync(0xffffffffu, h, d);
                const unsigned int mo = __shfl_up_sync(0xffffffffu, m, d);
                if (lane >= static_cast<unsigned int>(d)) {
                    h += ho;
                    m += mo;
                }
            }
            const unsigned int hTot = __shfl_sync(0xffffffffu, h, 31), mTot = __shfl_sync(0xffffffffu, m, 31);
            sHit[2 * lane] = h - h0 - h1;
            sHit[2 * lane + 1] = h - h1;
            sMiss[2 * lane] = m - m0 - m1;
            sMiss[2 * lane + 1] = m - m1;
            if (lane == 0) {
                sBase[0] = hTot ? atomicAdd(&c.q.counts[5 + 2 * par], hTot) : 0u;
                sBase[1] = mTot ? atomicAdd(&c.q.counts[4 + 2 * par], mTot) : 0u;
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kRouteRows; ++r) {
            if ((hitMask[r] >> lane) & 1u) {
                c.q.hitQueue[sBase[0] + sHit[r * 8 + warp] + __popc(hitMask[r] & below)] = e[r];
            } else if ((missMask[r] >> lane) & 1u) {
                c.q.missQueue[sBase[1] + sMiss[r * 8 + warp] + __popc(missMask[r] & below)] = e[r] & 0x7FFFFFFFu;
            }
        }
        __syncthreads(); // the shared offsets are rewritten by the next tile
    }
}

// Slot-ordered mode: lists the slots the shade kernels marked as the next
// bounce's extend queue, in increasing slot order within tiles of 2048 (the
// tiles in the order they reserve their ranges), and clears the marks.  The
// extend and shade kernels then read the path state of consecutive slots.
__global__ void __launch_bounds__(256) k_next_queue(const LaunchCtx* __restrict__ cp, int sel)
{
    const LaunchCtx& c = *cp;
    const unsigned int n = static_cast<unsigned int>(c.q.batch->slotCount);
    uint8_t* flag = c.q.nextFlag;
    uint32_t* out = c.q.extend[sel ^ 1];
    __shared__ unsigned int sOff[kRouteRows * 8];
    __shared__ unsigned int sBase;
    const unsigned int lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned int below = (1u << lane) - 1u;
    const unsigned int tile = 256u * kRouteRows;
    for (unsigned int t0 = blockIdx.x * tile; t0 < n; t0 += gridDim.x * tile) {
        unsigned int mask[kRouteRows];
#pragma unroll
        for (int r = 0; r < kRouteRows; ++r) {
            const unsigned int k = t0 + static_cast<unsigned int>(r) * 256u + threadIdx.x;
            const bool on = k < n && flag[k] != 0;
            if (on) {
                flag[k] = 0;
            }
            mask[r] = __ballot_sync(0xffffffffu, on);
            if (lane == 0) {
                sOff[r * 8 + warp] = __popc(mask[r]);
            }
        }
        __syncthreads();
        if (warp == 0) {
            const unsigned int a0 = sOff[2 * lane], a1 = sOff[2 * lane + 1];
            unsigned int a = a0 + a1;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned int o = __shfl_up_sync(0xffffffffu, a, d);
                if (lane >= static_cast<unsigned int>(d)) {
                    a += o;
                }
            }
            const unsigned int tot = __shfl_sync(0xffffffffu, a, 31);
            sOff[2 * lane] = a - a0 - a1;
            sOff[2 * lane + 1] = a - a1;
            if (lane == 0) {
                sBase = tot ? atomicAdd(&c.q.counts[sel ^ 1], tot) : 0u;
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kRouteRows; ++r) {
            if ((mask[r] >> lane) & 1u) {
                out[sBase + sOff[r * 8 + warp] + __popc(mask[r] & below)] =
                    t0 + static_cast<unsigned int>(r) * 256u + threadIdx.x;
            }
        }
        __syncthreads();
    }
}

// Paths whose ray left the scene: previous bounce's NEE, then the
// environment / background term (PathIntegratorRandCore.h:215-216, 338-346).
#ifndef PT_SHADE_MISS_MIN_BLOCKS
#define PT_SHADE_MISS_MIN_BLOCKS 4
#endif
template <int NW>
__global__ void __launch_bounds__(256, PT_SHADE_MISS_MIN_BLOCKS) k_shade_miss(const LaunchCtx* __restrict__ cp, int iter, int sel)
{
    const LaunchCtx& c = *cp;
    const unsigned int count = c.q.counts[4 + 2 * (iter & 1)];
    unsigned int* nextCount = &c.q.counts[sel ^ 1];
    uint32_t* nextQueue = c.q.extend[sel ^ 1];
    for (unsigned int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t i = c.q.missQueue[k];
        const Waves<NW> wv = pathWaves<NW>(c, i);
        const float4 d4 = c.paths.dir[i];
        const float3 d = f3(d4.x, d4.y, d4.z);
        const float4 r4 = c.paths.rad[i];
        const int depth = __float_as_int(r4.w);
        Col<NW> L;
        const bool sunOn = c.sun.enabled != 0;
        if (depth == 0) {
            L = sunOn ? skyCol<NW>(c, d, wv) : envCol<NW>(c, d, wv);
        } else {
            L = loadCol<NW>(r4, c.paths.radS, c.paths.capacity, i);
            if (c.paths.visEnv[i]) {
                L = cadd(L, pendingEnv<NW>(c, i));
            }
            if (c.paths.visEmis[i]) {
                L = cadd(L, pendingEmis<NW>(c, i));
            }
            const Col<NW> T = loadCol<NW>(c.paths.thr[i], c.paths.thrS, c.paths.capacity, i);
            const Col<NW> Le = sunOn ? skyCol<NW>(c, d, wv) : envCol<NW>(c, d, wv);
            const float lp = sunOn ? skyPdf(c, d) : envPdf(c.env, d);
            const float w = misBalance(fabsf(d4.w), lp);
            L = cadd(L, cmul(T, cscl(Le, w)));
        }
        writeSample<NW>(c, i, L, wv);
        recyclePath<NW>(c, i, nextCount, nextQueue);
    }
}

// Shading of the paths that hit a triangle. One thread per queued path.
template <int NW>
__global__ void __launch_bounds__(256, NW == 0 ? PT_SHADE_MIN_BLOCKS : PT_SHADE_SPEC_MIN_BLOCKS)
    k_shade(const LaunchCtx* __restrict__ cp, int sel, int iter)
{
    const LaunchCtx& c = *cp;
    const unsigned int count = c.q.counts[5 + 2 * (iter & 1)];
    const uint32_t* queue = c.q.hitQueue;
    unsigned int* nextCount = &c.q.counts[sel ^ 1];
    uint32_t* nextQueue = c.q.extend[sel ^ 1];
    const int debugFlags = c.params.brdf_debug_flags;
    const int cap = c.paths.capacity;
    for (unsigned int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t i = queue[k];
        const DevScene& S = sceneOf(c, i);
        const Waves<NW> wv = pathWaves<NW>(c, i);
        const float4 r4 = c.paths.rad[i];
        const int depth = __float_as_int(r4.w);
        // RGB: the radiance stays in registers through the bounce.  Spectral: it
        // is updated in memory (NEE of the previous bounce and the emission, in
        // one read-modify-write below) and reloaded only by a path that ends.
        Col<NW> L = czero<NW>();
        if constexpr (NW == 0) {
            L = loadCol<NW>(r4, c.paths.radS, cap, i);
            // NEE contributions of the previous bounce, in the reference's order
            // (the flags are clear for a path that starts at this bounce).
            if (c.paths.visEnv[i]) {
                L = cadd(L, pendingEnv<NW>(c, i));
            }
            if (c.paths.visEmis[i]) {
                L = cadd(L, pendingEmis<NW>(c, i));
            }
        }
        const float4 h4 = c.paths.hit[i];
        const uint32_t tri = __float_as_uint(h4.w);
        const float4 d4 = c.paths.dir[i];
        const float3 d = f3(d4.x, d4.y, d4.z);
        bool done = false;
        bool pendEnv = false, pendEmis = false;
        bool cont = false;
        if (depth >= c.maxDepth) {
            done = true;
        } else {
            const float4 o4 = c.paths.orig[i];
            const float4 t4 = c.paths.thr[i];
            Col<NW> T;
            if constexpr (NW == 0) {
                T = loadCol<NW>(t4, c.paths.thrS, cap, i);
            } else {
                if (depth == 0) {
#pragma unroll
                    for (int q = 0; q < NW; ++q) {
                        T.v[q] = 1.0f;
                    }
                } else {
                    T = loadCol<NW>(t4, c.paths.thrS, cap, i);
                }
            }
            float eta = t4.w;
            const float t = h4.x;
            const float3 pos = xadd(f3(o4.x, o4.y, o4.z), xscl(d, t));
            const float3 dn = xnormalize(d);
            const TriShade sh = S.shade[tri];
            float3 n;
            float tu, tv;
            if (S.instanceCount == 0) {
                hitShading(sh, dn, h4.y, h4.z, n, tu, tv);
            } else {
                hitShadingAt(S, sh, c.paths.hitInst[i], dn, h4.y, h4.z, n, tu, tv);
            }
            const uint32_t mi = __float_as_uint(sh.d.w);
            const pt_material& srcMat =
                (S.materials != nullptr && mi < S.materialCount) ? S.materials[mi] : kFallbackMaterial;
            Ctx cx;
            cx.m = resolveMaterial(srcMat, tu, tv, S.textures, S.textureCount);
            cx.w = computeLobes(cx.m);
            cx.n = n;
            cx.wo = scl3(d, -1.0f);
            cx.eta = eta;
            cx.debug = 0;
            // Emitter MIS mode: at a vertex that takes part (emitterMisVertex), the
            // emissive NEE and the BSDF-sampled emitter hits share the light by the
            // balance heuristic, outside the transmit cones and above the surface;
            // elsewhere the reference's estimator is kept.
            const bool emitterMis = c.params.emitter_mis == 1;
            const bool misVertex = emitterMis && S.instanceCount == 0 && debugFlags == 0 && emitterMisVertex(cx);
            // weight of this hit's emission: the previous vertex took part (pdf > 0) and
            // emissive NEE can pick this point (front face of a listed emitter)
            float emitW = 1.0f;
            if (emitterMis && depth > 0 && d4.w > 0.0f && S.emitPdfArea != nullptr && cx.m.emission != 0.0f) {
                const float pa = S.emitPdfArea[tri];
                if (pa > 0.0f) {
                    const float3 ev0 = loadOrigVertex(S, tri, 0), ev1 = loadOrigVertex(S, tri, 1),
                                 ev2 = loadOrigVertex(S, tri, 2);
                    const float3 ng = normalize3(cross3(sub3(ev1, ev0), sub3(ev2, ev0)));
                    const float cl = fmax2(0.0f, -dot3(ng, dn));
                    if (cl > 0.0f) {
                        const float lp = pa * (t * t * dot3(d, d)) / cl;
                        emitW = misBalance(d4.w, lp);
                    }
                }
            }
            const float emission = cx.m.emission * emitW;
            // base colour at the path's wavelengths (spectral mode)
            Col<NW> rho;
            float4 scatterCoef = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if constexpr (NW == 0) {
                rho.c = f3(cx.m.r, cx.m.g, cx.m.b);
                // emission (PathIntegratorRandCore.h:248)
                L = cadd(L, cmul(T, Col<0>{f3(cx.m.r * emission, cx.m.g * emission, cx.m.b * emission)}));
            } else {
                float4 baseCoef;
                matCoefs(S, mi, srcMat, tu, tv, baseCoef, scatterCoef);
                rho = coefCol<NW>(baseCoef, wv);
                cx.m.r = 0.0f; // evalCol's affine form (the RGB base is not read again)
                cx.m.g = 1.0f;
                cx.m.b = 1.0f;
                Col<NW> Lm = depth == 0 ? czero<NW>() : loadCol<NW>(r4, c.paths.radS, cap, i);
                if (c.paths.visEnv[i]) {
                    Lm = cadd(Lm, pendingEnv<NW>(c, i));
                }
                if (c.paths.visEmis[i]) {
                    Lm = cadd(Lm, pendingEmis<NW>(c, i));
                }
                // emission (PathIntegratorRandCore.h:248)
#pragma unroll
                for (int q = 0; q < NW; ++q) {
                    Lm.v[q] = Lm.v[q] + T.v[q] * (rho.v[q] * emission);
                }
                storeCol<NW>(nullptr, c.paths.radS, cap, i, Lm, 0.0f);
            }
            curandStateXORWOW st;
            rngLoad(c.paths, i, st);
            // environment NEE (PathIntegratorRandCore.h:65-108); with a distant
            // light, one more draw first picks the light or the environment
            if (!skipsEnvNee(cx.m)) {
                const bool sunOn = c.sun.enabled != 0;
                const float uSel = sunOn ? curand_uniform(&st) : 0.0f;
                const float u1 = curand_uniform(&st);
                const float u2 = curand_uniform(&st);
                float lp = 0.0f;
                float3 wi;
                if (!sunOn) {
                    wi = envSample(c.env, u1, u2, lp);
                } else if (uSel < c.sun.select) {
                    wi = sunSample(c.sun, u1, u2);
                    lp = skyPdf(c, wi);
                } else {
                    wi = envSample(c.env, u1, u2, lp);
                    lp = lp > kMinPdf ? skyPdf(c, wi) : 0.0f;
                }
                if (lp > kMinPdf) {
                    const float ct = fmax2(0.0f, dot3(n, wi));
                    const Col<NW> Le = sunOn ? skyCol<NW>(c, wi, wv) : envCol<NW>(c, wi, wv);
                    // A light of exactly zero radiance (a black background) contributes
                    // exactly zero for any finite BSDF value: the BSDF is not evaluated.
                    if (ct > 0.0f && cnonzero(Le)) {
                        const Col<NW> f = evalCol<NW>(cx, wi, rho, scatterCoef, wv);
                        const float bp = bsdfPdf(cx, wi);
                        const float kw = misBalance(lp, bp) * ct / lp;
                        const Col<NW> contrib = cmul(T, cmul(f, cscl(Le, kw)));
                        // A contribution of exactly zero adds nothing whether or not the light
                        // is occluded, so its shadow ray is not traced (black backgrounds).
                        if (cnonzero(contrib)) {
                            storeCol<NW>(c.paths.neeEnv, c.paths.neeEnvS, cap, i, contrib, 0.0f);
                            const uint32_t s = warpPush(&c.q.counts[2]);
                            const float3 so = add3(pos, scl3(n, kShadowBias));
                            c.q.shadowPath[s] = i;
                            c.q.shadowOrig[s] = make_float4(so.x, so.y, so.z, 0.0f);
                            c.q.shadowDir[s] = make_float4(wi.x, wi.y, wi.z, 0.0f);
                            pendEnv = true;
                        }
                    }
                }
            }
            // emissive NEE (PathIntegratorRandCore.h:110-167)
            if (S.emissiveCount > 0) {
                const float uTri = curand_uniform(&st);
                const float u1 = curand_uniform(&st);
                const float u2 = curand_uniform(&st);
                float3 lpos, ln, LeRgb, ev0, ev1, ev2;
                float ap;
                uint32_t etri = 0u;
                if (sampleEmissive(S, &kFallbackMaterial, uTri, u1, u2, lpos, ln, LeRgb, ap, ev0, ev1, ev2, &etri)) {
                    const float3 tl = sub3(lpos, pos);
                    const float d2 = dot3(tl, tl);
                    if (d2 > kMinPdf) {
                        const float3 wi = normalize3(tl);
                        const float ct = fmax2(0.0f, dot3(n, wi));
                        const float cl = fmax2(0.0f, dot3(ln, scl3(wi, -1.0f)));
                        if (ct > 0.0f && cl > 0.0f) {
                            const float lp = ap * d2 / cl;
                            // The reference's emissive shadow ray runs to tMax = 1e6
                            // (LightSamplingCore.h:360-369), so the sampled emitter triangle
                            // itself occludes it whenever the ray hits that triangle.  An
                            // any-hit query is true as soon as one triangle is hit, so testing
                            // the emitter first (same origin, direction and rounding as the
                            // shadow stage) decides those rays without a traversal -- and
                            // without evaluating the BSDF for a term that adds nothing.
                            const float3 so = add3(pos, scl3(wi, kShadowBias));
                            const float3 sdn = xnormalize(wi);
                            bool occludedBySelf = false;
                            // emitter MIS: the shadow ray ends just short of the light
                            // sample, so the emitter (and coplanar neighbours) never block it
                            float shadowTMax = 0.0f; // 0: the reference's kRayTMax
                            if (misVertex && !inTransmitCones(cx, wi)) {
                                shadowTMax = (sqrtf(d2) - kShadowBias) * (1.0f - 1.0e-4f);
                            } else if (!isDegenerateDir(sdn)) {
                                float th, tu2, tv2;
                                occludedBySelf = intersectTriExact(so, sdn, ev0, ev1, ev2, kShadowBias, kRayTMax, th,
                                                     tu2, tv2) && th < kRayTMax;
                            }
                            if (lp > kMinPdf && !occludedBySelf) {
                                Col<NW> Le;
                                if constexpr (NW == 0) {
                                    Le.c = LeRgb;
                                } else {
                                    // the emitter's own material colour (no texture), as sampleEmissive
                                    const uint32_t emi = __float_as_uint(S.shade[etri].d.w);
                                    const bool ok = S.matSpec != nullptr && S.materials != nullptr &&
                                        emi < S.materialCount;
                                    const float4 q = ok ? S.matSpec[2 * emi] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                                    const float em = ok ? S.materials[emi].emission : 0.0f;
                                    Le = cscl(coefCol<NW>(q, wv), em);
                                }
                                const Col<NW> f = evalCol<NW>(cx, wi, rho, scatterCoef, wv);
                                const float bp = bsdfPdf(cx, wi);
                                const float kw = misBalance(lp, bp) * ct / lp;
                                const Col<NW> contrib = cmul(T, cmul(f, cscl(Le, kw)));
                                if (cnonzero(contrib)) {
                                    storeCol<NW>(c.paths.neeEmis, c.paths.neeEmisS, cap, i, contrib, 0.0f);
                                    const uint32_t s = warpPush(&c.q.counts[2]);
                                    c.q.shadowPath[s] = i | 0x80000000u;
                                    c.q.shadowOrig[s] = make_float4(so.x, so.y, so.z, 0.0f);
                                    c.q.shadowDir[s] = make_float4(wi.x, wi.y, wi.z, shadowTMax);
                                    pendEmis = true;
                                }
                            }
                        }
                    }
                }
            }
            // BSDF sample (PathIntegratorRandCore.h:280-321)
            cx.debug = debugFlags;
            const float u1 = curand_uniform(&st);
            const float u2 = curand_uniform(&st);
            const BsdfSample smp = bsdfSample(cx, u1, u2);
            if (!smp.valid || smp.pdf <= kMinPdf) {
                done = true;
            } else {
                const Col<NW> f = evalCol<NW>(cx, smp.dir, rho, scatterCoef, wv);
                T = throughCol<NW>(T, cx, smp, f, rho);
                if (smp.sss && smp.sssSteps > 0) {
                    // subsurface tier B (PathIntegratorRandCore.h:169-204)
                    const float maxR = maxScatter(cx.m);
                    if (maxR > kMinRadius) {
                        for (int stp = 0; stp < smp.sssSteps; ++stp) {
                            (void)curand_uniform(&st);
                            (void)curand_uniform(&st);
                            const float u3 = curand_uniform(&st);
                            const float mfp = maxR * (-logf(fmax2(1.0e-8f, u3)));
                            const float surv = expf(-mfp / maxR);
                            T = cmul(T, cscl(rho, surv));
                        }
                        const float ed = sqrtf(dot3(smp.exitOffset, smp.exitOffset));
                        if (ed > 0.0f) {
                            T = cscl(T, expf(-ed / maxR));
                        }
                    }
                }
                if constexpr (NW == 0) {
                    // debug tint of glass paths (RGB display aid; not applied to spectra)
                    if (debugFlags & kDbgTintGlass) {
                        T.c = smp.transmitted ? mul3(T.c, f3(0.2f, 1.0f, 0.2f)) : mul3(T.c, f3(1.0f, 0.2f, 0.2f));
                    }
                }
                const float tl = pathWeight<NW>(T);
                if (!isfinite(tl) || tl <= 0.0f || tl > 1.0e8f) {
                    done = true;
                } else {
                    bool survive = true;
                    if (depth >= c.rrMinDepth) {
                        const float surv = fmin2(0.95f, fmax2(tl, 0.05f));
                        if (curand_uniform(&st) > surv) {
                            survive = false;
                        } else {
                            T = cscl(T, 1.0f / surv);
                        }
                    }
                    if (!survive) {
                        done = true;
                    } else {
                        eta = smp.nextEta;
                        const float bias = fmax2(1.0e-4f, 1.0e-3f * t);
                        const float sign = dot3(n, smp.dir) >= 0.0f ? 1.0f : -1.0f;
                        const float3 no = xadd(pos, xscl(n, __fmul_rn(sign, bias)));
                        c.paths.orig[i] = make_float4(no.x, no.y, no.z, bias);
                        // emitter MIS mode: a negative pdf marks a vertex that does not
                        // take part (the next hit's emission keeps weight 1)
                        const bool misSample = misVertex && !smp.transmitted && !smp.sss &&
                            dot3(n, smp.dir) > 0.0f && !inTransmitCones(cx, smp.dir);
                        c.paths.dir[i] = make_float4(smp.dir.x, smp.dir.y, smp.dir.z,
                            (emitterMis && !misSample) ? -smp.pdf : smp.pdf);
                        storeCol<NW>(c.paths.thr, c.paths.thrS, cap, i, T, eta);
                        cont = true;
                    }
                }
            }
            rngStore(c.paths, i, st);
        }
        (void)done;
        if constexpr (NW == 0) {
            c.paths.visEnv[i] = 0;
            c.paths.visEmis[i] = 0;
            if (cont) {
                storeCol<NW>(c.paths.rad, c.paths.radS, cap, i, L, __int_as_float(depth + 1));
                queueNext(c, i, nextCount, nextQueue);
            } else if (pendEnv || pendEmis) {
                storeCol<NW>(c.paths.rad, c.paths.radS, cap, i, L, __int_as_float(depth));
                const uint32_t s = warpPush(&c.q.counts[3]);
                c.q.finish[s] = i;
            } else {
                writeSample<NW>(c, i, L, wv);
                recyclePath<NW>(c, i, nextCount, nextQueue);
            }
        } else {
            if (cont || pendEnv || pendEmis) {
                // the radiance is in radS already
                c.paths.rad[i] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(cont ? depth + 1 : depth));
                if (cont) {
                    queueNext(c, i, nextCount, nextQueue);
                } else {
                    const uint32_t s = warpPush(&c.q.counts[3]);
                    c.q.finish[s] = i;
                }
            } else {
                L = loadCol<NW>(r4, c.paths.radS, cap, i);
                if (depth >= c.maxDepth) {
                    // (no read-modify-write happened: add the previous bounce's NEE here)
                    if (c.paths.visEnv[i]) {
                        L = cadd(L, pendingEnv<NW>(c, i));
                    }
                    if (c.paths.visEmis[i]) {
                        L = cadd(L, pendingEmis<NW>(c, i));
                    }
                }
                writeSample<NW>(c, i, L, wv);
                recyclePath<NW>(c, i, nextCount, nextQueue);
            }
            c.paths.visEnv[i] = 0;
            c.paths.visEmis[i] = 0;
        }
    }
}

// Occlusion of the queued shadow rays (LightSamplingCore.h:187-197, 360-369).
template <bool Count, bool Inst>
__global__ void __launch_bounds__(256, 4) k_shadow(const LaunchCtx* __restrict__ cp, int iter)
{
    const LaunchCtx& c = *cp;
    extern __shared__ uint2 smemStack[];
    const unsigned int count = c.q.counts[2];
    const int par = iter & 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&c.q.rays[1], static_cast<unsigned long long>(count));
        c.q.counts[10 + (par ^ 1)] = 0u; // next shadow stage's fetch counter
    }
    unsigned int* fetch = &c.q.counts[10 + par];
    for (;;) {
        const unsigned int k = warpFetch(fetch);
        if (__shfl_sync(0xffffffffu, k, 0) >= count) {
            break;
        }
        if (k >= count) {
            continue;
        }
        const uint32_t e = c.q.shadowPath[k];
        const float4 o4 = c.q.shadowOrig[k];
        const float4 d4 = c.q.shadowDir[k];
        const float3 dn = xnormalize(f3(d4.x, d4.y, d4.z));
        HitRec h;
        const float tMax = d4.w > 0.0f ? d4.w : kRayTMax; // emitter MIS rays end short of the light
        const bool occluded = traceRay<true, Count, Inst>(sceneOf(c, e & 0x7FFFFFFFu), f3(o4.x, o4.y, o4.z), dn, kShadowBias, tMax, h,
            c.q.overflow, c.q.visits + 2, smemStack + threadIdx.x, blockDim.x);
        if (!occluded) {
            const uint32_t i = e & 0x7FFFFFFFu;
            if (e & 0x80000000u) {
                c.paths.visEmis[i] = 1;
            } else {
                c.paths.visEnv[i] = 1;
            }
        }
    }
}

// Paths that terminated while their NEE shadow rays were in flight.
template <int NW>
__global__ void __launch_bounds__(256) k_finalize(const LaunchCtx* __restrict__ cp, int sel)
{
    const LaunchCtx& c = *cp;
    const unsigned int count = c.q.counts[3];
    unsigned int* nextCount = &c.q.counts[sel ^ 1];
    uint32_t* nextQueue = c.q.extend[sel ^ 1];
    for (unsigned int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t i = c.q.finish[k];
        const Waves<NW> wv = pathWaves<NW>(c, i);
        Col<NW> L = loadCol<NW>(c.paths.rad[i], c.paths.radS, c.paths.capacity, i);
        if (c.paths.visEnv[i]) {
            L = cadd(L, pendingEnv<NW>(c, i));
        }
        if (c.paths.visEmis[i]) {
            L = cadd(L, pendingEmis<NW>(c, i));
        }
        writeSample<NW>(c, i, L, wv);
        recyclePath<NW>(c, i, nextCount, nextQueue);
    }
}

// Per pixel: fold the batch's samples in sample order (PathTracer.cu:232-272).
__global__ void __launch_bounds__(256) k_accumulate(const LaunchCtx* __restrict__ cp, int activeCount, int batch)
{
    const LaunchCtx& c = *cp;
    const int* active = c.acc.active[c.activeSel];
    const int maxSpp = c.params.max_samples_per_pixel;
    const int minSpp = c.params.min_samples;
    const float thr = c.params.relative_error_threshold;
    const bool stdErr = c.params.adaptive_criterion == 1 || c.params.adaptive_criterion == 2;
    // criterion 2: a pixel all of whose samples are black stops after max(min spp, 64) samples
    const bool blackStops = c.params.adaptive_criterion == 2;
    const uint32_t blackSpp = static_cast<uint32_t>(minSpp > 64 ? minSpp : 64);
    for (int li = blockIdx.x * blockDim.x + threadIdx.x; li < activeCount; li += gridDim.x * blockDim.x) {
        const int p = active[li];
        uint8_t conv = c.acc.converged[p];
        if (conv) {
            continue;
        }
        uint32_t n = c.acc.counts[p];
        float mean = c.acc.lumMean[p];
        float m2 = c.acc.m2[p];
        float4 a = c.acc.acc[p];
        for (int s = 0; s < batch && !conv; ++s) {
            const float4 smp = c.acc.samples[static_cast<size_t>(s) * activeCount + li];
            const float sl =
                __fadd_rn(__fadd_rn(__fmul_rn(smp.x, 0.2126f), __fmul_rn(smp.y, 0.7152f)), __fmul_rn(smp.z, 0.0722f));
            const float fn1 = static_cast<float>(n + 1);
            const float delta = __fsub_rn(sl, mean);
            const float nm = __fadd_rn(mean, __fdiv_rn(delta, fn1));
            m2 = __fadd_rn(m2, __fmul_rn(delta, __fsub_rn(sl, nm)));
            mean = nm;
            const float invN = __fdiv_rn(1.0f, fn1);
            const float fn = static_cast<float>(n);
            a.x = __fmul_rn(__fadd_rn(__fmul_rn(a.x, fn), smp.x), invN);
            a.y = __fmul_rn(__fadd_rn(__fmul_rn(a.y, fn), smp.y), invN);
            a.z = __fmul_rn(__fadd_rn(__fmul_rn(a.z, fn), smp.z), invN);
            a.w = 1.0f;
            ++n;
            if (maxSpp > 0 && n >= static_cast<uint32_t>(maxSpp)) {
                conv = 1;
                break;
            }
            if ((n % 4u) != 0u) {
                continue;
            }
            // isAdaptivePixelConverged (PathTracerAdaptiveSampling.h:16-40)
            if (n >= static_cast<uint32_t>(minSpp) && n > 0 && mean >= 1.0e-5f) {
                const float var = __fdiv_rn(m2, static_cast<float>(n));
                float rel = __fdiv_rn(__fsqrt_rn(var), fmaxf(mean, 1.0e-4f));
                if (stdErr) {
                    rel = __fdiv_rn(rel, __fsqrt_rn(static_cast<float>(n)));
                }
                if (rel < thr) {
                    conv = 1;
                }
            } else if (blackStops && n >= blackSpp && mean == 0.0f && m2 == 0.0f) {
                conv = 1;
            }
        }
        c.acc.counts[p] = n;
        c.acc.lumMean[p] = mean;
        c.acc.m2[p] = m2;
        c.acc.acc[p] = a;
        c.acc.converged[p] = conv;
    }
}

// Per-scene active ranges (the active list is sorted by pixel) and job
// offsets of the current batch: scene s owns active entries
// [sceneActiveStart[s], sceneActiveStart[s + 1]) and jobs
// [sceneJobStart[s], sceneJobStart[s + 1]).
__global__ void k_scene_jobs(const LaunchCtx* __restrict__ cp, int sceneCount, int waves)
{
    const LaunchCtx& c = *cp;
    const int n = c.q.batch->activeCount;
    const int* active = c.acc.active[c.activeSel];
    for (int s = threadIdx.x; s <= sceneCount; s += blockDim.x) {
        uint32_t pos = static_cast<uint32_t>(n);
        if (s < sceneCount) {
            const int key = static_cast<int>(c.views[s].pixelBase);
            int lo = 0, hi = n; // first entry >= key
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (active[mid] < key) {
                    lo = mid + 1;
                } else {
                    hi = mid;
                }
            }
            pos = static_cast<uint32_t>(lo);
        }
        c.sceneActiveStart[s] = pos;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long acc = 0;
        for (int s = 0; s < sceneCount; ++s) {
            c.sceneJobStart[s] = acc;
            acc += static_cast<unsigned long long>(c.sceneActiveStart[s + 1] - c.sceneActiveStart[s]) *
                static_cast<unsigned long long>(waves);
        }
        c.sceneJobStart[sceneCount] = acc;
    }
}

// A pixel stays on the active list until it converged or reached the sample
// cap (the tests of compactActiveListKernel, PathTracer.cu:385-391).
struct KeepActive {
    const uint8_t* converged;
    const uint32_t* counts;
    int maxSpp;
    __device__ __forceinline__ bool operator()(int p) const
    {
        return converged[p] == 0 && !(maxSpp > 0 && counts[p] >= static_cast<uint32_t>(maxSpp));
    }
};
// Select predicate / value over the entries of an active list.
struct KeepListed {
    const int* list;
    KeepActive keep;
    __device__ __forceinline__ bool operator()(long long i) const { return keep(list[i]); }
};
struct ListedPixel {
    const int* list;
    __device__ __forceinline__ int operator()(long long i) const { return list[i]; }
};

__global__ void k_reset(const LaunchCtx* __restrict__ cp, int pixels)
{
    const LaunchCtx& c = *cp;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < pixels; i += gridDim.x * blockDim.x) {
        c.acc.acc[i] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        c.acc.counts[i] = 0;
        c.acc.lumMean[i] = 0.0f;
        c.acc.m2[i] = 0.0f;
        c.acc.converged[i] = 0;
        c.acc.active[0][i] = i;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.acc.activeCount[0] = pixels;
        c.acc.activeCount[1] = 0;
    }
}

__global__ void __launch_bounds__(256) k_trace_rays(DevScene S, int n, const float* o, const float* d, const float* tmin,
    const float* tmax, uint8_t* hit, float* t, uint32_t* tri, float* normal, float* uv, unsigned int* overflow)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float3 ro = f3(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
        const float3 dn = xnormalize(f3(d[3 * i], d[3 * i + 1], d[3 * i + 2]));
        HitRec h;
        const bool ok = traceRay<false, false, true>(S, ro, dn, tmin[i], tmax[i], h, overflow);
        hit[i] = ok ? 1 : 0;
        float3 nn = f3(0.0f, 0.0f, 0.0f);
        float tu = 0.0f, tv = 0.0f;
        if (ok) {
            hitShadingAt(S, S.shade[h.tri], h.inst, dn, h.u, h.v, nn, tu, tv);
        }
        if (t) {
            t[i] = ok ? h.t : 0.0f;
        }
        if (tri) {
            tri[i] = ok ? h.tri : 0u;
        }
        if (normal) {
            normal[3 * i] = nn.x;
            normal[3 * i + 1] = nn.y;
            normal[3 * i + 2] = nn.z;
        }
        if (uv) {
            uv[2 * i] = tu;
            uv[2 * i + 1] = tv;
        }
    }
}

// Region render (clearRegionAccumulatorKernel, PathTracer.cu:305-344): clears
// the accumulators of the pixels in [minX, maxX] x [minY, maxY] when `clear`
// and makes them the active list, row by row (so it stays sorted).
__global__ void k_region(const LaunchCtx* __restrict__ cp, int width, int minX, int minY, int maxX, int maxY, bool clear)
{
    const LaunchCtx& c = *cp;
    const int rw = maxX - minX + 1, rh = maxY - minY + 1;
    const int n = rw * rh;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int idx = (minY + t / rw) * width + minX + t % rw;
        if (clear) {
            c.acc.acc[idx] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            c.acc.counts[idx] = 0;
            c.acc.lumMean[idx] = 0.0f;
            c.acc.m2[idx] = 0.0f;
            c.acc.converged[idx] = 0;
        }
        c.acc.active[0][t] = idx;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.acc.activeCount[0] = n;
        c.acc.activeCount[1] = 0;
    }
}

__global__ void k_rng_tape(int width, int height, int firstWave, int waves, int stride, int seedOffset, float* out)
{
    const long long P = static_cast<long long>(width) * height;
    const long long total = P * waves;
    for (long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; k < total;
         k += static_cast<long long>(gridDim.x) * blockDim.x) {
        const uint32_t w = static_cast<uint32_t>(k / P);
        const uint32_t p = static_cast<uint32_t>(k % P);
        const uint32_t wave = static_cast<uint32_t>(firstWave) + w;
        const uint32_t seed = p * 747796405u + wave + (wave + 1u + static_cast<uint32_t>(seedOffset)) * 2891336453u;
        curandStateXORWOW st;
        curand_init(seed, 0ull, 0ull, &st);
        float* row = out + k * stride;
        for (int j = 0; j < stride; ++j) {
            row[j] = curand_uniform(&st);
        }
    }
}

inline int gridFor(long long n, int block = 256, int cap = 148 * 16)
{
    long long g = (n + block - 1) / block;
    if (g < 1) {
        g = 1;
    }
    return static_cast<int>(g < cap ? g : cap);
}

} // namespace

void launchGenerate(const LaunchCtx* d, int count, int extendSel, int nw, cudaStream_t s, unsigned long long jobOffset)
{
    if (nw == 8) {
        k_generate<8><<<gridFor(count), 256, 0, s>>>(d, count, extendSel, jobOffset);
    } else if (nw == 4) {
        k_generate<4><<<gridFor(count), 256, 0, s>>>(d, count, extendSel, jobOffset);
    } else {
        k_generate<0><<<gridFor(count), 256, 0, s>>>(d, count, extendSel, jobOffset);
    }
}
void launchExtend(const LaunchCtx* c, int sel, bool identity, int iter, int grid, bool count, bool inst, bool lane,
    cudaStream_t s)
{
    const size_t smem = sizeof(uint2) * kSharedStack * 256;
    if (inst) {
        if (count) {
            k_extend<true, true><<<grid, 256, smem, s>>>(c, sel, identity, iter);
        } else if (lane) {
            k_extend_lane_inst<<<grid, PT_EXTEND_LANE_THREADS, sizeof(uint2) * kSharedStack * PT_EXTEND_LANE_THREADS,
                s>>>(c, sel, identity, iter);
            k_route<<<grid, 256, 0, s>>>(c, sel, iter);
        } else {
            k_extend<false, true><<<grid, 256, smem, s>>>(c, sel, identity, iter);
        }
    } else if (count) {
        k_extend<true, false><<<grid, 256, smem, s>>>(c, sel, identity, iter);
    } else if (lane) {
        k_extend_lane<<<grid, PT_EXTEND_LANE_THREADS, sizeof(uint2) * kSharedStack * PT_EXTEND_LANE_THREADS, s>>>(c, sel,
            identity, iter);
        k_route<<<grid, 256, 0, s>>>(c, sel, iter);
    } else {
        k_extend<false, false><<<grid, 256, smem, s>>>(c, sel, identity, iter);
    }
}
int extendKernels(bool count, bool inst, bool lane)
{
    return (!count && lane) ? 2 : 1;
}
void launchNextQueue(const LaunchCtx* c, int sel, int grid, cudaStream_t s)
{
    k_next_queue<<<grid, 256, 0, s>>>(c, sel);
}
int extendLaneInstOccupancy()
{
    int blocks = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_extend_lane_inst, PT_EXTEND_LANE_THREADS,
        sizeof(uint2) * kSharedStack * PT_EXTEND_LANE_THREADS);
    return blocks > 0 ? blocks : 1;
}
int shadowLaneInstOccupancy()
{
    int blocks = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_shadow_lane_inst, PT_EXTEND_LANE_THREADS,
        sizeof(uint2) * kSharedStack * PT_EXTEND_LANE_THREADS);
    return blocks > 0 ? blocks : 1;
}
int shadowLaneOccupancy()
{
    int blocks = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_shadow_lane, PT_EXTEND_LANE_THREADS,
        sizeof(uint2) * kSharedStack * PT_EXTEND_LANE_THREADS);
    return blocks > 0 ? blocks : 1;
}
int shadeMissOccupancy()
{
    int blocks = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_shade_miss<8>, 256, 0);
    return blocks > 0 ? blocks : 1;
}
int extendLaneOccupancy()
{
    int blocks = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_extend_lane, PT_EXTEND_LANE_THREADS,
        sizeof(uint2) * kSharedStack * PT_EXTEND_LANE_THREADS);
    return blocks > 0 ? blocks : 1;
}
void launchShadeMiss(const LaunchCtx* c, int iter, int sel, int grid, int nw, cudaStream_t s)
{
    if (nw == 8) {
        k_shade_miss<8><<<grid, 256, 0, s>>>(c, iter, sel);
    } else if (nw == 4) {
        k_shade_miss<4><<<grid, 256, 0, s>>>(c, iter, sel);
    } else {
        k_shade_miss<0><<<grid, 256, 0, s>>>(c, iter, sel);
    }
}
void launchShade(const LaunchCtx* c, int sel, int iter, int grid, int nw, cudaStream_t s)
{
    if (nw == 8) {
        k_shade<8><<<grid, 256, 0, s>>>(c, sel, iter);
    } else if (nw == 4) {
        k_shade<4><<<grid, 256, 0, s>>>(c, sel, iter);
    } else {
        k_shade<0><<<grid, 256, 0, s>>>(c, sel, iter);
    }
}
void launchShadow(const LaunchCtx* c, int iter, int grid, bool count, bool inst, bool lane, cudaStream_t s)
{
    const size_t smem = sizeof(uint2) * kSharedStack * 256;
    if (PT_SHADOW_LANE && lane && !count) {
        if (inst) {
            k_shadow_lane_inst<<<grid, PT_EXTEND_LANE_THREADS, sizeof(uint2) * kSharedStack * PT_EXTEND_LANE_THREADS,
                s>>>(c, iter);
        } else {
            k_shadow_lane<<<grid, PT_EXTEND_LANE_THREADS, sizeof(uint2) * kSharedStack * PT_EXTEND_LANE_THREADS, s>>>(c,
                iter);
        }
    } else if (inst) {
        if (count) {
            k_shadow<true, true><<<grid, 256, smem, s>>>(c, iter);
        } else {
            k_shadow<false, true><<<grid, 256, smem, s>>>(c, iter);
        }
    } else if (count) {
        k_shadow<true, false><<<grid, 256, smem, s>>>(c, iter);
    } else {
        k_shadow<false, false><<<grid, 256, smem, s>>>(c, iter);
    }
}
int shadeOccupancy(int nw)
{
    // (one value per instantiation, computed once per process; renderers on
    // several host threads may race to fill it, with the same value)
    static std::atomic<int> occ[3] = {{0}, {0}, {0}};
    const int k = nw == 8 ? 2 : (nw == 4 ? 1 : 0);
    if (occ[k].load(std::memory_order_relaxed) == 0) {
        int b = 1;
        if (nw == 8) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<8>, 256, 0);
        } else if (nw == 4) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<4>, 256, 0);
        } else {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<0>, 256, 0);
        }
        occ[k].store(b > 0 ? b : 1, std::memory_order_relaxed);
    }
    return occ[k].load(std::memory_order_relaxed);
}
void stageOccupancy(int& extendBlocks, int& shadeBlocks, int& shadowBlocks)
{
    extendBlocks = shadeBlocks = shadowBlocks = 1;
    const size_t smem = sizeof(uint2) * kSharedStack * 256;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&extendBlocks, k_extend<false, false>, 256, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shadeBlocks, k_shade<0>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shadowBlocks, k_shadow<false, false>, 256, smem);
}
void launchFinalize(const LaunchCtx* c, int sel, int grid, int nw, cudaStream_t s)
{
    if (nw == 8) {
        k_finalize<8><<<grid, 256, 0, s>>>(c, sel);
    } else if (nw == 4) {
        k_finalize<4><<<grid, 256, 0, s>>>(c, sel);
    } else {
        k_finalize<0><<<grid, 256, 0, s>>>(c, sel);
    }
}
void launchAccumulate(const LaunchCtx* c, int activeCount, int batch, cudaStream_t s)
{
    k_accumulate<<<gridFor(activeCount), 256, 0, s>>>(c, activeCount, batch);
}
size_t compactTempBytes(int n)
{
    return selectTempBytes(n);
}
cudaError_t launchCompactStable(const int* in, int* out, int* outCount, int n, const uint8_t* converged,
    const uint32_t* counts, int maxSpp, void* temp, size_t tempBytes, cudaStream_t s)
{
    return launchSelect(static_cast<long long>(n), KeepListed{in, KeepActive{converged, counts, maxSpp}},
        ListedPixel{in}, out, outCount, temp, tempBytes, s);
}
void launchSceneJobs(const LaunchCtx* c, int sceneCount, int waves, cudaStream_t s)
{
    k_scene_jobs<<<1, 1024, 0, s>>>(c, sceneCount, waves);
}
void launchResetAccum(const LaunchCtx* c, int pixels, cudaStream_t s) { k_reset<<<gridFor(pixels), 256, 0, s>>>(c, pixels); }
void launchTraceRays(const DevScene& S, int n, const float* o, const float* d, const float* tmin, const float* tmax,
    uint8_t* hit, float* t, uint32_t* tri, float* normal, float* uv, cudaStream_t s, unsigned int* overflow)
{
    k_trace_rays<<<gridFor(n), 256, 0, s>>>(S, n, o, d, tmin, tmax, hit, t, tri, normal, uv, overflow);
}
void launchRngTape(int width, int height, int firstWave, int waves, int stride, int seedOffset, float* out,
    cudaStream_t s)
{
    k_rng_tape<<<gridFor(static_cast<long long>(width) * height * waves), 256, 0, s>>>(width, height, firstWave, waves,
        stride, seedOffset, out);
}
void launchRegion(const LaunchCtx* c, int width, int minX, int minY, int maxX, int maxY, bool clear, cudaStream_t s)
{
    const long long n = static_cast<long long>(maxX - minX + 1) * (maxY - minY + 1);
    k_region<<<gridFor(n), 256, 0, s>>>(c, width, minX, minY, maxX, maxY, clear);
}

} // namespace pt
