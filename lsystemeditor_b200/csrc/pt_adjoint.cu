// Differentiable rendering: gradients of an image loss with respect to the
// per-material Principled parameters (base colour r, g, b, roughness,
// metallic, sheen) and the emission strength, by path replay
// backpropagation (Vicini, Speierer & Jakob, SIGGRAPH 2021).  No reference
// counterpart: the reference renders forward only.
//
// The image is the mean of `spp` samples per pixel drawn exactly as a fresh
// pt_render draws them (sample k of pixel p uses the reference seed of wave k),
// each sample being the reference estimator of the forward pipeline (same
// random-number order, same quirks; pt_render.cu).  For one sample, with
// throughput beta_j at vertex j and E_j the radiance the estimator adds at j
// (emission and the next-event terms), L = sum_j beta_j E_j and, with the
// sampling treated as fixed (detached),
//   dL/dtheta = sum_j beta_j dE_j/dtheta
//             + sum_j (dlog f_j/dtheta) * sum_{k>j} beta_k E_k ,
// f_j the BSDF at the direction sampled at j.  The inner sum is L minus what
// the path has collected up to and including vertex j, so two replays of the
// path (one for L, one that accumulates the gradient) need O(1) memory per
// path; when the forward render kept every sample's radiance
// (pt_record_samples), that record replaces the first replay.  The Russian-roulette probability and the MIS weights are detached; the
// firefly clamp is differentiated exactly.
//
// BSDF derivatives at a fixed direction: exact affine differences for the
// base colour and sheen (the BSDF is affine in both when the material has no
// transmission or subsurface lobe), central differences (step 1e-3) for
// roughness, metallic, and for colour / sheen otherwise (second-order one-sided
// at the bounds 0 and 1 of the clamped parameters).
//
// Accumulation: every thread keeps Kahan-compensated single-precision partial
// sums per (material, parameter); a block folds its threads' partials with
// error-free (two-sum) additions and adds one value per entry to the output
// with an atomic.
#include "pt_adjoint.cuh"

#include "pt_bsdf.cuh"
#include "pt_path.cuh"
#include "pt_trace.cuh"

#include <curand_kernel.h>

namespace pt {

namespace {

constexpr int kP = kGradParams;
constexpr int kEntries = kMaxGradMaterials * kGradParams;
constexpr float kFdStep = 1.0e-3f;

struct GradAcc {
    float sum[kEntries];
    float comp[kEntries];
    __device__ __forceinline__ void clear()
    {
        for (int e = 0; e < kEntries; ++e) {
            sum[e] = 0.0f;
            comp[e] = 0.0f;
        }
    }
    // Kahan summation (comp holds the rounding error of the last addition)
    __device__ __forceinline__ void add(int e, float v)
    {
        const float y = __fsub_rn(v, comp[e]);
        const float t = __fadd_rn(sum[e], y);
        comp[e] = __fsub_rn(__fsub_rn(t, sum[e]), y);
        sum[e] = t;
    }
};

// Which parameters of a material the gradient reaches (a textured channel is
// read from its texture, not from the material record).
struct FreeParams {
    bool rgb, roughness, metallic, emission;
};

__device__ __forceinline__ bool textured(uint32_t tex, uint32_t count) { return tex != 0u && tex < count; }

__device__ __forceinline__ FreeParams freeParams(const pt_material& m, uint32_t texCount)
{
    FreeParams f;
    f.rgb = !textured(m.albedo_tex, texCount);
    f.roughness = !textured(m.roughness_tex, texCount);
    f.metallic = !textured(m.metallic_tex, texCount);
    f.emission = !textured(m.emission_tex, texCount);
    return f;
}

// Derivative of g at x in [0, 1] from evaluations g(x + k h): central inside,
// second-order one-sided at a bound (the parameter is clamped to [0, 1]).
template <class Eval>
__device__ __forceinline__ float3 paramDerivative(float x, float3 g0, Eval g)
{
    const float h = kFdStep;
    if (x - h >= 0.0f && x + h <= 1.0f) {
        return scl3(sub3(g(x + h), g(x - h)), 0.5f / h);
    }
    if (x - h < 0.0f) {
        // (-3 g(x) + 4 g(x + h) - g(x + 2h)) / 2h
        return scl3(sub3(sub3(scl3(g(x + h), 4.0f), scl3(g0, 3.0f)), g(x + 2.0f * h)), 0.5f / h);
    }
    // (3 g(x) - 4 g(x - h) + g(x - 2h)) / 2h
    return scl3(add3(sub3(scl3(g0, 3.0f), scl3(g(x - h), 4.0f)), g(x - 2.0f * h)), 0.5f / h);
}

// d f / d p at direction wi for p = r, g, b, roughness, metallic, sheen (RGB each);
// f0 = f(wi).  roughFollows: the diffuse roughness is the roughness (material
// value < 0).
__device__ void bsdfGrad(const Ctx& cx, float3 wi, float3 f0, bool roughFollows, float3 g[6])
{
    if (cx.w.transmit == 0.0f && cx.w.subsurface == 0.0f) {
        Ctx t = cx;
        t.m.r = t.m.g = t.m.b = 0.0f;
        t.m.sheen = 0.0f;
        const float3 f00 = bsdfEval(t, wi);
        t.m.r = t.m.g = t.m.b = 1.0f;
        const float3 f11 = bsdfEval(t, wi);
        t.m.r = t.m.g = t.m.b = 0.0f;
        t.m.sheen = 1.0f;
        const float3 fs = bsdfEval(t, wi);
        const float3 dc = sub3(f11, f00);
        g[0] = f3(dc.x, 0.0f, 0.0f);
        g[1] = f3(0.0f, dc.y, 0.0f);
        g[2] = f3(0.0f, 0.0f, dc.z);
        g[5] = sub3(fs, f00);
    } else {
        g[0] = paramDerivative(cx.m.r, f0, [&](float v) { Ctx t = cx; t.m.r = v; return bsdfEval(t, wi); });
        g[1] = paramDerivative(cx.m.g, f0, [&](float v) { Ctx t = cx; t.m.g = v; return bsdfEval(t, wi); });
        g[2] = paramDerivative(cx.m.b, f0, [&](float v) { Ctx t = cx; t.m.b = v; return bsdfEval(t, wi); });
        g[5] = paramDerivative(cx.m.sheen, f0, [&](float v) { Ctx t = cx; t.m.sheen = v; return bsdfEval(t, wi); });
    }
    g[3] = paramDerivative(cx.m.roughness, f0, [&](float v) {
        Ctx t = cx;
        t.m.roughness = v;
        if (roughFollows) {
            t.m.diffuseRoughness = v;
        }
        return bsdfEval(t, wi);
    });
    g[4] = paramDerivative(cx.m.metallic, f0, [&](float v) {
        Ctx t = cx;
        t.m.metallic = v;
        t.w = computeLobes(t.m);
        return bsdfEval(t, wi);
    });
}

// Gradient of a next-event contribution beta (x) f (x) Le * k with respect to
// the BSDF parameters of material mi.
__device__ __forceinline__ void addNeeGrad(GradAcc& acc, int mi, const FreeParams& fp, const Ctx& cx, float3 wi,
    float3 f, bool roughFollows, float3 delta, float3 T, float3 Le, float k)
{
    float3 g[6];
    bsdfGrad(cx, wi, f, roughFollows, g);
    const float3 w = mul3(mul3(delta, T), scl3(Le, k));
    const bool use[6] = {fp.rgb, fp.rgb, fp.rgb, fp.roughness, fp.metallic, true};
    for (int q = 0; q < 6; ++q) {
        if (use[q]) {
            acc.add(mi * kP + q, dot3(w, g[q]));
        }
    }
}

struct AdjointArgs {
    const LaunchCtx* ctx;
    const float* dImage;   // dLoss/dImage, `channels` floats per pixel
    int channels;
    int spp;
    int pixels;
    int materialCount;
    unsigned long long jobs;
    float* grad;           // [materialCount][kGradParams]
    const float4* record;  // radiance of every sample from the forward render, or null
};

// One sample of pixel p (sample index k) through the reference estimator.  With
// Grad = false returns the sample's radiance L (before the firefly clamp); with
// Grad = true replays the same path and accumulates the gradient of
// dot(delta, L) into acc, using Ltot = the first replay's L.  The traversal
// stack is sstack (this thread's column of the block's shared array) and then
// local memory, as in the forward kernels.
// Where a path starts: pixel p of a width x height image, sample index and
// global seed of its random numbers, subpixel jitter or the pixel centre
// (tracePixelRadiance, PathTracer.cu:69-105), and the depth limit.
struct PathStart {
    uint32_t p;
    uint32_t width, height;
    uint32_t sampleIndex;
    uint32_t globalSeed;
    bool jitter;
    int maxDepth;
};

template <bool Grad, bool Inst = false>
__device__ float3 replayPath(const LaunchCtx& c, const PathStart& ps, float3 delta, float3 Ltot, GradAcc* acc,
    int materialCount, uint2* sstack)
{
    const DevScene& S = c.scene;
    const uint32_t p = ps.p, width = ps.width, height = ps.height;
    curandStateXORWOW st;
    curand_init(pathSeed(c.params, p, width, ps.sampleIndex, ps.globalSeed), 0ull, 0ull, &st);
    const uint32_t x = p % width, y = p / width;
    const float ju = ps.jitter ? curand_uniform(&st) : 0.5f;
    const float jv = ps.jitter ? curand_uniform(&st) : 0.5f;
    const float u = (static_cast<float>(x) + ju) / static_cast<float>(width);
    const float v = (static_cast<float>(y) + jv) / static_cast<float>(height);
    const float l1 = curand_uniform(&st);
    const float l2 = curand_uniform(&st);
    float3 ro, rd;
    cameraRay(c.cam, u, v, l1, l2, ro, rd);
    float tMin = 0.0f;
    float pdfPrev = 0.0f;
    float3 T = f3(1.0f, 1.0f, 1.0f);
    float eta = 1.0f;
    float3 L = f3(0.0f, 0.0f, 0.0f);
    const int debugFlags = c.params.brdf_debug_flags;
    for (int depth = 0;; ++depth) {
        // closest hit (k_extend)
        HitRec h;
        const bool hit =
            traceRay<false, false, Inst>(S, ro, xnormalize(rd), tMin, kRayTMax, h, nullptr, nullptr, sstack, kAdjointBlock);
        if (!hit) {
            // k_shade_miss: the pending next-event terms are already in L
            if (depth == 0) {
                L = envEval(c.env, c.params, rd);
            } else {
                const float3 Le = envEval(c.env, c.params, rd);
                const float lp = envPdf(c.env, rd);
                const float w = misBalance(pdfPrev, lp);
                L = add3(L, mul3(T, scl3(Le, w)));
            }
            break;
        }
        if (depth >= ps.maxDepth) {
            break;
        }
        // shading point (k_shade)
        const float3 pos = xadd(ro, xscl(rd, h.t));
        const float3 dn = xnormalize(rd);
        const TriShade sh = S.shade[h.tri];
        float3 n;
        float tu, tv;
        hitShadingAt(S, sh, h.inst, dn, h.u, h.v, n, tu, tv);
        const uint32_t mi = __float_as_uint(sh.d.w);
        const bool known = S.materials != nullptr && mi < S.materialCount;
        const pt_material& srcMat = known ? S.materials[mi] : kFallbackMaterial;
        const bool grad = Grad && known && static_cast<int>(mi) < materialCount;
        FreeParams fp{};
        if (grad) {
            fp = freeParams(srcMat, S.textureCount);
        }
        const bool roughFollows = srcMat.diffuse_roughness < 0.0f;
        Ctx cx;
        cx.m = resolveMaterial(srcMat, tu, tv, S.textures, S.textureCount);
        cx.w = computeLobes(cx.m);
        cx.n = n;
        cx.wo = scl3(rd, -1.0f);
        cx.eta = eta;
        cx.debug = 0;
        // emission (PathIntegratorRandCore.h:248)
        const float3 E = f3(cx.m.r * cx.m.emission, cx.m.g * cx.m.emission, cx.m.b * cx.m.emission);
        if (grad && cx.m.emission != 0.0f) {
            const float3 dT = mul3(delta, T);
            if (fp.emission) {
                acc->add(mi * kP + 6, dot3(dT, f3(cx.m.r, cx.m.g, cx.m.b)));
            }
            if (fp.rgb) {
                acc->add(mi * kP + 0, dT.x * cx.m.emission);
                acc->add(mi * kP + 1, dT.y * cx.m.emission);
                acc->add(mi * kP + 2, dT.z * cx.m.emission);
            }
        }
        L = add3(L, mul3(T, E));
        // environment NEE (PathIntegratorRandCore.h:65-108) with k_shadow's shadow ray
        if (!skipsEnvNee(cx.m)) {
            const float u1 = curand_uniform(&st);
            const float u2 = curand_uniform(&st);
            float lp = 0.0f;
            const float3 wi = envSample(c.env, u1, u2, lp);
            if (lp > kMinPdf) {
                const float ct = fmax2(0.0f, dot3(n, wi));
                const float3 Le = envEval(c.env, c.params, wi);
                if (ct > 0.0f && (Le.x != 0.0f || Le.y != 0.0f || Le.z != 0.0f)) {
                    const float3 f = bsdfEval(cx, wi);
                    const float bp = bsdfPdf(cx, wi);
                    const float kk = misBalance(lp, bp) * ct / lp;
                    const float3 contrib = mul3(T, mul3(f, scl3(Le, kk)));
                    if (contrib.x != 0.0f || contrib.y != 0.0f || contrib.z != 0.0f) {
                        const float3 so = add3(pos, scl3(n, kShadowBias));
                        HitRec hh;
                        if (!traceRay<true, false, Inst>(S, so, xnormalize(wi), kShadowBias, kRayTMax, hh, nullptr, nullptr,
                                sstack, kAdjointBlock)) {
                            if (grad) {
                                addNeeGrad(*acc, mi, fp, cx, wi, f, roughFollows, delta, T, Le, kk);
                            }
                            L = add3(L, contrib);
                        }
                    }
                }
            }
        }
        // emissive NEE (PathIntegratorRandCore.h:110-167)
        if (S.emissiveCount > 0) {
            const float uTri = curand_uniform(&st);
            const float u1 = curand_uniform(&st);
            const float u2 = curand_uniform(&st);
            float3 lpos, ln, Le, ev0, ev1, ev2;
            float ap;
            uint32_t lt = 0;
            if (sampleEmissive(S, &kFallbackMaterial, uTri, u1, u2, lpos, ln, Le, ap, ev0, ev1, ev2, &lt)) {
                const float3 tl = sub3(lpos, pos);
                const float d2 = dot3(tl, tl);
                if (d2 > kMinPdf) {
                    const float3 wi = normalize3(tl);
                    const float ct = fmax2(0.0f, dot3(n, wi));
                    const float cl = fmax2(0.0f, dot3(ln, scl3(wi, -1.0f)));
                    if (ct > 0.0f && cl > 0.0f) {
                        const float lpdf = ap * d2 / cl;
                        const float3 so = add3(pos, scl3(wi, kShadowBias));
                        const float3 sdn = xnormalize(wi);
                        bool occludedBySelf = false;
                        if (!isDegenerateDir(sdn)) {
                            float th, tu2, tv2;
                            occludedBySelf = intersectTriExact(so, sdn, ev0, ev1, ev2, kShadowBias, kRayTMax, th, tu2,
                                                 tv2) && th < kRayTMax;
                        }
                        if (lpdf > kMinPdf && !occludedBySelf) {
                            const float3 f = bsdfEval(cx, wi);
                            const float bp = bsdfPdf(cx, wi);
                            const float kk = misBalance(lpdf, bp) * ct / lpdf;
                            const float3 contrib = mul3(T, mul3(f, scl3(Le, kk)));
                            if (contrib.x != 0.0f || contrib.y != 0.0f || contrib.z != 0.0f) {
                                HitRec hh;
                                if (!traceRay<true, false, Inst>(S, so, sdn, kShadowBias, kRayTMax, hh, nullptr, nullptr,
                                        sstack, kAdjointBlock)) {
                                    if (grad) {
                                        addNeeGrad(*acc, mi, fp, cx, wi, f, roughFollows, delta, T, Le, kk);
                                    }
                                    // the light's own emission and colour
                                    const uint32_t lm = __float_as_uint(S.shade[lt].d.w);
                                    if (Grad && S.materials != nullptr && lm < S.materialCount &&
                                        static_cast<int>(lm) < materialCount) {
                                        const pt_material& l0 = S.materials[lm];
                                        const float3 w = mul3(mul3(delta, T), scl3(f, kk));
                                        acc->add(lm * kP + 6, dot3(w, f3(l0.r, l0.g, l0.b)));
                                        acc->add(lm * kP + 0, w.x * l0.emission);
                                        acc->add(lm * kP + 1, w.y * l0.emission);
                                        acc->add(lm * kP + 2, w.z * l0.emission);
                                    }
                                    L = add3(L, contrib);
                                }
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
            break;
        }
        const float3 f = bsdfEval(cx, smp.dir);
        if (grad) {
            // radiance still to come from this direction: L_total - L
            const float3 dRem = mul3(delta, sub3(Ltot, L));
            float3 g[6];
            bsdfGrad(cx, smp.dir, f, roughFollows, g);
            const float3 inv = f3(f.x != 0.0f ? 1.0f / f.x : 0.0f, f.y != 0.0f ? 1.0f / f.y : 0.0f,
                f.z != 0.0f ? 1.0f / f.z : 0.0f);
            const float3 wgt = mul3(dRem, inv);
            const bool use[6] = {fp.rgb, fp.rgb, fp.rgb, fp.roughness, fp.metallic, true};
            for (int q = 0; q < 6; ++q) {
                if (use[q]) {
                    acc->add(mi * kP + q, dot3(wgt, g[q]));
                }
            }
            if (fp.rgb) {
                // factors of the base colour outside f: thin transmission and subsurface steps
                const float trans = fmax2(0.0f, fmin2(1.0f, cx.m.transmission));
                const float thin = fmax2(0.0f, fmin2(1.0f, cx.m.thin));
                const bool pure = trans > 0.99f && cx.m.metallic < 0.01f;
                float extra = 0.0f;
                if (!(pure && thin < 0.5f) && smp.transmitted && thin > 0.5f) {
                    extra += 1.0f;
                }
                if (smp.sss && smp.sssSteps > 0 && maxScatter(cx.m) > kMinRadius) {
                    extra += static_cast<float>(smp.sssSteps);
                }
                if (extra != 0.0f) {
                    acc->add(mi * kP + 0, cx.m.r != 0.0f ? dRem.x * extra / cx.m.r : 0.0f);
                    acc->add(mi * kP + 1, cx.m.g != 0.0f ? dRem.y * extra / cx.m.g : 0.0f);
                    acc->add(mi * kP + 2, cx.m.b != 0.0f ? dRem.z * extra / cx.m.b : 0.0f);
                }
            }
        }
        T = applyThroughput(T, cx, smp, f);
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
                    T = mul3(T, scl3(f3(cx.m.r, cx.m.g, cx.m.b), surv));
                }
                const float ed = sqrtf(dot3(smp.exitOffset, smp.exitOffset));
                if (ed > 0.0f) {
                    T = scl3(T, expf(-ed / maxR));
                }
            }
        }
        if (debugFlags & kDbgTintGlass) {
            T = smp.transmitted ? mul3(T, f3(0.2f, 1.0f, 0.2f)) : mul3(T, f3(1.0f, 0.2f, 0.2f));
        }
        const float tl = lum709(T);
        if (!isfinite(tl) || tl <= 0.0f || tl > 1.0e8f) {
            break;
        }
        if (depth >= c.rrMinDepth) {
            const float surv = fmin2(0.95f, fmax2(tl, 0.05f));
            if (curand_uniform(&st) > surv) {
                break;
            }
            T = scl3(T, 1.0f / surv);
        }
        eta = smp.nextEta;
        const float bias = fmax2(1.0e-4f, 1.0e-3f * h.t);
        const float sign = dot3(n, smp.dir) >= 0.0f ? 1.0f : -1.0f;
        ro = xadd(pos, xscl(n, __fmul_rn(sign, bias)));
        rd = smp.dir;
        tMin = bias;
        pdfPrev = smp.pdf;
    }
    return L;
}

// Error-free sum of two (hi, lo) pairs (Knuth two-sum, then a fast renormalisation).
__device__ __forceinline__ void pairAdd(float& hi, float& lo, float bhi, float blo)
{
    const float s = __fadd_rn(hi, bhi);
    const float bb = __fsub_rn(s, hi);
    const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(bhi, bb));
    const float l = __fadd_rn(__fadd_rn(lo, blo), err);
    hi = __fadd_rn(s, l);
    lo = __fsub_rn(l, __fsub_rn(hi, s));
}

__global__ void __launch_bounds__(kAdjointBlock) k_adjoint(AdjointArgs a)
{
    const LaunchCtx& c = *a.ctx;
    extern __shared__ uint2 smemStack[];
    uint2* sstack = smemStack + threadIdx.x;
    GradAcc acc;
    acc.clear();
    const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
    for (unsigned long long j = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; j < a.jobs;
         j += stride) {
        const uint32_t p = static_cast<uint32_t>(j % static_cast<unsigned long long>(a.pixels));
        const uint32_t k = static_cast<uint32_t>(j / static_cast<unsigned long long>(a.pixels));
        const float* di = a.dImage + static_cast<size_t>(p) * a.channels;
        float3 delta = f3(di[0], di[1], di[2]);
        if (delta.x == 0.0f && delta.y == 0.0f && delta.z == 0.0f) {
            continue;
        }
        // sample k of pixel p as a fresh render draws it: wave k's seed
        const PathStart start{p, static_cast<uint32_t>(c.width), static_cast<uint32_t>(c.height), k,
            k + 1u + static_cast<uint32_t>(c.seedOffset), true, c.maxDepth};
        float3 Ltot;
        if (a.record != nullptr) {
            const float4 r = a.record[j];  // j = k * pixels + p
            Ltot = f3(r.x, r.y, r.z);
        } else {
            Ltot = replayPath<false>(c, start, f3(0.0f, 0.0f, 0.0f), f3(0.0f, 0.0f, 0.0f), nullptr, 0, sstack);
        }
        if (!isfinite(Ltot.x) || !isfinite(Ltot.y) || !isfinite(Ltot.z)) {
            continue; // the firefly clamp replaces a non-finite sample by zero
        }
        if (Ltot.x == 0.0f && Ltot.y == 0.0f && Ltot.z == 0.0f) {
            // nothing collected: every emission and next-event term of the path is
            // zero and so is the radiance behind every vertex (exact up to terms
            // whose BSDF value is exactly zero towards a visible light)
            continue;
        }
        // adjoint of the firefly clamp (PathTracer.cu:49-67): negative channels are
        // cut to zero (no gradient); above luminance 100, c -> c * 100 / lum(c),
        // whose Jacobian is (100 / lum) (I - c w^T / lum), w the Rec.709 weights
        delta = scl3(delta, 1.0f / static_cast<float>(a.spp));
        delta = f3(Ltot.x > 0.0f ? delta.x : 0.0f, Ltot.y > 0.0f ? delta.y : 0.0f, Ltot.z > 0.0f ? delta.z : 0.0f);
        const float3 cl = f3(fmax2(0.0f, Ltot.x), fmax2(0.0f, Ltot.y), fmax2(0.0f, Ltot.z));
        const float l = __fadd_rn(__fadd_rn(__fmul_rn(cl.x, 0.2126f), __fmul_rn(cl.y, 0.7152f)), __fmul_rn(cl.z, 0.0722f));
        if (l > 100.0f) {
            const float kc = __fdiv_rn(100.0f, l);
            const float dc = dot3(delta, cl) / l;
            const float3 w = f3(Ltot.x > 0.0f ? 0.2126f : 0.0f, Ltot.y > 0.0f ? 0.7152f : 0.0f,
                Ltot.z > 0.0f ? 0.0722f : 0.0f);
            delta = scl3(sub3(delta, scl3(w, dc)), kc);
        }
        replayPath<true>(c, start, delta, Ltot, &acc, a.materialCount, sstack);
    }
    // block reduction of the (sum, -compensation) pairs, then one atomic per entry
    __shared__ float sHi[kAdjointBlock / 32], sLo[kAdjointBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int entries = a.materialCount * kP;
    for (int e = 0; e < entries; ++e) {
        float hi = acc.sum[e], lo = __fsub_rn(0.0f, acc.comp[e]);
        for (int off = 16; off > 0; off >>= 1) {
            const float oh = __shfl_down_sync(0xffffffffu, hi, off);
            const float ol = __shfl_down_sync(0xffffffffu, lo, off);
            pairAdd(hi, lo, oh, ol);
        }
        if (lane == 0) {
            sHi[warp] = hi;
            sLo[warp] = lo;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            float bh = sHi[0], bl = sLo[0];
            for (int w = 1; w < kAdjointBlock / 32; ++w) {
                pairAdd(bh, bl, sHi[w], sLo[w]);
            }
            const float v = __fadd_rn(bh, bl);
            if (v != 0.0f) {
                atomicAdd(&a.grad[e], v);
            }
        }
        __syncthreads();
    }
}

size_t adjointSmemBytes() { return sizeof(uint2) * kSharedStack * kAdjointBlock; }

// Preview pass (sampleKernel with previewPass, PathTracer.cu:132-184): one
// sample per pixel of a width x height image at the pixel centre, sample index
// 0 and the given global seed, depth limit kPreviewMaxPathDepth
// (PathTracerPreviewLevels.h:13), firefly-clamped.
template <bool Inst>
__global__ void __launch_bounds__(kAdjointBlock) k_preview(const LaunchCtx* __restrict__ cp, int width, int height,
    uint32_t globalSeed, int maxDepth, float4* out)
{
    const LaunchCtx& c = *cp;
    extern __shared__ uint2 smemStack[];
    uint2* sstack = smemStack + threadIdx.x;
    const int n = width * height;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const PathStart start{static_cast<uint32_t>(p), static_cast<uint32_t>(width), static_cast<uint32_t>(height), 0u,
            globalSeed, false, maxDepth};
        const float3 L = clampFirefly(
            replayPath<false, Inst>(c, start, f3(0.0f, 0.0f, 0.0f), f3(0.0f, 0.0f, 0.0f), nullptr, 0, sstack));
        out[p] = make_float4(L.x, L.y, L.z, 1.0f);
    }
}

} // namespace

void launchPreview(const LaunchCtx* ctx, int width, int height, uint32_t globalSeed, int maxDepth, float4* out,
    int grid, bool inst, cudaStream_t s)
{
    if (inst) {
        k_preview<true><<<grid, kAdjointBlock, adjointSmemBytes(), s>>>(ctx, width, height, globalSeed, maxDepth, out);
    } else {
        k_preview<false><<<grid, kAdjointBlock, adjointSmemBytes(), s>>>(ctx, width, height, globalSeed, maxDepth, out);
    }
}

int adjointBlocksPerSm()
{
    int blocks = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_adjoint, kAdjointBlock, adjointSmemBytes());
    return blocks < 1 ? 1 : blocks;
}

void launchAdjoint(const LaunchCtx* ctx, const float* dImage, int channels, int spp, int pixels, int materialCount,
    float* grad, const float4* record, int grid, cudaStream_t s)
{
    AdjointArgs a;
    a.ctx = ctx;
    a.dImage = dImage;
    a.channels = channels;
    a.spp = spp;
    a.pixels = pixels;
    a.materialCount = materialCount;
    a.jobs = static_cast<unsigned long long>(pixels) * static_cast<unsigned long long>(spp);
    a.grad = grad;
    a.record = record;
    k_adjoint<<<grid, kAdjointBlock, adjointSmemBytes(), s>>>(a);
}

} // namespace pt
