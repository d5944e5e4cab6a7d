// Device-side Principled BSDF, lights, camera and material resolve for the
// wavefront shade stage.  Follows the reference formulas term by term:
//   Brdf/BrdfBase.h:76-280, Brdf/PrincipledBrdf.h:14-588,
//   Brdf/SubsurfaceCore.h:20-118, Brdf/BrdfDispatch.h:11-76,
//   Sampling/LightSamplingCore.h:25-313, Sampling/MisCore.h:11-21,
//   Texture/ProceduralTexture.h:27-207, CameraDevice.cuh:8-139.
// Lobes whose weight is exactly zero are skipped: they add +0 in the
// reference, so the result is unchanged.
#pragma once

#include "pt_common.cuh"

namespace pt {

struct Mat {
    float r, g, b, roughness, metallic, transmission, thin, ior, subsurface, emission, diffuseRoughness, scatterR,
        scatterG, scatterB, specular, sheen;
};

struct Lobes {
    float diffuse, specular, transmit, subsurface;
};

struct Ctx {
    float3 n, wo;
    Mat m;
    Lobes w;
    float eta;
    int debug;
};

struct BsdfSample {
    float3 dir;
    float pdf;
    float nextEta;
    float3 exitOffset;
    int sssSteps;
    bool valid, transmitted, sss;
};

constexpr int kDbgForceTransmit = 1 << 0;
constexpr int kDbgDisableRefract = 1 << 1;
constexpr int kDbgDisableReflect = 1 << 2;
constexpr int kDbgDisableTirFallback = 1 << 3;
constexpr int kDbgTintGlass = 1 << 4;
constexpr float kMinRadius = 1.0e-5f;

__device__ __forceinline__ float clamp01(float v) { return fmax2(0.0f, fmin2(1.0f, v)); }
__device__ __forceinline__ float absf(float v) { return v < 0.0f ? -v : v; }

// --- material resolve (ProceduralTexture.h:27-207) --------------------------
__device__ __forceinline__ float fractf(float v) { return v - floorf(v); }

// Scalar channels: Stripe1D reads u1d = uv.x, Grid2D reads uv (ProceduralTexture.h:37-63, 138-186).
__device__ __forceinline__ float texScalar(const pt_texture& t, float u, float v)
{
    switch (t.kind) {
    case 0:
        return t.p0[0];
    case 3: {
        const float c = fractf(u * t.p0[0]);
        return c < t.p0[1] ? t.p0[2] : t.p0[3];
    }
    case 2: {
        const float fx = fractf(u * t.p0[0]);
        const float fy = fractf(v * t.p0[1]);
        return (fx < t.p0[2] || fy < t.p0[2]) ? 1.0f : 0.0f;
    }
    default:
        return 0.0f;
    }
}

__device__ __forceinline__ float3 texRgb(const pt_texture& t, float u, float v)
{
    switch (t.kind) {
    case 1:
        return f3(t.p0[0], t.p0[1], t.p0[2]);
    case 2: {
        const float fx = fractf(u * t.p0[0]);
        const float fy = fractf(v * t.p0[1]);
        const float g = (fx < t.p0[2] || fy < t.p0[2]) ? 1.0f : 0.0f;
        return f3(t.p1[0] + (t.p2[0] - t.p1[0]) * g, t.p1[1] + (t.p2[1] - t.p1[1]) * g, t.p1[2] + (t.p2[2] - t.p1[2]) * g);
    }
    default:
        return f3(0.0f, 0.0f, 0.0f);
    }
}

__device__ __forceinline__ float clampTex01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

__device__ __forceinline__ Mat resolveMaterial(const pt_material& src, float u, float v, const pt_texture* bank,
    uint32_t count)
{
    Mat m;
    auto scalar = [&](float inl, uint32_t ti) -> float {
        if (ti == 0u || bank == nullptr || ti >= count) {
            return inl;
        }
        return texScalar(bank[ti], u, v);
    };
    if (src.albedo_tex == 0u || bank == nullptr || src.albedo_tex >= count) {
        m.r = src.r;
        m.g = src.g;
        m.b = src.b;
    } else {
        const float3 c = texRgb(bank[src.albedo_tex], u, v);
        m.r = c.x;
        m.g = c.y;
        m.b = c.z;
    }
    m.roughness = clampTex01(scalar(src.roughness, src.roughness_tex));
    m.metallic = clampTex01(scalar(src.metallic, src.metallic_tex));
    m.transmission = clampTex01(scalar(src.transmission, src.transmission_tex));
    m.thin = clampTex01(scalar(src.thin, src.thin_tex));
    m.ior = fmaxf(1.0e-3f, scalar(src.ior, src.ior_tex));
    m.subsurface = clampTex01(scalar(src.subsurface, src.subsurface_tex));
    m.emission = fmaxf(0.0f, scalar(src.emission, src.emission_tex));
    m.diffuseRoughness = src.diffuse_roughness < 0.0f ? m.roughness : clampTex01(src.diffuse_roughness);
    m.scatterR = fmaxf(0.0f, src.scatter_radius_r);
    m.scatterG = fmaxf(0.0f, src.scatter_radius_g);
    m.scatterB = fmaxf(0.0f, src.scatter_radius_b);
    m.specular = clampTex01(src.specular);
    m.sheen = clamp01(src.sheen);
    return m;
}

// --- BSDF building blocks (BrdfBase.h) --------------------------------------
__device__ __forceinline__ void basis(float3 n, float3& t, float3& b)
{
    const float3 up = fabsf(n.y) < 0.999f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
    t = normalize3(cross3(up, n));
    b = normalize3(cross3(n, t));
}
__device__ __forceinline__ float3 toWorld(float3 l, float3 n, float3 t, float3 b)
{
    return normalize3(add3(add3(scl3(t, l.x), scl3(b, l.y)), scl3(n, l.z)));
}
__device__ __forceinline__ float3 cosineHemi(float u1, float u2)
{
    const float phi = 2.0f * kPi * u1;
    const float r = sqrtf(u2);
    float s, c;
    sincosf(phi, &s, &c);
    return f3(r * c, r * s, sqrtf(fmax2(0.0f, 1.0f - u2)));
}
__device__ __forceinline__ float cosinePdf(float c) { return fmax2(0.0f, c) * kInvPi; }
__device__ __forceinline__ float alphaFromRoughness(float r)
{
    const float c = fmax2(r, 0.04f);
    return c * c;
}
__device__ __forceinline__ float ggxD(float cosH, float a)
{
    const float a2 = a * a;
    const float c2 = cosH * cosH;
    const float den = c2 * (a2 - 1.0f) + 1.0f;
    return a2 / (kPi * den * den);
}
__device__ __forceinline__ float smithG1(float c, float a)
{
    const float a2 = a * a;
    const float c2 = fmax2(c * c, 1.0e-8f);
    const float t2 = (1.0f - c2) / c2;
    return 2.0f / (1.0f + sqrtf(1.0f + a2 * t2));
}
__device__ __forceinline__ float3 schlick(float c, float3 f0)
{
    const float t = fmax2(0.0f, fmin2(1.0f, 1.0f - c));
    const float t2 = t * t;
    const float t5 = t2 * t2 * t;
    return add3(scl3(f0, 1.0f - t5), f3(t5, t5, t5));
}
__device__ __forceinline__ float3 ggxHalf(float a, float u1, float u2, float& pdf)
{
    const float phi = 2.0f * kPi * u1;
    const float a2 = a * a;
    const float ct = sqrtf((1.0f - u2) / (1.0f + (a2 - 1.0f) * u2));
    const float st = sqrtf(fmax2(0.0f, 1.0f - ct * ct));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    const float den = ct * ct * (a2 - 1.0f) + 1.0f;
    pdf = (a2 * ct) / (kPi * den * den);
    return f3(st * cp, st * sp, ct);
}
__device__ __forceinline__ float dielectricFresnel(float cosI_, float etaI, float etaT)
{
    float cosI = fmax2(-1.0f, fmin2(1.0f, cosI_));
    float eta = etaI / fmax2(etaT, 1.0e-8f);
    if (cosI < 0.0f) {
        cosI = -cosI;
        eta = 1.0f / eta;
    }
    const float s2 = eta * eta * (1.0f - cosI * cosI);
    if (s2 >= 1.0f) {
        return 1.0f;
    }
    const float cosT = sqrtf(fmax2(0.0f, 1.0f - s2));
    const float rp = (eta * cosI - cosT) / fmax2(eta * cosI + cosT, 1.0e-8f);
    const float rs = (cosI - eta * cosT) / fmax2(cosI + eta * cosT, 1.0e-8f);
    return 0.5f * (rp * rp + rs * rs);
}
__device__ __forceinline__ bool refractRel(float3 wo, float3 n_, float etaI, float etaT, float3& out)
{
    float cO = dot3(n_, wo);
    float3 n = n_;
    float er = etaI / fmax2(etaT, 1.0e-8f);
    if (cO > 0.0f) {
        n = scl3(n_, -1.0f);
        er = 1.0f / er;
        cO = -cO;
    }
    const float s2 = er * er * (1.0f - cO * cO);
    if (s2 >= 1.0f) {
        return false;
    }
    const float cT = sqrtf(fmax2(0.0f, 1.0f - s2));
    out = normalize3(sub3(scl3(wo, -er), scl3(n, er * cO + cT)));
    return true;
}
__device__ __forceinline__ float orenNayar(float sigma, float cI, float cO, float dWoWi)
{
    if (sigma <= 1.0e-4f) {
        return 1.0f;
    }
    const float s2 = sigma * sigma;
    const float A = 1.0f - 0.5f * s2 / (s2 + 0.33f);
    const float B = 0.45f * s2 / (s2 + 0.09f);
    const float sI = sqrtf(fmax2(0.0f, 1.0f - cI * cI));
    const float sO = sqrtf(fmax2(0.0f, 1.0f - cO * cO));
    float sA, sB;
    if (cI > cO) {
        sA = sI;
        sB = sO;
    } else {
        sA = sO;
        sB = sI;
    }
    float cosPhi = 1.0f;
    const float d = dWoWi - cI * cO;
    if (d <= 0.0f) {
        cosPhi = fmax2(-1.0f, fmin2(1.0f, d / fmax2(sA * sB, 1.0e-8f)));
    } else {
        sA = 0.0f;
        sB = 0.0f;
    }
    const float tB = sB / fmax2(cI, cO);
    return A + B * fmax2(0.0f, cosPhi) * sA * tB;
}
__device__ __forceinline__ float energyComp(float rough, float c)
{
    const float a = alphaFromRoughness(rough);
    const float cc = fmax2(c, 1.0e-4f);
    const float Ess = 1.0f - a * (0.3316f + 0.3237f * a);
    const float Ems = (1.0f - Ess) * (1.0f - cc);
    return 1.0f + Ems / fmax2(Ess, 1.0e-4f);
}
__device__ __forceinline__ float maxScatter(const Mat& m)
{
    return fmax2(fmax2(fmax2(0.0f, m.scatterR), fmax2(0.0f, m.scatterG)), fmax2(0.0f, m.scatterB));
}

// --- Burley subsurface (SubsurfaceCore.h) ------------------------------------
__device__ __forceinline__ float burleyRadius(float u, float d)
{
    const float sd = fmax2(d, kMinRadius);
    return sd * sqrtf(-logf(fmax2(1.0e-8f, 1.0f - u * (1.0f - expf(-1.0f / sd)))));
}
__device__ __forceinline__ float burleyProfile(float r, float d)
{
    const float sd = fmax2(d, kMinRadius);
    return (expf(-r / sd) + expf(-r / (3.0f * sd))) / (4.0f * kPi * sd);
}
__device__ __forceinline__ float burleyPdf(float r, float d)
{
    const float sd = fmax2(d, kMinRadius);
    const float t0 = expf(-r / sd);
    const float t1 = expf(-r / (3.0f * sd));
    const float nn = 1.0f - expf(-1.0f / sd);
    return fmax2(0.0f, (t0 + t1) / fmax2(2.0f * sd * nn, 1.0e-8f));
}
__device__ __forceinline__ float3 burleyEval(const Mat& m, float disk, float cI, float cO)
{
    const float rx = fmax2(0.0f, m.scatterR), ry = fmax2(0.0f, m.scatterG), rz = fmax2(0.0f, m.scatterB);
    const float sum = fmax2(rx + ry + rz, kMinRadius);
    const float pR = burleyProfile(disk, fmax2(rx, kMinRadius));
    const float pG = burleyProfile(disk, fmax2(ry, kMinRadius));
    const float pB = burleyProfile(disk, fmax2(rz, kMinRadius));
    const float df = fmax2(cI, 0.0f) * fmax2(cO, 0.0f);
    return f3(rx / sum * pR * df, ry / sum * pG * df, rz / sum * pB * df);
}
__device__ __forceinline__ float effectiveRadius(const Mat& m, float uc)
{
    const float rx = fmax2(0.0f, m.scatterR), ry = fmax2(0.0f, m.scatterG), rz = fmax2(0.0f, m.scatterB);
    if (maxScatter(m) <= kMinRadius) {
        return kMinRadius;
    }
    if (uc < rx / (rx + ry + rz + kMinRadius)) {
        return fmax2(rx, kMinRadius);
    }
    if (uc < (rx + ry) / (rx + ry + rz + kMinRadius)) {
        return fmax2(ry, kMinRadius);
    }
    return fmax2(rz, kMinRadius);
}

// --- Principled lobes (PrincipledBrdf.h) --------------------------------------
__device__ __forceinline__ Lobes computeLobes(const Mat& m)
{
    Lobes w;
    const float metal = clamp01(m.metallic);
    const float trans = clamp01(m.transmission);
    const float sss = clamp01(m.subsurface);
    const float diel = 1.0f - metal;
    w.transmit = diel * trans;
    w.subsurface = diel * (1.0f - trans) * sss;
    w.diffuse = diel * (1.0f - trans) * (1.0f - sss);
    w.specular = metal + diel * (1.0f - trans);
    const float sum = w.diffuse + w.specular + w.transmit + w.subsurface;
    if (sum <= kMinPdf) {
        w.diffuse = 1.0f;
        return w;
    }
    const float inv = 1.0f / sum;
    w.diffuse *= inv;
    w.specular *= inv;
    w.transmit *= inv;
    w.subsurface *= inv;
    return w;
}

__device__ __forceinline__ float matIor(const Ctx& c) { return fmax2(c.m.ior, 1.0e-3f); }

__device__ __forceinline__ float3 specF0(const Ctx& c)
{
    const float metal = clamp01(c.m.metallic);
    const float ior = matIor(c);
    const float f = (ior - 1.0f) / (ior + 1.0f);
    const float v = f * f * clamp01(clamp01(c.m.specular));
    return f3(v + (c.m.r - v) * metal, v + (c.m.g - v) * metal, v + (c.m.b - v) * metal);
}

__device__ __forceinline__ float3 mirrorOut(float3 wo, float3 n) { return normalize3(sub3(scl3(n, 2.0f * dot3(n, wo)), wo)); }

__device__ __forceinline__ float onFactor(const Ctx& c, float3 wi, float cI, float cO)
{
    const float dr = c.m.diffuseRoughness < 0.0f ? c.m.roughness : c.m.diffuseRoughness;
    const float sigma = fmax2(0.0f, fmin2(1.0f, dr)) * 0.5f * kPi;
    return orenNayar(sigma, cI, cO, dot3(wi, c.wo));
}

__device__ __forceinline__ bool transmitValid(const Ctx& c, float cOs)
{
    if (absf(cOs) <= kMinPdf) {
        return false;
    }
    return cOs > 0.0f || c.eta > 1.0f + 1.0e-4f;
}

__device__ __forceinline__ bool refractDir(const Ctx& c, float3& out, float& nextEta)
{
    const float cO = dot3(c.n, c.wo);
    const float ior = matIor(c);
    float etaT;
    if (cO > 0.0f) {
        etaT = ior;
        nextEta = ior;
    } else {
        etaT = 1.0f;
        nextEta = 1.0f;
    }
    return refractRel(c.wo, c.n, c.eta, etaT, out);
}

__device__ __forceinline__ float3 evalDiffuse(const Ctx& c, float3 wi)
{
    const float cI = fmax2(0.0f, dot3(c.n, wi));
    const float cO = fmax2(0.0f, dot3(c.n, c.wo));
    if (cI <= 0.0f || cO <= 0.0f) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    const float on = onFactor(c, wi, cI, cO);
    float3 r = scl3(f3(c.m.r, c.m.g, c.m.b), c.w.diffuse * on * kInvPi);
    if (c.m.sheen > 0.0f) {
        // extension (no reference counterpart): white sheen sheen * (1 - cos theta_d)^5
        // on the diffuse lobe, theta_d between wi and the half vector (the Disney
        // BRDF's sheen term); 0 leaves the reference BSDF unchanged
        const float3 h = normalize3(add3(wi, c.wo));
        const float x = 1.0f - fmax2(0.0f, dot3(wi, h));
        const float x2 = x * x;
        const float sh = c.w.diffuse * c.m.sheen * (x2 * x2 * x);
        r = add3(r, f3(sh, sh, sh));
    }
    return r;
}

__device__ __forceinline__ float3 evalSpecular(const Ctx& c, float3 wi)
{
    const float cO = fmax2(0.0f, dot3(c.n, c.wo));
    const float cI = fmax2(0.0f, dot3(c.n, wi));
    if (cO <= 0.0f || cI <= 0.0f) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    const float3 h = normalize3(add3(wi, c.wo));
    const float cH = fmax2(0.0f, dot3(c.n, h));
    const float cHo = fmax2(0.0f, dot3(h, c.wo));
    if (cHo <= 0.0f) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    const float a = alphaFromRoughness(c.m.roughness);
    const float D = ggxD(cH, a);
    const float G = smithG1(cO, a) * smithG1(cI, a);
    const float3 F = schlick(cHo, specF0(c));
    const float ec = energyComp(c.m.roughness, cO);
    const float den = fmax2(4.0f * cO * cI, 1.0e-8f);
    const float s = c.w.specular * ec * (D * G) / den;
    return f3(F.x * s, F.y * s, F.z * s);
}

__device__ __forceinline__ float3 evalTransmit(const Ctx& c, float3 wi)
{
    const float cOs = dot3(c.n, c.wo);
    if (!transmitValid(c, cOs)) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    const float thin = clamp01(c.m.thin);
    const float3 base = f3(c.m.r, c.m.g, c.m.b);
    const float ior = matIor(c);
    const float etaT = cOs > 0.0f ? ior : 1.0f;
    const float refl = dielectricFresnel(cOs, c.eta, etaT);
    const float trans = 1.0f - refl;
    const float3 reflected = mirrorOut(c.wo, c.n);
    if (dot3(wi, reflected) > 0.999f) {
        const float cI = absf(dot3(c.n, wi));
        return scl3(base, c.w.transmit * refl / fmax2(cI, 1.0e-8f));
    }
    float3 td;
    float ne = 1.0f;
    if (thin > 0.5f) {
        td = normalize3(scl3(c.wo, -1.0f));
    } else if (!refractDir(c, td, ne)) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    if (dot3(wi, td) > 0.999f) {
        const float cI = absf(dot3(c.n, td));
        const float3 tint = thin > 0.5f ? base : f3(1.0f, 1.0f, 1.0f);
        return f3(tint.x * c.w.transmit * trans / fmax2(cI, 1.0e-8f), tint.y * c.w.transmit * trans / fmax2(cI, 1.0e-8f),
            tint.z * c.w.transmit * trans / fmax2(cI, 1.0e-8f));
    }
    const float a = alphaFromRoughness(c.m.roughness);
    if (a > 0.04f) {
        const float3 h = normalize3(add3(wi, c.wo));
        const float cH = fmax2(0.0f, absf(dot3(c.n, h)));
        const float rp = ggxD(cH, a) * cH;
        if (rp > kMinPdf) {
            const float3 tint = thin > 0.5f ? base : f3(1.0f, 1.0f, 1.0f);
            const float s = c.w.transmit * trans * rp;
            return f3(tint.x * s, tint.y * s, tint.z * s);
        }
    }
    return f3(0.0f, 0.0f, 0.0f);
}

__device__ __forceinline__ float3 evalSubsurface(const Ctx& c, float3 wi)
{
    const float cI = fmax2(0.0f, dot3(c.n, wi));
    const float cO = fmax2(0.0f, dot3(c.n, c.wo));
    if (cI <= 0.0f || cO <= 0.0f) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    const float3 base = f3(c.m.r, c.m.g, c.m.b);
    if (maxScatter(c.m) <= kMinRadius) {
        const float on = onFactor(c, wi, cI, cO);
        return scl3(base, c.w.subsurface * on * kInvPi);
    }
    float3 t, b;
    basis(c.n, t, b);
    const float3 wt = add3(scl3(t, dot3(wi, t)), scl3(b, dot3(wi, b)));
    const float disk = sqrtf(dot3(wt, wt));
    const float3 bu = burleyEval(c.m, disk, cI, cO);
    return f3(base.x * c.w.subsurface * bu.x, base.y * c.w.subsurface * bu.y, base.z * c.w.subsurface * bu.z);
}

__device__ __forceinline__ float pdfDiffuse(const Ctx& c, float3 wi) { return c.w.diffuse * cosinePdf(fmax2(0.0f, dot3(c.n, wi))); }

__device__ __forceinline__ float pdfSpecular(const Ctx& c, float3 wi)
{
    const float cO = fmax2(0.0f, dot3(c.n, c.wo));
    const float cI = fmax2(0.0f, dot3(c.n, wi));
    if (cO <= 0.0f || cI <= 0.0f) {
        return 0.0f;
    }
    const float3 h = normalize3(add3(wi, c.wo));
    const float cH = fmax2(0.0f, dot3(c.n, h));
    const float cHo = fmax2(0.0f, dot3(h, c.wo));
    if (cHo <= 0.0f) {
        return 0.0f;
    }
    const float a = alphaFromRoughness(c.m.roughness);
    return c.w.specular * (ggxD(cH, a) * cH) / fmax2(4.0f * cHo, 1.0e-8f);
}

// The reference's transmit lobe is a pair of narrow cones (cosine > 0.999
// with the mirror and with the transmitted direction; evalTransmit and
// pdfTransmit) that its sampler produces as exact directions.  The emitter MIS
// mode leaves directions in those cones to BSDF sampling alone.
__device__ __forceinline__ bool inTransmitCones(const Ctx& c, float3 wi)
{
    if (c.w.transmit == 0.0f) {
        return false;
    }
    const float cOs = dot3(c.n, c.wo);
    if (!transmitValid(c, cOs)) {
        return false;
    }
    if (dot3(wi, mirrorOut(c.wo, c.n)) > 0.999f) {
        return true;
    }
    float3 td;
    float ne = 1.0f;
    if (clamp01(c.m.thin) > 0.5f) {
        td = normalize3(scl3(c.wo, -1.0f));
    } else if (!refractDir(c, td, ne)) {
        return false;
    }
    return dot3(wi, td) > 0.999f;
}

__device__ __forceinline__ float pdfTransmit(const Ctx& c, float3 wi)
{
    const float cOs = dot3(c.n, c.wo);
    if (!transmitValid(c, cOs)) {
        return 0.0f;
    }
    const float thin = clamp01(c.m.thin);
    const float ior = matIor(c);
    const float etaT = cOs > 0.0f ? ior : 1.0f;
    const float refl = dielectricFresnel(cOs, c.eta, etaT);
    const float trans = 1.0f - refl;
    float pdf = 0.0f;
    const float3 reflected = mirrorOut(c.wo, c.n);
    if (dot3(wi, reflected) > 0.999f) {
        const float cI = absf(dot3(c.n, wi));
        pdf += c.w.transmit * refl / fmax2(cI, 1.0e-8f);
    }
    float3 td;
    if (thin > 0.5f) {
        td = normalize3(scl3(c.wo, -1.0f));
    } else {
        float ne;
        if (!refractDir(c, td, ne)) {
            return pdf;
        }
    }
    if (dot3(wi, td) > 0.999f) {
        const float cI = absf(dot3(c.n, td));
        pdf += c.w.transmit * trans / fmax2(cI, 1.0e-8f);
    }
    return pdf;
}

__device__ __forceinline__ float pdfSubsurface(const Ctx& c, float3 wi)
{
    const float cp = cosinePdf(fmax2(0.0f, dot3(c.n, wi)));
    const float mr = maxScatter(c.m);
    if (mr <= kMinRadius) {
        return c.w.subsurface * cp;
    }
    float3 t, b;
    basis(c.n, t, b);
    const float3 wt = add3(scl3(t, dot3(wi, t)), scl3(b, dot3(wi, b)));
    const float disk = sqrtf(dot3(wt, wt));
    return c.w.subsurface * fmax2(cp, burleyPdf(disk, mr) * 0.5f);
}

// The BSDF is evaluated at up to four call sites per shading point (two NEE
// estimators, the sampled direction, and the pdf inside sampling).  Keeping one
// out-of-line copy of eval, pdf and sample keeps the shade kernel small enough
// for the instruction cache (inlining every site made it fetch-bound).
__device__ __forceinline__ float3 bsdfEvalImpl(const Ctx& c, float3 wi)
{
    const float3 d = evalDiffuse(c, wi);
    const float3 s = evalSpecular(c, wi);
    float3 r = add3(d, s);
    if (c.w.transmit != 0.0f || c.w.subsurface != 0.0f) {
        const float3 t = c.w.transmit != 0.0f ? evalTransmit(c, wi) : f3(0.0f, 0.0f, 0.0f);
        const float3 ss = c.w.subsurface != 0.0f ? evalSubsurface(c, wi) : f3(0.0f, 0.0f, 0.0f);
        r = add3(r, add3(t, ss));
    }
    return r;
}

__device__ __forceinline__ float bsdfPdfImpl(const Ctx& c, float3 wi)
{
    float p = pdfDiffuse(c, wi) + pdfSpecular(c, wi);
    if (c.w.transmit != 0.0f) {
        p = p + pdfTransmit(c, wi);
    }
    if (c.w.subsurface != 0.0f) {
        p = p + pdfSubsurface(c, wi);
    }
    return p;
}

static __device__ __noinline__ float3 bsdfEval(const Ctx& c, float3 wi) { return bsdfEvalImpl(c, wi); }
static __device__ __noinline__ float bsdfPdf(const Ctx& c, float3 wi) { return bsdfPdfImpl(c, wi); }

__device__ __forceinline__ BsdfSample emptySample(const Ctx& c)
{
    BsdfSample s;
    s.dir = f3(0.0f, 0.0f, 0.0f);
    s.pdf = 0.0f;
    s.nextEta = 1.0f;
    s.exitOffset = f3(0.0f, 0.0f, 0.0f);
    s.sssSteps = 0;
    s.valid = s.transmitted = s.sss = false;
    (void)c;
    return s;
}

__device__ __forceinline__ BsdfSample sampleDiffuse(const Ctx& c, float u1, float u2)
{
    BsdfSample s = emptySample(c);
    float3 t, b;
    basis(c.n, t, b);
    s.dir = toWorld(cosineHemi(u1, u2), c.n, t, b);
    s.pdf = bsdfPdf(c, s.dir);
    s.valid = dot3(c.n, s.dir) > 0.0f && s.pdf > kMinPdf;
    s.nextEta = c.eta;
    return s;
}

static __device__ __noinline__ BsdfSample sampleSubsurface(const Ctx& c, float u1, float u2)
{
    if (maxScatter(c.m) <= kMinRadius) {
        return sampleDiffuse(c, u1, u2);
    }
    BsdfSample s = emptySample(c);
    float3 t, b;
    basis(c.n, t, b);
    const float u3 = u1 * 0.318f + u2 * 0.682f;
    const float er = effectiveRadius(c.m, u3);
    const float r = burleyRadius(u1, er);
    const float phi = 2.0f * kPi * u2;
    s.exitOffset = add3(scl3(t, r * cosf(phi)), scl3(b, r * sinf(phi)));
    const float3 l = cosineHemi(fmax2(kMinPdf, u1 * 0.5f + 0.25f), fmax2(kMinPdf, u2 * 0.5f + 0.25f));
    s.dir = toWorld(l, c.n, t, b);
    s.sss = true;
    s.sssSteps = clamp01(c.m.thin) > 0.5f ? 0 : 2;
    s.pdf = bsdfPdf(c, s.dir);
    s.valid = dot3(c.n, s.dir) > 0.0f && s.pdf > kMinPdf;
    s.nextEta = c.eta;
    return s;
}

__device__ __forceinline__ BsdfSample sampleSpecular(const Ctx& c, float u1, float u2)
{
    BsdfSample s = emptySample(c);
    const float cO = fmax2(0.0f, dot3(c.n, c.wo));
    if (cO <= 0.0f) {
        return s;
    }
    const float a = alphaFromRoughness(c.m.roughness);
    float3 t, b;
    basis(c.n, t, b);
    float hp = 0.0f;
    const float3 h = toWorld(ggxHalf(a, u1, u2, hp), c.n, t, b);
    const float cHo = fmax2(0.0f, dot3(h, c.wo));
    if (cHo <= 0.0f || hp <= kMinPdf) {
        return s;
    }
    s.dir = normalize3(sub3(scl3(h, 2.0f * cHo), c.wo));
    if (fmax2(0.0f, dot3(c.n, s.dir)) <= 0.0f) {
        return s;
    }
    s.pdf = bsdfPdf(c, s.dir);
    s.valid = s.pdf > kMinPdf;
    s.nextEta = c.eta;
    return s;
}

static __device__ __noinline__ BsdfSample sampleTransmit(const Ctx& c, float u1, float u2)
{
    BsdfSample s = emptySample(c);
    const float cOs = dot3(c.n, c.wo);
    if (!transmitValid(c, cOs)) {
        return s;
    }
    const float thin = clamp01(c.m.thin);
    const float ior = matIor(c);
    const float etaT = cOs > 0.0f ? ior : 1.0f;
    const float refl = dielectricFresnel(cOs, c.eta, etaT);
    const float trans = 1.0f - refl;
    bool refr = u1 < trans;
    if (c.debug & kDbgDisableRefract) {
        refr = false;
    }
    if (c.debug & kDbgDisableReflect) {
        refr = true;
    }
    Ctx rc = c;
    const float a = alphaFromRoughness(c.m.roughness);
    if (refr && thin < 0.5f && a > 0.04f) {
        float3 t, b;
        basis(c.n, t, b);
        float hp = 0.0f;
        rc.n = toWorld(ggxHalf(a, u2, u1 * 0.413f + u2 * 0.587f, hp), c.n, t, b);
    }
    if (refr) {
        if (thin > 0.5f) {
            s.dir = normalize3(scl3(c.wo, -1.0f));
            s.nextEta = c.eta;
        } else if (!refractDir(rc, s.dir, s.nextEta)) {
            if (c.debug & kDbgDisableTirFallback) {
                return s;
            }
            s.dir = mirrorOut(c.wo, c.n);
            s.transmitted = false;
            s.nextEta = c.eta;
        } else {
            s.transmitted = true;
        }
        if (thin > 0.5f) {
            s.transmitted = true;
        }
        if (absf(dot3(c.n, s.dir)) <= 0.0f) {
            return s;
        }
    } else {
        s.dir = mirrorOut(c.wo, c.n);
        if (absf(dot3(c.n, s.dir)) <= 0.0f) {
            return s;
        }
        s.transmitted = false;
        s.nextEta = c.eta;
    }
    s.pdf = bsdfPdf(c, s.dir);
    s.valid = s.pdf > kMinPdf;
    return s;
}

static __device__ __noinline__ BsdfSample bsdfSample(const Ctx& c, float u1, float u2)
{
    if (c.debug & kDbgForceTransmit) {
        return sampleTransmit(c, u1, u2);
    }
    const Lobes& w = c.w;
    if (u1 < w.diffuse) {
        return sampleDiffuse(c, u1 / fmax2(w.diffuse, kMinPdf), u2);
    }
    float u = u1 - w.diffuse;
    if (u < w.specular) {
        return sampleSpecular(c, (u1 - w.diffuse) / fmax2(w.specular, kMinPdf), u2);
    }
    u -= w.specular;
    if (u < w.transmit) {
        return sampleTransmit(c, (u1 - w.diffuse - w.specular) / fmax2(w.transmit, kMinPdf), u2);
    }
    return sampleSubsurface(c, (u1 - w.diffuse - w.specular - w.transmit) / fmax2(w.subsurface, kMinPdf), u2);
}

__device__ __forceinline__ bool skipsEnvNee(const Mat& m)
{
    return fmax2(0.0f, fmin2(1.0f, m.transmission)) > 0.99f && fmax2(0.0f, fmin2(1.0f, m.metallic)) < 0.01f;
}

// Emitter MIS mode: a vertex takes part when its BSDF samples the upper
// hemisphere with the mixture pdf the NEE weight uses and its throughput is
// f cos / pdf: no subsurface lobe, not the pure transmit lobe (whose throughput
// drops the cosine), outside any medium.  Directions in the transmit cones and
// below the surface stay with BSDF sampling alone.
__device__ __forceinline__ bool emitterMisVertex(const Ctx& c)
{
    return c.w.subsurface <= 0.0f && !skipsEnvNee(c.m) && c.eta == 1.0f;
}

// Throughput rule of the sampled lobe (BrdfDispatch.h:42-76): the new
// throughput is tp * f * k, times the base colour when `tint` (thin
// transmission); false when the sample ends the path.
__device__ __forceinline__ bool throughputFactor(const Ctx& c, const BsdfSample& s, float& k, bool& tint)
{
    tint = false;
    if (!s.valid || s.pdf <= kMinPdf) {
        return false;
    }
    const float trans = fmax2(0.0f, fmin2(1.0f, c.m.transmission));
    const float thin = fmax2(0.0f, fmin2(1.0f, c.m.thin));
    const bool pure = trans > 0.99f && c.m.metallic < 0.01f;
    if (pure && thin < 0.5f) {
        k = 1.0f / s.pdf;
    } else if (s.transmitted) {
        k = absf(dot3(c.n, s.dir)) / s.pdf;
        tint = thin > 0.5f;
    } else if (s.sss) {
        k = fmax2(0.0f, dot3(c.n, s.dir)) / s.pdf;
    } else {
        const float ct = c.eta > 1.0f + 1.0e-4f ? absf(dot3(c.n, s.dir)) : fmax2(0.0f, dot3(c.n, s.dir));
        k = ct / s.pdf;
    }
    return true;
}

__device__ __forceinline__ float3 applyThroughput(float3 tp, const Ctx& c, const BsdfSample& s, float3 f)
{
    float k;
    bool tint;
    if (!throughputFactor(c, s, k, tint)) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    float3 sc = scl3(f, k);
    if (tint) {
        sc = f3(sc.x * c.m.r, sc.y * c.m.g, sc.z * c.m.b);
    }
    return f3(tp.x * sc.x, tp.y * sc.y, tp.z * sc.z);
}

// --- lights (LightSamplingCore.h, MisCore.h) ----------------------------------
__device__ __forceinline__ float misBalance(float a, float b)
{
    if (a <= 0.0f) {
        return 0.0f;
    }
    const float d = a + b;
    if (d <= 0.0f) {
        return 0.0f;
    }
    return a / d;
}

__device__ __forceinline__ float3 latLongToDir(float u, float v)
{
    const float phi = u * 2.0f * kPi - kPi;
    const float theta = v * kPi;
    const float st = sinf(theta);
    return normalize3(f3(st * sinf(phi), cosf(theta), st * cosf(phi)));
}

__device__ __forceinline__ void dirToLatLong(float3 d, float& u, float& v)
{
    const float3 w = normalize3(d);
    const float phi = atan2f(w.x, w.z);
    const float theta = acosf(fmax2(-1.0f, fmin2(w.y, 1.0f)));
    u = (phi + kPi) / (2.0f * kPi);
    v = theta / kPi;
}

__device__ __forceinline__ float3 envEval(const DevEnv& e, const pt_render_params& p, float3 d)
{
    if (!e.valid) {
        const float k = p.environment_intensity;
        return f3(p.background_r * k, p.background_g * k, p.background_b * k);
    }
    float u, v;
    dirToLatLong(d, u, v);
    const int x = min(max(static_cast<int>(u * static_cast<float>(e.width)), 0), e.width - 1);
    const int y = min(max(static_cast<int>(v * static_cast<float>(e.height)), 0), e.height - 1);
    const float* px = e.pixels + (static_cast<size_t>(y) * e.width + x) * 3;
    return f3(px[0], px[1], px[2]);
}

__device__ __forceinline__ int cdfFind(const float* cdf, int count, float u)
{
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (cdf[mid] < u) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

__device__ __forceinline__ float envPdfTable(const DevEnv& e, int x, int y, float v)
{
    const int off = y * (e.width + 1);
    const float rp = e.row[off + x + 1] - e.row[off + x];
    const float mp = e.marginal[y + 1] - e.marginal[y];
    const float st = fmax2(1.0e-4f, sinf(v * kPi));
    return (mp * rp) * static_cast<float>(e.width * e.height) / (2.0f * kPi * kPi * st);
}

__device__ __forceinline__ float3 envSample(const DevEnv& e, float u1, float u2, float& pdf)
{
    if (!e.valid) {
        pdf = 1.0f / (4.0f * kPi);
        return latLongToDir(u1, u2);
    }
    const int y = cdfFind(e.marginal, e.height, u1);
    const int x = cdfFind(e.row + y * (e.width + 1), e.width, u2);
    const float u = (static_cast<float>(x) + 0.5f) / static_cast<float>(e.width);
    const float v = (static_cast<float>(y) + 0.5f) / static_cast<float>(e.height);
    const float3 d = latLongToDir(u, v);
    const float* px = e.pixels + (static_cast<size_t>(y) * e.width + x) * 3;
    pdf = envPdfTable(e, x, y, v);
    if (fmax2(fmax2(px[0], px[1]), px[2]) <= 0.0f) {
        pdf = 0.0f;
    }
    return d;
}

__device__ __forceinline__ float envPdf(const DevEnv& e, float3 d)
{
    if (!e.valid) {
        return 1.0f / (4.0f * kPi);
    }
    float u, v;
    dirToLatLong(d, u, v);
    const int x = min(max(static_cast<int>(u * static_cast<float>(e.width)), 0), e.width - 1);
    const int y = min(max(static_cast<int>(v * static_cast<float>(e.height)), 0), e.height - 1);
    return envPdfTable(e, x, y, v);
}

__device__ __forceinline__ float3 loadOrigVertex(const DevScene& S, uint32_t tri, int k)
{
    const float* p = reinterpret_cast<const float*>(S.origVerts) + 9ull * tri + 3 * k;
    return f3(p[0], p[1], p[2]);
}

__device__ __forceinline__ const pt_material* fetchMaterial(const DevScene& S, uint32_t tri, const pt_material* fallback)
{
    if (S.materials == nullptr || tri >= S.triCount) {
        return fallback;
    }
    const uint32_t mi = __float_as_uint(S.shade[tri].d.w);
    return mi < S.materialCount ? &S.materials[mi] : fallback;
}

// Emissive triangle sampling (LightSamplingCore.h:257-313).
__device__ __forceinline__ bool sampleEmissive(const DevScene& S, const pt_material* fallback, float uTri, float u1,
    float u2, float3& pos, float3& n, float3& L, float& pdf, float3& v0, float3& v1, float3& v2,
    uint32_t* triOut = nullptr)
{
    pdf = 0.0f;
    const uint32_t E = S.emissiveCount;
    const float total = S.emissiveCdf[E];
    if (total <= kMinPdf) {
        return false;
    }
    const float target = uTri * total;
    int lo = 0, hi = static_cast<int>(E) - 1;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (S.emissiveCdf[mid + 1] < target) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    const uint32_t tri = S.emissiveIdx[lo];
    if (triOut != nullptr) {
        *triOut = tri;
    }
    const pt_material& m = *fetchMaterial(S, tri, fallback);
    v0 = loadOrigVertex(S, tri, 0);
    v1 = loadOrigVertex(S, tri, 1);
    v2 = loadOrigVertex(S, tri, 2);
    const float su = sqrtf(fmax2(0.0f, u1));
    const float b0 = 1.0f - su;
    const float b1 = u2 * su;
    const float b2 = 1.0f - b0 - b1;
    pos = add3(add3(scl3(v0, b0), scl3(v1, b1)), scl3(v2, b2));
    const float3 e1 = sub3(v1, v0), e2 = sub3(v2, v0);
    const float3 cr = cross3(e1, e2);
    n = normalize3(cr);
    L = f3(m.r * m.emission, m.g * m.emission, m.b * m.emission);
    const float area = 0.5f * sqrtf(dot3(cr, cr));
    if (area <= kMinPdf) {
        return false;
    }
    pdf = ((S.emissiveCdf[lo + 1] - S.emissiveCdf[lo]) / total) / area;
    return pdf > kMinPdf;
}

// --- camera (CameraDevice.cuh:8-139) ---------------------------------------------
__device__ __forceinline__ float3 rotq(const float* q, float3 v)
{
    const float s = q[0];
    const float3 u = f3(q[1], q[2], q[3]);
    const float3 c1 = cross3(u, v);
    const float3 c2 = cross3(u, c1);
    return f3(v.x + 2.0f * c1.x * s + 2.0f * c2.x, v.y + 2.0f * c1.y * s + 2.0f * c2.y, v.z + 2.0f * c1.z * s + 2.0f * c2.z);
}

__device__ __forceinline__ float3 filmLocal(const pt_camera& c, float u, float v)
{
    const float nx = 2.0f * u - 1.0f;
    const float ny = 1.0f - 2.0f * v;
    const float th = tanf(c.fov_y * 0.5f);
    const float top = c.near_plane * th;
    return f3(nx * (top * c.aspect), ny * top, -c.near_plane);
}

__device__ __forceinline__ void cameraRay(const pt_camera& c, float u, float v, float l1, float l2, float3& ro, float3& rd)
{
    const float3 pos = f3(c.position[0], c.position[1], c.position[2]);
    if (c.focus_valid == 0 || c.aperture_radius <= 0.0f || c.focus_distance <= 0.0f || c.near_plane <= 0.0f) {
        ro = pos;
        rd = normalize3(rotq(c.orientation, filmLocal(c, u, v)));
        return;
    }
    const float3 right = normalize3(rotq(c.orientation, f3(1.0f, 0.0f, 0.0f)));
    const float3 up = normalize3(rotq(c.orientation, f3(0.0f, 1.0f, 0.0f)));
    const float3 pf = filmLocal(c, u, v);
    const float fs = c.focus_distance / c.near_plane;
    const float3 r = rotq(c.orientation, f3(pf.x * fs, pf.y * fs, -c.focus_distance));
    const float3 pfw = add3(pos, r);
    const float a = 2.0f * l1 - 1.0f;
    const float b = 2.0f * l2 - 1.0f;
    float dx = 0.0f, dy = 0.0f;
    if (!(a == 0.0f && b == 0.0f)) {
        float rr, th;
        if (fabsf(a) > fabsf(b)) {
            rr = a;
            th = (3.14159265358979323846f * 0.25f) * (b / a);
        } else {
            rr = b;
            th = (3.14159265358979323846f * 0.5f) - (3.14159265358979323846f * 0.25f) * (a / b);
        }
        dx = rr * cosf(th);
        dy = rr * sinf(th);
    }
    const float ox = dx * c.aperture_radius, oy = dy * c.aperture_radius;
    ro = f3(pos.x + right.x * ox + up.x * oy, pos.y + right.y * ox + up.y * oy, pos.z + right.z * ox + up.z * oy);
    rd = normalize3(sub3(pfw, ro));
}

} // namespace pt
