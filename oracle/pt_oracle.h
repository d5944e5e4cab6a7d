// CPU ORACLE for the path-tracer parity tests -- test infrastructure, never
// linked into the product.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it (through oracle/libpt_oracle.so).
//
// This is a restatement, in this project's own code, of the reference render
// path (ipilter/LSystemEditor PathTracerLib).  Every function names the
// reference file:line it follows.  It is templated on the scalar type:
//   Real = float  : follows the reference's FP32 operation order so that it
//                   can be compared bit-for-bit with the reference compiled
//                   for the host (oracle/_ref) when both are built without
//                   floating-point contraction;
//   Real = double : the same estimator in FP64, used as the "FP64 host oracle"
//                   that every GPU result states its error against.
// Constants are the reference's float literals, widened for FP64.
//
// Quirks of the reference that are kept on purpose (see the product's design
// notes): Q1 zero direction components disable the slab test, Q2 emission at
// BSDF-sampled hits is added without MIS, Q3 different shadow-ray offsets,
// Q4 firefly clamp, Q5 relative std-dev convergence test, Q6 shading normal
// only, Q7 lens draws always consumed.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// Plain-old-data records with the reference's byte layouts
// (MeshAccel/MeshAccelTypes.h:49-151, RenderTypes.h:5-28, CameraGpu.h:5-16).
// ---------------------------------------------------------------------------
struct alignas(16) MaterialRec {
    float r, g, b, roughness, metallic, transmission, thin, ior, subsurface, emission,
        diffuseRoughness, scatterR, scatterG, scatterB, specular;
    uint32_t albedoTex, roughnessTex, metallicTex, transmissionTex, thinTex, iorTex, subsurfaceTex,
        emissionTex;
    float sheen; // tail padding in the reference layout; this project's extension
};
static_assert(sizeof(MaterialRec) == 96, "material record is 96 bytes");

struct alignas(16) TextureRec {
    uint32_t kind;
    uint32_t pad[3];
    float p0[4], p1[4], p2[4];
};
static_assert(sizeof(TextureRec) == 64, "texture record is 64 bytes");

struct alignas(16) CameraRec {
    float position[3];
    float pad0;
    float orientation[4]; // (w, x, y, z)
    float fovY, aspect, nearPlane, farPlane, apertureRadius, focusDistance;
    float focusPoint[3];
    int focusValid;
    float pad1[2];
};
static_assert(sizeof(CameraRec) == 80, "camera record is 80 bytes");

struct ParamsRec {
    float backgroundR, backgroundG, backgroundB, environmentIntensity;
    int maxPathDepth, russianRouletteMinDepth, minSamples, maxSamplesPerPixel, debugOverlayMode,
        brdfDebugFlags;
    float relativeErrorThreshold;
};
static_assert(sizeof(ParamsRec) == 44, "params record is 44 bytes");

// ---------------------------------------------------------------------------
// Vector helpers (Geometry/MathCore.h:13-120).
// ---------------------------------------------------------------------------
template <class R>
struct V3 {
    R x, y, z;
};
template <class R>
struct V2 {
    R x, y;
};

template <class R> inline V3<R> mk(R x, R y, R z) { return V3<R>{x, y, z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> add(V3<R> a, V3<R> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class R> inline V3<R> sub(V3<R> a, V3<R> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class R> inline V3<R> scl(V3<R> v, R s) { return mk(v.x * s, v.y * s, v.z * s); }
template <class R> inline V3<R> mul(V3<R> a, V3<R> b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
template <class R> inline R len(V3<R> v) { using std::sqrt; return sqrt(dot(v, v)); }
template <class R> inline R mx(R a, R b) { return a > b ? a : b; }
template <class R> inline R mn(R a, R b) { return a < b ? a : b; }
template <class R> inline R clampv(R v, R lo, R hi) { return mx(lo, mn(v, hi)); }
template <class R> inline R absv(R v) { return v < R(0) ? -v : v; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// MathCore.h:67-75: zero-length vectors normalise to (0,0,-1).
template <class R> inline V3<R> nrm(V3<R> v)
{
    const R l = len(v);
    if (l <= R(0)) {
        return mk(R(0), R(0), R(-1));
    }
    const R inv = R(1) / l;
    return scl(v, inv);
}
template <class R> inline R lum709(V3<R> c) { return R(0.2126f) * c.x + R(0.7152f) * c.y + R(0.0722f) * c.z; }

template <class R> struct Kc {
    static constexpr R pi = R(3.14159265f);          // BrdfBase.h:16, LightSamplingCore.h:18
    static constexpr R invPi = R(1.0f / 3.14159265f); // BrdfBase.h:17 (computed in float)
    static constexpr R minPdf = R(1.0e-8f);
};

// ---------------------------------------------------------------------------
// Scene in the reference's host representation.
// ---------------------------------------------------------------------------
struct TriRec {
    float v[3][3];
    float n[3][3];
    float uv[3][2];
    uint32_t mat;
};

struct BvhNode {
    float bmin[3], bmax[3];
    uint32_t left, right, triStart, triCount;
};

// Distant light (an extension with no reference counterpart), restated from
// the product's definition: constant radiance in a cone around `dir`; the
// sky's next-event sample picks it with probability select (1/2, or 1 when the
// sky is black) after one extra draw, else the environment; MIS against BSDF
// sampling uses the mixture density; escaping rays see environment + light.
struct SunSetup {
    bool enabled = false;
    float dir[3] = {0, 0, 0}, t[3] = {0, 0, 0}, b[3] = {0, 0, 0};
    float omc = 0.0f, sin2 = 0.0f, pdf = 0.0f;
    float rgb[3] = {0, 0, 0};
    float temperature = 0.0f, scale = 0.0f;
    float coef[4] = {0, 0, 0, 0};
};

struct Scene {
    SunSetup sun;
    std::vector<TriRec> tris;
    std::vector<MaterialRec> materials;
    std::vector<TextureRec> textures;
    std::vector<BvhNode> nodes;
    uint32_t root = 0;
    std::vector<uint32_t> emissiveIdx;
    std::vector<float> emissiveCdf;
    // Emitter MIS mode (extension; no reference counterpart): at opaque
    // vertices emissive NEE's shadow ray stops short of the light sample and
    // BSDF-sampled emitter hits are balance-weighted against it.  emitIndex[t]
    // is triangle t's position in the emissive list (-1 if none).
    bool emitterMis = false;
    std::vector<int> emitIndex;
    // the product's stop-test extensions (isConverged); 0 = the reference's
    int adaptiveCriterion = 0;
};

struct Env {
    int width = 0, height = 0;
    std::vector<float> pixels, marginal, row;
};

template <class R> inline V3<R> vtx(const TriRec& t, int k) { return mk(R(t.v[k][0]), R(t.v[k][1]), R(t.v[k][2])); }
template <class R> inline V3<R> nml(const TriRec& t, int k) { return mk(R(t.n[k][0]), R(t.n[k][1]), R(t.n[k][2])); }

// ---------------------------------------------------------------------------
// Ray / box and ray / triangle (MeshAccel/MeshAccelIntersectCore.h:12-108).
// ---------------------------------------------------------------------------
template <class R>
inline bool rayBox(V3<R> o, V3<R> inv, const float* bmin, const float* bmax, R tMin, R tMax, R& tEnter, R& tExit)
{
    R te = tMin, tx = tMax;
    const R oo[3] = {o.x, o.y, o.z};
    const R ii[3] = {inv.x, inv.y, inv.z};
    for (int a = 0; a < 3; ++a) {
        R t0 = (R(bmin[a]) - oo[a]) * ii[a];
        R t1 = (R(bmax[a]) - oo[a]) * ii[a];
        if (ii[a] < R(0)) {
            std::swap(t0, t1);
        }
        te = mx(te, t0);
        tx = mn(tx, t1);
        if (te > tx) {
            return false;
        }
    }
    tEnter = te;
    tExit = tx;
    return tx >= tMin;
}

template <class R>
struct Hit {
    bool hit = false;
    R t = R(0);
    V3<R> normal{R(0), R(0), R(0)};
    V2<R> uv{R(0), R(0)};
    uint32_t tri = 0;
};

template <class R>
inline bool rayTri(V3<R> o, V3<R> d, const TriRec& tri, R tMin, R tMax, R& outT, V3<R>& outN, V2<R>& outUv)
{
    using std::fabs;
    const V3<R> v0 = vtx<R>(tri, 0), v1 = vtx<R>(tri, 1), v2 = vtx<R>(tri, 2);
    const V3<R> e1 = sub(v1, v0);
    const V3<R> e2 = sub(v2, v0);
    const V3<R> p = mk(d.y * e2.z - d.z * e2.y, d.z * e2.x - d.x * e2.z, d.x * e2.y - d.y * e2.x);
    const R det = dot(e1, p);
    if (fabs(det) < R(1.0e-8f)) {
        return false;
    }
    const R invDet = R(1) / det;
    const V3<R> tv = sub(o, v0);
    const R bu = dot(tv, p) * invDet;
    if (bu < R(0) || bu > R(1)) {
        return false;
    }
    const V3<R> q = mk(tv.y * e1.z - tv.z * e1.y, tv.z * e1.x - tv.x * e1.z, tv.x * e1.y - tv.y * e1.x);
    const R bv = dot(d, q) * invDet;
    if (bv < R(0) || bu + bv > R(1)) {
        return false;
    }
    const R t = dot(e2, q) * invDet;
    if (t < tMin || t > tMax) {
        return false;
    }
    const R bw = R(1) - bu - bv;
    outT = t;
    V3<R> n = nrm(add(add(scl(nml<R>(tri, 0), bw), scl(nml<R>(tri, 1), bu)), scl(nml<R>(tri, 2), bv)));
    if (dot(n, d) > R(0)) {
        n = scl(n, R(-1));
    }
    outN = n;
    outUv = V2<R>{R(tri.uv[0][0]) * bw + R(tri.uv[1][0]) * bu + R(tri.uv[2][0]) * bv,
        R(tri.uv[0][1]) * bw + R(tri.uv[1][1]) * bu + R(tri.uv[2][1]) * bv};
    return true;
}

// Stack traversal, near child first, 64-entry stack (MeshAccelIntersectCore.h:110-221).
template <class R>
inline Hit<R> traceRay(const Scene& s, V3<R> o, V3<R> d, R tMin, R tMax)
{
    using std::fabs;
    Hit<R> res;
    if (s.nodes.empty() || s.tris.empty()) {
        return res;
    }
    d = nrm(d);
    const V3<R> inv = mk(fabs(d.x) > R(1.0e-8f) ? R(1) / d.x : R(0), fabs(d.y) > R(1.0e-8f) ? R(1) / d.y : R(0),
        fabs(d.z) > R(1.0e-8f) ? R(1) / d.z : R(0));
    int stack[64];
    int sp = 0;
    stack[sp++] = static_cast<int>(s.root);
    R closest = tMax;
    V3<R> cn{R(0), R(0), R(0)};
    V2<R> cuv{R(0), R(0)};
    uint32_t ctri = 0;
    const int nodeCount = static_cast<int>(s.nodes.size());
    while (sp > 0) {
        const int ni = stack[--sp];
        if (ni < 0 || ni >= nodeCount) {
            continue;
        }
        const BvhNode& node = s.nodes[static_cast<size_t>(ni)];
        R te, tx;
        if (!rayBox(o, inv, node.bmin, node.bmax, tMin, closest, te, tx)) {
            continue;
        }
        if (node.triCount > 0) {
            const uint32_t end = node.triStart + node.triCount;
            for (uint32_t ti = node.triStart; ti < end; ++ti) {
                if (ti >= s.tris.size()) {
                    break;
                }
                R th;
                V3<R> n;
                V2<R> uv;
                if (rayTri(o, d, s.tris[ti], tMin, closest, th, n, uv)) {
                    closest = th;
                    cn = n;
                    cuv = uv;
                    ctri = ti;
                }
            }
            continue;
        }
        if (sp + 2 > 64) {
            continue;
        }
        const int l = static_cast<int>(node.left), r = static_cast<int>(node.right);
        R le = R(0), lx = R(0), re = R(0), rx = R(0);
        bool lh = false, rh = false;
        if (l >= 0 && l < nodeCount) {
            lh = rayBox(o, inv, s.nodes[l].bmin, s.nodes[l].bmax, tMin, closest, le, lx);
        }
        if (r >= 0 && r < nodeCount) {
            rh = rayBox(o, inv, s.nodes[r].bmin, s.nodes[r].bmax, tMin, closest, re, rx);
        }
        if (lh && rh) {
            if (le < re) {
                stack[sp++] = r;
                stack[sp++] = l;
            } else {
                stack[sp++] = l;
                stack[sp++] = r;
            }
        } else if (lh) {
            stack[sp++] = l;
        } else if (rh) {
            stack[sp++] = r;
        }
    }
    if (closest < tMax) {
        res.hit = true;
        res.t = closest;
        res.normal = nrm(cn);
        res.uv = cuv;
        res.tri = ctri;
    }
    return res;
}

// ---------------------------------------------------------------------------
// Procedural textures and material resolve (Texture/ProceduralTexture.h:27-207).
// ---------------------------------------------------------------------------
template <class R> inline R fract(R v) { using std::floor; return v - floor(v); }
template <class R> inline R clamp01f(R v) { using std::fmax; using std::fmin; return fmin(fmax(v, R(0)), R(1)); }

template <class R>
inline R texScalar(const TextureRec& t, V2<R> uv, R u1d)
{
    switch (t.kind) {
    case 0: // ConstantScalar
        return R(t.p0[0]);
    case 3: { // Stripe1D
        const R c = fract(u1d * R(t.p0[0]));
        return c < R(t.p0[1]) ? R(t.p0[2]) : R(t.p0[3]);
    }
    case 2: { // Grid2D
        const R fx = fract(uv.x * R(t.p0[0]));
        const R fy = fract(uv.y * R(t.p0[1]));
        return (fx < R(t.p0[2]) || fy < R(t.p0[2])) ? R(1) : R(0);
    }
    default:
        return R(0);
    }
}

template <class R>
inline V3<R> texRgb(const TextureRec& t, V2<R> uv)
{
    switch (t.kind) {
    case 1: // ConstantRgb
        return mk(R(t.p0[0]), R(t.p0[1]), R(t.p0[2]));
    case 2: { // Grid2D
        const R fx = fract(uv.x * R(t.p0[0]));
        const R fy = fract(uv.y * R(t.p0[1]));
        const R g = (fx < R(t.p0[2]) || fy < R(t.p0[2])) ? R(1) : R(0);
        return mk(R(t.p1[0]) + (R(t.p2[0]) - R(t.p1[0])) * g, R(t.p1[1]) + (R(t.p2[1]) - R(t.p1[1])) * g,
            R(t.p1[2]) + (R(t.p2[2]) - R(t.p1[2])) * g);
    }
    default:
        return mk(R(0), R(0), R(0));
    }
}

// Resolved material in Real precision (the fields of MaterialGpu that the BSDF reads).
template <class R>
struct Mat {
    R r, g, b, roughness, metallic, transmission, thin, ior, subsurface, emission, diffuseRoughness, scatterR,
        scatterG, scatterB, specular;
    R sheen; // extension (no reference counterpart): white sheen lobe, 0 = the reference BSDF
};

template <class R>
inline Mat<R> matFromRec(const MaterialRec& m)
{
    return Mat<R>{R(m.r), R(m.g), R(m.b), R(m.roughness), R(m.metallic), R(m.transmission), R(m.thin), R(m.ior),
        R(m.subsurface), R(m.emission), R(m.diffuseRoughness), R(m.scatterR), R(m.scatterG), R(m.scatterB),
        R(m.specular), R(m.sheen)};
}

// ProceduralTexture.h:138-207 (resolveMaterial + materialFromResolved).
template <class R>
inline Mat<R> resolve(const MaterialRec& m, V2<R> uv, const std::vector<TextureRec>& bank)
{
    using std::fmax;
    const uint32_t n = static_cast<uint32_t>(bank.size());
    auto scalar = [&](float inl, uint32_t ti) -> R {
        if (ti == 0u || n == 0u || ti >= n) {
            return R(inl);
        }
        return texScalar<R>(bank[ti], uv, uv.x);
    };
    Mat<R> o{};
    if (m.albedoTex == 0u || n == 0u || m.albedoTex >= n) {
        o.r = R(m.r);
        o.g = R(m.g);
        o.b = R(m.b);
    } else {
        const V3<R> c = texRgb<R>(bank[m.albedoTex], uv);
        o.r = c.x;
        o.g = c.y;
        o.b = c.z;
    }
    o.roughness = clamp01f(scalar(m.roughness, m.roughnessTex));
    o.metallic = clamp01f(scalar(m.metallic, m.metallicTex));
    o.transmission = clamp01f(scalar(m.transmission, m.transmissionTex));
    o.thin = clamp01f(scalar(m.thin, m.thinTex));
    o.ior = fmax(R(1.0e-3f), scalar(m.ior, m.iorTex));
    o.subsurface = clamp01f(scalar(m.subsurface, m.subsurfaceTex));
    o.emission = fmax(R(0), scalar(m.emission, m.emissionTex));
    o.diffuseRoughness = R(m.diffuseRoughness);
    if (o.diffuseRoughness < R(0)) {
        o.diffuseRoughness = o.roughness;
    } else {
        o.diffuseRoughness = clamp01f(o.diffuseRoughness);
    }
    o.scatterR = fmax(R(0), R(m.scatterR));
    o.scatterG = fmax(R(0), R(m.scatterG));
    o.scatterB = fmax(R(0), R(m.scatterB));
    o.specular = clamp01f(R(m.specular));
    o.sheen = clamp01f(R(m.sheen));
    return o;
}

// ---------------------------------------------------------------------------
// BSDF building blocks (Brdf/BrdfBase.h:76-280) and Burley subsurface
// (Brdf/SubsurfaceCore.h:20-118).
// ---------------------------------------------------------------------------
template <class R>
struct Ctx {
    V3<R> n, wo;
    Mat<R> m;
    R eta;
    int debug;
};

template <class R>
struct Sample {
    V3<R> dir{R(0), R(0), R(0)};
    R pdf = R(0);
    bool valid = false, transmitted = false;
    R nextEta = R(1);
    bool sss = false;
    V3<R> exitOffset{R(0), R(0), R(0)};
    int sssSteps = 0;
};

template <class R> inline void basis(V3<R> n, V3<R>& t, V3<R>& b)
{
    using std::fabs;
    const V3<R> up = fabs(n.y) < R(0.999f) ? mk(R(0), R(1), R(0)) : mk(R(1), R(0), R(0));
    t = nrm(cross(up, n));
    b = nrm(cross(n, t));
}
template <class R> inline V3<R> toWorld(V3<R> l, V3<R> n, V3<R> t, V3<R> b)
{
    return nrm(add(add(scl(t, l.x), scl(b, l.y)), scl(n, l.z)));
}
template <class R> inline V3<R> cosineHemi(R u1, R u2)
{
    using std::cos; using std::sin; using std::sqrt;
    const R phi = R(2) * Kc<R>::pi * u1;
    const R r = sqrt(u2);
    return mk(r * cos(phi), r * sin(phi), sqrt(mx(R(0), R(1) - u2)));
}
template <class R> inline R cosinePdf(R c) { return mx(R(0), c) * Kc<R>::invPi; }
template <class R> inline R alphaFromRoughness(R r) { const R c = mx(r, R(0.04f)); return c * c; }
template <class R> inline R ggxD(R cosH, R a)
{
    const R a2 = a * a;
    const R c2 = cosH * cosH;
    const R den = c2 * (a2 - R(1)) + R(1);
    return a2 / (Kc<R>::pi * den * den);
}
template <class R> inline R smithG1(R c, R a)
{
    using std::sqrt;
    const R a2 = a * a;
    const R c2 = mx(c * c, R(1.0e-8f));
    const R t2 = (R(1) - c2) / c2;
    return R(2) / (R(1) + sqrt(R(1) + a2 * t2));
}
template <class R> inline V3<R> schlick(R c, V3<R> f0)
{
    const R t = mx(R(0), mn(R(1), R(1) - c));
    const R t2 = t * t;
    const R t5 = t2 * t2 * t;
    return add(scl(f0, R(1) - t5), mk(t5, t5, t5));
}
template <class R> inline V3<R> ggxHalf(R a, R u1, R u2, R& pdf)
{
    using std::cos; using std::sin; using std::sqrt;
    const R phi = R(2) * Kc<R>::pi * u1;
    const R a2 = a * a;
    const R ct = sqrt((R(1) - u2) / (R(1) + (a2 - R(1)) * u2));
    const R st = sqrt(mx(R(0), R(1) - ct * ct));
    const R cp = cos(phi);
    const R sp = sin(phi);
    pdf = (a2 * ct) / (Kc<R>::pi * (ct * ct * (a2 - R(1)) + R(1)) * (ct * ct * (a2 - R(1)) + R(1)));
    return mk(st * cp, st * sp, ct);
}
template <class R> inline R dielectricFresnel(R cosI_, R etaI, R etaT)
{
    using std::sqrt;
    R cosI = mx(R(-1), mn(R(1), cosI_));
    R eta = etaI / mx(etaT, R(1.0e-8f));
    if (cosI < R(0)) {
        cosI = -cosI;
        eta = R(1) / eta;
    }
    const R s2 = eta * eta * (R(1) - cosI * cosI);
    if (s2 >= R(1)) {
        return R(1);
    }
    const R cosT = sqrt(mx(R(0), R(1) - s2));
    const R rp = (eta * cosI - cosT) / mx(eta * cosI + cosT, R(1.0e-8f));
    const R rs = (cosI - eta * cosT) / mx(cosI + eta * cosT, R(1.0e-8f));
    return R(0.5f) * (rp * rp + rs * rs);
}
template <class R> inline bool refractRel(V3<R> wo, V3<R> n_, R etaI, R etaT, V3<R>& out)
{
    using std::sqrt;
    R cO = dot(n_, wo);
    V3<R> n = n_;
    R er = etaI / mx(etaT, R(1.0e-8f));
    if (cO > R(0)) {
        n = scl(n_, R(-1));
        er = R(1) / er;
        cO = -cO;
    }
    const R s2 = er * er * (R(1) - cO * cO);
    if (s2 >= R(1)) {
        return false;
    }
    const R cT = sqrt(mx(R(0), R(1) - s2));
    out = nrm(sub(scl(wo, -er), scl(n, er * cO + cT)));
    return true;
}
template <class R> inline R diffuseRough(const Mat<R>& m)
{
    const R v = m.diffuseRoughness < R(0) ? m.roughness : m.diffuseRoughness;
    return mx(R(0), mn(R(1), v));
}
template <class R> inline R orenNayar(R sigma, R cI, R cO, R dWoWi)
{
    using std::sqrt;
    if (sigma <= R(1.0e-4f)) {
        return R(1);
    }
    const R s2 = sigma * sigma;
    const R A = R(1) - R(0.5f) * s2 / (s2 + R(0.33f));
    const R B = R(0.45f) * s2 / (s2 + R(0.09f));
    const R sI = sqrt(mx(R(0), R(1) - cI * cI));
    const R sO = sqrt(mx(R(0), R(1) - cO * cO));
    R sA, sB;
    if (cI > cO) {
        sA = sI;
        sB = sO;
    } else {
        sA = sO;
        sB = sI;
    }
    R cosPhi = R(1);
    const R d = dWoWi - cI * cO;
    if (d <= R(0)) {
        const R den = mx(sA * sB, R(1.0e-8f));
        cosPhi = mx(R(-1), mn(R(1), d / den));
    } else {
        sA = R(0);
        sB = R(0);
    }
    const R tB = sB / mx(cI, cO);
    return A + B * mx(R(0), cosPhi) * sA * tB;
}
template <class R> inline R energyComp(R rough, R c)
{
    const R a = alphaFromRoughness(rough);
    const R cc = mx(c, R(1.0e-4f));
    const R Ess = R(1) - a * (R(0.3316f) + R(0.3237f) * a);
    const R Ems = (R(1) - Ess) * (R(1) - cc);
    return R(1) + Ems / mx(Ess, R(1.0e-4f));
}
template <class R> inline V3<R> scatterRadius(const Mat<R>& m)
{
    return mk(mx(R(0), m.scatterR), mx(R(0), m.scatterG), mx(R(0), m.scatterB));
}
template <class R> inline R maxScatter(const Mat<R>& m)
{
    const V3<R> r = scatterRadius(m);
    return mx(mx(r.x, r.y), r.z);
}

constexpr float kMinRadius = 1.0e-5f; // SubsurfaceCore.h:15

template <class R> inline R burleyRadius(R u, R d)
{
    using std::exp; using std::log; using std::sqrt;
    const R sd = mx(d, R(kMinRadius));
    return sd * sqrt(-log(mx(R(1.0e-8f), R(1) - u * (R(1) - exp(R(-1) / sd)))));
}
template <class R> inline R burleyProfile(R r, R d)
{
    using std::exp;
    const R sd = mx(d, R(kMinRadius));
    return (exp(-r / sd) + exp(-r / (R(3) * sd))) / (R(4) * Kc<R>::pi * sd);
}
template <class R> inline R burleyPdf(R r, R d)
{
    using std::exp;
    const R sd = mx(d, R(kMinRadius));
    const R t0 = exp(-r / sd);
    const R t1 = exp(-r / (R(3) * sd));
    const R nn = R(1) - exp(R(-1) / sd);
    return mx(R(0), (t0 + t1) / mx(R(2) * sd * nn, R(1.0e-8f)));
}
template <class R> inline V3<R> burleyEval(const Mat<R>& m, R disk, R cI, R cO)
{
    const V3<R> rad = scatterRadius(m);
    const R sum = mx(rad.x + rad.y + rad.z, R(kMinRadius));
    const V3<R> w = mk(rad.x / sum, rad.y / sum, rad.z / sum);
    const R pR = burleyProfile(disk, mx(rad.x, R(kMinRadius)));
    const R pG = burleyProfile(disk, mx(rad.y, R(kMinRadius)));
    const R pB = burleyProfile(disk, mx(rad.z, R(kMinRadius)));
    const R df = mx(cI, R(0)) * mx(cO, R(0));
    return mk(w.x * pR * df, w.y * pG * df, w.z * pB * df);
}
template <class R> inline R effectiveRadius(const Mat<R>& m, R uc)
{
    const V3<R> rad = scatterRadius(m);
    const R mr = maxScatter(m);
    if (mr <= R(kMinRadius)) {
        return R(kMinRadius);
    }
    if (uc < rad.x / (rad.x + rad.y + rad.z + R(kMinRadius))) {
        return mx(rad.x, R(kMinRadius));
    }
    if (uc < (rad.x + rad.y) / (rad.x + rad.y + rad.z + R(kMinRadius))) {
        return mx(rad.y, R(kMinRadius));
    }
    return mx(rad.z, R(kMinRadius));
}
template <class R> inline void exitOffset(const Ctx<R>& c, R u1, R u2, R u3, V3<R>& off, R& disk, R& pdf)
{
    using std::cos; using std::sin;
    V3<R> t, b;
    basis(c.n, t, b);
    const R er = effectiveRadius(c.m, u3);
    const R r = burleyRadius(u1, er);
    const R phi = R(2) * Kc<R>::pi * u2;
    off = add(scl(t, r * cos(phi)), scl(b, r * sin(phi)));
    disk = r;
    pdf = burleyPdf(r, er) / mx(R(2) * Kc<R>::pi * r, R(1.0e-8f));
}

// ---------------------------------------------------------------------------
// Principled BSDF (Brdf/PrincipledBrdf.h:14-588).
// ---------------------------------------------------------------------------
template <class R> struct Lobes {
    R diffuse, specular, transmit, subsurface;
};

template <class R> inline R clamp01(R v) { return mx(R(0), mn(R(1), v)); }
template <class R> inline R matIor(const Ctx<R>& c) { return mx(c.m.ior, R(1.0e-3f)); } // SpectralCore.h:221-225

template <class R> inline Lobes<R> lobes(const Ctx<R>& c)
{
    Lobes<R> w{};
    const R metal = clamp01(c.m.metallic);
    const R trans = clamp01(c.m.transmission);
    const R sss = clamp01(c.m.subsurface);
    const R diel = R(1) - metal;
    w.transmit = diel * trans;
    w.subsurface = diel * (R(1) - trans) * sss;
    w.diffuse = diel * (R(1) - trans) * (R(1) - sss);
    w.specular = metal + diel * (R(1) - trans);
    const R sum = w.diffuse + w.specular + w.transmit + w.subsurface;
    if (sum <= Kc<R>::minPdf) {
        w.diffuse = R(1);
        return w;
    }
    const R inv = R(1) / sum;
    w.diffuse *= inv;
    w.specular *= inv;
    w.transmit *= inv;
    w.subsurface *= inv;
    return w;
}

template <class R> inline V3<R> specF0(const Ctx<R>& c)
{
    const R metal = clamp01(c.m.metallic);
    const R ior = matIor(c);
    const R f = (ior - R(1)) / (ior + R(1));
    const R v = f * f * clamp01(clamp01(c.m.specular));
    return mk(v + (c.m.r - v) * metal, v + (c.m.g - v) * metal, v + (c.m.b - v) * metal);
}

template <class R> inline V3<R> mirrorOut(V3<R> wo, V3<R> n)
{
    return nrm(sub(scl(n, R(2) * dot(n, wo)), wo));
}

template <class R> inline R onFactor(const Ctx<R>& c, V3<R> wi)
{
    const R cI = mx(R(0), dot(c.n, wi));
    const R cO = mx(R(0), dot(c.n, c.wo));
    if (cI <= R(0) || cO <= R(0)) {
        return R(0);
    }
    const R sigma = diffuseRough(c.m) * R(0.5f) * Kc<R>::pi;
    return orenNayar(sigma, cI, cO, dot(wi, c.wo));
}

template <class R> inline V3<R> evalDiffuse(const Ctx<R>& c, V3<R> wi)
{
    const R cI = mx(R(0), dot(c.n, wi));
    const R cO = mx(R(0), dot(c.n, c.wo));
    if (cI <= R(0) || cO <= R(0)) {
        return mk(R(0), R(0), R(0));
    }
    const Lobes<R> w = lobes(c);
    const R on = onFactor(c, wi);
    V3<R> r = scl(mk(c.m.r, c.m.g, c.m.b), w.diffuse * on * Kc<R>::invPi);
    if (c.m.sheen > R(0)) {
        // extension: white sheen sheen * (1 - cos theta_d)^5 on the diffuse lobe
        // (theta_d between wi and the half vector; the Disney BRDF's sheen term)
        const V3<R> h = nrm(add(wi, c.wo));
        const R x = R(1) - mx(R(0), dot(wi, h));
        const R x2 = x * x;
        const R sh = w.diffuse * c.m.sheen * (x2 * x2 * x);
        r = add(r, mk(sh, sh, sh));
    }
    return r;
}

template <class R> inline V3<R> evalSubsurface(const Ctx<R>& c, V3<R> wi)
{
    using std::sqrt;
    const R cI = mx(R(0), dot(c.n, wi));
    const R cO = mx(R(0), dot(c.n, c.wo));
    if (cI <= R(0) || cO <= R(0)) {
        return mk(R(0), R(0), R(0));
    }
    const Lobes<R> w = lobes(c);
    const V3<R> base = mk(c.m.r, c.m.g, c.m.b);
    if (maxScatter(c.m) <= R(kMinRadius)) {
        const R on = onFactor(c, wi);
        return scl(base, w.subsurface * on * Kc<R>::invPi);
    }
    V3<R> t, b;
    basis(c.n, t, b);
    const V3<R> wt = add(scl(t, dot(wi, t)), scl(b, dot(wi, b)));
    const R disk = sqrt(dot(wt, wt));
    const V3<R> bu = burleyEval(c.m, disk, cI, cO);
    return mk(base.x * w.subsurface * bu.x, base.y * w.subsurface * bu.y, base.z * w.subsurface * bu.z);
}

template <class R> inline V3<R> evalSpecular(const Ctx<R>& c, V3<R> wi)
{
    const R cO = mx(R(0), dot(c.n, c.wo));
    const R cI = mx(R(0), dot(c.n, wi));
    if (cO <= R(0) || cI <= R(0)) {
        return mk(R(0), R(0), R(0));
    }
    const V3<R> h = nrm(add(wi, c.wo));
    const R cH = mx(R(0), dot(c.n, h));
    const R cHo = mx(R(0), dot(h, c.wo));
    if (cHo <= R(0)) {
        return mk(R(0), R(0), R(0));
    }
    const Lobes<R> w = lobes(c);
    const R a = alphaFromRoughness(c.m.roughness);
    const R D = ggxD(cH, a);
    const R G = smithG1(cO, a) * smithG1(cI, a);
    const V3<R> F = schlick(cHo, specF0(c));
    const R ec = energyComp(c.m.roughness, cO);
    const R den = mx(R(4) * cO * cI, R(1.0e-8f));
    const R s = w.specular * ec * (D * G) / den;
    return mk(F.x * s, F.y * s, F.z * s);
}

template <class R> inline bool refractDir(const Ctx<R>& c, V3<R>& out, R& nextEta)
{
    const R cO = dot(c.n, c.wo);
    const R ior = matIor(c);
    const R etaI = c.eta;
    R etaT;
    if (cO > R(0)) {
        etaT = ior;
        nextEta = ior;
    } else {
        etaT = R(1);
        nextEta = R(1);
    }
    return refractRel(c.wo, c.n, etaI, etaT, out);
}

template <class R> inline bool transmitValid(const Ctx<R>& c, R cOs)
{
    if (absv(cOs) <= Kc<R>::minPdf) {
        return false;
    }
    return cOs > R(0) || c.eta > R(1.0f + 1.0e-4f);
}

template <class R> inline V3<R> evalTransmit(const Ctx<R>& c, V3<R> wi)
{
    const R cOs = dot(c.n, c.wo);
    if (!transmitValid(c, cOs)) {
        return mk(R(0), R(0), R(0));
    }
    const Lobes<R> w = lobes(c);
    const R thin = clamp01(c.m.thin);
    const V3<R> base = mk(c.m.r, c.m.g, c.m.b);
    const R ior = matIor(c);
    const R etaT = cOs > R(0) ? ior : R(1);
    const R refl = dielectricFresnel(cOs, c.eta, etaT);
    const R trans = R(1) - refl;
    const V3<R> reflected = mirrorOut(c.wo, c.n);
    if (dot(wi, reflected) > R(0.999f)) {
        const R cI = absv(dot(c.n, wi));
        return scl(base, w.transmit * refl / mx(cI, R(1.0e-8f)));
    }
    V3<R> td{R(0), R(0), R(0)};
    R ne = R(1);
    if (thin > R(0.5f)) {
        td = nrm(scl(c.wo, R(-1)));
    } else if (!refractDir(c, td, ne)) {
        return mk(R(0), R(0), R(0));
    }
    if (dot(wi, td) > R(0.999f)) {
        const R cI = absv(dot(c.n, td));
        const V3<R> tint = thin > R(0.5f) ? base : mk(R(1), R(1), R(1));
        return mk(tint.x * w.transmit * trans / mx(cI, R(1.0e-8f)), tint.y * w.transmit * trans / mx(cI, R(1.0e-8f)),
            tint.z * w.transmit * trans / mx(cI, R(1.0e-8f)));
    }
    const R a = alphaFromRoughness(c.m.roughness);
    if (a > R(0.04f)) {
        const V3<R> h = nrm(add(wi, c.wo));
        const R cH = mx(R(0), absv(dot(c.n, h)));
        const R D = ggxD(cH, a);
        const R rp = D * cH;
        if (rp > Kc<R>::minPdf) {
            const V3<R> tint = thin > R(0.5f) ? base : mk(R(1), R(1), R(1));
            const R s = w.transmit * trans * rp;
            return mk(tint.x * s, tint.y * s, tint.z * s);
        }
    }
    return mk(R(0), R(0), R(0));
}

template <class R> inline R pdfDiffuse(const Ctx<R>& c, V3<R> wi)
{
    return lobes(c).diffuse * cosinePdf(mx(R(0), dot(c.n, wi)));
}

template <class R> inline R pdfSubsurface(const Ctx<R>& c, V3<R> wi)
{
    using std::sqrt;
    const Lobes<R> w = lobes(c);
    const R cp = cosinePdf(mx(R(0), dot(c.n, wi)));
    if (maxScatter(c.m) <= R(kMinRadius)) {
        return w.subsurface * cp;
    }
    V3<R> t, b;
    basis(c.n, t, b);
    const V3<R> wt = add(scl(t, dot(wi, t)), scl(b, dot(wi, b)));
    const R disk = sqrt(dot(wt, wt));
    const R rp = burleyPdf(disk, maxScatter(c.m));
    return w.subsurface * mx(cp, rp * R(0.5f));
}

template <class R> inline R pdfSpecular(const Ctx<R>& c, V3<R> wi)
{
    const R cO = mx(R(0), dot(c.n, c.wo));
    const R cI = mx(R(0), dot(c.n, wi));
    if (cO <= R(0) || cI <= R(0)) {
        return R(0);
    }
    const V3<R> h = nrm(add(wi, c.wo));
    const R cH = mx(R(0), dot(c.n, h));
    const R cHo = mx(R(0), dot(h, c.wo));
    if (cHo <= R(0)) {
        return R(0);
    }
    const Lobes<R> w = lobes(c);
    const R a = alphaFromRoughness(c.m.roughness);
    const R hp = ggxD(cH, a) * cH;
    return w.specular * hp / mx(R(4) * cHo, R(1.0e-8f));
}

template <class R> inline R pdfTransmit(const Ctx<R>& c, V3<R> wi)
{
    const R cOs = dot(c.n, c.wo);
    if (!transmitValid(c, cOs)) {
        return R(0);
    }
    const Lobes<R> w = lobes(c);
    const R thin = clamp01(c.m.thin);
    const R ior = matIor(c);
    const R etaT = cOs > R(0) ? ior : R(1);
    const R refl = dielectricFresnel(cOs, c.eta, etaT);
    const R trans = R(1) - refl;
    R pdf = R(0);
    const V3<R> reflected = mirrorOut(c.wo, c.n);
    if (dot(wi, reflected) > R(0.999f)) {
        const R cI = absv(dot(c.n, wi));
        pdf += w.transmit * refl / mx(cI, R(1.0e-8f));
    }
    V3<R> td{R(0), R(0), R(0)};
    if (thin > R(0.5f)) {
        td = nrm(scl(c.wo, R(-1)));
    } else {
        R ne = R(1);
        if (!refractDir(c, td, ne)) {
            return pdf;
        }
    }
    if (dot(wi, td) > R(0.999f)) {
        const R cI = absv(dot(c.n, td));
        pdf += w.transmit * trans / mx(cI, R(1.0e-8f));
    }
    return pdf;
}

template <class R> inline V3<R> bsdfEval(const Ctx<R>& c, V3<R> wi)
{
    const V3<R> d = evalDiffuse(c, wi);
    const V3<R> s = evalSpecular(c, wi);
    const V3<R> t = evalTransmit(c, wi);
    const V3<R> ss = evalSubsurface(c, wi);
    return add(add(d, s), add(t, ss));
}

template <class R> inline R bsdfPdf(const Ctx<R>& c, V3<R> wi)
{
    return pdfDiffuse(c, wi) + pdfSpecular(c, wi) + pdfTransmit(c, wi) + pdfSubsurface(c, wi);
}

template <class R> inline Sample<R> sampleDiffuse(const Ctx<R>& c, R u1, R u2)
{
    Sample<R> s;
    V3<R> t, b;
    basis(c.n, t, b);
    s.dir = toWorld(cosineHemi(u1, u2), c.n, t, b);
    s.pdf = bsdfPdf(c, s.dir);
    s.valid = dot(c.n, s.dir) > R(0) && s.pdf > Kc<R>::minPdf;
    s.transmitted = false;
    s.nextEta = c.eta;
    return s;
}

template <class R> inline Sample<R> sampleSubsurface(const Ctx<R>& c, R u1, R u2)
{
    Sample<R> s;
    if (maxScatter(c.m) <= R(kMinRadius)) {
        return sampleDiffuse(c, u1, u2);
    }
    V3<R> off;
    R disk, opdf;
    const R u3 = u1 * R(0.318f) + u2 * R(0.682f);
    exitOffset(c, u1, u2, u3, off, disk, opdf);
    V3<R> t, b;
    basis(c.n, t, b);
    const V3<R> l = cosineHemi(mx(Kc<R>::minPdf, u1 * R(0.5f) + R(0.25f)), mx(Kc<R>::minPdf, u2 * R(0.5f) + R(0.25f)));
    s.dir = toWorld(l, c.n, t, b);
    s.sss = true;
    s.exitOffset = off;
    s.sssSteps = clamp01(c.m.thin) > R(0.5f) ? 0 : 2;
    s.pdf = bsdfPdf(c, s.dir);
    s.valid = dot(c.n, s.dir) > R(0) && s.pdf > Kc<R>::minPdf;
    s.transmitted = false;
    s.nextEta = c.eta;
    return s;
}

template <class R> inline Sample<R> sampleSpecular(const Ctx<R>& c, R u1, R u2)
{
    Sample<R> s;
    const R cO = mx(R(0), dot(c.n, c.wo));
    if (cO <= R(0)) {
        return s;
    }
    const R a = alphaFromRoughness(c.m.roughness);
    V3<R> t, b;
    basis(c.n, t, b);
    R hp = R(0);
    const V3<R> hl = ggxHalf(a, u1, u2, hp);
    const V3<R> h = toWorld(hl, c.n, t, b);
    const R cHo = mx(R(0), dot(h, c.wo));
    if (cHo <= R(0) || hp <= Kc<R>::minPdf) {
        return s;
    }
    s.dir = nrm(sub(scl(h, R(2) * cHo), c.wo));
    const R cI = mx(R(0), dot(c.n, s.dir));
    if (cI <= R(0)) {
        return s;
    }
    s.pdf = bsdfPdf(c, s.dir);
    s.valid = s.pdf > Kc<R>::minPdf;
    s.transmitted = false;
    s.nextEta = c.eta;
    return s;
}

constexpr int kForceTransmitLobeOnly = 1 << 0; // Brdf/BrdfDebug.h:6-19
constexpr int kDisableRefract = 1 << 1;
constexpr int kDisableReflect = 1 << 2;
constexpr int kDisableTirFallback = 1 << 3;
constexpr int kTintGlassPaths = 1 << 4;

template <class R> inline Sample<R> sampleTransmit(const Ctx<R>& c, R u1, R u2)
{
    Sample<R> s;
    const R cOs = dot(c.n, c.wo);
    if (!transmitValid(c, cOs)) {
        return s;
    }
    const R thin = clamp01(c.m.thin);
    const R ior = matIor(c);
    const R etaT = cOs > R(0) ? ior : R(1);
    const R refl = dielectricFresnel(cOs, c.eta, etaT);
    const R trans = R(1) - refl;
    bool refr = u1 < trans;
    if ((c.debug & kDisableRefract) != 0) {
        refr = false;
    }
    if ((c.debug & kDisableReflect) != 0) {
        refr = true;
    }
    Ctx<R> rc = c;
    const R a = alphaFromRoughness(c.m.roughness);
    if (refr && thin < R(0.5f) && a > R(0.04f)) {
        V3<R> t, b;
        basis(c.n, t, b);
        R hp = R(0);
        const V3<R> hl = ggxHalf(a, u2, u1 * R(0.413f) + u2 * R(0.587f), hp);
        rc.n = toWorld(hl, c.n, t, b);
    }
    if (refr) {
        if (thin > R(0.5f)) {
            s.dir = nrm(scl(c.wo, R(-1)));
            s.nextEta = c.eta;
        } else {
            if (!refractDir(rc, s.dir, s.nextEta)) {
                if ((c.debug & kDisableTirFallback) != 0) {
                    return s;
                }
                s.dir = mirrorOut(c.wo, c.n);
                s.transmitted = false;
                s.nextEta = c.eta;
            } else {
                s.transmitted = true;
            }
        }
        if (thin > R(0.5f)) {
            s.transmitted = true;
        }
        if (absv(dot(c.n, s.dir)) <= R(0)) {
            return s;
        }
    } else {
        s.dir = mirrorOut(c.wo, c.n);
        if (absv(dot(c.n, s.dir)) <= R(0)) {
            return s;
        }
        s.transmitted = false;
        s.nextEta = c.eta;
    }
    s.pdf = bsdfPdf(c, s.dir);
    s.valid = s.pdf > Kc<R>::minPdf;
    return s;
}

template <class R> inline Sample<R> bsdfSample(const Ctx<R>& c, R u1, R u2)
{
    if ((c.debug & kForceTransmitLobeOnly) != 0) {
        return sampleTransmit(c, u1, u2);
    }
    const Lobes<R> w = lobes(c);
    int lobe;
    {
        R u = u1;
        if (u < w.diffuse) {
            lobe = 0;
        } else {
            u -= w.diffuse;
            if (u < w.specular) {
                lobe = 1;
            } else {
                u -= w.specular;
                lobe = u < w.transmit ? 2 : 3;
            }
        }
    }
    switch (lobe) {
    case 0:
        return sampleDiffuse(c, u1 / mx(w.diffuse, Kc<R>::minPdf), u2);
    case 1:
        return sampleSpecular(c, (u1 - w.diffuse) / mx(w.specular, Kc<R>::minPdf), u2);
    case 2:
        return sampleTransmit(c, (u1 - w.diffuse - w.specular) / mx(w.transmit, Kc<R>::minPdf), u2);
    default:
        return sampleSubsurface(c, (u1 - w.diffuse - w.specular - w.transmit) / mx(w.subsurface, Kc<R>::minPdf), u2);
    }
}

// Brdf/BrdfDispatch.h:35-40.
template <class R> inline bool skipsEnvNee(const Mat<R>& m)
{
    return mx(R(0), mn(R(1), m.transmission)) > R(0.99f) && mx(R(0), mn(R(1), m.metallic)) < R(0.01f);
}

// Brdf/BrdfDispatch.h:42-76.
template <class R> inline V3<R> applyThroughput(V3<R> tp, const Ctx<R>& c, const Sample<R>& s, V3<R> f)
{
    if (!s.valid || s.pdf <= Kc<R>::minPdf) {
        return mk(R(0), R(0), R(0));
    }
    const R trans = mx(R(0), mn(R(1), c.m.transmission));
    const R thin = mx(R(0), mn(R(1), c.m.thin));
    const bool pure = trans > R(0.99f) && c.m.metallic < R(0.01f);
    V3<R> sc;
    if (pure && thin < R(0.5f)) {
        sc = scl(f, R(1) / s.pdf);
    } else if (s.transmitted) {
        const R ct = absv(dot(c.n, s.dir));
        sc = scl(f, ct / s.pdf);
        if (thin > R(0.5f)) {
            sc = mk(sc.x * c.m.r, sc.y * c.m.g, sc.z * c.m.b);
        }
    } else if (s.sss) {
        const R ct = mx(R(0), dot(c.n, s.dir));
        sc = scl(f, ct / s.pdf);
    } else {
        const R ct = c.eta > R(1.0f + 1.0e-4f) ? absv(dot(c.n, s.dir)) : mx(R(0), dot(c.n, s.dir));
        sc = scl(f, ct / s.pdf);
    }
    return mk(tp.x * sc.x, tp.y * sc.y, tp.z * sc.z);
}

// ---------------------------------------------------------------------------
// Lights (Sampling/LightSamplingCore.h:25-369) and MIS (Sampling/MisCore.h:11-21).
// ---------------------------------------------------------------------------
template <class R> inline R misBalance(R a, R b)
{
    if (a <= R(0)) {
        return R(0);
    }
    const R d = a + b;
    if (d <= R(0)) {
        return R(0);
    }
    return a / d;
}

template <class R> inline V3<R> dirToLatLong(V3<R> d)
{
    using std::acos; using std::atan2;
    const V3<R> w = nrm(d);
    const R phi = atan2(w.x, w.z);
    const R theta = acos(clampv(w.y, R(-1), R(1)));
    return mk((phi + Kc<R>::pi) / (R(2) * Kc<R>::pi), theta / Kc<R>::pi, R(0));
}

template <class R> inline V3<R> latLongToDir(R u, R v)
{
    using std::cos; using std::sin;
    const R phi = u * R(2) * Kc<R>::pi - Kc<R>::pi;
    const R theta = v * Kc<R>::pi;
    const R st = sin(theta);
    return nrm(mk(st * sin(phi), cos(theta), st * cos(phi)));
}

template <class R> inline V3<R> solidEnv(const ParamsRec* p)
{
    if (p == nullptr) {
        return mk(R(0.04f), R(0.04f), R(0.04f));
    }
    const R k = R(p->environmentIntensity);
    return mk(R(p->backgroundR) * k, R(p->backgroundG) * k, R(p->backgroundB) * k);
}

inline bool envValid(const Env* e) { return e != nullptr && e->width > 0 && e->height > 0 && !e->pixels.empty(); }

template <class R> inline V3<R> envEval(const Env* e, const ParamsRec* p, V3<R> d)
{
    if (!envValid(e)) {
        return solidEnv<R>(p);
    }
    const V3<R> uv = dirToLatLong(d);
    const int x = clampv(static_cast<int>(uv.x * R(e->width)), 0, e->width - 1);
    const int y = clampv(static_cast<int>(uv.y * R(e->height)), 0, e->height - 1);
    const size_t i = (static_cast<size_t>(y) * e->width + x) * 3;
    return mk(R(e->pixels[i]), R(e->pixels[i + 1]), R(e->pixels[i + 2]));
}

inline int cdfFind(const float* cdf, int count, float u)
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

template <class R> inline R envPdfTable(const Env* e, int x, int y, R v)
{
    using std::sin;
    const int off = y * (e->width + 1);
    const R rp = R(e->row[static_cast<size_t>(off + x + 1)]) - R(e->row[static_cast<size_t>(off + x)]);
    const R mp = R(e->marginal[static_cast<size_t>(y + 1)]) - R(e->marginal[static_cast<size_t>(y)]);
    const R st = mx(R(1.0e-4f), sin(v * Kc<R>::pi));
    return (mp * rp) * R(e->width * e->height) / (R(2) * Kc<R>::pi * Kc<R>::pi * st);
}

template <class R> inline V3<R> envSample(const Env* e, R u1, R u2, R& pdf)
{
    if (!envValid(e)) {
        pdf = R(1) / (R(4) * Kc<R>::pi);
        return latLongToDir(u1, u2);
    }
    pdf = R(0);
    const int y = cdfFind(e->marginal.data(), e->height, static_cast<float>(u1));
    const int off = y * (e->width + 1);
    const int x = cdfFind(e->row.data() + off, e->width, static_cast<float>(u2));
    const R u = (R(x) + R(0.5f)) / R(e->width);
    const R v = (R(y) + R(0.5f)) / R(e->height);
    const V3<R> d = latLongToDir(u, v);
    const size_t i = (static_cast<size_t>(y) * e->width + x) * 3;
    const R L = mx(mx(R(e->pixels[i]), R(e->pixels[i + 1])), R(e->pixels[i + 2]));
    pdf = envPdfTable(e, x, y, v);
    if (L <= R(0)) {
        pdf = R(0);
    }
    return d;
}

template <class R> inline R envPdf(const Env* e, V3<R> d)
{
    if (!envValid(e)) {
        return R(1) / (R(4) * Kc<R>::pi);
    }
    const V3<R> uv = dirToLatLong(d);
    const int x = clampv(static_cast<int>(uv.x * R(e->width)), 0, e->width - 1);
    const int y = clampv(static_cast<int>(uv.y * R(e->height)), 0, e->height - 1);
    return envPdfTable(e, x, y, uv.y);
}

template <class R> inline bool sunIn(const SunSetup& l, V3<R> d)
{
    const V3<R> sd = mk(R(l.dir[0]), R(l.dir[1]), R(l.dir[2]));
    const V3<R> x = cross(d, sd);
    return dot(d, sd) > R(0) && dot(x, x) <= R(l.sin2) * dot(d, d);
}

template <class R> inline V3<R> sunSampleDir(const SunSetup& l, R u1, R u2)
{
    using std::cos; using std::sin; using std::sqrt;
    const R h = u1 * R(l.omc);
    const R ct = R(1) - h;
    const R st = sqrt(mx(R(0), h * (R(2) - h)));
    const R ph = R(2) * Kc<R>::pi * u2;
    const V3<R> t = mk(R(l.t[0]), R(l.t[1]), R(l.t[2])), b = mk(R(l.b[0]), R(l.b[1]), R(l.b[2]));
    const V3<R> d = mk(R(l.dir[0]), R(l.dir[1]), R(l.dir[2]));
    return nrm(add(add(scl(t, st * cos(ph)), scl(b, st * sin(ph))), scl(d, ct)));
}

inline float sunSelect(const Env* e, const ParamsRec* p)
{
    const float k = p->environmentIntensity;
    const bool lit = envValid(e) || p->backgroundR * k != 0.0f || p->backgroundG * k != 0.0f || p->backgroundB * k != 0.0f;
    return lit ? 0.5f : 1.0f;
}

template <class R> inline R skyPdfAt(const Scene& s, const Env* e, const ParamsRec* p, V3<R> d)
{
    const R sel = R(sunSelect(e, p));
    const R ls = sunIn(s.sun, d) ? R(s.sun.pdf) : R(0);
    return sel * ls + (R(1) - sel) * envPdf(e, d);
}

template <class R> inline V3<R> skyEval(const Scene& s, const Env* e, const ParamsRec* p, V3<R> d)
{
    V3<R> L = envEval(e, p, d);
    if (s.sun.enabled && sunIn(s.sun, d)) {
        L = add(L, mk(R(s.sun.rgb[0]), R(s.sun.rgb[1]), R(s.sun.rgb[2])));
    }
    return L;
}

template <class R> inline bool occluded(const Scene& s, V3<R> origin, V3<R> wi, R tMax = R(1.0e6f))
{
    return traceRay(s, origin, wi, R(1.0e-4f), tMax).hit;
}

inline const MaterialRec& fetchMaterial(const Scene& s, uint32_t tri, MaterialRec& fallback)
{
    if (s.materials.empty() || tri >= s.tris.size()) {
        return fallback;
    }
    const uint32_t mi = s.tris[tri].mat;
    if (mi >= s.materials.size()) {
        return fallback;
    }
    return s.materials[mi];
}

inline MaterialRec defaultFetchMaterial()
{
    // LightSamplingCore.h:199-213 fallback: a MaterialGpu{} with rgb 0.8.
    MaterialRec m{};
    m.r = m.g = m.b = 0.8f;
    m.roughness = 0.5f;
    m.ior = 1.5f;
    m.diffuseRoughness = -1.0f;
    m.specular = 1.0f;
    return m;
}

template <class R> inline R triArea(const TriRec& t)
{
    const V3<R> e1 = sub(vtx<R>(t, 1), vtx<R>(t, 0));
    const V3<R> e2 = sub(vtx<R>(t, 2), vtx<R>(t, 0));
    return R(0.5f) * len(cross(e1, e2));
}

template <class R>
inline bool sampleEmissive(const Scene& s, R uTri, R u1, R u2, V3<R>& pos, V3<R>& n, V3<R>& L, R& pdf,
    uint32_t* triOut = nullptr)
{
    using std::sqrt;
    pdf = R(0);
    const uint32_t E = static_cast<uint32_t>(s.emissiveIdx.size());
    if (E == 0 || s.tris.empty()) {
        return false;
    }
    const R total = R(s.emissiveCdf[E]);
    if (total <= Kc<R>::minPdf) {
        return false;
    }
    const R target = uTri * total;
    int lo = 0, hi = static_cast<int>(E) - 1;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (R(s.emissiveCdf[static_cast<size_t>(mid + 1)]) < target) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    const uint32_t tri = s.emissiveIdx[static_cast<size_t>(lo)];
    if (triOut != nullptr) {
        *triOut = tri;
    }
    const TriRec& t = s.tris[tri];
    MaterialRec fb = defaultFetchMaterial();
    const MaterialRec& m = fetchMaterial(s, tri, fb);
    const R su = sqrt(mx(R(0), u1));
    const R b0 = R(1) - su;
    const R b1 = u2 * su;
    const R b2 = R(1) - b0 - b1;
    pos = add(add(scl(vtx<R>(t, 0), b0), scl(vtx<R>(t, 1), b1)), scl(vtx<R>(t, 2), b2));
    n = nrm(cross(sub(vtx<R>(t, 1), vtx<R>(t, 0)), sub(vtx<R>(t, 2), vtx<R>(t, 0))));
    L = mk(R(m.r) * R(m.emission), R(m.g) * R(m.emission), R(m.b) * R(m.emission));
    const R area = triArea<R>(t);
    if (area <= Kc<R>::minPdf) {
        return false;
    }
    const R sel = (R(s.emissiveCdf[static_cast<size_t>(lo) + 1]) - R(s.emissiveCdf[static_cast<size_t>(lo)])) / total;
    pdf = sel / area;
    return pdf > Kc<R>::minPdf;
}

// ---------------------------------------------------------------------------
// Camera (CameraDevice.cuh:8-139).
// ---------------------------------------------------------------------------
template <class R> inline V3<R> rotq(const float* q, V3<R> v)
{
    const R s = R(q[0]);
    const V3<R> u = mk(R(q[1]), R(q[2]), R(q[3]));
    const V3<R> c1 = mk(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
    const V3<R> c2 = mk(u.y * c1.z - u.z * c1.y, u.z * c1.x - u.x * c1.z, u.x * c1.y - u.y * c1.x);
    return mk(v.x + R(2) * c1.x * s + R(2) * c2.x, v.y + R(2) * c1.y * s + R(2) * c2.y,
        v.z + R(2) * c1.z * s + R(2) * c2.z);
}

template <class R> inline V3<R> filmLocal(const CameraRec& c, R u, R v)
{
    using std::tan;
    const R nx = R(2) * u - R(1);
    const R ny = R(1) - R(2) * v;
    const R th = tan(R(c.fovY) * R(0.5f));
    const R top = R(c.nearPlane) * th;
    const R right = top * R(c.aspect);
    return mk(nx * right, ny * top, -R(c.nearPlane));
}

template <class R> inline void concentricDisk(R u1, R u2, R& dx, R& dy)
{
    using std::cos; using std::fabs; using std::sin;
    const R a = R(2) * u1 - R(1);
    const R b = R(2) * u2 - R(1);
    if (a == R(0) && b == R(0)) {
        dx = dy = R(0);
        return;
    }
    R r, th;
    if (fabs(a) > fabs(b)) {
        r = a;
        th = R(3.14159265358979323846f * 0.25f) * (b / a);
    } else {
        r = b;
        th = R(3.14159265358979323846f * 0.5f) - R(3.14159265358979323846f * 0.25f) * (a / b);
    }
    dx = r * cos(th);
    dy = r * sin(th);
}

template <class R> inline void cameraRay(const CameraRec& c, R u, R v, R l1, R l2, V3<R>& ro, V3<R>& rd)
{
    const V3<R> pos = mk(R(c.position[0]), R(c.position[1]), R(c.position[2]));
    if (c.focusValid == 0 || c.apertureRadius <= 0.0f || c.focusDistance <= 0.0f || c.nearPlane <= 0.0f) {
        ro = pos;
        rd = nrm(rotq(c.orientation, filmLocal(c, u, v)));
        return;
    }
    const V3<R> right = nrm(rotq(c.orientation, mk(R(1), R(0), R(0))));
    const V3<R> up = nrm(rotq(c.orientation, mk(R(0), R(1), R(0))));
    const V3<R> pf = filmLocal(c, u, v);
    const R fs = R(c.focusDistance) / R(c.nearPlane);
    const V3<R> pfl = mk(pf.x * fs, pf.y * fs, -R(c.focusDistance));
    const V3<R> r = rotq(c.orientation, pfl);
    const V3<R> pfw = mk(pos.x + r.x, pos.y + r.y, pos.z + r.z);
    R dx, dy;
    concentricDisk(l1, l2, dx, dy);
    const R ox = dx * R(c.apertureRadius);
    const R oy = dy * R(c.apertureRadius);
    ro = mk(pos.x + right.x * ox + up.x * oy, pos.y + right.y * ox + up.y * oy, pos.z + right.z * ox + up.z * oy);
    rd = nrm(mk(pfw.x - ro.x, pfw.y - ro.y, pfw.z - ro.z));
}

// ---------------------------------------------------------------------------
// Random-number source: a tape row or PCG32.
// ---------------------------------------------------------------------------
struct Rng {
    const float* row = nullptr;
    int length = 0;
    int cursor = 0;
    int underruns = 0;
    bool pcg = false;
    uint64_t state = 0, inc = 0;

    static uint32_t pcgNext(uint64_t& st, uint64_t in)
    {
        const uint64_t old = st;
        st = old * 6364136223846793005ULL + in;
        const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = static_cast<uint32_t>(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
    void seedPcg(uint64_t seed, uint64_t stream)
    {
        pcg = true;
        state = 0u;
        inc = (stream << 1u) | 1u;
        pcgNext(state, inc);
        state += seed;
        pcgNext(state, inc);
    }
    float next()
    {
        if (pcg) {
            const uint32_t bits = pcgNext(state, inc);
            return (static_cast<float>(bits >> 8) + 1.0f) * (1.0f / 16777216.0f);
        }
        if (row == nullptr || cursor >= length) {
            ++underruns;
            return 0.5f;
        }
        return row[cursor++];
    }
};

// ---------------------------------------------------------------------------
// Path integrator (PathIntegratorRandCore.h:38-363).
// ---------------------------------------------------------------------------
template <class R>
inline V3<R> neeEnvironment(const Scene& s, const Env* e, const ParamsRec* p, V3<R> pos, V3<R> n, V3<R> wo,
    const Mat<R>& m, R eta, Rng& rng)
{
    if (skipsEnvNee(m)) {
        return mk(R(0), R(0), R(0));
    }
    const bool sunOn = s.sun.enabled;
    const R uSel = sunOn ? R(rng.next()) : R(0);
    const R u1 = R(rng.next());
    const R u2 = R(rng.next());
    R lp = R(0);
    V3<R> wi;
    if (!sunOn) {
        wi = envSample(e, u1, u2, lp);
    } else if (uSel < R(sunSelect(e, p))) {
        wi = sunSampleDir(s.sun, u1, u2);
        lp = skyPdfAt(s, e, p, wi);
    } else {
        wi = envSample(e, u1, u2, lp);
        lp = lp > Kc<R>::minPdf ? skyPdfAt(s, e, p, wi) : R(0);
    }
    if (lp <= Kc<R>::minPdf) {
        return mk(R(0), R(0), R(0));
    }
    if (occluded(s, add(pos, scl(n, R(1.0e-4f))), wi)) {
        return mk(R(0), R(0), R(0));
    }
    const R ct = mx(R(0), dot(n, wi));
    if (ct <= R(0)) {
        return mk(R(0), R(0), R(0));
    }
    const Ctx<R> c{n, wo, m, eta, 0};
    const V3<R> L = sunOn ? skyEval(s, e, p, wi) : envEval(e, p, wi);
    const V3<R> f = bsdfEval(c, wi);
    const R bp = bsdfPdf(c, wi);
    const R w = misBalance(lp, bp);
    const R k = w * ct / lp;
    return mul(f, scl(L, k));
}

template <class R>
inline V3<R> neeEmissive(const Scene& s, V3<R> pos, V3<R> n, V3<R> wo, const Mat<R>& m, R eta, Rng& rng,
    bool misVertex = false)
{
    if (s.emissiveIdx.empty()) {
        return mk(R(0), R(0), R(0));
    }
    const R uTri = R(rng.next());
    const R u1 = R(rng.next());
    const R u2 = R(rng.next());
    V3<R> lpos, ln, L;
    R ap = R(0);
    if (!sampleEmissive(s, uTri, u1, u2, lpos, ln, L, ap)) {
        return mk(R(0), R(0), R(0));
    }
    const V3<R> tl = sub(lpos, pos);
    const R d2 = dot(tl, tl);
    if (d2 <= Kc<R>::minPdf) {
        return mk(R(0), R(0), R(0));
    }
    const V3<R> wi = nrm(tl);
    const R ct = mx(R(0), dot(n, wi));
    const R cl = mx(R(0), dot(ln, scl(wi, R(-1))));
    if (ct <= R(0) || cl <= R(0)) {
        return mk(R(0), R(0), R(0));
    }
    // Q12: the reference's shadow ray runs to 1e6 and meets the sampled emitter;
    // in emitter MIS mode it ends just short of the light sample
    const bool misLight = misVertex && !inTransmitCones(Ctx<R>{n, wo, m, eta, 0}, wi);
    const R tMax = misLight ? (std::sqrt(d2) - R(1.0e-4f)) * (R(1) - R(1.0e-4f)) : R(1.0e6f);
    if (occluded(s, add(pos, scl(wi, R(1.0e-4f))), wi, tMax)) {
        return mk(R(0), R(0), R(0));
    }
    const R lp = ap * d2 / cl;
    if (lp <= Kc<R>::minPdf) {
        return mk(R(0), R(0), R(0));
    }
    const Ctx<R> c{n, wo, m, eta, 0};
    const V3<R> f = bsdfEval(c, wi);
    const R bp = bsdfPdf(c, wi);
    const R w = misBalance(lp, bp);
    const R k = w * ct / lp;
    return mul(f, scl(L, k));
}

template <class R>
inline V3<R> subsurfaceTierB(V3<R> tp, const Mat<R>& m, V3<R> n, const Sample<R>& s, Rng& rng)
{
    using std::cos; using std::exp; using std::log; using std::sin; using std::sqrt;
    if (!s.sss || s.sssSteps <= 0) {
        return tp;
    }
    const R maxR = maxScatter(m);
    if (maxR <= R(kMinRadius)) {
        return tp;
    }
    const V3<R> albedo = mk(m.r, m.g, m.b);
    for (int step = 0; step < s.sssSteps; ++step) {
        const R a = R(rng.next());
        const R b = R(rng.next());
        const R c = R(rng.next());
        (void)a;
        (void)b; // the internal step direction is computed and discarded by the reference
        const R mfp = maxR * (-log(mx(R(1.0e-8f), c)));
        const R surv = exp(-mfp / maxR);
        tp = mul(tp, scl(albedo, surv));
    }
    const R ed = len(s.exitOffset);
    if (ed > R(0)) {
        tp = scl(tp, exp(-ed / maxR));
    }
    return tp;
}

// Emitter MIS mode: a vertex takes part when its BSDF samples the upper
// hemisphere with the mixture pdf the NEE weight uses and its throughput is
// f cos / pdf: no subsurface lobe, not the pure transmit lobe (whose throughput
// drops the cosine), outside any medium, no BRDF debug flags.
template <class R> inline bool emitterMisVertex(const Scene& s, const Ctx<R>& c)
{
    if (!s.emitterMis || c.debug != 0) {
        return false;
    }
    const Lobes<R> w = lobes(c);
    return w.subsurface <= R(0) && !skipsEnvNee(c.m) && c.eta == R(1);
}

// The transmit lobe's two narrow cones (evalTransmit: cosine > 0.999 with the
// mirror and the transmitted direction), left to BSDF sampling alone.
template <class R> inline bool inTransmitCones(const Ctx<R>& c, V3<R> wi)
{
    const Lobes<R> w = lobes(c);
    if (w.transmit == R(0)) {
        return false;
    }
    const R cOs = dot(c.n, c.wo);
    if (!transmitValid(c, cOs)) {
        return false;
    }
    if (dot(wi, mirrorOut(c.wo, c.n)) > R(0.999f)) {
        return true;
    }
    V3<R> td{R(0), R(0), R(0)};
    R ne = R(1);
    if (clamp01(c.m.thin) > R(0.5f)) {
        td = nrm(scl(c.wo, R(-1)));
    } else if (!refractDir(c, td, ne)) {
        return false;
    }
    return dot(wi, td) > R(0.999f);
}

// Balance weight of the emission of an emitter hit at distance t along the
// BSDF-sampled direction d (pdf bsdfPdfPrev) against emissive NEE's density
// of picking that point: pick probability / area * t^2 |d|^2 / cos at the light.
template <class R> inline R emitterHitWeight(const Scene& s, uint32_t tri, V3<R> d, R t, R bsdfPdfPrev)
{
    using std::sqrt;
    if (tri >= s.emitIndex.size() || s.emitIndex[tri] < 0) {
        return R(1);
    }
    const size_t e = static_cast<size_t>(s.emitIndex[tri]);
    const uint32_t E = static_cast<uint32_t>(s.emissiveIdx.size());
    const R total = R(s.emissiveCdf[E]);
    const TriRec& tr = s.tris[tri];
    const V3<R> cr = cross(sub(vtx<R>(tr, 1), vtx<R>(tr, 0)), sub(vtx<R>(tr, 2), vtx<R>(tr, 0)));
    const R area = R(0.5f) * len(cr);
    if (total <= Kc<R>::minPdf || area <= Kc<R>::minPdf) {
        return R(1);
    }
    const R pa = ((R(s.emissiveCdf[e + 1]) - R(s.emissiveCdf[e])) / total) / area;
    const R cl = mx(R(0), -dot(nrm(cr), nrm(d)));
    if (pa <= R(0) || cl <= R(0)) {
        return R(1);
    }
    const R lp = pa * (t * t * dot(d, d)) / cl;
    return misBalance(bsdfPdfPrev, lp);
}

inline void setEmitterMis(Scene& s, bool on)
{
    s.emitterMis = on;
    s.emitIndex.assign(s.tris.size(), -1);
    for (size_t e = 0; e < s.emissiveIdx.size(); ++e) {
        if (s.emissiveIdx[e] < s.tris.size()) {
            s.emitIndex[s.emissiveIdx[e]] = static_cast<int>(e);
        }
    }
}

template <class R>
inline V3<R> tracePath(const Scene& s, const Env* e, const ParamsRec* p, V3<R> ro, V3<R> rd, Rng& rng)
{
    using std::isfinite;
    const Hit<R> first = traceRay(s, ro, rd, R(0), R(1.0e6f));
    if (!first.hit) {
        return s.sun.enabled ? skyEval(s, e, p, rd) : envEval(e, p, rd);
    }
    int maxDepth = 32, rrMin = 3, debug = 0;
    if (p != nullptr) {
        if (p->maxPathDepth > 0) {
            maxDepth = p->maxPathDepth;
        } else if (p->maxPathDepth == 0) {
            maxDepth = 256;
        }
        if (p->russianRouletteMinDepth >= 0) {
            rrMin = p->russianRouletteMinDepth;
        }
        debug = p->brdfDebugFlags;
    }
    V3<R> L = mk(R(0), R(0), R(0));
    V3<R> T = mk(R(1), R(1), R(1));
    V3<R> o = ro, d = rd;
    Hit<R> h = first;
    R eta = R(1);
    MaterialRec fb = defaultFetchMaterial();
    R prevPdf = R(0);
    bool prevMis = false;
    for (int depth = 0; depth < maxDepth; ++depth) {
        const V3<R> pos = add(o, scl(d, h.t));
        const V3<R> n = h.normal;
        const V3<R> wo = scl(d, R(-1));
        const Mat<R> m = resolve<R>(fetchMaterial(s, h.tri, fb), h.uv, s.textures);
        const Ctx<R> c{n, wo, m, eta, debug};
        const bool misV = emitterMisVertex(s, c);
        const R ew = (prevMis && depth > 0 && m.emission != R(0)) ? emitterHitWeight(s, h.tri, d, h.t, prevPdf) : R(1);
        const R em = m.emission * ew;
        L = add(L, mul(T, mk(m.r * em, m.g * em, m.b * em)));
        L = add(L, mul(T, neeEnvironment(s, e, p, pos, n, wo, m, eta, rng)));
        L = add(L, mul(T, neeEmissive(s, pos, n, wo, m, eta, rng, misV)));
        const R u1 = R(rng.next());
        const R u2 = R(rng.next());
        const Sample<R> smp = bsdfSample(c, u1, u2);
        if (!smp.valid || smp.pdf <= Kc<R>::minPdf) {
            break;
        }
        const V3<R> f = bsdfEval(c, smp.dir);
        T = applyThroughput(T, c, smp, f);
        T = subsurfaceTierB(T, m, n, smp, rng);
        if ((debug & kTintGlassPaths) != 0) {
            T = smp.transmitted ? mul(T, mk(R(0.2f), R(1), R(0.2f))) : mul(T, mk(R(1), R(0.2f), R(0.2f)));
        }
        const R tl = lum709(T);
        if (!isfinite(tl) || tl <= R(0) || tl > R(1.0e8f)) {
            break;
        }
        if (depth >= rrMin) {
            const R surv = mn(R(0.95f), mx(tl, R(0.05f)));
            if (R(rng.next()) > surv) {
                break;
            }
            T = scl(T, R(1) / surv);
        }
        eta = smp.nextEta;
        prevPdf = smp.pdf;
        prevMis = misV && !smp.transmitted && !smp.sss && dot(n, smp.dir) > R(0) && !inTransmitCones(c, smp.dir);
        const R bias = mx(R(1.0e-4f), R(1.0e-3f) * h.t);
        const R sign = dot(n, smp.dir) >= R(0) ? R(1) : R(-1);
        o = add(pos, scl(n, sign * bias));
        d = smp.dir;
        h = traceRay(s, o, d, bias, R(1.0e6f));
        if (!h.hit) {
            const V3<R> Le = s.sun.enabled ? skyEval(s, e, p, d) : envEval(e, p, d);
            const R lp = s.sun.enabled ? skyPdfAt(s, e, p, d) : envPdf(e, d);
            const R w = misBalance(smp.pdf, lp);
            L = add(L, mul(T, scl(Le, w)));
            break;
        }
    }
    return L;
}

// PathTracer.cu:49-67.
template <class R> inline V3<R> clampFirefly(V3<R> c)
{
    using std::isfinite;
    if (!isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z)) {
        return mk(R(0), R(0), R(0));
    }
    c = mk(mx(R(0), c.x), mx(R(0), c.y), mx(R(0), c.z));
    const R l = c.x * R(0.2126f) + c.y * R(0.7152f) + c.z * R(0.0722f);
    if (l <= R(100)) {
        return c;
    }
    const R k = R(100) / l;
    return mk(c.x * k, c.y * k, c.z * k);
}

// PathTracer.cu:69-105 with the seed formula of Sampling/RandCore.h:7-12.
inline uint32_t referenceSeed(int pixel, int sampleIndex, uint32_t globalSeed)
{
    return static_cast<uint32_t>(pixel) * 747796405u + static_cast<uint32_t>(sampleIndex) + globalSeed * 2891336453u;
}

template <class R>
inline V3<R> tracePixel(const Scene& s, const Env* e, const CameraRec& cam, const ParamsRec& p, int idx, int width,
    int height, Rng& rng)
{
    const int x = idx % width;
    const int y = idx / width;
    const R ju = R(rng.next());
    const R jv = R(rng.next());
    const R u = (R(x) + ju) / R(width);
    const R v = (R(y) + jv) / R(height);
    const R l1 = R(rng.next());
    const R l2 = R(rng.next());
    V3<R> ro, rd;
    cameraRay(cam, u, v, l1, l2, ro, rd);
    return clampFirefly(tracePath(s, e, &p, ro, rd, rng));
}

// ---------------------------------------------------------------------------
// Hero-wavelength spectral mode: an extension with no reference counterpart on
// the render path (the reference's Spectral/ helpers are not called by its
// integrator).  Restated here from the product's definition:
//   * spectrum of a colour: scale * (1/2 + x / (2 sqrt(1 + x^2))),
//     x = c0 l^2 + c1 l + c2 (the function of Spectral/Rgb2Spec.h:58-66);
//   * NW wavelengths 380 + 400 frac(u + k / NW), u from a hash of the path seed;
//   * the BSDF at lambda is the RGB BSDF of the material with every colour
//     channel set to the colour's spectrum at lambda; sampling, pdfs, MIS and
//     the random-number draws are those of the RGB material;
//   * Russian roulette weighs the mean throughput over the wavelengths;
//   * a sample's sRGB = sum_k L_k response(lambda_k) 400 / NW, then the
//     firefly clamp without zeroing negative channels.
// The coefficient records and the response table are inputs (they come from
// the product's host functions, which other tests check on their own).
// ---------------------------------------------------------------------------
constexpr int kSpecMax = 8;

struct SpecSetup {
    int nw = 0;
    const float* resp = nullptr;  // 401 x 3, 1 nm apart from 380 nm
    const float* mat = nullptr;   // per material: base colour, scatter radii (4 floats each)
    size_t matCount = 0;
    const float* tex = nullptr;   // per texture: colour A, colour B (4 floats each)
    size_t texCount = 0;
    const float* env = nullptr;   // per environment texel (4 floats), or null
    float bg[4] = {0.0f, 0.0f, 0.0f, 0.0f}; // background x intensity
};

template <class R> inline R specEval(const float* c, R lambda)
{
    using std::sqrt;
    const R x = R(c[0]) * lambda * lambda + R(c[1]) * lambda + R(c[2]);
    const R y = R(1) / sqrt(x * x + R(1));
    return (R(0.5f) * x * y + R(0.5f)) * R(c[3]);
}

inline float heroU(uint32_t seed)
{
    uint32_t x = seed ^ 0x9E3779B9u;
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return static_cast<float>(x >> 8) * (1.0f / 16777216.0f);
}

inline float heroLambda(float u, int k, int nw)
{
    float t = u + static_cast<float>(k) / static_cast<float>(nw);
    if (t >= 1.0f) {
        t = t - 1.0f;
    }
    return 380.0f + 400.0f * t;
}

template <class R> inline V3<R> specResponse(const float* resp, R lambda)
{
    const R x = lambda - R(380);
    const int i = clampv(static_cast<int>(x), 0, 399);
    const R w = x - R(i);
    const R v = R(1) - w;
    const float* a = resp + 3 * i;
    const float* b = resp + 3 * (i + 1);
    return mk(R(a[0]) * v + R(b[0]) * w, R(a[1]) * v + R(b[1]) * w, R(a[2]) * v + R(b[2]) * w);
}

// Spectral radiance of the distant light at lambda (Planck's law in
// micrometres times the scale, or the spectrum of its RGB radiance).
template <class R> inline R specSun(const SunSetup& l, R lambda)
{
    using std::expm1;
    if (l.temperature > 0.0f) {
        const R lu = lambda * R(1.0e-3f);
        const R l2 = lu * lu;
        return R(l.scale) / (l2 * l2 * lu * expm1(R(14387.769f) / (lu * R(l.temperature))));
    }
    return specEval(l.coef, lambda);
}

template <class R> inline const float* specEnvCoef(const Env* e, const SpecSetup& sp, V3<R> d)
{
    if (!envValid(e) || sp.env == nullptr) {
        return sp.bg;
    }
    const V3<R> uv = dirToLatLong(d);
    const int x = clampv(static_cast<int>(uv.x * R(e->width)), 0, e->width - 1);
    const int y = clampv(static_cast<int>(uv.y * R(e->height)), 0, e->height - 1);
    return sp.env + 4 * (static_cast<size_t>(y) * e->width + x);
}

// Coefficient records of the material at a hit (base colour after the albedo
// texture rules of resolve(), scatter radii).
template <class R>
inline void specMatCoefs(const Scene& s, const SpecSetup& sp, uint32_t tri, V2<R> uv, const float*& base,
    const float*& scatter)
{
    static const float kGrey[4] = {0.0f, 0.0f, 0.0f, 1.6f}; // the fallback material's 0.8
    static const float kZero[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    base = kGrey;
    scatter = kZero;
    if (s.materials.empty() || tri >= s.tris.size()) {
        return;
    }
    const uint32_t mi = s.tris[tri].mat;
    if (mi >= s.materials.size() || mi >= sp.matCount) {
        return;
    }
    base = sp.mat + 8 * static_cast<size_t>(mi);
    scatter = base + 4;
    const MaterialRec& m = s.materials[mi];
    const uint32_t n = static_cast<uint32_t>(s.textures.size());
    if (m.albedoTex != 0u && n != 0u && m.albedoTex < n && m.albedoTex < sp.texCount) {
        const TextureRec& t = s.textures[m.albedoTex];
        const float* tc = sp.tex + 8 * static_cast<size_t>(m.albedoTex);
        if (t.kind == 1) {
            base = tc;
        } else if (t.kind == 2) {
            const R fx = fract(uv.x * R(t.p0[0]));
            const R fy = fract(uv.y * R(t.p0[1]));
            base = (fx < R(t.p0[2]) || fy < R(t.p0[2])) ? tc + 4 : tc;
        } else {
            base = kZero;
        }
    }
}

// The material of a hit at wavelength k: every colour channel set to its spectrum there.
template <class R> inline Mat<R> greyAt(const Mat<R>& m, R rho, R radius)
{
    Mat<R> g = m;
    g.r = g.g = g.b = rho;
    g.scatterR = g.scatterG = g.scatterB = radius;
    return g;
}

template <class R>
inline void tracePathSpectral(const Scene& s, const Env* e, const ParamsRec* p, const SpecSetup& sp, const R* lam,
    V3<R> ro, V3<R> rd, Rng& rng, R* L)
{
    using std::exp; using std::isfinite; using std::log;
    const int NW = sp.nw;
    for (int k = 0; k < NW; ++k) {
        L[k] = R(0);
    }
    const bool sunOn = s.sun.enabled;
    const Hit<R> first = traceRay(s, ro, rd, R(0), R(1.0e6f));
    if (!first.hit) {
        const float* q = specEnvCoef(e, sp, rd);
        const bool inS = sunOn && sunIn(s.sun, rd);
        for (int k = 0; k < NW; ++k) {
            L[k] = specEval(q, lam[k]);
            if (inS) {
                L[k] = L[k] + specSun(s.sun, lam[k]);
            }
        }
        return;
    }
    int maxDepth = 32, rrMin = 3, debug = 0;
    if (p->maxPathDepth > 0) {
        maxDepth = p->maxPathDepth;
    } else if (p->maxPathDepth == 0) {
        maxDepth = 256;
    }
    if (p->russianRouletteMinDepth >= 0) {
        rrMin = p->russianRouletteMinDepth;
    }
    debug = p->brdfDebugFlags;
    R T[kSpecMax];
    for (int k = 0; k < NW; ++k) {
        T[k] = R(1);
    }
    V3<R> o = ro, d = rd;
    Hit<R> h = first;
    R eta = R(1);
    MaterialRec fb = defaultFetchMaterial();
    for (int depth = 0; depth < maxDepth; ++depth) {
        const V3<R> pos = add(o, scl(d, h.t));
        const V3<R> n = h.normal;
        const V3<R> wo = scl(d, R(-1));
        const Mat<R> m = resolve<R>(fetchMaterial(s, h.tri, fb), h.uv, s.textures);
        const float* baseC;
        const float* scatC;
        specMatCoefs<R>(s, sp, h.tri, h.uv, baseC, scatC);
        R rho[kSpecMax], rad[kSpecMax];
        for (int k = 0; k < NW; ++k) {
            rho[k] = specEval(baseC, lam[k]);
            rad[k] = specEval(scatC, lam[k]);
            L[k] = L[k] + T[k] * (rho[k] * m.emission);
        }
        auto bsdfAt = [&](int k, V3<R> wi) -> R {
            const Ctx<R> ck{n, wo, greyAt(m, rho[k], rad[k]), eta, 0};
            return bsdfEval(ck, wi).x;
        };
        // environment NEE (the geometry of neeEnvironment)
        R add1[kSpecMax], add2[kSpecMax];
        bool has1 = false, has2 = false;
        if (!skipsEnvNee(m)) {
            const R uSel = sunOn ? R(rng.next()) : R(0);
            const R u1 = R(rng.next());
            const R u2 = R(rng.next());
            R lp = R(0);
            V3<R> wi;
            if (!sunOn) {
                wi = envSample(e, u1, u2, lp);
            } else if (uSel < R(sunSelect(e, p))) {
                wi = sunSampleDir(s.sun, u1, u2);
                lp = skyPdfAt(s, e, p, wi);
            } else {
                wi = envSample(e, u1, u2, lp);
                lp = lp > Kc<R>::minPdf ? skyPdfAt(s, e, p, wi) : R(0);
            }
            if (lp > Kc<R>::minPdf && !occluded(s, add(pos, scl(n, R(1.0e-4f))), wi)) {
                const R ct = mx(R(0), dot(n, wi));
                if (ct > R(0)) {
                    const float* q = specEnvCoef(e, sp, wi);
                    const bool inS = sunOn && sunIn(s.sun, wi);
                    const R bp = bsdfPdf(Ctx<R>{n, wo, m, eta, 0}, wi);
                    const R kw = misBalance(lp, bp) * ct / lp;
                    for (int k = 0; k < NW; ++k) {
                        R Le = specEval(q, lam[k]);
                        if (inS) {
                            Le = Le + specSun(s.sun, lam[k]);
                        }
                        add1[k] = T[k] * (bsdfAt(k, wi) * (Le * kw));
                    }
                    has1 = true;
                }
            }
        }
        // emissive NEE (the geometry of neeEmissive)
        if (!s.emissiveIdx.empty()) {
            const R uTri = R(rng.next());
            const R u1 = R(rng.next());
            const R u2 = R(rng.next());
            V3<R> lpos, ln, Lrgb;
            R ap = R(0);
            uint32_t etri = 0;
            if (sampleEmissive(s, uTri, u1, u2, lpos, ln, Lrgb, ap, &etri)) {
                const V3<R> tl = sub(lpos, pos);
                const R d2 = dot(tl, tl);
                if (d2 > Kc<R>::minPdf) {
                    const V3<R> wi = nrm(tl);
                    const R ct = mx(R(0), dot(n, wi));
                    const R cl = mx(R(0), dot(ln, scl(wi, R(-1))));
                    const R lp = ap * d2 / cl;
                    if (ct > R(0) && cl > R(0) && !occluded(s, add(pos, scl(wi, R(1.0e-4f))), wi) &&
                        lp > Kc<R>::minPdf) {
                        static const float kZero[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                        const uint32_t emi = s.tris[etri].mat;
                        const bool ok = emi < s.materials.size() && emi < sp.matCount;
                        const float* q = ok ? sp.mat + 8 * static_cast<size_t>(emi) : kZero;
                        const R em = ok ? R(s.materials[emi].emission) : R(0);
                        const R bp = bsdfPdf(Ctx<R>{n, wo, m, eta, 0}, wi);
                        const R kw = misBalance(lp, bp) * ct / lp;
                        for (int k = 0; k < NW; ++k) {
                            add2[k] = T[k] * (bsdfAt(k, wi) * ((specEval(q, lam[k]) * em) * kw));
                        }
                        has2 = true;
                    }
                }
            }
        }
        for (int k = 0; k < NW; ++k) {
            if (has1) {
                L[k] = L[k] + add1[k];
            }
            if (has2) {
                L[k] = L[k] + add2[k];
            }
        }
        const Ctx<R> c{n, wo, m, eta, debug};
        const R u1 = R(rng.next());
        const R u2 = R(rng.next());
        const Sample<R> smp = bsdfSample(c, u1, u2);
        if (!smp.valid || smp.pdf <= Kc<R>::minPdf) {
            break;
        }
        for (int k = 0; k < NW; ++k) {
            const Mat<R> gk = greyAt(m, rho[k], rad[k]);
            const Ctx<R> ck{n, wo, gk, eta, 0};
            const R fk = bsdfEval(ck, smp.dir).x;
            T[k] = applyThroughput(mk(T[k], T[k], T[k]), ck, smp, mk(fk, fk, fk)).x;
        }
        if (smp.sss && smp.sssSteps > 0) {
            // subsurfaceTierB with the base colour at each wavelength
            const R maxR = maxScatter(m);
            if (maxR > R(kMinRadius)) {
                for (int step = 0; step < smp.sssSteps; ++step) {
                    (void)rng.next();
                    (void)rng.next();
                    const R c3 = R(rng.next());
                    const R mfp = maxR * (-log(mx(R(1.0e-8f), c3)));
                    const R surv = exp(-mfp / maxR);
                    for (int k = 0; k < NW; ++k) {
                        T[k] = T[k] * (rho[k] * surv);
                    }
                }
                const R ed = len(smp.exitOffset);
                if (ed > R(0)) {
                    for (int k = 0; k < NW; ++k) {
                        T[k] = T[k] * exp(-ed / maxR);
                    }
                }
            }
        }
        R tl = R(0);
        for (int k = 0; k < NW; ++k) {
            tl = tl + T[k];
        }
        tl = tl * (R(1) / R(NW));
        if (!isfinite(tl) || tl <= R(0) || tl > R(1.0e8f)) {
            break;
        }
        if (depth >= rrMin) {
            const R surv = mn(R(0.95f), mx(tl, R(0.05f)));
            if (R(rng.next()) > surv) {
                break;
            }
            for (int k = 0; k < NW; ++k) {
                T[k] = T[k] * (R(1) / surv);
            }
        }
        eta = smp.nextEta;
        const R bias = mx(R(1.0e-4f), R(1.0e-3f) * h.t);
        const R sign = dot(n, smp.dir) >= R(0) ? R(1) : R(-1);
        o = add(pos, scl(n, sign * bias));
        d = smp.dir;
        h = traceRay(s, o, d, bias, R(1.0e6f));
        if (!h.hit) {
            const float* q = specEnvCoef(e, sp, d);
            const R lp = sunOn ? skyPdfAt(s, e, p, d) : envPdf(e, d);
            const R w = misBalance(smp.pdf, lp);
            const bool inS = sunOn && sunIn(s.sun, d);
            for (int k = 0; k < NW; ++k) {
                R Le = specEval(q, lam[k]);
                if (inS) {
                    Le = Le + specSun(s.sun, lam[k]);
                }
                L[k] = L[k] + T[k] * (Le * w);
            }
            break;
        }
    }
}

// sRGB of a spectral sample, then the firefly clamp without zeroing negative channels.
template <class R> inline V3<R> spectralSampleRgb(const SpecSetup& sp, const R* lam, const R* L)
{
    using std::isfinite;
    V3<R> a = mk(R(0), R(0), R(0));
    for (int k = 0; k < sp.nw; ++k) {
        a = add(a, scl(specResponse(sp.resp, lam[k]), L[k]));
    }
    V3<R> c = scl(a, R(400.0f) / R(sp.nw));
    if (!isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z)) {
        return mk(R(0), R(0), R(0));
    }
    const R l = c.x * R(0.2126f) + c.y * R(0.7152f) + c.z * R(0.0722f);
    if (l <= R(100)) {
        return c;
    }
    const R kk = R(100) / l;
    return mk(c.x * kk, c.y * kk, c.z * kk);
}

template <class R>
inline V3<R> tracePixelSpectral(const Scene& s, const Env* e, const CameraRec& cam, const ParamsRec& p,
    const SpecSetup& sp, uint32_t seed, int idx, int width, int height, Rng& rng)
{
    const int x = idx % width;
    const int y = idx / width;
    const R ju = R(rng.next());
    const R jv = R(rng.next());
    const R u = (R(x) + ju) / R(width);
    const R v = (R(y) + jv) / R(height);
    const R l1 = R(rng.next());
    const R l2 = R(rng.next());
    V3<R> ro, rd;
    cameraRay(cam, u, v, l1, l2, ro, rd);
    const float hu = heroU(seed);
    R lam[kSpecMax], L[kSpecMax];
    for (int k = 0; k < sp.nw; ++k) {
        lam[k] = R(heroLambda(hu, k, sp.nw));
    }
    tracePathSpectral(s, e, &p, sp, lam, ro, rd, rng, L);
    return spectralSampleRgb(sp, lam, L);
}

// PathTracerAdaptiveSampling.h:16-40 (criterion 0).  The product's extensions:
// criterion 1 divides the relative std-dev by sqrt(n) (relative std-error);
// criterion 2 is criterion 1 plus: a pixel all of whose samples are black
// (mean and M2 exactly 0) stops after max(minSamples, 64) samples.
inline bool isConverged(uint32_t n, float mean, float m2, int minSamples, float thr, int criterion = 0)
{
    if (n < static_cast<uint32_t>(minSamples) || n == 0) {
        return false;
    }
    if (mean < 1.0e-5f) {
        const uint32_t blackSpp = static_cast<uint32_t>(minSamples > 64 ? minSamples : 64);
        return criterion == 2 && n >= blackSpp && mean == 0.0f && m2 == 0.0f;
    }
    const float var = m2 / static_cast<float>(n);
    const float sd = std::sqrt(var);
    const float den = std::fmax(mean, 1.0e-4f);
    float rel = sd / den;
    if (criterion == 1 || criterion == 2) {
        rel = rel / std::sqrt(static_cast<float>(n));
    }
    return rel < thr;
}

// ---------------------------------------------------------------------------
// Scene build: median-split binary BVH with one triangle per leaf
// (MeshAccel/MeshBvhBuilder.cpp:52-142) and the emissive CDF
// (MeshAccel/MeshAccelScene.cpp:62-95).
// ---------------------------------------------------------------------------
void buildScene(Scene& s);

// ---------------------------------------------------------------------------
// Path-replay gradient of an image loss (the product's adjoint kernel,
// pt_adjoint.cu, restated): per sample, L from a first replay, then a second
// replay that adds beta_j dE_j/dtheta for the emission and next-event terms
// and (L - collected so far) * dlog f_j/dtheta at every BSDF vertex, sampling,
// Russian roulette and MIS weights held constant.  BSDF derivatives at a
// fixed direction by central differences (step 1e-6 in FP64; second-order
// one-sided at the bounds 0 and 1 of the clamped parameters).  Gradients go to
// G[m * 7 + j], j = r, g, b, roughness, metallic, sheen, emission.
// ---------------------------------------------------------------------------
struct FreeParams {
    bool rgb, roughness, metallic, emission;
};

inline FreeParams freeParams(const MaterialRec& m, size_t texCount)
{
    auto tex = [texCount](uint32_t t) { return t != 0u && t < texCount; };
    return FreeParams{!tex(m.albedoTex), !tex(m.roughnessTex), !tex(m.metallicTex), !tex(m.emissionTex)};
}

template <class R>
inline void bsdfGradFd(const Ctx<R>& c, V3<R> wi, bool roughFollows, V3<R> g[6])
{
    const R h = sizeof(R) == 8 ? R(1.0e-6) : R(1.0e-3f);
    const V3<R> f0 = bsdfEval(c, wi);
    for (int q = 0; q < 6; ++q) {
        auto at = [&](R x) {
            Ctx<R> t = c;
            R* v = q == 0 ? &t.m.r : q == 1 ? &t.m.g : q == 2 ? &t.m.b : q == 3 ? &t.m.roughness
                 : q == 4 ? &t.m.metallic : &t.m.sheen;
            *v = x;
            if (q == 3 && roughFollows) {
                t.m.diffuseRoughness = x;
            }
            return bsdfEval(t, wi);
        };
        const R x = q == 0 ? c.m.r : q == 1 ? c.m.g : q == 2 ? c.m.b : q == 3 ? c.m.roughness
                  : q == 4 ? c.m.metallic : c.m.sheen;
        if (x - h >= R(0) && x + h <= R(1)) {
            g[q] = scl(sub(at(x + h), at(x - h)), R(0.5) / h);
        } else if (x - h < R(0)) {
            g[q] = scl(sub(sub(scl(at(x + h), R(4)), scl(f0, R(3))), at(x + R(2) * h)), R(0.5) / h);
        } else {
            g[q] = scl(add(sub(scl(f0, R(3)), scl(at(x - h), R(4))), at(x - R(2) * h)), R(0.5) / h);
        }
    }
}

template <class R>
inline void gradAdd(double* G, int M, uint32_t mi, int j, R v)
{
    if (static_cast<int>(mi) < M) {
        G[mi * 7u + static_cast<uint32_t>(j)] += static_cast<double>(v);
    }
}

template <class R>
inline void neeGrad(double* G, int M, uint32_t mi, const FreeParams& fp, const Ctx<R>& c, V3<R> wi, bool roughFollows,
    V3<R> w)
{
    V3<R> g[6];
    bsdfGradFd(c, wi, roughFollows, g);
    const bool use[6] = {fp.rgb, fp.rgb, fp.rgb, fp.roughness, fp.metallic, true};
    for (int q = 0; q < 6; ++q) {
        if (use[q]) {
            gradAdd(G, M, mi, q, dot(w, g[q]));
        }
    }
}

// tracePath with gradient accumulation (G == nullptr: forward only).
template <class R>
inline V3<R> tracePathGrad(const Scene& s, const Env* e, const ParamsRec* p, V3<R> ro, V3<R> rd, Rng& rng,
    V3<R> delta, V3<R> Ltot, double* G, int M)
{
    using std::isfinite;
    const Hit<R> first = traceRay(s, ro, rd, R(0), R(1.0e6f));
    if (!first.hit) {
        return envEval(e, p, rd);
    }
    int maxDepth = 32, rrMin = 3, debug = 0;
    if (p != nullptr) {
        if (p->maxPathDepth > 0) {
            maxDepth = p->maxPathDepth;
        } else if (p->maxPathDepth == 0) {
            maxDepth = 256;
        }
        if (p->russianRouletteMinDepth >= 0) {
            rrMin = p->russianRouletteMinDepth;
        }
        debug = p->brdfDebugFlags;
    }
    V3<R> L = mk(R(0), R(0), R(0));
    V3<R> T = mk(R(1), R(1), R(1));
    V3<R> o = ro, d = rd;
    Hit<R> h = first;
    R eta = R(1);
    MaterialRec fb = defaultFetchMaterial();
    for (int depth = 0; depth < maxDepth; ++depth) {
        const V3<R> pos = add(o, scl(d, h.t));
        const V3<R> n = h.normal;
        const V3<R> wo = scl(d, R(-1));
        const MaterialRec& rec = fetchMaterial(s, h.tri, fb);
        const uint32_t mi = (s.materials.empty() || h.tri >= s.tris.size() || s.tris[h.tri].mat >= s.materials.size())
            ? 0xFFFFFFFFu : s.tris[h.tri].mat;
        const bool grad = G != nullptr && mi != 0xFFFFFFFFu;
        const FreeParams fp = freeParams(rec, s.textures.size());
        const bool roughFollows = rec.diffuseRoughness < 0.0f;
        const Mat<R> m = resolve<R>(rec, h.uv, s.textures);
        // emission
        if (grad && m.emission != R(0)) {
            const V3<R> dT = mul(delta, T);
            if (fp.emission) {
                gradAdd(G, M, mi, 6, dot(dT, mk(m.r, m.g, m.b)));
            }
            if (fp.rgb) {
                gradAdd(G, M, mi, 0, dT.x * m.emission);
                gradAdd(G, M, mi, 1, dT.y * m.emission);
                gradAdd(G, M, mi, 2, dT.z * m.emission);
            }
        }
        L = add(L, mul(T, mk(m.r * m.emission, m.g * m.emission, m.b * m.emission)));
        // environment NEE (neeEnvironment with the gradient of f)
        if (!skipsEnvNee(m)) {
            const R u1 = R(rng.next());
            const R u2 = R(rng.next());
            R lp = R(0);
            const V3<R> wi = envSample(e, u1, u2, lp);
            if (lp > Kc<R>::minPdf && !occluded(s, add(pos, scl(n, R(1.0e-4f))), wi)) {
                const R ct = mx(R(0), dot(n, wi));
                if (ct > R(0)) {
                    const Ctx<R> c{n, wo, m, eta, 0};
                    const V3<R> Le = envEval(e, p, wi);
                    const V3<R> f = bsdfEval(c, wi);
                    const R bp = bsdfPdf(c, wi);
                    const R k = misBalance(lp, bp) * ct / lp;
                    if (grad) {
                        neeGrad(G, M, mi, fp, c, wi, roughFollows, mul(mul(delta, T), scl(Le, k)));
                    }
                    L = add(L, mul(T, mul(f, scl(Le, k))));
                }
            }
        }
        // emissive NEE (neeEmissive with the gradient of f and of the light)
        if (!s.emissiveIdx.empty()) {
            const R uTri = R(rng.next());
            const R u1 = R(rng.next());
            const R u2 = R(rng.next());
            V3<R> lpos, ln, Le;
            R ap = R(0);
            uint32_t lt = 0;
            if (sampleEmissive(s, uTri, u1, u2, lpos, ln, Le, ap, &lt)) {
                const V3<R> tl = sub(lpos, pos);
                const R d2 = dot(tl, tl);
                if (d2 > Kc<R>::minPdf) {
                    const V3<R> wi = nrm(tl);
                    const R ct = mx(R(0), dot(n, wi));
                    const R cl = mx(R(0), dot(ln, scl(wi, R(-1))));
                    if (ct > R(0) && cl > R(0) && !occluded(s, add(pos, scl(wi, R(1.0e-4f))), wi)) {
                        const R lpdf = ap * d2 / cl;
                        if (lpdf > Kc<R>::minPdf) {
                            const Ctx<R> c{n, wo, m, eta, 0};
                            const V3<R> f = bsdfEval(c, wi);
                            const R bp = bsdfPdf(c, wi);
                            const R k = misBalance(lpdf, bp) * ct / lpdf;
                            if (grad) {
                                neeGrad(G, M, mi, fp, c, wi, roughFollows, mul(mul(delta, T), scl(Le, k)));
                            }
                            if (G != nullptr && lt < s.tris.size() && s.tris[lt].mat < s.materials.size()) {
                                const uint32_t lm = s.tris[lt].mat;
                                const MaterialRec& l0 = s.materials[lm];
                                const V3<R> w = mul(mul(delta, T), scl(f, k));
                                gradAdd(G, M, lm, 6, dot(w, mk(R(l0.r), R(l0.g), R(l0.b))));
                                gradAdd(G, M, lm, 0, w.x * R(l0.emission));
                                gradAdd(G, M, lm, 1, w.y * R(l0.emission));
                                gradAdd(G, M, lm, 2, w.z * R(l0.emission));
                            }
                            L = add(L, mul(T, mul(f, scl(Le, k))));
                        }
                    }
                }
            }
        }
        const Ctx<R> c{n, wo, m, eta, debug};
        const R u1 = R(rng.next());
        const R u2 = R(rng.next());
        const Sample<R> smp = bsdfSample(c, u1, u2);
        if (!smp.valid || smp.pdf <= Kc<R>::minPdf) {
            break;
        }
        const V3<R> f = bsdfEval(c, smp.dir);
        if (grad) {
            const V3<R> dRem = mul(delta, sub(Ltot, L));
            V3<R> g[6];
            bsdfGradFd(c, smp.dir, roughFollows, g);
            const V3<R> wgt = mk(f.x != R(0) ? dRem.x / f.x : R(0), f.y != R(0) ? dRem.y / f.y : R(0),
                f.z != R(0) ? dRem.z / f.z : R(0));
            const bool use[6] = {fp.rgb, fp.rgb, fp.rgb, fp.roughness, fp.metallic, true};
            for (int q = 0; q < 6; ++q) {
                if (use[q]) {
                    gradAdd(G, M, mi, q, dot(wgt, g[q]));
                }
            }
            if (fp.rgb) {
                const R trans = clampv(m.transmission, R(0), R(1));
                const R thin = clampv(m.thin, R(0), R(1));
                const bool pure = trans > R(0.99f) && m.metallic < R(0.01f);
                R extra = R(0);
                if (!(pure && thin < R(0.5f)) && smp.transmitted && thin > R(0.5f)) {
                    extra += R(1);
                }
                if (smp.sss && smp.sssSteps > 0 && maxScatter(m) > R(kMinRadius)) {
                    extra += R(smp.sssSteps);
                }
                if (extra != R(0)) {
                    gradAdd(G, M, mi, 0, m.r != R(0) ? dRem.x * extra / m.r : R(0));
                    gradAdd(G, M, mi, 1, m.g != R(0) ? dRem.y * extra / m.g : R(0));
                    gradAdd(G, M, mi, 2, m.b != R(0) ? dRem.z * extra / m.b : R(0));
                }
            }
        }
        T = applyThroughput(T, c, smp, f);
        T = subsurfaceTierB(T, m, n, smp, rng);
        if ((debug & kTintGlassPaths) != 0) {
            T = smp.transmitted ? mul(T, mk(R(0.2f), R(1), R(0.2f))) : mul(T, mk(R(1), R(0.2f), R(0.2f)));
        }
        const R tl = lum709(T);
        if (!isfinite(tl) || tl <= R(0) || tl > R(1.0e8f)) {
            break;
        }
        if (depth >= rrMin) {
            const R surv = mn(R(0.95f), mx(tl, R(0.05f)));
            if (R(rng.next()) > surv) {
                break;
            }
            T = scl(T, R(1) / surv);
        }
        eta = smp.nextEta;
        const R bias = mx(R(1.0e-4f), R(1.0e-3f) * h.t);
        const R sign = dot(n, smp.dir) >= R(0) ? R(1) : R(-1);
        o = add(pos, scl(n, sign * bias));
        d = smp.dir;
        h = traceRay(s, o, d, bias, R(1.0e6f));
        if (!h.hit) {
            const V3<R> Le = envEval(e, p, d);
            const R lp = envPdf(e, d);
            const R w = misBalance(smp.pdf, lp);
            L = add(L, mul(T, scl(Le, w)));
            break;
        }
    }
    return L;
}

// Camera ray of pixel idx (the first four draws of tracePixel).
template <class R>
inline void pixelRay(const CameraRec& cam, int idx, int width, int height, Rng& rng, V3<R>& ro, V3<R>& rd)
{
    const int x = idx % width;
    const int y = idx / width;
    const R ju = R(rng.next());
    const R jv = R(rng.next());
    const R u = (R(x) + ju) / R(width);
    const R v = (R(y) + jv) / R(height);
    const R l1 = R(rng.next());
    const R l2 = R(rng.next());
    cameraRay(cam, u, v, l1, l2, ro, rd);
}

} // namespace orc
