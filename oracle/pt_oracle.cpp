// CPU ORACLE (test infrastructure) -- extern "C" surface of pt_oracle.h.
// The entry points mirror oracle/ref_harness.cpp one for one (prefix orc_ for
// FP32, orc64_ for the FP64 estimator) so that tests can run the same case
// through the reference, this restatement and the GPU product.
#include "pt_oracle.h"

#include <omp.h>

namespace orc {

namespace {

// MeshBvhBuilder.cpp:10-29.
V3<float> centroid(const TriRec& t)
{
    const V3<float> s = add(add(vtx<float>(t, 0), vtx<float>(t, 1)), vtx<float>(t, 2));
    return scl(s, 1.0f / 3.0f);
}

// MeshBvhBuilder.cpp:52-114: bounds of the range, one triangle per leaf,
// median split (nth_element) along the longest axis of the bounds.
int buildRecursive(const std::vector<TriRec>& tris, std::vector<int>& idx, int begin, int end,
    std::vector<BvhNode>& nodes)
{
    float bmin[3], bmax[3];
    {
        const TriRec& t = tris[static_cast<size_t>(idx[static_cast<size_t>(begin)])];
        for (int a = 0; a < 3; ++a) {
            bmin[a] = mn(mn(t.v[0][a], t.v[1][a]), t.v[2][a]);
            bmax[a] = mx(mx(t.v[0][a], t.v[1][a]), t.v[2][a]);
        }
    }
    for (int i = begin + 1; i < end; ++i) {
        const TriRec& t = tris[static_cast<size_t>(idx[static_cast<size_t>(i)])];
        for (int a = 0; a < 3; ++a) {
            bmin[a] = mn(bmin[a], mn(mn(t.v[0][a], t.v[1][a]), t.v[2][a]));
            bmax[a] = mx(bmax[a], mx(mx(t.v[0][a], t.v[1][a]), t.v[2][a]));
        }
    }
    const int ni = static_cast<int>(nodes.size());
    BvhNode node{};
    std::memcpy(node.bmin, bmin, sizeof(bmin));
    std::memcpy(node.bmax, bmax, sizeof(bmax));
    nodes.push_back(node);
    const int count = end - begin;
    if (count == 1) {
        nodes[static_cast<size_t>(ni)].triStart = static_cast<uint32_t>(idx[static_cast<size_t>(begin)]);
        nodes[static_cast<size_t>(ni)].triCount = 1u;
        return ni;
    }
    const float ex = bmax[0] - bmin[0], ey = bmax[1] - bmin[1], ez = bmax[2] - bmin[2];
    const int axis = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
    const int mid = begin + count / 2;
    std::nth_element(idx.begin() + begin, idx.begin() + mid, idx.begin() + end, [&tris, axis](int l, int r) {
        const V3<float> cl = centroid(tris[static_cast<size_t>(l)]);
        const V3<float> cr = centroid(tris[static_cast<size_t>(r)]);
        return axis == 0 ? cl.x < cr.x : (axis == 1 ? cl.y < cr.y : cl.z < cr.z);
    });
    const int left = buildRecursive(tris, idx, begin, mid, nodes);
    const int right = buildRecursive(tris, idx, mid, end, nodes);
    nodes[static_cast<size_t>(ni)].left = static_cast<uint32_t>(left);
    nodes[static_cast<size_t>(ni)].right = static_cast<uint32_t>(right);
    nodes[static_cast<size_t>(ni)].triCount = 0;
    return ni;
}

} // namespace

void buildScene(Scene& s)
{
    s.nodes.clear();
    s.root = 0;
    if (s.materials.empty()) {
        s.materials.push_back(defaultFetchMaterial()); // MeshAccelScene.cpp:27-46
    }
    if (!s.tris.empty()) {
        std::vector<int> idx(s.tris.size());
        for (size_t i = 0; i < idx.size(); ++i) {
            idx[i] = static_cast<int>(i);
        }
        s.root = static_cast<uint32_t>(buildRecursive(s.tris, idx, 0, static_cast<int>(s.tris.size()), s.nodes));
    }
    // MeshAccelScene.cpp:62-95: sequential float prefix sum of area x emitted luminance.
    s.emissiveIdx.clear();
    s.emissiveCdf.assign(1, 0.0f);
    float total = 0.0f;
    for (uint32_t i = 0; i < s.tris.size(); ++i) {
        const TriRec& t = s.tris[i];
        if (t.mat >= s.materials.size()) {
            continue;
        }
        const MaterialRec& m = s.materials[t.mat];
        const float l = m.emission * (0.2126f * m.r + 0.7152f * m.g + 0.0722f * m.b);
        if (l <= 0.0f) {
            continue;
        }
        const float w = triArea<float>(t) * l;
        if (w <= 0.0f) {
            continue;
        }
        s.emissiveIdx.push_back(i);
        total += w;
        s.emissiveCdf.push_back(total);
    }
    if (total <= 0.0f) {
        s.emissiveCdf.assign(1, 0.0f);
    }
}

} // namespace orc

using namespace orc;

namespace {

template <class R>
int renderImpl(void* sceneHandle, void* envHandle, const void* cameraBytes, const void* paramsBytes, int width,
    int height, int waves, unsigned int seedBase, const float* tape, int tapeStride, const int* pixelList,
    int pixelListCount, R* acc, uint32_t* counts, R* lumMean, R* m2, uint8_t* converged, int threads)
{
    const Scene& s = *static_cast<Scene*>(sceneHandle);
    const Env* e = static_cast<Env*>(envHandle);
    CameraRec cam;
    std::memcpy(&cam, cameraBytes, sizeof(cam));
    ParamsRec p;
    std::memcpy(&p, paramsBytes, sizeof(p));
    const int P = width * height;
    const int listCount = pixelList ? pixelListCount : P;
    if (threads > 0) {
        omp_set_num_threads(threads);
    }
    int errors = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : errors)
    for (int li = 0; li < listCount; ++li) {
        const int idx = pixelList ? pixelList[li] : li;
        for (int w = 0; w < waves; ++w) {
            if (converged[idx] != 0) {
                break;
            }
            const uint32_t gs = seedBase + static_cast<uint32_t>(w);
            const uint32_t n = counts[idx];
            Rng rng;
            if (tape != nullptr) {
                rng.row = tape + (static_cast<size_t>(w) * P + idx) * static_cast<size_t>(tapeStride);
                rng.length = tapeStride;
            } else {
                rng.seedPcg(referenceSeed(idx, static_cast<int>(n), gs), 0x9e3779b97f4a7c15ULL);
            }
            const V3<R> smp = tracePixel<R>(s, e, cam, p, idx, width, height, rng);
            errors += rng.underruns;
            // sampleAdaptiveKernel accumulation (PathTracer.cu:232-272).
            const R sl = smp.x * R(0.2126f) + smp.y * R(0.7152f) + smp.z * R(0.0722f);
            const R pm = lumMean[idx];
            const R delta = sl - pm;
            const R nm = pm + delta / R(n + 1);
            m2[idx] = m2[idx] + delta * (sl - nm);
            lumMean[idx] = nm;
            R* a = acc + 4 * static_cast<size_t>(idx);
            const R invN = R(1) / R(n + 1);
            a[0] = (a[0] * R(n) + smp.x) * invN;
            a[1] = (a[1] * R(n) + smp.y) * invN;
            a[2] = (a[2] * R(n) + smp.z) * invN;
            a[3] = R(1);
            const uint32_t nc = n + 1;
            counts[idx] = nc;
            if (p.maxSamplesPerPixel > 0 && nc >= static_cast<uint32_t>(p.maxSamplesPerPixel)) {
                converged[idx] = 1;
                continue;
            }
            if ((nc % 4u) != 0) {
                continue;
            }
            if (isConverged(nc, static_cast<float>(nm), static_cast<float>(m2[idx]), p.minSamples,
                    p.relativeErrorThreshold, s.adaptiveCriterion)) {
                converged[idx] = 1;
            }
        }
    }
    return errors;
}

// renderImpl in spectral mode: each sample is a hero-wavelength sample whose
// wavelengths come from the reference seed of (pixel, sample index, wave).
template <class R>
int renderSpectralImpl(void* sceneHandle, void* envHandle, const void* cameraBytes, const void* paramsBytes, int width,
    int height, int waves, unsigned int seedBase, const float* tape, int tapeStride, const SpecSetup& sp, R* acc,
    uint32_t* counts, R* lumMean, R* m2, uint8_t* converged, int threads)
{
    const Scene& s = *static_cast<Scene*>(sceneHandle);
    const Env* e = static_cast<Env*>(envHandle);
    CameraRec cam;
    std::memcpy(&cam, cameraBytes, sizeof(cam));
    ParamsRec p;
    std::memcpy(&p, paramsBytes, sizeof(p));
    const int P = width * height;
    if (threads > 0) {
        omp_set_num_threads(threads);
    }
    int errors = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : errors)
    for (int idx = 0; idx < P; ++idx) {
        for (int w = 0; w < waves; ++w) {
            if (converged[idx] != 0) {
                break;
            }
            const uint32_t gs = seedBase + static_cast<uint32_t>(w);
            const uint32_t n = counts[idx];
            const uint32_t seed = referenceSeed(idx, static_cast<int>(n), gs);
            Rng rng;
            if (tape != nullptr) {
                rng.row = tape + (static_cast<size_t>(w) * P + idx) * static_cast<size_t>(tapeStride);
                rng.length = tapeStride;
            } else {
                rng.seedPcg(seed, 0x9e3779b97f4a7c15ULL);
            }
            const V3<R> smp = tracePixelSpectral<R>(s, e, cam, p, sp, seed, idx, width, height, rng);
            errors += rng.underruns;
            const R sl = smp.x * R(0.2126f) + smp.y * R(0.7152f) + smp.z * R(0.0722f);
            const R pm = lumMean[idx];
            const R delta = sl - pm;
            const R nm = pm + delta / R(n + 1);
            m2[idx] = m2[idx] + delta * (sl - nm);
            lumMean[idx] = nm;
            R* a = acc + 4 * static_cast<size_t>(idx);
            const R invN = R(1) / R(n + 1);
            a[0] = (a[0] * R(n) + smp.x) * invN;
            a[1] = (a[1] * R(n) + smp.y) * invN;
            a[2] = (a[2] * R(n) + smp.z) * invN;
            a[3] = R(1);
            const uint32_t nc = n + 1;
            counts[idx] = nc;
            if (p.maxSamplesPerPixel > 0 && nc >= static_cast<uint32_t>(p.maxSamplesPerPixel)) {
                converged[idx] = 1;
                continue;
            }
            if ((nc % 4u) != 0) {
                continue;
            }
            if (isConverged(nc, static_cast<float>(nm), static_cast<float>(m2[idx]), p.minSamples,
                    p.relativeErrorThreshold, s.adaptiveCriterion)) {
                converged[idx] = 1;
            }
        }
    }
    return errors;
}

SpecSetup makeSpecSetup(int nw, const float* resp, const float* matCoef, int matCount, const float* texCoef,
    int texCount, const float* envCoef, const float* bgCoef)
{
    SpecSetup sp;
    sp.nw = nw;
    sp.resp = resp;
    sp.mat = matCoef;
    sp.matCount = static_cast<size_t>(matCount);
    sp.tex = texCoef;
    sp.texCount = static_cast<size_t>(texCount);
    sp.env = envCoef;
    for (int k = 0; k < 4; ++k) {
        sp.bg[k] = bgCoef[k];
    }
    return sp;
}

Ctx<float> makeCtx(const float* normal, const float* wo, const void* material, float eta, int debug)
{
    MaterialRec m;
    std::memcpy(&m, material, sizeof(m));
    return Ctx<float>{mk(normal[0], normal[1], normal[2]), mk(wo[0], wo[1], wo[2]), matFromRec<float>(m), eta, debug};
}

} // namespace

extern "C" {

void* orc_scene_create(int triCount, const float* positions, const float* normals, const float* uvs,
    const uint32_t* materialIds, int materialCount, const void* materials, int textureCount, const void* textures)
{
    Scene* s = new Scene();
    s->tris.resize(static_cast<size_t>(triCount));
    for (int i = 0; i < triCount; ++i) {
        TriRec& t = s->tris[static_cast<size_t>(i)];
        std::memcpy(t.v, positions + 9 * static_cast<size_t>(i), sizeof(t.v));
        std::memcpy(t.n, normals + 9 * static_cast<size_t>(i), sizeof(t.n));
        std::memcpy(t.uv, uvs + 6 * static_cast<size_t>(i), sizeof(t.uv));
        t.mat = materialIds[i];
    }
    s->materials.resize(static_cast<size_t>(materialCount));
    if (materialCount > 0) {
        std::memcpy(s->materials.data(), materials, sizeof(MaterialRec) * static_cast<size_t>(materialCount));
    }
    s->textures.resize(static_cast<size_t>(textureCount));
    if (textureCount > 0) {
        std::memcpy(s->textures.data(), textures, sizeof(TextureRec) * static_cast<size_t>(textureCount));
    }
    buildScene(*s);
    return s;
}

void orc_scene_destroy(void* h) { delete static_cast<Scene*>(h); }

int orc_scene_bvh_node_count(void* h) { return static_cast<int>(static_cast<Scene*>(h)->nodes.size()); }

int orc_scene_emissive(void* h, uint32_t* outIdx, float* outCdf)
{
    const Scene* s = static_cast<Scene*>(h);
    if (outIdx) {
        std::memcpy(outIdx, s->emissiveIdx.data(), s->emissiveIdx.size() * sizeof(uint32_t));
    }
    if (outCdf) {
        std::memcpy(outCdf, s->emissiveCdf.data(), s->emissiveCdf.size() * sizeof(float));
    }
    return static_cast<int>(s->emissiveIdx.size());
}

void orc_trace_rays(void* h, int n, const float* o, const float* d, const float* tmin, const float* tmax,
    uint8_t* hit, float* t, uint32_t* tri, float* normal, float* uv)
{
    const Scene& s = *static_cast<Scene*>(h);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const Hit<float> r = traceRay<float>(s, mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]),
            mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]), tmin[i], tmax[i]);
        hit[i] = r.hit ? 1 : 0;
        t[i] = r.t;
        tri[i] = r.tri;
        normal[3 * i] = r.normal.x;
        normal[3 * i + 1] = r.normal.y;
        normal[3 * i + 2] = r.normal.z;
        uv[2 * i] = r.uv.x;
        uv[2 * i + 1] = r.uv.y;
    }
}

// Closest hit by testing every triangle (BVH-independent check of the BVH path;
// the reference's zero-direction quirk is not modelled here).
void orc_trace_rays_bruteforce(void* h, int n, const float* o, const float* d, const float* tmin, const float* tmax,
    uint8_t* hit, float* t, uint32_t* tri)
{
    const Scene& s = *static_cast<Scene*>(h);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const V3<float> ro = mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
        const V3<float> rd = nrm(mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]));
        float closest = tmax[i];
        uint32_t best = 0;
        for (uint32_t k = 0; k < s.tris.size(); ++k) {
            float th;
            V3<float> nn;
            V2<float> uv;
            if (rayTri<float>(ro, rd, s.tris[k], tmin[i], closest, th, nn, uv)) {
                closest = th;
                best = k;
            }
        }
        hit[i] = closest < tmax[i] ? 1 : 0;
        t[i] = hit[i] ? closest : 0.0f;
        tri[i] = hit[i] ? best : 0u;
    }
}

void* orc_env_create(int width, int height, const float* rgb)
{
    Env* e = new Env();
    e->width = width;
    e->height = height;
    e->pixels.assign(rgb, rgb + static_cast<size_t>(width) * height * 3);
    // EnvironmentMap.cpp:76-128.
    e->marginal.assign(static_cast<size_t>(height) + 1, 0.0f);
    e->row.assign(static_cast<size_t>(height) * (width + 1), 0.0f);
    std::vector<float> rowW(static_cast<size_t>(height), 0.0f);
    for (int y = 0; y < height; ++y) {
        const float v = (static_cast<float>(y) + 0.5f) / static_cast<float>(height);
        const float st = std::sin(v * 3.14159265f);
        float sum = 0.0f;
        const size_t off = static_cast<size_t>(y) * (width + 1);
        for (int x = 0; x < width; ++x) {
            const size_t i = (static_cast<size_t>(y) * width + x) * 3;
            const float l = std::max(e->pixels[i], std::max(e->pixels[i + 1], e->pixels[i + 2]));
            sum += std::max(l, 1.0e-6f) * st;
            e->row[off + x + 1] = sum;
        }
        if (sum > 0.0f) {
            for (int x = 0; x < width; ++x) {
                e->row[off + x + 1] /= sum;
            }
        }
        rowW[static_cast<size_t>(y)] = sum;
    }
    float total = 0.0f;
    for (int y = 0; y < height; ++y) {
        total += rowW[static_cast<size_t>(y)];
        e->marginal[static_cast<size_t>(y) + 1] = total;
    }
    if (total > 0.0f) {
        for (int y = 0; y < height; ++y) {
            e->marginal[static_cast<size_t>(y) + 1] /= total;
        }
    }
    return e;
}

void orc_env_destroy(void* h) { delete static_cast<Env*>(h); }

void orc_env_tables(void* h, float* marginal, float* row)
{
    const Env* e = static_cast<Env*>(h);
    std::memcpy(marginal, e->marginal.data(), e->marginal.size() * sizeof(float));
    std::memcpy(row, e->row.data(), e->row.size() * sizeof(float));
}

int orc_render(void* scene, void* env, const void* cam, const void* params, int width, int height, int waves,
    unsigned int seedBase, const float* tape, int tapeStride, const int* pixelList, int pixelListCount, float* acc,
    uint32_t* counts, float* lumMean, float* m2, uint8_t* converged, int threads)
{
    return renderImpl<float>(scene, env, cam, params, width, height, waves, seedBase, tape, tapeStride, pixelList,
        pixelListCount, acc, counts, lumMean, m2, converged, threads);
}

int orc64_render(void* scene, void* env, const void* cam, const void* params, int width, int height, int waves,
    unsigned int seedBase, const float* tape, int tapeStride, const int* pixelList, int pixelListCount, double* acc,
    uint32_t* counts, double* lumMean, double* m2, uint8_t* converged, int threads)
{
    return renderImpl<double>(scene, env, cam, params, width, height, waves, seedBase, tape, tapeStride, pixelList,
        pixelListCount, acc, counts, lumMean, m2, converged, threads);
}

// Spectral-mode render (FP32 and FP64): nw wavelengths per sample; resp 401 x 3;
// matCoef: per material base and scatter records (8 floats); texCoef: per
// texture two colour records (8 floats); envCoef: per texel (4 floats) or null;
// bgCoef: background x intensity (4 floats).  Returns tape underruns.
int orc_render_spectral(void* scene, void* env, const void* cam, const void* params, int width, int height, int waves,
    unsigned int seedBase, const float* tape, int tapeStride, int nw, const float* resp, const float* matCoef,
    int matCount, const float* texCoef, int texCount, const float* envCoef, const float* bgCoef, float* acc,
    uint32_t* counts, float* lumMean, float* m2, uint8_t* converged, int threads)
{
    const SpecSetup sp = makeSpecSetup(nw, resp, matCoef, matCount, texCoef, texCount, envCoef, bgCoef);
    return renderSpectralImpl<float>(scene, env, cam, params, width, height, waves, seedBase, tape, tapeStride, sp,
        acc, counts, lumMean, m2, converged, threads);
}

int orc64_render_spectral(void* scene, void* env, const void* cam, const void* params, int width, int height,
    int waves, unsigned int seedBase, const float* tape, int tapeStride, int nw, const float* resp,
    const float* matCoef, int matCount, const float* texCoef, int texCount, const float* envCoef, const float* bgCoef,
    double* acc, uint32_t* counts, double* lumMean, double* m2, uint8_t* converged, int threads)
{
    const SpecSetup sp = makeSpecSetup(nw, resp, matCoef, matCount, texCoef, texCount, envCoef, bgCoef);
    return renderSpectralImpl<double>(scene, env, cam, params, width, height, waves, seedBase, tape, tapeStride, sp,
        acc, counts, lumMean, m2, converged, threads);
}

// Distant light of a scene (restated from the product's definition): frame,
// cone constants in double, radiance RGB as given or a blackbody of the given
// temperature scaled to Rec. 709 luminance `luminance` through the response
// table resp (401 x 3, 1 nm from 380 nm); spectral coefficients of the RGB
// radiance `coef` (4 floats) for temperature <= 0.  enabled = 0 removes it.
// Emitter MIS mode of the renders of this scene (extension; the product's
// pt_render_params.emitter_mis = 1): 0 = the reference estimator.
void orc_scene_set_emitter_mis(void* h, int on)
{
    setEmitterMis(*static_cast<Scene*>(h), on != 0);
}

// Stop test of this scene's adaptive renders (the product's
// pt_render_params.adaptive_criterion): 0 = the reference's.
void orc_scene_set_adaptive_criterion(void* h, int criterion)
{
    static_cast<Scene*>(h)->adaptiveCriterion = criterion;
}

void orc_scene_set_sun(void* h, int enabled, const float* dir, float halfAngle, const float* rgb, float temperature,
    float luminance, const float* resp, const float* coef)
{
    Scene& s = *static_cast<Scene*>(h);
    s.sun = SunSetup{};
    if (!enabled) {
        return;
    }
    SunSetup& l = s.sun;
    const double len = std::sqrt(double(dir[0]) * dir[0] + double(dir[1]) * dir[1] + double(dir[2]) * dir[2]);
    const double d[3] = {dir[0] / len, dir[1] / len, dir[2] / len};
    const double up[3] = {std::fabs(d[1]) < 0.999 ? 0.0 : 1.0, std::fabs(d[1]) < 0.999 ? 1.0 : 0.0, 0.0};
    double t[3] = {up[1] * d[2] - up[2] * d[1], up[2] * d[0] - up[0] * d[2], up[0] * d[1] - up[1] * d[0]};
    const double tl = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    for (double& x : t) {
        x /= tl;
    }
    const double b[3] = {d[1] * t[2] - d[2] * t[1], d[2] * t[0] - d[0] * t[2], d[0] * t[1] - d[1] * t[0]};
    for (int k = 0; k < 3; ++k) {
        l.dir[k] = static_cast<float>(d[k]);
        l.t[k] = static_cast<float>(t[k]);
        l.b[k] = static_cast<float>(b[k]);
    }
    const double omc = 2.0 * std::sin(0.5 * halfAngle) * std::sin(0.5 * halfAngle);
    l.omc = static_cast<float>(omc);
    l.sin2 = static_cast<float>(std::sin(double(halfAngle)) * std::sin(double(halfAngle)));
    l.pdf = static_cast<float>(1.0 / (2.0 * 3.14159265358979323846 * omc));
    l.temperature = temperature;
    if (temperature > 0.0f) {
        double c[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < 401; ++i) {
            const double lu = (380.0 + i) * 1.0e-3;
            const double B = 1.0 / (lu * lu * lu * lu * lu * std::expm1(14387.769 / (lu * temperature)));
            const double w = (i == 0 || i == 400) ? 0.5 : 1.0;
            for (int k = 0; k < 3; ++k) {
                c[k] += w * B * resp[3 * i + k];
            }
        }
        const double K = 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2];
        const double scale = luminance / K;
        l.scale = static_cast<float>(scale);
        for (int k = 0; k < 3; ++k) {
            l.rgb[k] = static_cast<float>(c[k] * scale);
        }
    } else {
        for (int k = 0; k < 3; ++k) {
            l.rgb[k] = rgb[k];
        }
        for (int k = 0; k < 4; ++k) {
            l.coef[k] = coef != nullptr ? coef[k] : 0.0f;
        }
    }
    l.enabled = true;
}

// The spectrum of coefficient record c at lambda (FP32, the product's operation order).
float orc_spec_eval(const float* c, float lambda) { return specEval<float>(c, lambda); }

// Hero draw and wavelength k of nw for a path seed.
float orc_hero_lambda(unsigned int seed, int k, int nw) { return heroLambda(heroU(seed), k, nw); }

// d loss / d material parameters of the image drawn with `spp` samples per
// pixel (sample k of pixel p replays tape row (k, p)); dImage: 3 floats per
// pixel; grad: materialCount x 7 doubles (zeroed here).  Returns tape underruns.
int orc64_backward(void* sceneHandle, void* envHandle, const void* cameraBytes, const void* paramsBytes, int width,
    int height, int spp, const float* tape, int tapeStride, const float* dImage, double* grad, int materialCount,
    int threads)
{
    const Scene& s = *static_cast<Scene*>(sceneHandle);
    const Env* e = static_cast<Env*>(envHandle);
    CameraRec cam;
    std::memcpy(&cam, cameraBytes, sizeof(cam));
    ParamsRec p;
    std::memcpy(&p, paramsBytes, sizeof(p));
    const int P = width * height;
    const size_t G = static_cast<size_t>(materialCount) * 7;
    std::fill(grad, grad + G, 0.0);
    if (threads > 0) {
        omp_set_num_threads(threads);
    }
    int errors = 0;
#pragma omp parallel reduction(+ : errors)
    {
        std::vector<double> local(G, 0.0);
#pragma omp for schedule(dynamic, 16)
        for (int idx = 0; idx < P; ++idx) {
            const V3<double> d0 = mk(double(dImage[3 * idx]), double(dImage[3 * idx + 1]), double(dImage[3 * idx + 2]));
            if (d0.x == 0.0 && d0.y == 0.0 && d0.z == 0.0) {
                continue;
            }
            for (int k = 0; k < spp; ++k) {
                const float* row = tape + (static_cast<size_t>(k) * P + idx) * static_cast<size_t>(tapeStride);
                Rng r1;
                r1.row = row;
                r1.length = tapeStride;
                V3<double> ro, rd;
                pixelRay(cam, idx, width, height, r1, ro, rd);
                const V3<double> Lt = tracePathGrad<double>(s, e, &p, ro, rd, r1, mk(0.0, 0.0, 0.0),
                    mk(0.0, 0.0, 0.0), nullptr, 0);
                errors += r1.underruns;
                if (!std::isfinite(Lt.x) || !std::isfinite(Lt.y) || !std::isfinite(Lt.z)) {
                    continue;
                }
                if (Lt.x == 0.0 && Lt.y == 0.0 && Lt.z == 0.0) {
                    continue; // nothing collected: no gradient (as the product's adjoint)
                }
                // adjoint of the firefly clamp (PathTracer.cu:49-67)
                V3<double> delta = mk(Lt.x > 0.0 ? d0.x / spp : 0.0, Lt.y > 0.0 ? d0.y / spp : 0.0,
                    Lt.z > 0.0 ? d0.z / spp : 0.0);
                const V3<double> cl = mk(mx(0.0, Lt.x), mx(0.0, Lt.y), mx(0.0, Lt.z));
                const double l = cl.x * 0.2126 + cl.y * 0.7152 + cl.z * 0.0722;
                if (l > 100.0) {
                    const double kc = 100.0 / l;
                    const double dc = dot(delta, cl) / l;
                    const V3<double> w =
                        mk(Lt.x > 0.0 ? 0.2126 : 0.0, Lt.y > 0.0 ? 0.7152 : 0.0, Lt.z > 0.0 ? 0.0722 : 0.0);
                    delta = scl(sub(delta, scl(w, dc)), kc);
                }
                Rng r2;
                r2.row = row;
                r2.length = tapeStride;
                pixelRay(cam, idx, width, height, r2, ro, rd);
                tracePathGrad<double>(s, e, &p, ro, rd, r2, delta, Lt, local.data(), materialCount);
            }
        }
#pragma omp critical
        for (size_t i = 0; i < G; ++i) {
            grad[i] += local[i];
        }
    }
    return errors;
}

int orc_trace_pixel(void* scene, void* env, const void* camBytes, const void* paramsBytes, int width, int height,
    int idx, int sampleIndex, unsigned int globalSeed, const float* tapeRow, int tapeLength, float* outRgb)
{
    (void)sampleIndex;
    (void)globalSeed;
    CameraRec cam;
    std::memcpy(&cam, camBytes, sizeof(cam));
    ParamsRec p;
    std::memcpy(&p, paramsBytes, sizeof(p));
    Rng rng;
    rng.row = tapeRow;
    rng.length = tapeLength;
    const V3<float> c = tracePixel<float>(*static_cast<Scene*>(scene), static_cast<Env*>(env), cam, p, idx, width,
        height, rng);
    outRgb[0] = c.x;
    outRgb[1] = c.y;
    outRgb[2] = c.z;
    return rng.underruns != 0 ? -1 : rng.cursor;
}

// One preview pass (sampleKernel with previewPass, PathTracer.cu:132-184): per
// pixel, tape row idx, no jitter draws (pixel centre), lens draws, the path
// with the given params (the caller sets the preview depth), firefly clamp.
int orc_render_preview(void* scene, void* env, const void* camBytes, const void* paramsBytes, int width, int height,
    const float* tape, int tapeStride, float* outRgba)
{
    CameraRec cam;
    std::memcpy(&cam, camBytes, sizeof(cam));
    ParamsRec p;
    std::memcpy(&p, paramsBytes, sizeof(p));
    const Scene& s = *static_cast<Scene*>(scene);
    const Env* e = static_cast<Env*>(env);
    int errors = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : errors)
    for (int idx = 0; idx < width * height; ++idx) {
        Rng rng;
        rng.row = tape + static_cast<size_t>(idx) * tapeStride;
        rng.length = tapeStride;
        const int x = idx % width, y = idx / width;
        const float u = (static_cast<float>(x) + 0.5f) / static_cast<float>(width);
        const float v = (static_cast<float>(y) + 0.5f) / static_cast<float>(height);
        const float l1 = rng.next();
        const float l2 = rng.next();
        V3<float> ro, rd;
        cameraRay(cam, u, v, l1, l2, ro, rd);
        const V3<float> c = clampFirefly(tracePath(s, e, &p, ro, rd, rng));
        outRgba[4 * idx] = c.x;
        outRgba[4 * idx + 1] = c.y;
        outRgba[4 * idx + 2] = c.z;
        outRgba[4 * idx + 3] = 1.0f;
        errors += rng.underruns;
    }
    return errors;
}

void orc_brdf_eval(const float* normal, const float* wo, const void* material, float eta, int debug, const float* wi,
    float* outRgb)
{
    const Ctx<float> c = makeCtx(normal, wo, material, eta, debug);
    const V3<float> f = bsdfEval(c, mk(wi[0], wi[1], wi[2]));
    outRgb[0] = f.x;
    outRgb[1] = f.y;
    outRgb[2] = f.z;
}

float orc_brdf_pdf(const float* normal, const float* wo, const void* material, float eta, int debug, const float* wi)
{
    return bsdfPdf(makeCtx(normal, wo, material, eta, debug), mk(wi[0], wi[1], wi[2]));
}

int orc_brdf_sample(const float* normal, const float* wo, const void* material, float eta, int debug, float u1,
    float u2, float* outDir, float* outPdf, float* outNextEta, float* outExitOffset, int* outFlags)
{
    const Sample<float> r = bsdfSample(makeCtx(normal, wo, material, eta, debug), u1, u2);
    outDir[0] = r.dir.x;
    outDir[1] = r.dir.y;
    outDir[2] = r.dir.z;
    *outPdf = r.pdf;
    *outNextEta = r.nextEta;
    outExitOffset[0] = r.exitOffset.x;
    outExitOffset[1] = r.exitOffset.y;
    outExitOffset[2] = r.exitOffset.z;
    *outFlags = (r.valid ? 1 : 0) | (r.transmitted ? 2 : 0) | (r.sss ? 4 : 0);
    return r.sssSteps;
}

void orc_brdf_apply_throughput(const float* tp, const float* normal, const float* wo, const void* material, float eta,
    float u1, float u2, float* outTp)
{
    const Ctx<float> c = makeCtx(normal, wo, material, eta, 0);
    const Sample<float> r = bsdfSample(c, u1, u2);
    const V3<float> f = bsdfEval(c, r.dir);
    const V3<float> t = applyThroughput(mk(tp[0], tp[1], tp[2]), c, r, f);
    outTp[0] = t.x;
    outTp[1] = t.y;
    outTp[2] = t.z;
}

void orc_camera_ray(const void* camBytes, float u, float v, float l1, float l2, float* outO, float* outD)
{
    CameraRec cam;
    std::memcpy(&cam, camBytes, sizeof(cam));
    V3<float> o, d;
    cameraRay<float>(cam, u, v, l1, l2, o, d);
    outO[0] = o.x;
    outO[1] = o.y;
    outO[2] = o.z;
    outD[0] = d.x;
    outD[1] = d.y;
    outD[2] = d.z;
}

void orc_env_sample(void* env, const void* paramsBytes, float u1, float u2, float* outDir, float* outPdf)
{
    (void)paramsBytes;
    float pdf = 0.0f;
    const V3<float> d = envSample<float>(static_cast<Env*>(env), u1, u2, pdf);
    outDir[0] = d.x;
    outDir[1] = d.y;
    outDir[2] = d.z;
    *outPdf = pdf;
}

float orc_env_pdf(void* env, const void* paramsBytes, const float* dir)
{
    (void)paramsBytes;
    return envPdf<float>(static_cast<Env*>(env), mk(dir[0], dir[1], dir[2]));
}

void orc_env_eval(void* env, const void* paramsBytes, const float* dir, float* outRgb)
{
    ParamsRec p;
    std::memcpy(&p, paramsBytes, sizeof(p));
    const V3<float> c = envEval<float>(static_cast<Env*>(env), &p, mk(dir[0], dir[1], dir[2]));
    outRgb[0] = c.x;
    outRgb[1] = c.y;
    outRgb[2] = c.z;
}

int orc_sample_emissive(void* scene, float uTri, float u1, float u2, float* outPos, float* outNormal,
    float* outRadiance, float* outPdf)
{
    V3<float> p{0, 0, 0}, n{0, 0, 0}, L{0, 0, 0};
    float pdf = 0.0f;
    const bool ok = sampleEmissive<float>(*static_cast<Scene*>(scene), uTri, u1, u2, p, n, L, pdf);
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

int orc_brdf_sample_transmit(const float* normal, const float* wo, const void* material, float eta, int debug,
    float u1, float u2, float* outDir, float* outPdf, float* outNextEta, int* outFlags)
{
    const Sample<float> r = sampleTransmit(makeCtx(normal, wo, material, eta, debug), u1, u2);
    outDir[0] = r.dir.x;
    outDir[1] = r.dir.y;
    outDir[2] = r.dir.z;
    *outPdf = r.pdf;
    *outNextEta = r.nextEta;
    *outFlags = (r.valid ? 1 : 0) | (r.transmitted ? 2 : 0) | (r.sss ? 4 : 0);
    return r.sssSteps;
}

void orc_lobe_weights(const void* material, float* out)
{
    const float zero[3] = {0.0f, 0.0f, 1.0f};
    const Lobes<float> w = lobes(makeCtx(zero, zero, material, 1.0f, 0));
    out[0] = w.diffuse;
    out[1] = w.specular;
    out[2] = w.transmit;
    out[3] = w.subsurface;
}

void orc_resolve_material(const void* material, float u, float v, const void* textures, int textureCount, float* out)
{
    MaterialRec m;
    std::memcpy(&m, material, sizeof(m));
    std::vector<TextureRec> bank(static_cast<size_t>(textureCount > 0 ? textureCount : 0));
    if (textureCount > 0) {
        std::memcpy(bank.data(), textures, sizeof(TextureRec) * static_cast<size_t>(textureCount));
    }
    const Mat<float> r = resolve<float>(m, V2<float>{u, v}, bank);
    const float vals[15] = {r.r, r.g, r.b, r.roughness, r.metallic, r.transmission, r.thin, r.ior, r.subsurface,
        r.emission, r.diffuseRoughness, r.scatterR, r.scatterG, r.scatterB, r.specular};
    std::memcpy(out, vals, sizeof(vals));
}

int orc_is_converged(uint32_t n, float mean, float m2, int minSamples, float thr)
{
    return isConverged(n, mean, m2, minSamples, thr) ? 1 : 0;
}

unsigned int orc_reference_seed(int pixel, int sampleIndex, unsigned int globalSeed)
{
    return referenceSeed(pixel, sampleIndex, globalSeed);
}

int orc_max_threads() { return omp_get_max_threads(); }

} // extern "C"
