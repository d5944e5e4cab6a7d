// Scene construction on the device.
//
// Tube loft: the turtle's branch polylines become tubes of `sides`-gons, one
// ring per polyline state, with two triangles per side quad and flat caps at
// both ends (the loft of Application/src/Procedural/Loft.cpp:108-155 as the
// scene generator in lsystemeditor_b200/scene.py writes it).  The arithmetic is
// IEEE double with every operation rounded on its own (no contraction), in the
// generator's order, so the device mesh is bit-identical to the host one.
//
// Emissive list: per-triangle weight area x Rec.709 luminance x emission and a
// prefix sum over the emissive triangles in triangle order, in single
// precision and summed sequentially exactly like MeshAccelScene.cpp:62-95, so
// light sampling picks the same triangle as the reference for every uniform.
#include "pt_scene.cuh"

#include "pt_select.cuh"

namespace pt {

namespace {

constexpr int kBlock = 256;

inline int gridFor(uint64_t n)
{
    const uint64_t g = (n + kBlock - 1) / kBlock;
    return static_cast<int>(g < 1 ? 1 : (g > 148ull * 32ull ? 148ull * 32ull : g));
}

struct D3 {
    double x, y, z;
};

__device__ __forceinline__ D3 dload(const double* p) { return D3{p[0], p[1], p[2]}; }
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return D3{__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return D3{__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y), __dadd_rn(a.z, b.z)}; }
__device__ __forceinline__ D3 dscl(D3 a, double s) { return D3{__dmul_rn(a.x, s), __dmul_rn(a.y, s), __dmul_rn(a.z, s)}; }
__device__ __forceinline__ D3 ddiv(D3 a, double s) { return D3{__ddiv_rn(a.x, s), __ddiv_rn(a.y, s), __ddiv_rn(a.z, s)}; }
__device__ __forceinline__ D3 dneg(D3 a) { return D3{-a.x, -a.y, -a.z}; }
// numpy.cross: (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0)
__device__ __forceinline__ D3 dcross(D3 a, D3 b)
{
    return D3{__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
        __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}
// numpy.linalg.norm over the last axis: sqrt((x^2 + y^2) + z^2)
__device__ __forceinline__ double dnorm(D3 a)
{
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y)), __dmul_rn(a.z, a.z)));
}

__device__ __forceinline__ void put3(float* p, D3 a)
{
    p[0] = __double2float_rn(a.x);
    p[1] = __double2float_rn(a.y);
    p[2] = __double2float_rn(a.z);
}

// Tube of ring g: the last t with ringStart[t] <= g.
__device__ __forceinline__ uint32_t tubeOfRing(const uint32_t* ringStart, uint32_t tubes, uint32_t g)
{
    uint32_t lo = 0, hi = tubes - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (ringStart[mid] <= g) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

// frames[9 g ..]: unit tangent u, side axes a, b of ring g.  The last ring of
// a tube takes the tangent of the ring before it; a = normalize(ref x u) with
// ref = +Y unless u is within acos(0.99) of it (then +X); b = u x a.
__global__ void k_ring_frames(TubeSetDev T, double* frames)
{
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < T.ringCount; g += gridDim.x * blockDim.x) {
        D3 u, a, b;
        if (T.frames != nullptr) {
            // given frames (the spline's): the ring's own unit tangent, normal and binormal
            const D3 tan = dload(T.tangents + 3ull * g);
            u = ddiv(tan, dnorm(tan));
            a = dload(T.frames + 6ull * g);
            b = dload(T.frames + 6ull * g + 3);
        } else {
            const uint32_t t = tubeOfRing(T.ringStart, T.tubeCount, g);
            const uint32_t first = T.ringStart[t], last = T.ringStart[t + 1] - 1;
            const uint32_t src = (g == last && last > first) ? g - 1 : g;
            const D3 tan = dload(T.tangents + 3ull * src);
            u = ddiv(tan, dnorm(tan));
            const D3 ref = fabs(u.y) < 0.99 ? D3{0.0, 1.0, 0.0} : D3{1.0, 0.0, 0.0};
            a = dcross(ref, u);
            a = ddiv(a, dnorm(a));
            b = dcross(u, a);
        }
        double* f = frames + 9ull * g;
        f[0] = u.x;
        f[1] = u.y;
        f[2] = u.z;
        f[3] = a.x;
        f[4] = a.y;
        f[5] = a.z;
        f[6] = b.x;
        f[7] = b.y;
        f[8] = b.z;
    }
}

// Radial direction a cos + b sin of side k at ring g, and the ring vertex.
__device__ __forceinline__ void ringVertex(const TubeSetDev& T, const double* frames, uint32_t g, uint32_t k, D3& dir,
    D3& pos)
{
    const double* f = frames + 9ull * g;
    const double c = T.cosSin[2 * k], s = T.cosSin[2 * k + 1];
    dir = dadd(dscl(D3{f[3], f[4], f[5]}, c), dscl(D3{f[6], f[7], f[8]}, s));
    pos = dadd(dload(T.points + 3ull * g), dscl(dir, T.radii[g]));
}

__global__ void k_loft(TubeSetDev T, const double* frames, float* positions, float* normals, float* uvs,
    uint32_t* materialIds)
{
    const uint64_t sides2 = 2ull * T.sides;
    const uint64_t tubeTris = sides2 * T.ringCount;
    const uint64_t total = tubeTris + 2ull * T.leafCount;
    for (uint64_t g = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; g < total;
         g += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        D3 p[3], n[3];
        float uv[6];
        uint32_t mat;
        if (g < tubeTris) {
            const uint32_t t = tubeOfRing(T.ringStart, T.tubeCount, static_cast<uint32_t>(g / sides2));
            const uint32_t first = T.ringStart[t];
            const uint32_t R = T.ringStart[t + 1] - first;
            const uint64_t local = g - sides2 * first;
            mat = T.materials[t];
            if (local < sides2 * (R - 1)) {
                // side quad (ring r, side k): (r,k) (r,k+1) (r+1,k) | (r,k+1) (r+1,k+1) (r+1,k)
                const uint32_t r = static_cast<uint32_t>(local / sides2);
                const uint32_t rem = static_cast<uint32_t>(local % sides2);
                const uint32_t k = rem >> 1;
                const uint32_t k1 = (k + 1 == T.sides) ? 0u : k + 1; // the seam vertex is side 0's
                const double u0 = __ddiv_rn(static_cast<double>(k), static_cast<double>(T.sides));
                const double u1 = __ddiv_rn(static_cast<double>(k + 1), static_cast<double>(T.sides));
                const double span = static_cast<double>(R - 1 > 1 ? R - 1 : 1);
                const double v0 = __ddiv_rn(static_cast<double>(r), span);
                const double v1 = __ddiv_rn(static_cast<double>(r + 1), span);
                if ((rem & 1u) == 0u) {
                    ringVertex(T, frames, first + r, k, n[0], p[0]);
                    ringVertex(T, frames, first + r, k1, n[1], p[1]);
                    ringVertex(T, frames, first + r + 1, k, n[2], p[2]);
                    const float q[6] = {__double2float_rn(u0), __double2float_rn(v0), __double2float_rn(u1),
                        __double2float_rn(v0), __double2float_rn(u0), __double2float_rn(v1)};
                    for (int i = 0; i < 6; ++i) {
                        uv[i] = q[i];
                    }
                } else {
                    ringVertex(T, frames, first + r, k1, n[0], p[0]);
                    ringVertex(T, frames, first + r + 1, k1, n[1], p[1]);
                    ringVertex(T, frames, first + r + 1, k, n[2], p[2]);
                    const float q[6] = {__double2float_rn(u1), __double2float_rn(v0), __double2float_rn(u1),
                        __double2float_rn(v1), __double2float_rn(u0), __double2float_rn(v1)};
                    for (int i = 0; i < 6; ++i) {
                        uv[i] = q[i];
                    }
                }
            } else {
                // caps, interleaved per side (Loft.cpp:141-152): start (centre, k+1, k)
                // facing -u, end (centre, k, k+1) facing +u; rim uvs 0.5 + 0.5 (sin, cos)
                const uint32_t c = static_cast<uint32_t>(local - sides2 * (R - 1));
                const bool start = (c & 1u) == 0u;
                const uint32_t k = c >> 1;
                const uint32_t k1 = (k + 1 == T.sides) ? 0u : k + 1;
                const uint32_t ring = start ? first : first + R - 1;
                D3 d0, d1, r0, r1;
                ringVertex(T, frames, ring, k, d0, r0);
                ringVertex(T, frames, ring, k1, d1, r1);
                p[0] = dload(T.points + 3ull * ring);
                p[1] = start ? r1 : r0;
                p[2] = start ? r0 : r1;
                const double* f = frames + 9ull * ring;
                const D3 u = D3{f[0], f[1], f[2]};
                n[0] = n[1] = n[2] = start ? dneg(u) : u;
                const float ua = __double2float_rn(__dadd_rn(0.5, __dmul_rn(0.5, T.cosSin[2 * k + 1])));
                const float va = __double2float_rn(__dadd_rn(0.5, __dmul_rn(0.5, T.cosSin[2 * k])));
                const float ub = __double2float_rn(__dadd_rn(0.5, __dmul_rn(0.5, T.cosSin[2 * k1 + 1])));
                const float vb = __double2float_rn(__dadd_rn(0.5, __dmul_rn(0.5, T.cosSin[2 * k1])));
                uv[0] = 0.5f;
                uv[1] = 0.5f;
                uv[2] = start ? ub : ua;
                uv[3] = start ? vb : va;
                uv[4] = start ? ua : ub;
                uv[5] = start ? va : vb;
            }
        } else {
            // leaf quad spanning (tangent x up) and the tangent: (p00 p10 p11) (p00 p11 p01)
            const uint64_t l = (g - tubeTris) >> 1;
            const bool second = ((g - tubeTris) & 1ull) != 0ull;
            const double* L = T.leaves + 10ull * l;
            const D3 P = dload(L), Tn = dload(L + 3), U = dload(L + 6);
            const double s = __dmul_rn(L[9], T.leafSize);
            D3 w = dcross(Tn, U);
            w = ddiv(w, dnorm(w));
            const D3 half = dscl(dscl(w, s), 0.5);
            const D3 p00 = dsub(P, half), p10 = dadd(P, half);
            const D3 ts = dscl(Tn, s);
            const D3 p01 = dadd(p00, ts), p11 = dadd(p10, ts);
            const D3 nn = ddiv(U, dnorm(U));
            n[0] = n[1] = n[2] = nn;
            mat = T.leafMaterial;
            p[0] = p00;
            if (!second) {
                p[1] = p10;
                p[2] = p11;
                const float q[6] = {0.0f, 0.0f, 1.0f, 0.0f, 1.0f, 1.0f};
                for (int i = 0; i < 6; ++i) {
                    uv[i] = q[i];
                }
            } else {
                p[1] = p11;
                p[2] = p01;
                const float q[6] = {0.0f, 0.0f, 1.0f, 1.0f, 0.0f, 1.0f};
                for (int i = 0; i < 6; ++i) {
                    uv[i] = q[i];
                }
            }
        }
        for (int v = 0; v < 3; ++v) {
            put3(positions + 9ull * g + 3 * v, p[v]);
            put3(normals + 9ull * g + 3 * v, n[v]);
        }
        for (int i = 0; i < 6; ++i) {
            uvs[6ull * g + i] = uv[i];
        }
        materialIds[g] = mat;
    }
}

__global__ void k_emissive_weights(const float* positions, const uint32_t* materialIds, uint32_t n,
    const pt_material* materials, uint32_t materialCount, float* weights, uint8_t* flags)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float w = 0.0f;
        uint8_t f = 0;
        const uint32_t mi = materialIds[i];
        if (mi < materialCount) {
            const pt_material m = materials[mi];
            const float lum = __fmul_rn(m.emission,
                __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, m.r), __fmul_rn(0.7152f, m.g)), __fmul_rn(0.0722f, m.b)));
            if (!(lum <= 0.0f)) { // as the reference's `lum <= 0 -> skip` (a NaN passes)
                const float* p = positions + 9ull * i;
                const float e1x = __fsub_rn(p[3], p[0]), e1y = __fsub_rn(p[4], p[1]), e1z = __fsub_rn(p[5], p[2]);
                const float e2x = __fsub_rn(p[6], p[0]), e2y = __fsub_rn(p[7], p[1]), e2z = __fsub_rn(p[8], p[2]);
                const float cx = __fsub_rn(__fmul_rn(e1y, e2z), __fmul_rn(e1z, e2y));
                const float cy = __fsub_rn(__fmul_rn(e1z, e2x), __fmul_rn(e1x, e2z));
                const float cz = __fsub_rn(__fmul_rn(e1x, e2y), __fmul_rn(e1y, e2x));
                const float area = __fmul_rn(0.5f,
                    __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz))));
                w = __fmul_rn(area, lum);
                f = (w <= 0.0f) ? 0 : 1;
            }
        }
        weights[i] = w;
        flags[i] = f;
    }
}

// One thread: the sequential single-precision running sum.
__global__ void k_emissive_cdf(const float* weights, const uint32_t* idx, const uint32_t* dCount, float* cdf,
    uint32_t* out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) {
        return;
    }
    const uint32_t count = *dCount;
    float total = 0.0f;
    cdf[0] = 0.0f;
    for (uint32_t k = 0; k < count; ++k) {
        total = __fadd_rn(total, weights[idx[k]]);
        cdf[k + 1] = total;
    }
    out[0] = count;
    out[1] = __float_as_uint(total);
}

__global__ void k_build_shade(const float* nrm, const float* uv, const uint32_t* mat, uint32_t n, TriShade* out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* a = nrm + 9ull * i;
        const float* t = uv + 6ull * i;
        TriShade s;
        s.a = make_float4(a[0], a[1], a[2], t[0]);
        s.b = make_float4(a[3], a[4], a[5], t[1]);
        s.c = make_float4(a[6], a[7], a[8], t[2]);
        s.d = make_float4(t[3], t[4], t[5], __uint_as_float(mat[i]));
        out[i] = s;
    }
}

__global__ void k_unpack_shade(const TriShade* shade, uint32_t n, float* nrm, float* uv, uint32_t* mat)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const TriShade s = shade[i];
        float* a = nrm + 9ull * i;
        float* t = uv + 6ull * i;
        a[0] = s.a.x;
        a[1] = s.a.y;
        a[2] = s.a.z;
        a[3] = s.b.x;
        a[4] = s.b.y;
        a[5] = s.b.z;
        a[6] = s.c.x;
        a[7] = s.c.y;
        a[8] = s.c.z;
        t[0] = s.a.w;
        t[1] = s.b.w;
        t[2] = s.c.w;
        t[3] = s.d.x;
        t[4] = s.d.y;
        t[5] = s.d.z;
        mat[i] = __float_as_uint(s.d.w);
    }
}

// std::max as the reference uses it: (a < b) ? b : a.
__device__ __forceinline__ float stdMax(float a, float b) { return a < b ? b : a; }

// Environment importance tables (EnvironmentMap.cpp:76-128), one thread per
// row: the row's running sum of max(r, g, b) (at least 1e-6) times sin(theta)
// in single precision, in column order, then divided by the row total.
__global__ void k_env_rows(const float* rgb, int width, int height, const float* sinTheta, float* row, float* rowW)
{
    for (int y = blockIdx.x * blockDim.x + threadIdx.x; y < height; y += gridDim.x * blockDim.x) {
        const float st = sinTheta[y];
        const size_t off = static_cast<size_t>(y) * (width + 1);
        const float* px = rgb + static_cast<size_t>(y) * width * 3;
        float sum = 0.0f;
        row[off] = 0.0f;
        for (int x = 0; x < width; ++x) {
            const float l = stdMax(px[3 * x], stdMax(px[3 * x + 1], px[3 * x + 2]));
            sum = __fadd_rn(sum, __fmul_rn(stdMax(l, 1.0e-6f), st));
            row[off + x + 1] = sum;
        }
        if (sum > 0.0f) {
            for (int x = 0; x < width; ++x) {
                row[off + x + 1] = __fdiv_rn(row[off + x + 1], sum);
            }
        }
        rowW[y] = sum;
    }
}

// The marginal over rows, summed in row order by one thread.
__global__ void k_env_marginal(const float* rowW, int height, float* marginal)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) {
        return;
    }
    float total = 0.0f;
    marginal[0] = 0.0f;
    for (int y = 0; y < height; ++y) {
        total = __fadd_rn(total, rowW[y]);
        marginal[y + 1] = total;
    }
    if (total > 0.0f) {
        for (int y = 0; y < height; ++y) {
            marginal[y + 1] = __fdiv_rn(marginal[y + 1], total);
        }
    }
}

} // namespace

void launchEnvTables(const float* rgb, int width, int height, const float* sinTheta, float* marginal, float* row,
    float* rowW, cudaStream_t s)
{
    k_env_rows<<<(height + 127) / 128, 128, 0, s>>>(rgb, width, height, sinTheta, row, rowW);
    k_env_marginal<<<1, 32, 0, s>>>(rowW, height, marginal);
}

void launchRingFrames(const TubeSetDev& t, double* frames, cudaStream_t s)
{
    if (t.ringCount > 0) {
        k_ring_frames<<<gridFor(t.ringCount), kBlock, 0, s>>>(t, frames);
    }
}

void launchLoft(const TubeSetDev& t, const double* frames, float* positions, float* normals, float* uvs,
    uint32_t* materialIds, cudaStream_t s)
{
    const uint64_t n = tubeTriangles(t.sides, t.ringCount, t.leafCount);
    if (n > 0) {
        k_loft<<<gridFor(n), kBlock, 0, s>>>(t, frames, positions, normals, uvs, materialIds);
    }
}

void launchEmissiveWeights(const float* positions, const uint32_t* materialIds, uint32_t n,
    const pt_material* materials, uint32_t materialCount, float* weights, uint8_t* flags, cudaStream_t s)
{
    if (n > 0) {
        k_emissive_weights<<<gridFor(n), kBlock, 0, s>>>(positions, materialIds, n, materials, materialCount, weights,
            flags);
    }
}

namespace {
struct FlaggedTriangle {
    const uint8_t* flags;
    __device__ __forceinline__ bool operator()(long long i) const { return flags[i] != 0; }
};
struct TriangleIndex {
    __device__ __forceinline__ uint32_t operator()(long long i) const { return static_cast<uint32_t>(i); }
};
} // namespace

size_t emissiveSelectTempBytes(uint32_t n)
{
    return selectTempBytes(n);
}

// The emissive list in increasing triangle order (MeshAccelScene.cpp:62-95
// walks the triangles in order and appends every emitter).
cudaError_t emissiveSelect(void* temp, size_t tempBytes, const uint8_t* flags, uint32_t n, uint32_t* idx,
    uint32_t* dCount, cudaStream_t s)
{
    return launchSelect(static_cast<long long>(n), FlaggedTriangle{flags}, TriangleIndex{}, idx, dCount, temp,
        tempBytes, s);
}

namespace {
// Per emitter of the list: the area density with which sampleEmissive picks a
// point of it, ((cdf[e+1] - cdf[e]) / total) / area, in the same operations.
__global__ void k_emitter_pdf(const float* __restrict__ positions, const uint32_t* __restrict__ idx,
    const float* __restrict__ cdf, uint32_t count, float* __restrict__ out)
{
    const float total = cdf[count];
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        const uint32_t tri = idx[e];
        const float* p = positions + 9ull * tri;
        const float3 v0 = f3(p[0], p[1], p[2]), v1 = f3(p[3], p[4], p[5]), v2 = f3(p[6], p[7], p[8]);
        const float3 cr = cross3(sub3(v1, v0), sub3(v2, v0));
        const float area = 0.5f * sqrtf(dot3(cr, cr));
        out[tri] = (total > kMinPdf && area > kMinPdf) ? ((cdf[e + 1] - cdf[e]) / total) / area : 0.0f;
    }
}
} // namespace

void launchEmitterPdf(const float* positions, const uint32_t* idx, const float* cdf, uint32_t count, float* out,
    cudaStream_t s)
{
    if (count > 0) {
        k_emitter_pdf<<<gridFor(count), kBlock, 0, s>>>(positions, idx, cdf, count, out);
    }
}

void launchEmissiveCdf(const float* weights, const uint32_t* idx, const uint32_t* dCount, float* cdf, uint32_t* out,
    cudaStream_t s)
{
    k_emissive_cdf<<<1, 32, 0, s>>>(weights, idx, dCount, cdf, out);
}

void launchBuildShade(const float* normals, const float* uvs, const uint32_t* materialIds, uint32_t n, TriShade* out,
    cudaStream_t s)
{
    if (n > 0) {
        k_build_shade<<<gridFor(n), kBlock, 0, s>>>(normals, uvs, materialIds, n, out);
    }
}

void launchUnpackShade(const TriShade* shade, uint32_t n, float* normals, float* uvs, uint32_t* materialIds,
    cudaStream_t s)
{
    if (n > 0) {
        k_unpack_shade<<<gridFor(n), kBlock, 0, s>>>(shade, n, normals, uvs, materialIds);
    }
}

} // namespace pt
