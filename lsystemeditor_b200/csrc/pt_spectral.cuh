// Hero-wavelength spectral rendering (an extension: the reference's
// integrator is RGB; its spectral helpers in PathTracerLib/src/Spectral/ are
// not on any render path).
//
// A path carries NW radiance / throughput values at NW wavelengths spread
// evenly over [380, 780] nm from one uniformly drawn hero wavelength
// (Wilkie, Nawaz, Droske, Weidlich, Hanika, "Hero Wavelength Spectral
// Sampling", EGSR 2014).  Path sampling does not depend on the wavelength
// (the BSDF's lobe probabilities and index of refraction are colour- and
// wavelength-independent, as in the reference: SpectralCore.h:221-225), so
// every wavelength shares the path and the hero MIS weights are all 1/NW.
//
// Colours become spectra through the reference's function space,
// s(lambda) = 1/2 + x / (2 sqrt(1 + x^2)), x = c0 lambda^2 + c1 lambda + c2
// (Jakob and Hanika, "A Low-Dimensional Function Space for Efficient
// Spectral Upsampling", Eurographics 2019; evaluated as Rgb2Spec.h:58-66).
// The reference reads (c0, c1, c2) from a precomputed coefficient cube whose
// file is absent from its tree; here they are solved per colour (upliftSolve,
// Gauss-Newton with Levenberg-Marquardt damping along a path from grey to the
// target), so no table is needed.  A radiance colour brighter than 1 is
// scaled by its largest channel first (as rgb2specEvalRadiance does).
//
// A spectral sample becomes linear sRGB through the CIE 1931 2-degree
// colour-matching functions weighted by the D65 illuminant (the reference's
// spectralRgbResponseAtWavelength, SpectralCore.h:128-139) and the XYZ ->
// linear sRGB matrix derived from the sRGB primaries and white point
// (IEC 61966-2-1), normalised per channel so that a constant spectrum of 1
// maps to RGB (1, 1, 1) -- the role of the reference's white normalisation
// (SpectralState.cpp:15-45).  The response is tabulated every 1 nm.
#pragma once

#include "pt_common.cuh"

#include <cmath>

#if defined(__CUDACC__)
#define PT_HD __host__ __device__
#else
#define PT_HD
#endif

namespace pt {
namespace spectral {

constexpr float kLambdaMin = 380.0f;
constexpr float kLambdaMax = 780.0f;
constexpr float kLambdaRange = kLambdaMax - kLambdaMin;
constexpr int kRespCount = 401; // response table entries, 1 nm apart
constexpr int kMaxWavelengths = 8;

// Coefficient record of one colour: spectrum(lambda) = scale * s(lambda).
// A grey g is stored exactly as c = 0, scale = 2 g (s = 1/2 everywhere).
struct Coef {
    float c0, c1, c2, scale;
};

// --- host: tables ------------------------------------------------------------

// Response table: out[4 * i + ch] = sRGB response of channel ch at
// 380 + i nm, normalised so that the trapezoid sum over the table (1 nm
// steps) is 1 per channel; out[4 * i + 3] = 0.
void buildResponseTable(float* out);
// The data it is built from: x-bar, y-bar, z-bar, D65 at 380 .. 780 nm every
// 10 nm (41 x 4, cie may be null) and the XYZ -> linear sRGB matrix (row-major,
// m may be null).
void spectralSourceTables(float* cie, float* m);

// --- host + device: the uplift ------------------------------------------------

PT_HD inline double sigmoidD(double z) { return 0.5 + z / (2.0 * sqrt(1.0 + z * z)); }

// RGB of spectrum s(c0 t^2 + c1 t + c2), t = (lambda - 380) / 400, against the
// response table (trapezoid over its 401 nodes); with J the Jacobian.
PT_HD inline void upliftRgb(const float* resp, const double c[3], double rgb[3], double J[3][3], bool wantJ)
{
    for (int k = 0; k < 3; ++k) {
        rgb[k] = 0.0;
        J[k][0] = J[k][1] = J[k][2] = 0.0;
    }
    for (int i = 0; i < kRespCount; ++i) {
        const double t = static_cast<double>(i) / static_cast<double>(kRespCount - 1);
        const double z = (c[0] * t + c[1]) * t + c[2];
        const double q = 1.0 + z * z;
        const double rq = sqrt(q);
        const double s = 0.5 + z / (2.0 * rq);
        const double w = (i == 0 || i == kRespCount - 1) ? 0.5 : 1.0;
        const double ds = wantJ ? w / (2.0 * q * rq) : 0.0;
        for (int k = 0; k < 3; ++k) {
            const double rk = static_cast<double>(resp[4 * i + k]);
            rgb[k] += w * s * rk;
            if (wantJ) {
                J[k][0] += ds * t * t * rk;
                J[k][1] += ds * t * rk;
                J[k][2] += ds * rk;
            }
        }
    }
}

PT_HD inline bool solve3(const double A[3][3], const double b[3], double x[3])
{
    const double d = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
        A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) + A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    if (!(fabs(d) > 1.0e-300)) {
        return false;
    }
    for (int col = 0; col < 3; ++col) {
        double M[3][3];
        for (int r = 0; r < 3; ++r) {
            for (int k = 0; k < 3; ++k) {
                M[r][k] = k == col ? b[r] : A[r][k];
            }
        }
        x[col] = (M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                     M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0])) /
            d;
    }
    return true;
}

PT_HD inline double sq3(const double r[3]) { return r[0] * r[0] + r[1] * r[1] + r[2] * r[2]; }

// Coefficients of a reflectance (radiance = false: channels clamped to [0, 1])
// or a radiance colour (radiance = true: negative channels clamped to 0,
// scaled by the largest channel when that exceeds 1).  Deterministic; the
// same code runs on the host (materials, textures, background) and on the
// device (environment-map texels).
PT_HD inline Coef upliftSolve(const float* resp, float r, float g, float b, bool radiance)
{
    double tgt[3] = {r, g, b};
    double scale = 1.0;
    for (int k = 0; k < 3; ++k) {
        if (!(tgt[k] > 0.0)) {
            tgt[k] = 0.0; // also NaN
        }
        if (!radiance && tgt[k] > 1.0) {
            tgt[k] = 1.0;
        }
    }
    if (radiance) {
        const double m = fmax(tgt[0], fmax(tgt[1], tgt[2]));
        if (m > 1.0) {
            scale = m;
            for (int k = 0; k < 3; ++k) {
                tgt[k] /= m;
            }
        }
    }
    Coef out{0.0f, 0.0f, 0.0f, 0.0f};
    if (tgt[0] == tgt[1] && tgt[1] == tgt[2]) {
        out.scale = static_cast<float>(2.0 * tgt[0] * scale);
        return out;
    }
    // start: the grey of the target's mean, then move the target there-to in steps
    double g0 = (tgt[0] + tgt[1] + tgt[2]) / 3.0;
    g0 = fmin(fmax(g0, 0.02), 0.98);
    const double y0 = 2.0 * g0 - 1.0;
    double c[3] = {0.0, 0.0, y0 / sqrt(1.0 - y0 * y0)};
    const int kSteps = 8;
    double mu = 1.0e-3;
    for (int step = 1; step <= kSteps; ++step) {
        const double a = static_cast<double>(step) / kSteps;
        const double tk[3] = {g0 + (tgt[0] - g0) * a, g0 + (tgt[1] - g0) * a, g0 + (tgt[2] - g0) * a};
        const int iters = step == kSteps ? 60 : 12;
        double rgb[3], J[3][3];
        upliftRgb(resp, c, rgb, J, true);
        double res[3] = {rgb[0] - tk[0], rgb[1] - tk[1], rgb[2] - tk[2]};
        double e = sq3(res);
        for (int it = 0; it < iters && e > 1.0e-22; ++it) {
            // normal equations (J^T J + mu diag) d = -J^T r
            double A[3][3], gr[3];
            for (int p = 0; p < 3; ++p) {
                gr[p] = -(J[0][p] * res[0] + J[1][p] * res[1] + J[2][p] * res[2]);
                for (int q = 0; q < 3; ++q) {
                    A[p][q] = J[0][p] * J[0][q] + J[1][p] * J[1][q] + J[2][p] * J[2][q];
                }
            }
            bool improved = false;
            for (int tries = 0; tries < 24 && !improved; ++tries) {
                double Ad[3][3];
                for (int p = 0; p < 3; ++p) {
                    for (int q = 0; q < 3; ++q) {
                        Ad[p][q] = A[p][q];
                    }
                    Ad[p][p] = A[p][p] * (1.0 + mu) + 1.0e-30;
                }
                double d[3];
                if (solve3(Ad, gr, d)) {
                    const double cn[3] = {c[0] + d[0], c[1] + d[1], c[2] + d[2]};
                    double rn[3], Jn[3][3];
                    upliftRgb(resp, cn, rn, Jn, true);
                    const double resn[3] = {rn[0] - tk[0], rn[1] - tk[1], rn[2] - tk[2]};
                    const double en = sq3(resn);
                    if (en < e) {
                        for (int k = 0; k < 3; ++k) {
                            c[k] = cn[k];
                            res[k] = resn[k];
                            for (int q = 0; q < 3; ++q) {
                                J[k][q] = Jn[k][q];
                            }
                        }
                        e = en;
                        mu = fmax(mu * 0.25, 1.0e-12);
                        improved = true;
                    }
                }
                if (!improved) {
                    mu *= 8.0;
                }
            }
            if (!improved) {
                break;
            }
        }
    }
    // coefficients in nanometres: t = (lambda - a) / s
    const double s = static_cast<double>(kLambdaRange), a = static_cast<double>(kLambdaMin);
    out.c0 = static_cast<float>(c[0] / (s * s));
    out.c1 = static_cast<float>(c[1] / s - 2.0 * a * c[0] / (s * s));
    out.c2 = static_cast<float>(c[0] * a * a / (s * s) - c[1] * a / s + c[2]);
    out.scale = static_cast<float>(scale);
    return out;
}

#if defined(__CUDACC__)
// --- device: per-path evaluation ------------------------------------------------

// s(lambda) in the reference's operation order (Rgb2Spec.h:58-66), times scale.
__device__ __forceinline__ float evalCoef(float4 c, float lambda)
{
    const float x = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(c.x, lambda), lambda), __fmul_rn(c.y, lambda)), c.z);
    const float y = __fdiv_rn(1.0f, __fsqrt_rn(__fadd_rn(__fmul_rn(x, x), 1.0f)));
    return __fmul_rn(__fadd_rn(__fmul_rn(__fmul_rn(0.5f, x), y), 0.5f), c.w);
}

// Hero draw of a path from its seed: lowbias32 (C. Wellons, "Prospecting for
// Hash Functions", 2018) of the seed, top 24 bits.  It draws nothing from the
// path's random-number stream, so a path takes the same decisions in RGB and
// spectral mode.
__host__ __device__ inline float heroU(uint32_t seed)
{
    uint32_t x = seed ^ 0x9E3779B9u;
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return static_cast<float>(x >> 8) * (1.0f / 16777216.0f);
}

// Wavelength k of NW: 380 + 400 frac(u + k / NW) (k / NW is exact for NW = 4, 8).
__device__ __forceinline__ float heroLambda(float u, int k, int nw)
{
    float t = __fadd_rn(u, static_cast<float>(k) / static_cast<float>(nw));
    if (t >= 1.0f) {
        t = __fsub_rn(t, 1.0f);
    }
    return __fadd_rn(kLambdaMin, __fmul_rn(kLambdaRange, t));
}

// Linear interpolation of the response table at lambda.
__device__ __forceinline__ float3 responseAt(const float4* tab, float lambda)
{
    const float x = __fsub_rn(lambda, kLambdaMin);
    int i = static_cast<int>(x);
    i = i < 0 ? 0 : (i > kRespCount - 2 ? kRespCount - 2 : i);
    const float w = __fsub_rn(x, static_cast<float>(i));
    const float4 a = __ldg(tab + i);
    const float4 b = __ldg(tab + i + 1);
    const float v = __fsub_rn(1.0f, w);
    return f3(__fadd_rn(__fmul_rn(a.x, v), __fmul_rn(b.x, w)), __fadd_rn(__fmul_rn(a.y, v), __fmul_rn(b.y, w)),
        __fadd_rn(__fmul_rn(a.z, v), __fmul_rn(b.z, w)));
}

// Environment-map texels to radiance coefficients (one thread per texel).
void launchUpliftTexels(const float* rgb, size_t count, const float* resp, float4* out, cudaStream_t s);
#endif

} // namespace spectral
} // namespace pt

#undef PT_HD
