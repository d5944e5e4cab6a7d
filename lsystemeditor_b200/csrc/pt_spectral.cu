// Spectral tables (host) and the environment-map uplift kernel.
#include "pt_spectral.cuh"

namespace pt {
namespace spectral {

namespace {

// CIE 1931 2-degree standard observer (x-bar, y-bar, z-bar) and CIE standard
// illuminant D65 (relative, 100 at 560 nm), 380 .. 780 nm every 10 nm
// (CIE 015:2018 tables).
constexpr int kCieCount = 41;
const double kCie[kCieCount][4] = {
    {0.001368, 0.000039, 0.006450, 49.9755},  {0.004243, 0.000120, 0.020050, 54.6482},
    {0.014310, 0.000396, 0.067850, 82.7549},  {0.043510, 0.001210, 0.207400, 91.4860},
    {0.134380, 0.004000, 0.645600, 93.4318},  {0.283900, 0.011600, 1.385600, 86.6823},
    {0.348280, 0.023000, 1.747060, 104.8650}, {0.336200, 0.038000, 1.772110, 117.0080},
    {0.290800, 0.060000, 1.669200, 117.8120}, {0.195360, 0.090980, 1.287640, 114.8610},
    {0.095640, 0.139020, 0.812950, 115.9230}, {0.032010, 0.208020, 0.465180, 108.8110},
    {0.004900, 0.323000, 0.272000, 109.3540}, {0.009300, 0.503000, 0.158200, 107.8020},
    {0.063270, 0.710000, 0.078250, 104.7900}, {0.165500, 0.862000, 0.042160, 107.6890},
    {0.290400, 0.954000, 0.020300, 104.4050}, {0.433450, 0.994950, 0.008750, 104.0460},
    {0.594500, 0.995000, 0.003900, 100.0000}, {0.762100, 0.952000, 0.002100, 96.3342},
    {0.916300, 0.870000, 0.001650, 95.7880},  {1.026300, 0.757000, 0.001100, 88.6856},
    {1.062200, 0.631000, 0.000800, 90.0062},  {1.002600, 0.503000, 0.000340, 89.5991},
    {0.854450, 0.381000, 0.000190, 87.6987},  {0.642400, 0.265000, 0.000050, 83.2886},
    {0.447900, 0.175000, 0.000020, 83.6992},  {0.283500, 0.107000, 0.000000, 80.0268},
    {0.164900, 0.061000, 0.000000, 80.2146},  {0.087400, 0.032000, 0.000000, 82.2778},
    {0.046770, 0.017000, 0.000000, 78.2842},  {0.022700, 0.008210, 0.000000, 69.7213},
    {0.011359, 0.004102, 0.000000, 71.6091},  {0.005790, 0.002091, 0.000000, 74.3490},
    {0.002899, 0.001047, 0.000000, 61.6040},  {0.001440, 0.000520, 0.000000, 69.8856},
    {0.000690, 0.000249, 0.000000, 75.0870},  {0.000332, 0.000120, 0.000000, 63.5927},
    {0.000166, 0.000060, 0.000000, 46.4182},  {0.000083, 0.000030, 0.000000, 66.8054},
    {0.000042, 0.000015, 0.000000, 63.3828},
};

// XYZ -> linear sRGB: the inverse of the matrix whose columns are the sRGB
// primaries' XYZ (chromaticities R 0.64/0.33, G 0.30/0.60, B 0.15/0.06)
// scaled so that RGB (1, 1, 1) is the D65 white (0.3127, 0.3290).
void xyzToSrgb(double M[3][3])
{
    const double xy[3][2] = {{0.64, 0.33}, {0.30, 0.60}, {0.15, 0.06}};
    double P[3][3];
    for (int k = 0; k < 3; ++k) {
        P[0][k] = xy[k][0] / xy[k][1];
        P[1][k] = 1.0;
        P[2][k] = (1.0 - xy[k][0] - xy[k][1]) / xy[k][1];
    }
    const double W[3] = {0.3127 / 0.3290, 1.0, (1.0 - 0.3127 - 0.3290) / 0.3290};
    double S[3];
    solve3(P, W, S);
    double RX[3][3];
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k) {
            RX[r][k] = P[r][k] * S[k];
        }
    }
    // inverse column by column
    for (int col = 0; col < 3; ++col) {
        const double e[3] = {col == 0 ? 1.0 : 0.0, col == 1 ? 1.0 : 0.0, col == 2 ? 1.0 : 0.0};
        double x[3];
        solve3(RX, e, x);
        for (int r = 0; r < 3; ++r) {
            M[r][col] = x[r];
        }
    }
}

} // namespace

void buildResponseTable(float* out)
{
    double M[3][3];
    xyzToSrgb(M);
    double resp[kRespCount][3];
    double norm[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < kRespCount; ++i) {
        // linear interpolation of the 10 nm tables at 380 + i nm
        const int j = i / 10 < kCieCount - 1 ? i / 10 : kCieCount - 2;
        const double w = (static_cast<double>(i) - 10.0 * j) / 10.0;
        double v[4];
        for (int k = 0; k < 4; ++k) {
            v[k] = kCie[j][k] * (1.0 - w) + kCie[j + 1][k] * w;
        }
        const double X = v[0] * v[3], Y = v[1] * v[3], Z = v[2] * v[3];
        const double wt = (i == 0 || i == kRespCount - 1) ? 0.5 : 1.0;
        for (int c = 0; c < 3; ++c) {
            resp[i][c] = M[c][0] * X + M[c][1] * Y + M[c][2] * Z;
            norm[c] += wt * resp[i][c];
        }
    }
    for (int i = 0; i < kRespCount; ++i) {
        for (int c = 0; c < 3; ++c) {
            out[4 * i + c] = static_cast<float>(resp[i][c] / norm[c]);
        }
        out[4 * i + 3] = 0.0f;
    }
}

void spectralSourceTables(float* cie, float* m)
{
    if (cie != nullptr) {
        for (int i = 0; i < kCieCount; ++i) {
            for (int k = 0; k < 4; ++k) {
                cie[4 * i + k] = static_cast<float>(kCie[i][k]);
            }
        }
    }
    if (m != nullptr) {
        double M[3][3];
        xyzToSrgb(M);
        for (int r = 0; r < 3; ++r) {
            for (int k = 0; k < 3; ++k) {
                m[3 * r + k] = static_cast<float>(M[r][k]);
            }
        }
    }
}

namespace {

__global__ void k_uplift_texels(const float* rgb, size_t count, const float* resp, float4* out)
{
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const Coef c = upliftSolve(resp, rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2], true);
        out[i] = make_float4(c.c0, c.c1, c.c2, c.scale);
    }
}

} // namespace

void launchUpliftTexels(const float* rgb, size_t count, const float* resp, float4* out, cudaStream_t s)
{
    if (count == 0) {
        return;
    }
    size_t grid = (count + 127) / 128;
    if (grid > 148 * 64) {
        grid = 148 * 64;
    }
    k_uplift_texels<<<static_cast<unsigned>(grid), 128, 0, s>>>(rgb, count, resp, out);
}

} // namespace spectral
} // namespace pt
