// LSD radix sort of (key, value) pairs of 32-bit unsigned integers, used for
// the BVH builder's 30-bit Morton keys.  Stable, 8-bit digits, one pass per
// digit of the requested bit range (4 passes for 30 bits), each pass three
// launches with no atomics on global memory and no inter-block waits:
//   k_radix_hist    one block per tile of kRadixTile keys: the tile's digit
//                   histogram (shared-memory counters), stored digit-major;
//   k_radix_rows    one block per digit: exclusive scan of that digit's counts
//                   over the tiles (in place) and the digit's total;
//   k_radix_scatter one block per tile: the digit totals' exclusive scan gives
//                   each digit's global start, the tile's row entry its start
//                   within that digit, and __match_any_sync ranks equal digits
//                   within a warp; warps and rounds are combined in index order
//                   through shared counters, so equal keys keep their order.
// Per pass the keys and values are read twice and written once (16 B per
// pair) plus 1 KB of counters per tile.  Passes ping-pong through the scratch
// pair so the input arrays are left unchanged.
#include "pt_bvh.cuh"
#include "pt_select.cuh"

namespace pt {
namespace {

constexpr int kRadixBits = 8;
constexpr int kRadixDigits = 1 << kRadixBits;
constexpr int kRadixBlock = 256;
constexpr int kRadixRounds = 8;
constexpr int kRadixTile = kRadixBlock * kRadixRounds;

static_assert(kRadixDigits == kRadixBlock, "one thread per digit");

int radixTiles(uint32_t n)
{
    return static_cast<int>((static_cast<uint64_t>(n) + kRadixTile - 1) / kRadixTile);
}

size_t align256(size_t b)
{
    return (b + 255) & ~size_t(255);
}

__global__ void __launch_bounds__(kRadixBlock) k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n, int shift,
    uint32_t* __restrict__ tileHist, int tiles)
{
    __shared__ uint32_t h[kRadixDigits];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kRadixTile;
#pragma unroll
    for (int r = 0; r < kRadixRounds; ++r) {
        const uint64_t i = base + r * kRadixBlock + threadIdx.x;
        if (i < n) {
            atomicAdd(&h[(keys[i] >> shift) & (kRadixDigits - 1)], 1u);
        }
    }
    __syncthreads();
    tileHist[static_cast<size_t>(threadIdx.x) * tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kRadixBlock) k_radix_rows(uint32_t* __restrict__ tileHist, int tiles,
    uint32_t* __restrict__ digitTotal)
{
    __shared__ uint32_t warpSums[kRadixBlock / 32];
    uint32_t* row = tileHist + static_cast<size_t>(blockIdx.x) * tiles;
    uint32_t carry = 0;
    for (int start = 0; start < tiles; start += kRadixBlock) {
        const int i = start + threadIdx.x;
        const uint32_t v = i < tiles ? row[i] : 0u;
        uint32_t total = 0;
        const uint32_t ex = blockExclusiveScan(v, warpSums, &total);
        if (i < tiles) {
            row[i] = carry + ex;
        }
        carry += total;
    }
    if (threadIdx.x == 0) {
        digitTotal[blockIdx.x] = carry;
    }
}

__global__ void __launch_bounds__(kRadixBlock) k_radix_scatter(const uint32_t* __restrict__ kin,
    const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, uint32_t n, int shift,
    const uint32_t* __restrict__ tileHist, const uint32_t* __restrict__ digitTotal, int tiles)
{
    __shared__ uint32_t warpSums[kRadixBlock / 32];
    __shared__ uint32_t digitBase[kRadixDigits];
    __shared__ uint32_t warpCount[kRadixBlock / 32][kRadixDigits];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int t = threadIdx.x; // also the digit whose counters this thread keeps
    uint32_t total = 0;
    const uint32_t start = blockExclusiveScan(digitTotal[t], warpSums, &total);
    digitBase[t] = start + tileHist[static_cast<size_t>(t) * tiles + blockIdx.x];
    uint32_t run = 0; // keys of digit t in earlier rounds of this tile
    const unsigned lt = laneMaskLt();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kRadixTile;
    for (int r = 0; r < kRadixRounds; ++r) {
        const uint64_t i = base + r * kRadixBlock + threadIdx.x;
        const bool valid = i < n;
        const uint32_t key = valid ? kin[i] : 0u;
        const uint32_t val = valid ? vin[i] : 0u;
        const uint32_t d = valid ? (key >> shift) & (kRadixDigits - 1) : uint32_t(kRadixDigits); // sentinel
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & lt);
        for (int j = lane; j < kRadixDigits; j += 32) {
            warpCount[warp][j] = 0;
        }
        __syncwarp();
        if (valid && rank == 0) {
            warpCount[warp][d] = __popc(peers);
        }
        __syncthreads();
        {
            uint32_t acc = run;
#pragma unroll
            for (int w = 0; w < kRadixBlock / 32; ++w) {
                const uint32_t c = warpCount[w][t];
                warpCount[w][t] = acc;
                acc += c;
            }
            run = acc;
        }
        __syncthreads();
        if (valid) {
            const uint32_t pos = digitBase[d] + warpCount[warp][d] + rank;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
    }
}

} // namespace

size_t radixSortTempBytes(uint32_t n)
{
    const size_t tiles = static_cast<size_t>(radixTiles(n) > 0 ? radixTiles(n) : 1);
    const size_t pairs = static_cast<size_t>(n > 0 ? n : 1);
    return align256(sizeof(uint32_t) * kRadixDigits * tiles) + align256(sizeof(uint32_t) * kRadixDigits) +
        2 * align256(sizeof(uint32_t) * pairs);
}

cudaError_t radixSortPairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keysOut, uint32_t* valsOut, uint32_t n,
    int bits, void* temp, size_t tempBytes, cudaStream_t s)
{
    if (n == 0) {
        return cudaSuccess;
    }
    if (temp == nullptr || tempBytes < radixSortTempBytes(n) || bits < 1 || bits > 32) {
        return cudaErrorInvalidValue;
    }
    const int tiles = radixTiles(n);
    unsigned char* p = static_cast<unsigned char*>(temp);
    uint32_t* tileHist = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * kRadixDigits * static_cast<size_t>(tiles));
    uint32_t* digitTotal = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * kRadixDigits);
    uint32_t* ktmp = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * n);
    uint32_t* vtmp = reinterpret_cast<uint32_t*>(p);
    const int passes = (bits + kRadixBits - 1) / kRadixBits;
    // the last pass lands in keysOut: passes alternate between it and the scratch pair
    const uint32_t* kin = keys;
    const uint32_t* vin = vals;
    for (int pass = 0; pass < passes; ++pass) {
        const bool toOut = ((passes - 1 - pass) % 2) == 0;
        uint32_t* ko = toOut ? keysOut : ktmp;
        uint32_t* vo = toOut ? valsOut : vtmp;
        const int shift = pass * kRadixBits;
        k_radix_hist<<<tiles, kRadixBlock, 0, s>>>(kin, n, shift, tileHist, tiles);
        k_radix_rows<<<kRadixDigits, kRadixBlock, 0, s>>>(tileHist, tiles, digitTotal);
        k_radix_scatter<<<tiles, kRadixBlock, 0, s>>>(kin, vin, ko, vo, n, shift, tileHist, digitTotal, tiles);
        kin = ko;
        vin = vo;
    }
    return cudaGetLastError();
}

} // namespace pt

// C ABI over device buffers (declared in include/pt_b200.h).
extern "C" size_t pt_radix_sort_temp_bytes(uint32_t n)
{
    return pt::radixSortTempBytes(n);
}

extern "C" int pt_radix_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out, uint32_t* vals_out,
    uint32_t n, int bits, void* temp, size_t temp_bytes, void* stream)
{
    if (n == 0) {
        return PT_OK;
    }
    if (keys == nullptr || vals == nullptr || keys_out == nullptr || vals_out == nullptr || temp == nullptr ||
        bits < 1 || bits > 32 || temp_bytes < pt::radixSortTempBytes(n) || keys_out == keys || vals_out == vals) {
        return PT_ERR_INVALID_ARGUMENT;
    }
    const cudaError_t e = pt::radixSortPairs(keys, vals, keys_out, vals_out, n, bits, temp, temp_bytes,
        static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PT_OK : PT_ERR_CUDA;
}
