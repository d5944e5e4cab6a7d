// Order-preserving stream compaction (stable select) and the block scan it
// shares with the radix sort.
//
// A select keeps the entries i < n for which keep(i) holds and writes value(i)
// for them, in increasing i, to out[0 .. count).  It runs in three launches
// with no atomics and no inter-block waits:
//   1. k_select_count: one block per tile of kSelectTile entries counts the
//      kept entries with one ballot per warp and round;
//   2. k_select_scan: one block turns the tile counts into exclusive tile
//      offsets and writes the total;
//   3. k_select_write: every block re-evaluates its tile, ranks each kept
//      entry by (round, warp, lane) -- which is index order -- and writes it.
// Traffic per entry: the predicate's reads twice, 4 B out per kept entry, 8 B
// per tile of offsets.  This replaces compactActiveListKernel's one atomicAdd
// per surviving pixel (PathTracer.cu:372-411), whose output order is the
// order in which threads win the atomic.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pt {

constexpr int kSelectBlock = 256;
constexpr int kSelectRounds = 8;
constexpr int kSelectTile = kSelectBlock * kSelectRounds; // 2048 entries per block

__host__ __device__ inline int selectTiles(long long n)
{
    return static_cast<int>((n + kSelectTile - 1) / kSelectTile);
}

// Scratch of a select over n entries: one int per tile.
inline size_t selectTempBytes(long long n)
{
    return sizeof(int) * static_cast<size_t>(selectTiles(n) > 0 ? selectTiles(n) : 1);
}

__device__ __forceinline__ unsigned laneMaskLt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread over a block of blockDim.x <= 1024
// threads (a multiple of 32); returns the thread's exclusive prefix, *total
// the block sum.  `warpSums` needs blockDim.x / 32 entries.  Ends with a
// __syncthreads, so the scratch can be reused right away.
template <class T>
__device__ __forceinline__ T blockExclusiveScan(T v, T* warpSums, T* total)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    T x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) {
            x += y;
        }
    }
    if (lane == 31) {
        warpSums[warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        T s = lane < warps ? warpSums[lane] : T(0);
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) {
                s += y;
            }
        }
        if (lane < warps) {
            warpSums[lane] = s; // inclusive over warps
        }
    }
    __syncthreads();
    const T before = warp > 0 ? warpSums[warp - 1] : T(0);
    *total = warpSums[warps - 1];
    __syncthreads();
    return before + x - v;
}

template <class Keep>
__global__ void __launch_bounds__(kSelectBlock) k_select_count(long long n, Keep keep, int* tileCount)
{
    __shared__ int warpCount[kSelectBlock / 32];
    const long long base = static_cast<long long>(blockIdx.x) * kSelectTile;
    int c = 0;
#pragma unroll
    for (int r = 0; r < kSelectRounds; ++r) {
        const long long i = base + r * kSelectBlock + threadIdx.x;
        const bool k = i < n && keep(i);
        c += __popc(__ballot_sync(0xffffffffu, k));
    }
    if ((threadIdx.x & 31) == 0) {
        warpCount[threadIdx.x >> 5] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kSelectBlock / 32; ++w) {
            s += warpCount[w];
        }
        tileCount[blockIdx.x] = s;
    }
}

// One block of 1024 threads: tile counts -> exclusive tile offsets (in place),
// the total to *outCount.
template <class CountT>
__global__ void __launch_bounds__(1024) k_select_scan(int tiles, int* tileOffset, CountT* outCount)
{
    __shared__ int warpSums[32];
    int carry = 0;
    for (int start = 0; start < tiles; start += blockDim.x) {
        const int i = start + threadIdx.x;
        const int v = i < tiles ? tileOffset[i] : 0;
        int total = 0;
        const int ex = blockExclusiveScan(v, warpSums, &total);
        if (i < tiles) {
            tileOffset[i] = carry + ex;
        }
        carry += total;
    }
    if (threadIdx.x == 0) {
        *outCount = static_cast<CountT>(carry);
    }
}

template <class Keep, class Value, class OutT>
__global__ void __launch_bounds__(kSelectBlock) k_select_write(long long n, Keep keep, Value value,
    const int* tileOffset, OutT* out)
{
    __shared__ int prefix[kSelectRounds][kSelectBlock / 32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long base = static_cast<long long>(blockIdx.x) * kSelectTile;
    unsigned masks[kSelectRounds];
#pragma unroll
    for (int r = 0; r < kSelectRounds; ++r) {
        const long long i = base + r * kSelectBlock + threadIdx.x;
        masks[r] = __ballot_sync(0xffffffffu, i < n && keep(i));
        if (lane == 0) {
            prefix[r][warp] = __popc(masks[r]);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // exclusive prefix in index order: round-major, then warp
        int s = tileOffset[blockIdx.x];
        for (int r = 0; r < kSelectRounds; ++r) {
            for (int w = 0; w < kSelectBlock / 32; ++w) {
                const int c = prefix[r][w];
                prefix[r][w] = s;
                s += c;
            }
        }
    }
    __syncthreads();
    const unsigned lt = laneMaskLt();
#pragma unroll
    for (int r = 0; r < kSelectRounds; ++r) {
        if ((masks[r] >> lane) & 1u) {
            const long long i = base + r * kSelectBlock + threadIdx.x;
            out[prefix[r][warp] + __popc(masks[r] & lt)] = value(i);
        }
    }
}

// Stable select of n entries; temp needs selectTempBytes(n).  Writes the kept
// count to *outCount (device memory) and the kept values to out.
template <class Keep, class Value, class OutT, class CountT>
cudaError_t launchSelect(long long n, Keep keep, Value value, OutT* out, CountT* outCount, void* temp,
    size_t tempBytes, cudaStream_t s)
{
    if (tempBytes < selectTempBytes(n)) {
        return cudaErrorInvalidValue;
    }
    const int tiles = selectTiles(n);
    int* tileOffset = static_cast<int*>(temp);
    if (tiles > 0) {
        k_select_count<<<tiles, kSelectBlock, 0, s>>>(n, keep, tileOffset);
    }
    k_select_scan<<<1, 1024, 0, s>>>(tiles, tileOffset, outCount);
    if (tiles > 0) {
        k_select_write<<<tiles, kSelectBlock, 0, s>>>(n, keep, value, tileOffset, out);
    }
    return cudaGetLastError();
}

} // namespace pt
