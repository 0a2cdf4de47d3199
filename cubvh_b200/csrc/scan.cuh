// Exclusive prefix sum of a uint32 array in place (n + 1 entries; entry n
// receives the total) in three launches: per-chunk sums, a single-block scan
// of the chunk sums, per-chunk scans.  Scratch: (ceil(n / kScanChunk) + 1)
// uint32 for the chunk sums.
#pragma once
#include "launches.h"
#include <cstdint>
#include <cuda_runtime.h>

namespace cubvh {
namespace scan {
namespace {  // internal linkage: every translation unit gets its own copy

constexpr int kScanChunk = 2048;  // entries per block (1024 threads x 2)

inline int64_t num_chunks(int64_t n) { return (n + kScanChunk - 1) / kScanChunk; }

__global__ void k_chunk_sums(const uint32_t* __restrict__ cnt, uint32_t* __restrict__ bsum, int64_t n) {
    __shared__ uint32_t sh[32];
    const int64_t base = (int64_t)blockIdx.x * kScanChunk;
    uint32_t s = 0;
    for (int i = threadIdx.x; i < kScanChunk; i += blockDim.x)
        if (base + i < n) s += cnt[base + i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
        if (threadIdx.x == 0) bsum[blockIdx.x] = v;
    }
}

// single block of 1024 threads; each thread scans a contiguous slice
__global__ void k_top(uint32_t* __restrict__ bsum, int64_t nblk) {
    __shared__ uint32_t sh[1024];
    const int64_t per = (nblk + 1023) / 1024;
    const int64_t b0 = threadIdx.x * per, b1 = min(b0 + per, nblk);
    uint32_t s = 0;
    for (int64_t i = b0; i < b1; ++i) s += bsum[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const uint32_t v = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = threadIdx.x ? sh[threadIdx.x - 1] : 0;
    for (int64_t i = b0; i < b1; ++i) { const uint32_t v = bsum[i]; bsum[i] = run; run += v; }
    if (threadIdx.x == 1023) bsum[nblk] = sh[1023];
}

__global__ void k_apply(uint32_t* __restrict__ cnt, const uint32_t* __restrict__ bsum, int64_t n) {
    __shared__ uint32_t sh[1024];
    const int64_t base = (int64_t)blockIdx.x * kScanChunk;
    const int64_t i0 = base + 2 * threadIdx.x;
    const uint32_t a = i0 < n ? cnt[i0] : 0, b = i0 + 1 < n ? cnt[i0 + 1] : 0;
    sh[threadIdx.x] = a + b;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const uint32_t v = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += v;
        __syncthreads();
    }
    const uint32_t excl = (threadIdx.x ? sh[threadIdx.x - 1] : 0) + bsum[blockIdx.x];
    if (i0 < n) cnt[i0] = excl;
    if (i0 + 1 < n) cnt[i0 + 1] = excl + a;
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) cnt[n] = bsum[gridDim.x];
}

// cnt: n + 1 entries; bsum: num_chunks(n) + 1 entries.  n >= 1.
inline void exclusive(uint32_t* cnt, uint32_t* bsum, int64_t n, cudaStream_t s) {
    const int64_t nblk = num_chunks(n);
    k_chunk_sums<<<(unsigned)nblk, 256, 0, s>>>(cnt, bsum, n); count_launch();
    k_top<<<1, 1024, 0, s>>>(bsum, nblk); count_launch();
    k_apply<<<(unsigned)nblk, 1024, 0, s>>>(cnt, bsum, n); count_launch();
}

}  // namespace
}  // namespace scan
}  // namespace cubvh
