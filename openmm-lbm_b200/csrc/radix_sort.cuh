// Stable LSD radix sort of 32-bit keys with 32-bit values on the device, 8 bits per pass: a per-block histogram
// of the digit, one exclusive scan over (digit, block), and a stable scatter in which each block ranks its items
// by warp (match_any) and by the counts of the earlier warps.  Used to order particles by node or cell.
#pragma once

#include <cuda_runtime.h>

namespace lbm {
namespace {

const int kSortItems = 1024;     // items per block (one per thread)

__global__ void __launch_bounds__(kSortItems) radixHistogram(const unsigned* keys, int n, int shift, unsigned* hist, int numBlocks) {
    __shared__ unsigned counts[256];
    for (int b = threadIdx.x; b < 256; b += blockDim.x)
        counts[b] = 0;
    __syncthreads();
    int i = blockIdx.x*kSortItems + threadIdx.x;
    if (i < n)
        atomicAdd(&counts[(keys[i] >> shift) & 255u], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x)
        hist[b*numBlocks + blockIdx.x] = counts[b];
}

// Exclusive scan of hist (256 x numBlocks, digit-major) in one block.
__global__ void __launch_bounds__(1024) radixScan(unsigned* hist, int count) {
    __shared__ unsigned partial[1024];
    int per = (count + blockDim.x - 1)/blockDim.x;
    int begin = threadIdx.x*per, end = min(count, begin + per);
    unsigned sum = 0;
    for (int i = begin; i < end; i++)
        sum += hist[i];
    // Exclusive scan of the per-thread sums: inclusive scans within the warps (shuffles), then over the warp totals.
    int lane = threadIdx.x%32, warp = threadIdx.x/32;
    unsigned inclusive = sum;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned v = __shfl_up_sync(0xffffffffu, inclusive, o);
        if (lane >= o)
            inclusive += v;
    }
    if (lane == 31)
        partial[warp] = inclusive;
    __syncthreads();
    if (warp == 0) {
        unsigned total = lane < (int) blockDim.x/32 ? partial[lane] : 0u, scan = total;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned v = __shfl_up_sync(0xffffffffu, scan, o);
            if (lane >= o)
                scan += v;
        }
        partial[32 + lane] = scan - total;       // exclusive prefix of the warp totals
    }
    __syncthreads();
    unsigned run = partial[32 + warp] + inclusive - sum;
    for (int i = begin; i < end; i++) {
        unsigned v = hist[i];
        hist[i] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(kSortItems) radixScatter(const unsigned* keys, const int* values, int n, int shift,
                                                           const unsigned* hist, int numBlocks, unsigned* keysOut, int* valuesOut) {
    __shared__ unsigned warpCount[256][kSortItems/32];
    int lane = threadIdx.x%32, warp = threadIdx.x/32;
    for (int k = threadIdx.x; k < 256*(kSortItems/32); k += blockDim.x)
        warpCount[k/(kSortItems/32)][k%(kSortItems/32)] = 0;
    __syncthreads();
    int i = blockIdx.x*kSortItems + threadIdx.x;
    bool valid = i < n;
    unsigned key = valid ? keys[i] : 0u;
    unsigned digit = valid ? ((key >> shift) & 255u) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, digit);
    int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0)
        warpCount[digit][warp] = __popc(peers);
    __syncthreads();
    // Exclusive prefix over the warps of each digit (warps are in item order, so the sort is stable).
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
        unsigned run = 0;
        for (int w = 0; w < kSortItems/32; w++) {
            unsigned v = warpCount[d][w];
            warpCount[d][w] = run;
            run += v;
        }
    }
    __syncthreads();
    if (valid) {
        unsigned dest = hist[digit*numBlocks + blockIdx.x] + warpCount[digit][warp] + rank;
        keysOut[dest] = key;
        valuesOut[dest] = values[i];
    }
}

// Sorts keys[0]/values[0] (n items, keys < 2^bits) with keys[1]/values[1] as the other buffers and hist of
// 256*ceil(n/1024) words; returns the index of the buffers that hold the result.  Launches 3 kernels per 8 bits.
inline int radixSortByKey(unsigned* keys[2], int* values[2], unsigned* hist, int n, int bits, cudaStream_t stream) {
    int blocks = (n + kSortItems - 1)/kSortItems;
    int cur = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        radixHistogram<<<blocks, kSortItems, 0, stream>>>(keys[cur], n, shift, hist, blocks);
        radixScan<<<1, 1024, 0, stream>>>(hist, 256*blocks);
        radixScatter<<<blocks, kSortItems, 0, stream>>>(keys[cur], values[cur], n, shift, hist, blocks, keys[1-cur], values[1-cur]);
        cur = 1 - cur;
    }
    return cur;
}

} // namespace
} // namespace lbm
