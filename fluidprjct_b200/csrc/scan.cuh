// scan.cuh -- block-level exclusive scan and a single-block scan of tile sums,
// the building blocks of the three-pass device scans (tile sums -> scan of
// tile sums -> tile scan) used by the cell sort and the fluid compaction.
#pragma once

#include <cuda_runtime.h>

namespace fp {

// Exclusive scan of one int per thread over a block of BLOCK threads.
// Returns the thread's exclusive prefix; *total receives the block sum.
template <int BLOCK>
__device__ __forceinline__ int block_exclusive_scan(int v, int& total) {
    static_assert(BLOCK % 32 == 0 && BLOCK <= 1024, "block size");
    __shared__ int warp_sums[BLOCK / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < BLOCK / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < BLOCK / 32) warp_sums[lane] = s;  // inclusive warp prefix
    }
    __syncthreads();
    total = warp_sums[BLOCK / 32 - 1];
    int before = wid > 0 ? warp_sums[wid - 1] : 0;
    __syncthreads();  // warp_sums may be reused by the caller's next scan
    return before + x - v;
}

// In-place exclusive scan of n ints by one block of 1024 threads; the grand
// total is written to *total (if non-null).
__global__ void k_scan_single_block(int* data, int n, int* total);

}  // namespace fp
