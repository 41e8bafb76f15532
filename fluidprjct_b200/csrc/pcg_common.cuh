// pcg_common.cuh -- device helpers shared by the persistent PCG kernels:
// a bounded grid barrier for cooperative launches and deterministic FP64
// block / grid reductions.
#pragma once

#include "kernels.hpp"

namespace fp {
namespace {

// ---------------------------------------------------------------- grid barrier
// Grid barrier for a cooperative launch on one 32-bit word: every block adds
// 1 except block 0, which adds 2^31 - (nblocks - 1), so the word's top bit
// flips exactly when the last block arrives and no reset is needed between
// barriers.  The block whose arrival flips the bit knows it from the
// atomic's result and does not poll.  The wait is bounded: after bar->limit
// polls (kDefaultWaitPolls = 2^27 unless the solver's owner set another
// limit) the block records DEV_TIMEOUT and leaves; callers check the status
// after every barrier and return, so no block waits forever.  The arrival is
// an acquire-release atomic and the poll an acquire load (the pattern of a
// release-acquire grid barrier), so plain loads after it see every write made
// before it by any block.
__device__ __forceinline__ bool grid_barrier(GridBar* bar, unsigned nblocks, int* status) {
    __shared__ int s_ok;
    __syncthreads();
    // A one-block launch (a small grid) has no other block to wait for: the
    // block barrier alone orders its threads' global writes and reads.
    if (nblocks == 1u) return true;
    if (threadIdx.x == 0) {
        // The status and limit loads are issued before the arrival so that
        // their latency overlaps the atomic; a timeout recorded by another
        // block is seen at this or the next barrier, and every wait below is
        // bounded.
        const int st0 = *(volatile int*)status;
        const unsigned limit = *(volatile unsigned*)&bar->limit;  // at least 1
        const unsigned inc = blockIdx.x == 0 ? 0x80000000u - (nblocks - 1u) : 1u;
        // arrival with release semantics: after the block barrier above it
        // publishes every write this block made before the grid barrier
        unsigned old;
        // acquire as well: the last block to arrive reads the value the
        // other arrivals' release RMWs wrote, so it has their writes and need
        // not poll.  That takes one L2 round trip off the barrier's critical
        // path: 0.974 -> 0.964 ms per warm-started MG solve at 128^3.
        asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;\n"
                     : "=r"(old)
                     : "l"(&bar->count), "r"(inc)
                     : "memory");
        const bool last = ((old ^ (old + inc)) & 0x80000000u) != 0u;
        bool ok = st0 == DEV_OK;
        unsigned polls = 0;
        for (; !last;) {
            // acquire load: writes published by the other blocks' arrivals are
            // visible to this block once the top bit has flipped
            unsigned cur;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(cur) : "l"(&bar->count) : "memory");
            if (((old ^ cur) & 0x80000000u) != 0u) break;
            if (++polls >= limit) {
                atomicExch(status, DEV_TIMEOUT);
                ok = false;
                break;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Block sum of two doubles (fixed tree, deterministic); result valid in thread 0.
__device__ __forceinline__ double2 block_sum2(double a, double b) {
    __shared__ double2 sh[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = make_double2(a, b);
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (wid == 0) {
        r = lane < int(blockDim.x >> 5) ? sh[lane] : make_double2(0.0, 0.0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r.x += __shfl_down_sync(0xffffffffu, r.x, o);
            r.y += __shfl_down_sync(0xffffffffu, r.y, o);
        }
    }
    __syncthreads();
    return r;
}

// Sum of per-block partials part[0..nb) (pairs), identical in every block.
__device__ __forceinline__ double2 grid_sum2(const double2* part, int nb) {
    __shared__ double2 res;
    if (threadIdx.x < 32) {
        double2 s = make_double2(0.0, 0.0);
        for (int t = threadIdx.x; t < nb; t += 32) {
            // Written by other CTAs in this launch: read through L2.
            double2 v = __ldcg(part + t);
            s.x += v.x;
            s.y += v.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s.x += __shfl_down_sync(0xffffffffu, s.x, o);
            s.y += __shfl_down_sync(0xffffffffu, s.y, o);
        }
        if (threadIdx.x == 0) res = s;
    }
    __syncthreads();
    double2 r = res;
    __syncthreads();
    return r;
}

// Sum of three per-block partial arrays part[0..nb), part[nb..2nb),
// part[2nb..3nb), returned to every thread of every block.  All threads load
// (one L2 round trip when nb <= blockDim) and reduce with a fixed tree, so
// every block obtains the same bits.
__device__ __forceinline__ double3 grid_sum3(const double* part, int nb) {
    __shared__ double3 red3[32];
    __shared__ double3 res3;
    double a = 0.0, b = 0.0, c = 0.0;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        a += __ldcg(part + t);
        b += __ldcg(part + nb + t);
        c += __ldcg(part + 2 * nb + t);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red3[wid] = make_double3(a, b, c);
    __syncthreads();
    if (wid == 0) {
        double3 r = lane < int(blockDim.x >> 5) ? red3[lane] : make_double3(0.0, 0.0, 0.0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r.x += __shfl_down_sync(0xffffffffu, r.x, o);
            r.y += __shfl_down_sync(0xffffffffu, r.y, o);
            r.z += __shfl_down_sync(0xffffffffu, r.z, o);
        }
        if (lane == 0) res3 = r;
    }
    __syncthreads();
    double3 r = res3;
    __syncthreads();
    return r;
}

// Block sum of three doubles; result valid in thread 0.
__device__ __forceinline__ double3 block_sum3(double a, double b, double c) {
    __shared__ double3 sh3[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh3[wid] = make_double3(a, b, c);
    __syncthreads();
    double3 r = make_double3(0.0, 0.0, 0.0);
    if (wid == 0) {
        r = lane < int(blockDim.x >> 5) ? sh3[lane] : make_double3(0.0, 0.0, 0.0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r.x += __shfl_down_sync(0xffffffffu, r.x, o);
            r.y += __shfl_down_sync(0xffffffffu, r.y, o);
            r.z += __shfl_down_sync(0xffffffffu, r.z, o);
        }
    }
    __syncthreads();
    return r;
}


}  // namespace
}  // namespace fp
