// noalloc.cu -- an allocation-free variant of the stand-alone CSR solve.
//
// fp_solve_csr_upper_noalloc solves the same system as fp_solve_csr_upper (an
// SPD matrix given by its upper-triangle CSR, Jacobi-preconditioned CG with
// FP64 vectors), with two differences: the matrix, right-hand side and
// solution are device buffers owned by the caller, and every work vector lives
// in g_csr_scratch, one file-scope device array of fixed size.  The call makes
// no cudaMalloc, no cudaFree and no call into an allocating library.
//
// It is meant for callers that must not allocate device memory while they
// run: a host application whose own pool allocator owns the GPU memory (a
// stray cudaMalloc there can fail once the pool has reserved the device, and
// it synchronises the whole device), and time-bounded loops that cannot afford
// the unbounded latency of cudaMalloc/cudaFree between steps.
//
// Rules that follow from the fixed scratch:
//   * it holds systems of at most FP_NOALLOC_MAX_N unknowns (5 double vectors
//     of that length, 10 MiB); larger systems are rejected with FP_ERR_ARG
//     before any GPU work;
//   * every call on a device uses the same array, so the calls on one device
//     take turns: each holds that device's host mutex from its first launch
//     until its stream has drained (the call is synchronous; on an error path
//     the stream is synchronised before the mutex is released), and calls
//     from several host threads, on any streams, are serialised in-process
//     (separate processes have separate contexts, each with its own array);
//   * each call clears the scratch it relies on: the argument-check flag and
//     the product vector before every SpMV; x starts at zero;
//   * the first call on each device, with that device current, looks up the
//     array's device address with cudaGetSymbolAddress (the host-side symbol
//     is not a device address) and caches it; make that first call before any
//     stream capture begins on that device.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/fluidprjct.h"

namespace {

constexpr int kMaxN = FP_NOALLOC_MAX_N;
constexpr int kDotBlocks = 64;
constexpr int kMaxDevices = 64;
// Layout in doubles: diag, r, d, q, z (kMaxN each), kDotBlocks dot partials,
// one dot result, one argument-check flag.
constexpr size_t kScratchDoubles = size_t(5) * kMaxN + kDotBlocks + 2;

static __device__ __align__(256) double g_csr_scratch[kScratchDoubles];

std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {nullptr};  // device address of g_csr_scratch, per device ordinal
std::mutex g_call_mutex[kMaxDevices];            // held by the one call that owns a device's scratch

int current_device(int* dev) {
    return cudaGetDevice(dev) == cudaSuccess && *dev >= 0 && *dev < kMaxDevices ? FP_OK : FP_ERR_CUDA;
}

int scratch_for_device(int dev, double** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_csr_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "fp_solve_csr_upper_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                         cudaGetErrorString(e));
            return FP_ERR_CUDA;
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return FP_OK;
}

// The checks fp_solve_csr_upper makes on the host, made on the device: row
// offsets start at 0 and never decrease (first kernel), column indices lie in
// [0, n) (second kernel, run only after the first passed, so its loop bounds
// are trusted).  Any failure sets *bad to 1.
__global__ void na_check_offsets(int n, const int* __restrict__ off, double* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if ((i == 0 && off[0] != 0) || off[i + 1] < off[i]) *bad = 1.0;
}
__global__ void na_check_cols(int n, const int* __restrict__ off, const int* __restrict__ cols,
                              double* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int e = off[i]; e < off[i + 1]; ++e)
        if (cols[e] < 0 || cols[e] >= n) *bad = 1.0;
}
__global__ void na_diag(int n, const int* __restrict__ off, const int* __restrict__ cols,
                        const double* __restrict__ vals, double* __restrict__ dg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 1.0;
    for (int e = off[i]; e < off[i + 1]; ++e) if (cols[e] == i) d = vals[e];
    dg[i] = d;
}
// y = U x + U^T x - diag(U) x for the stored upper triangle U; y is zero on entry.
__global__ void na_spmv(int n, const int* __restrict__ off, const int* __restrict__ cols,
                        const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int e = off[i]; e < off[i + 1]; ++e) {
        const int c = cols[e];
        s += vals[e] * x[c];
        if (c != i) atomicAdd(&y[c], vals[e] * x[i]);
    }
    atomicAdd(&y[i], s);
}
// Dot product in a fixed order: a grid-stride sum per thread, a shared-memory
// tree per block, then one thread adds the block partials in block order.
__global__ void __launch_bounds__(128) na_dot_partials(int n, const double* __restrict__ a,
                                                       const double* __restrict__ b, double* __restrict__ part) {
    __shared__ double sh[128];
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = 64; w > 0; w >>= 1) {
        if (int(threadIdx.x) < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void na_dot_sum(const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[b];
    *out = s;
}
__global__ void na_init(int n, const double* __restrict__ b, const double* __restrict__ dg, double* __restrict__ x,
                        double* __restrict__ r, double* __restrict__ z, double* __restrict__ d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = 0.0;
    r[i] = b[i];
    z[i] = b[i] / dg[i];
    d[i] = z[i];
}
__global__ void na_update(int n, double alpha, const double* __restrict__ d, const double* __restrict__ q,
                          double* __restrict__ x, double* __restrict__ r, const double* __restrict__ dg,
                          double* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] += alpha * d[i];
    r[i] -= alpha * q[i];
    z[i] = r[i] / dg[i];
}
__global__ void na_direction(int n, const double* __restrict__ z, double beta, double* __restrict__ d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = z[i] + beta * d[i];
}

// The solve proper, run by one call at a time per device on scratch base.
int solve_on_scratch(double* base, int n, const int* d_offsets, const int* d_cols, const double* d_vals,
                     const double* d_b, double* d_x, double tol, int max_iters, int* iters, double* relres,
                     cudaStream_t st) {
    double* dg = base;
    double* r = base + size_t(kMaxN);
    double* d = base + 2 * size_t(kMaxN);
    double* q = base + 3 * size_t(kMaxN);
    double* z = base + 4 * size_t(kMaxN);
    double* part = base + 5 * size_t(kMaxN);
    double* res = part + kDotBlocks;
    double* bad = res + 1;
    const int blk = 128, grd = (n + blk - 1) / blk;

    auto read = [&](const double* src, double& out) {
        return cudaMemcpyAsync(&out, src, sizeof(double), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
               cudaStreamSynchronize(st) == cudaSuccess;
    };
    auto dot = [&](const double* a, const double* b, double& out) {
        na_dot_partials<<<kDotBlocks, 128, 0, st>>>(n, a, b, part);
        na_dot_sum<<<1, 32, 0, st>>>(part, kDotBlocks, res);
        return read(res, out);
    };

    double flag = 0.0;
    if (cudaMemsetAsync(bad, 0, sizeof(double), st) != cudaSuccess) return FP_ERR_CUDA;
    na_check_offsets<<<grd, blk, 0, st>>>(n, d_offsets, bad);
    if (!read(bad, flag)) return FP_ERR_CUDA;
    if (flag == 0.0) {
        na_check_cols<<<grd, blk, 0, st>>>(n, d_offsets, d_cols, bad);
        if (!read(bad, flag)) return FP_ERR_CUDA;
    }
    if (flag != 0.0) {
        std::fprintf(stderr, "fp_solve_csr_upper_noalloc: malformed CSR (offsets or column indices)\n");
        return FP_ERR_ARG;
    }

    na_diag<<<grd, blk, 0, st>>>(n, d_offsets, d_cols, d_vals, dg);
    na_init<<<grd, blk, 0, st>>>(n, d_b, dg, d_x, r, z, d);
    double bb = 0.0, rz = 0.0;
    if (!dot(r, r, bb) || !dot(r, z, rz)) return FP_ERR_CUDA;
    double rr = bb;
    int it = 0;
    while (bb > 0.0 && rr > tol * tol * bb && it < max_iters) {
        if (cudaMemsetAsync(q, 0, sizeof(double) * size_t(n), st) != cudaSuccess) return FP_ERR_CUDA;
        na_spmv<<<grd, blk, 0, st>>>(n, d_offsets, d_cols, d_vals, d, q);
        double dq = 0.0;
        if (!dot(d, q, dq)) return FP_ERR_CUDA;
        if (!(dq > 0.0)) break;
        const double alpha = rz / dq;
        na_update<<<grd, blk, 0, st>>>(n, alpha, d, q, d_x, r, dg, z);
        double rz2 = 0.0;
        if (!dot(r, z, rz2) || !dot(r, r, rr)) return FP_ERR_CUDA;
        na_direction<<<grd, blk, 0, st>>>(n, z, rz2 / rz, d);
        rz = rz2;
        ++it;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return FP_ERR_CUDA;
    if (iters) *iters = it;
    if (relres) *relres = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
    return FP_OK;
}

}  // namespace

extern "C" int fp_solve_csr_upper_noalloc(int n, const int* d_offsets, const int* d_cols, const double* d_vals,
                                          const double* d_b, double* d_x, double tol, int max_iters, int* iters,
                                          double* relres, void* stream) {
    if (n <= 0 || !d_offsets || !d_cols || !d_vals || !d_b || !d_x) return FP_ERR_ARG;
    if (n > kMaxN) {
        std::fprintf(stderr, "fp_solve_csr_upper_noalloc: n = %d exceeds the scratch limit of %d unknowns\n", n,
                     kMaxN);
        return FP_ERR_ARG;
    }
    int dev = 0;
    double* base = nullptr;
    if (const int rc = current_device(&dev)) return rc;
    if (const int rc = scratch_for_device(dev, &base)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(g_call_mutex[dev]);
    // A launch error of this call is one that appears during it: an error the
    // calling thread left pending before the call is neither reported as this
    // call's failure nor cleared.
    const bool clean_before = cudaPeekAtLastError() == cudaSuccess;
    int rc = solve_on_scratch(base, n, d_offsets, d_cols, d_vals, d_b, d_x, tol, max_iters, iters, relres, st);
    // An early error return may leave launches queued on st: let them finish
    // before the next call takes the scratch.
    if (rc != FP_OK) cudaStreamSynchronize(st);
    if (clean_before && cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();  // this call's launch error: report it and clear it
        if (rc == FP_OK) rc = FP_ERR_CUDA;
    }
    return rc;
}
