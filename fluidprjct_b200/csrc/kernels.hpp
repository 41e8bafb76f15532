// kernels.hpp -- host launchers of the PIC/FLIP kernels (implemented in *.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace fp {

// Scratch of the persistent PCG kernel: a grid barrier and FP64 partials.
struct GridBar {
    unsigned count;
    unsigned gen;
};

struct PcgOut {
    int iters;
    int status;     // DEV_*
    double rr;      // ||r||^2 of the recurrence at exit
    double bb;      // ||b||^2
    double rz;
};

// Device buffers of the pressure system (compact over FLUID cells, except dd).
struct PressureBufs {
    int* nf;              // [1] number of FLUID cells
    int* fidx;            // [nc] cell index of the n-th FLUID cell
    uint8_t* diag;        // [nc] diagonal of the unit operator (compact)
    float* b;             // [nc] right-hand side (compact)
    float* bin;           // [nc] right-hand side of an inner refinement solve
    float* x;             // [nc] solution (compact)
    float* r;             // [nc] residual (compact)
    float* q;             // [nc] A*d (compact)
    float* dd;            // [nc] search direction (dense, zero off FLUID)
    double* x64;          // [nc] refinement accumulator (compact)
    double* part;         // [3 * max_blocks] per-block partial sums
    GridBar* bar;         // [1]
    PcgOut* out;          // [1]
    int* tile_sums;       // scan scratch
    double* red;          // [2] FP64 reduction results (true residual)
};

// -------- labelling and the particle sort (kernels_sort.cu) --------
// counts[nc] must be zero on entry.  Writes key/rank per particle.
void launch_bin(const float4* pos, int64_t np, Dims g, int* counts, int* key, int* rank, cudaStream_t st);
// Labels from the SOLID map, the body mark and counts; exclusive scan of counts
// into start[nc+1]; start[nc] = np.
void launch_label_scan(const uint8_t* base, const uint8_t* body_mark, const int* counts, uint8_t* labels, int* start,
                       int* tile_sums, Dims g, cudaStream_t st);
void launch_scatter(const float4* pos, const float4* vel, const int* key, const int* rank, const int* start, int64_t np,
                    float4* pos2, float4* vel2, cudaStream_t st);

// -------- P2G with the fused normalise / save / gravity epilogue (kernels_p2g.cu) --------
void launch_p2g(const float4* pos, const float4* vel, const int* start, Dims g, float dt, float3 gravity, float* u,
                float* v, float* w, float* us, float* vs, float* ws, int fused_forces, cudaStream_t st);
void launch_forces(float* u, float* v, float* w, Dims g, float dt, float3 gravity, cudaStream_t st);
void launch_copy(const float* src, float* dst, int64_t n, cudaStream_t st);

// -------- pressure (kernels_pressure.cu) --------
// Compacts FLUID cells, builds rhs (FluidSolver3D.cu:1360-1474) and diagonals,
// zeroes p and dd off the fluid.  If rhs_dense is non-null it replaces the
// computed rhs (caller-provided system).
void launch_pressure_setup(const uint8_t* labels, const float* u, const float* v, const float* w, Dims g, float dt,
                           BodyKin body, const float* rhs_dense, float* p, PressureBufs& pb, cudaStream_t st);
// Persistent cooperative PCG (Jacobi).  x starts at zero; solves A x = b to
// ||r||/||b|| <= tol.  Results in pb.out.
int launch_pcg(Dims g, PressureBufs& pb, const float* rhs, double tol, int maxit, int max_blocks, cudaStream_t st);
int pcg_max_blocks();
// p[fidx[n]] = x[n] (x64 when use64).
void launch_scatter_p(const PressureBufs& pb, float* p, int use64, Dims g, cudaStream_t st);
// ||b - A p||^2 and ||b||^2 in FP64 into pb.red[0..1] (p dense float).
void launch_true_residual(const PressureBufs& pb, const float* p, Dims g, cudaStream_t st);
// Iterative refinement helpers: r = b - A x64 (FP64, via the dense double
// scratch xd), and x64 += x.
void launch_ir_residual(PressureBufs& pb, double* xd, Dims g, cudaStream_t st);
void launch_ir_update(PressureBufs& pb, double* xd, Dims g, cudaStream_t st);

// -------- projection (kernels_pressure.cu) --------
void launch_project(float* u, float* v, float* w, const float* p, const uint8_t* labels, Dims g, float dt, BodyKin b,
                    cudaStream_t st);

// -------- G2P + advection (kernels_advect.cu) --------
void launch_g2p_advect(float4* pos, float4* vel, int64_t np, const float* u, const float* v, const float* w,
                       const float* us, const float* vs, const float* ws, const uint8_t* labels, Dims g, float alpha,
                       float dt, float cfl, int do_g2p, int do_advect, int rk2, cudaStream_t st);

// -------- particle order helpers --------
// out[pid] = in[slot] for the xyz part of float4 arrays (pid in pos.w bits).
void launch_unsort(const float4* pos, const float4* vel, int64_t np, float* pos_out, float* vel_out, cudaStream_t st);
void launch_pack(const float* pos, const float* vel, int64_t np, float4* pos4, float4* vel4, cudaStream_t st);

// -------- generic CSR CG with FP64 vectors (kernels_pressure.cu) --------
int csr_cg_solve(int n, const int* offsets, const int* cols, const double* vals, const double* b, double* x, double tol,
                 int maxit, int* iters, double* relres, cudaStream_t st);

}  // namespace fp
