// kernels.hpp -- host launchers of the PIC/FLIP kernels (implemented in *.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace fp {

// Scratch of the persistent PCG kernel: a grid barrier and FP64 partials.
struct GridBar {
    unsigned count;
    unsigned limit;  // polls after which a wait gives up (set at launch)
};

// Polls after which a grid-barrier wait of the persistent solvers gives up
// and reports DEV_TIMEOUT (fp_set_wait_limit lowers it for tests).  Each
// launch stores it in its GridBar, where the polling thread reads it.
constexpr unsigned kDefaultWaitPolls = 1u << 27;

struct PcgOut {
    int iters;
    int status;     // DEV_*
    double rr;      // ||r||^2 of the recurrence at exit
    double bb;      // ||b||^2
    double rz;
    double rr0;     // ||b - A x0||^2 of the initial iterate (MG kernel)
};

// Device buffers of the pressure system.  Compact arrays are indexed by the
// fluid number n (i-fastest order of FLUID cells); padded dense grids have a
// one-cell zero halo, (W+2)*(H+2)*(D+2) entries.  Vector storage is sized for
// FP64 and reinterpreted as FP32 by the mixed-precision solves.
struct PressureBufs {
    int* nf;              // [1] number of FLUID cells
    int* fidx;            // [nc] padded index of the n-th FLUID cell
    uint8_t* diag;        // [nc] diagonal of the unit operator (compact)
    float* b;             // [nc] right-hand side (compact)
    float* bin;           // [nc] right-hand side of an inner refinement solve
    void* R[2];           // padded dense residual (double-buffered)
    void* Wv[2];          // padded dense w = A M^-1 r
    void* S[2];           // padded dense s = A p
    void* invd;           // padded dense 1/diag
    void* P;              // [nc] compact search direction
    void* X;              // [nc] compact solution
    double* x64;          // [nc] refinement accumulator (compact)
    double* xd;           // padded dense FP64 copy of x64
    double* part;         // [6 * max_blocks] per-block partial sums
    GridBar* bar;         // [1]
    PcgOut* out;          // [1]
    int* tile_sums;       // scan scratch
    double* red;          // [2] FP64 reduction results (true residual)
};

// -------- multigrid-preconditioned PCG (kernels_mg.cu) --------
constexpr int MG_MAX_LEVELS = 8;
constexpr int MG_BLOCK_CELLS = 4096;           // levels at most this big are solved by one block ...
constexpr int MG_SMEM_BUDGET = 180 * 1024;     // ... in shared memory, when their copies fit in this
// One multigrid level: padded dense grids with a SOLID / zero halo.
struct MgLevel {
    int W, H, D;    // interior cells
    int sy, sz;     // padded strides: W+2 and (W+2)*(H+2)
    uint8_t* lab;   // labels (BODY folded into SOLID)
    float* x;       // correction (level 0: the preconditioned residual z)
    float* b;       // right-hand side (level 0: the residual r)
    uint8_t* code;  // per solve: FLUID cells 1 + diagonal, every other cell 0
};
// Fills lv[].W/H/D/sy/sz of the level hierarchy for a W x H x D grid (down to
// at most 2 cells per axis, or MG_MAX_LEVELS levels); returns L.
int mg_levels_for(int W, int H, int D, MgLevel* lv);
int mg_max_blocks();
// First block-solved level G of the hierarchy and the shared memory its
// copies take (0: the block levels stay in global memory).
int mg_split(const MgLevel* lv, int L, int* smem_bytes);
// Level labels from the cell labels (per solve): the grid-wide coarse levels;
// the solver kernel coarsens the shared-memory levels itself.  With l1list
// (room for level 1's W*H*D cells) it also lists level 1's FLUID cells there
// and their number in *l1n.  Returns the number of launches.
int launch_mg_setup(const uint8_t* labels, Dims g, MgLevel* lv, int L, int* l1list, int* l1n, cudaStream_t st);
// MG-preconditioned PCG (FP32 V-cycle, FP64 Krylov vectors and reductions) for
// A x = rhs (compact) to ||r||/||rhs|| <= tol; solution in pb.X (FP64
// compact).  p, q, xs, r are level-0 padded dense FP64 work grids, zero at
// entry and on exit.
// x0: compact initial guess (scaled on the device by its energy-optimal
// factor), or null to start from x = 0.
// nu0: red-black sweep pairs before and after the coarse correction on the
// finest level (coarser levels take one pair; the cycle stays symmetric).
// pprev: without x0, a dense W x H x D guess (the previous step's pressure),
// gathered at the FLUID cells and scaled like x0; null to start from zero.
// pout: the dense W x H x D pressure out (its non-FLUID cells must be zero),
// or null.  The kernel also writes the true residual's ||rhs - A x||^2 and
// ||rhs||^2 (FP64) to pb.red.  l1list / l1n: level 1's FLUID cells from
// launch_mg_setup (or null), whose x and b the kernel leaves zero again.
int launch_pcg_mg(Dims g, PressureBufs& pb, MgLevel* lv, int L, const int* l1list, const int* l1n, double* p,
                  double* q, double* xs, double* r, const float* rhs, double tol, int maxit, cudaStream_t st, const float* x0 = nullptr, int nu0 = 2,
                  const float* pprev = nullptr, float* pout = nullptr, unsigned wait_polls = kDefaultWaitPolls);

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
// acc: [nu + nv + nw] (num, den) pairs, zero on entry and left zero (four launches).
void launch_p2g(const float4* pos, const float4* vel, const int* start, Dims g, float dt, float3 gravity,
                float2* acc, float* u, float* v, float* w, float* us, float* vs, float* ws, int fused_forces,
                cudaStream_t st);
void launch_forces(float* u, float* v, float* w, Dims g, float dt, float3 gravity, cudaStream_t st);
void launch_copy(const float* src, float* dst, int64_t n, cudaStream_t st);

// -------- pressure (kernels_pressure.cu) --------
// Compacts FLUID cells, builds rhs (FluidSolver3D.cu:1360-1474) and diagonals,
// zeroes p and dd off the fluid.  If rhs_dense is non-null it replaces the
// computed rhs (caller-provided system).
void launch_pressure_setup(const uint8_t* labels, const float* u, const float* v, const float* w, Dims g, float dt,
                           BodyKin body, const float* rhs_dense, float* p, PressureBufs& pb, cudaStream_t st);
// Persistent cooperative Jacobi PCG (Chronopoulos-Gear form, one grid barrier
// per iteration) from x0 = 0 for A x = rhs to ||r||/||rhs|| <= tol; vectors in
// FP64 (fp64 = 1) or FP32 (0), reductions always FP64.  Solution in pb.X,
// diagnostics in pb.out.  The padded work grids must be zero on entry;
// launch_pcg_clear restores that after a solve.
int launch_pcg(Dims g, PressureBufs& pb, const float* rhs, int fp64, double tol, int maxit, cudaStream_t st,
               unsigned wait_polls = kDefaultWaitPolls);
void launch_pcg_clear(PressureBufs& pb, int fp64, int with_invd, cudaStream_t st);
// Barrier word to zero with its poll limit, status word to DEV_OK (before
// every persistent-solver launch).
void launch_reset_barrier(GridBar* bar, int* status, unsigned wait_polls, cudaStream_t st);
int pcg_max_blocks();
// p[cell] = X[n] (src 0: FP32 X, 1: FP64 X, 2: x64).
void launch_scatter_p(const PressureBufs& pb, float* p, int src, Dims g, cudaStream_t st);
// ||b - A X||^2 and ||b||^2 in FP64 into pb.red[0..1] (uses R[0] as scratch).
void launch_true_residual(PressureBufs& pb, int fp64, Dims g, cudaStream_t st);
// Iterative refinement: bin = float(b - A x64) with the FP64 residual norms in
// pb.red; x64 += X (FP32) and its padded copy xd.
void launch_ir_residual(PressureBufs& pb, Dims g, cudaStream_t st);
void launch_ir_update(PressureBufs& pb, Dims g, cudaStream_t st);
// Scales the refinement's starting point x64 (and xd) by its energy-optimal
// factor (x, b) / (x, A x), computed in FP64 on the device (3 launches).
void launch_guess_scale(PressureBufs& pb, Dims g, cudaStream_t st);

// -------- projection (kernels_pressure.cu) --------
// guard: the status word of the solve that produced p, or null; the kernel
// does nothing when that solve failed (solve_failed).
void launch_project(float* u, float* v, float* w, const float* p, const uint8_t* labels, Dims g, float dt, BodyKin b,
                    cudaStream_t st, const int* guard = nullptr);

// -------- G2P + advection (kernels_advect.cu) --------
void launch_g2p_advect(float4* pos, float4* vel, int64_t np, const float* u, const float* v, const float* w,
                       const float* us, const float* vs, const float* ws, const uint8_t* labels, Dims g, float alpha,
                       float dt, float cfl, int do_g2p, int do_advect, int rk2, cudaStream_t st,
                       const int* guard = nullptr, const BodyShape* collide = nullptr);
// collide: the body for SDF collision projection (sdf_push_out, eps = dx/4),
// or null for the reference's label search alone.

// -------- rigid body (kernels_body.cu) --------
// mark[c] = 1 where the cell centre is inside the body (SDF <= 0).
void launch_mark_body(uint8_t* mark, Dims g, const BodyShape& b, cudaStream_t st);
// labels[c] = BODY where mark[c] and labels[c] != SOLID (init-time marking).
void launch_apply_mark(uint8_t* labels, const uint8_t* mark, Dims g, cudaStream_t st);
// Fluid force and torque on the body (FP64): out[0..2] force, out[3..5]
// torque about b.com; part holds body_force_partials() doubles.
void launch_body_force(const float* p, const uint8_t* labels, Dims g, const BodyShape& b, double* part, double* out,
                       cudaStream_t st);
int body_force_partials();
// The reference's body forces: out[0..5] = panel drag + lift force and torque
// about cm, out[6..7] = body volume and submerged volume from the SDF voxels.
// part holds body_force_partials() doubles; pos/start are the cell-sorted
// particles.  sdf = null samples the analytic sphere |x - local_com| - radius.
struct RefBuoyancy {
    const float* sdf;
    int sw, sh, sd;
    float cs;
    float3 origin, local_com, com;
    float radius;
    float rot[9];
};
void launch_ref_body_forces(const uint8_t* labels, const float* u, const float* v, const float* w, Dims g, float3 cm,
                            float3 bvel, const RefBuoyancy& b, const float4* pos, const int* start, double* part,
                            double* out, cudaStream_t st);

// -------- particle order helpers --------
// out[pid] = in[slot] for the xyz part of float4 arrays (pid in pos.w bits).
void launch_unsort(const float4* pos, const float4* vel, int64_t np, float* pos_out, float* vel_out, cudaStream_t st);
// rec[6 pid + 0..5] = x y z vx vy vz (frame records in the original order).
void launch_unsort_records(const float4* pos, const float4* vel, int64_t np, float* rec, cudaStream_t st);
// AoS to float4 (w = original index); the lowest index holding a non-finite
// value goes to *bad (set to INT_MAX before the call), if bad is not null.
void launch_pack(const float* pos, const float* vel, int64_t np, float4* pos4, float4* vel4, int* bad,
                 cudaStream_t st);

// -------- generic CSR CG with FP64 vectors (kernels_pressure.cu) --------
int csr_cg_solve(int n, const int* offsets, const int* cols, const double* vals, const double* b, double* x, double tol,
                 int maxit, int* iters, double* relres, cudaStream_t st);

// -------- velocity extrapolation (kernels_extrap.cu) --------
// Values equal to VEL_UNKNOWN on an nx x ny face grid, depth waves; the first
// front reads neighbour markers at row stride front_stride.  mark: nx*ny ints.
// Returns the number of launches.
int launch_extrapolate_unknown(float* v, int nx, int ny, int depth, int front_stride, int* mark, cudaStream_t st);
// Faces of component axis (0 u, 1 v, 2 w) with no FLUID side, depth waves.
int launch_extrapolate_from_fluid(float* v, int axis, const uint8_t* labels, Dims g, int depth, int* mark,
                                  cudaStream_t st);

// -------- scene generation (kernels_scene.cu) --------
void launch_seabed_labels(uint8_t* labels, int W, int H, int D, double dx, double level, double bed_base,
                          double bed_amp, uint64_t seed, double water_xmin, cudaStream_t st);
void launch_levelset_labels(const float* solid, const float* fluid, int64_t n, uint8_t* labels, cudaStream_t st);

// -------- the reference's own 2D step, scheme "ref2d" (kernels_ref2d.cu) --------
// Scratch: start[(W+4)*(H+4)+1] (bins of cells -2..W+1 x -2..H+1), list, key,
// rank [np], keep [np+1], misc[3] (non-finite u and v velocities, capped
// substep loops).
struct R2Scratch {
    int *start, *list, *key, *rank, *keep, *misc;
};
void launch_r2_label(const uint8_t* base, uint8_t* labels, const float4* pos, int64_t np, Dims g, float dx,
                     cudaStream_t st);
// mode 0: u, v = P2G; mode 1: u*, v* = P2G and u, v = P2G + gravity (5 launches)
void launch_r2_p2g(const float4* pos, const float4* vel, int64_t np, Dims g, float dx, float dt, int mode,
                   R2Scratch& sc, float* u, float* v, float* us, float* vs, cudaStream_t st);
void launch_r2_forces(float* u, float* v, Dims g, float dt, cudaStream_t st);
void launch_r2_project(float* u, float* v, const float* p, const uint8_t* labels, Dims g, float dx, float dt,
                       cudaStream_t st);
// flags: 1 G2P, 2 advection, 4 clean-up (sets sc.keep)
void launch_r2_particles(float4* pos, float4* vel, int64_t np, const float* u, const float* v, const float* us,
                         const float* vs, const uint8_t* labels, Dims g, float dx, float dt, float alpha, int flags,
                         R2Scratch& sc, cudaStream_t st);
// kept particles of sc.keep, in order, to pos2/vel2 (w = new index); the
// count lands in sc.keep[np] (2 launches)
void launch_r2_compact(const float4* pos, const float4* vel, int64_t np, R2Scratch& sc, float4* pos2, float4* vel2,
                       cudaStream_t st);

}  // namespace fp
