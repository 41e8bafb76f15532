/*
 * fluidprjct.h -- C ABI of the B200-native PIC/FLIP solver.
 *
 * Drop-in replacement for the per-step solve path of Ship-Vano/FluidPrjct,
 * whose interface is the C++ class FluidSolver3D
 * (src/FluidSim/FluidSolver3D.cuh:13-186) driven by main.cpp:9-58.
 * The class becomes an opaque handle; its public knobs become fp_config
 * fields; init()/run()/frameStep() become fp_load_labels()+fp_seed_particles()
 * / fp_run() / fp_step().
 *
 * Conventions
 *   - Every entry point returns an int status (FP_OK = 0) and never throws.
 *     fp_last_error() gives the message of the last failure on a handle.
 *   - One solver per host thread; each solver owns one CUDA stream and all of
 *     its device memory.  Buffers passed in or out are host memory owned by
 *     the caller and are copied.
 *   - fp_create makes fp_config.device current on the calling thread, which
 *     then makes the solver's calls.  A process may drive solvers on several
 *     GPUs at once, one thread each; launch set-up is kept per device.
 *   - Grids use the reference's layouts: cell (i,j,k) at i + j*W + k*W*H;
 *     u is (W+1) x H x D, v is W x (H+1) x D, w is W x H x (D+1), each with
 *     i fastest.  Labels: FP_SOLID 0, FP_FLUID 1, FP_AIR 2, FP_BODY 3
 *     (utility.cuh:65-68).
 *   - Particles are n x 3 interleaved float32 (x y z), returned in the order
 *     they were given (the solver keeps them sorted by cell internally).
 *   - Cells outside the grid count as SOLID walls.
 */
#ifndef FLUIDPRJCT_H
#define FLUIDPRJCT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference's pressureSolve returns -1 (no fluid cells),
 * -2 (empty matrix) and -4 (matrix creation failure)
 * (FluidSolver3D.cu:1875-1951); those map to FP_ERR_NO_FLUID / FP_ERR_SOLVER. */
enum {
    FP_OK = 0,
    FP_ERR_ARG = -1,        /* bad argument or size                        */
    FP_ERR_IO = -2,         /* file missing, truncated or malformed        */
    FP_ERR_CUDA = -3,       /* CUDA runtime error                          */
    FP_ERR_STATE = -4,      /* call out of order (e.g. step before labels) */
    FP_ERR_NO_FLUID = -5,   /* pressure solve found no FLUID cell          */
    FP_ERR_SOLVER = -6,     /* PCG breakdown, NaN, or iteration cap        */
    FP_ERR_TIMEOUT = -7     /* a bounded device-side wait gave up          */
};

enum { FP_SOLID = 0, FP_FLUID = 1, FP_AIR = 2, FP_BODY = 3 };

/* Frame output format of fp_run (FileOutputFormat, utility.cuh:58-61, plus
 * binary little-endian PLY and "no output"). */
enum { FP_OUT_PLY = 0, FP_OUT_OFF = 1, FP_OUT_PLY_BINARY = 2, FP_OUT_NONE = 3 };

/* Pressure solver variants (all matrix-free 7-point PCG on the GPU):
 *   FP_SOLVER_PCG         FP64 vectors and reductions, Jacobi preconditioner
 *                         ("plain" PCG);
 *   FP_SOLVER_PCG_MIXED   FP32 stencil and vectors with FP64 reductions, inside
 *                         an FP64 iterative-refinement loop (true residual
 *                         recomputed in FP64);
 *   FP_SOLVER_PCG_MG      flexible PCG with an FP32 geometric-multigrid V-cycle
 *                         preconditioner, FP64 Krylov vectors and reductions;
 *                         its first direction is the previous step's pressure
 *                         (warm_start);
 *   FP_SOLVER_PCG_LEARNED flexible PCG whose first preconditioner application
 *                         is a learned U-Net (z0 = N(b)) and whose later ones
 *                         are the V-cycle; plain PCG fallback;
 *   FP_SOLVER_PCG_LEARNED_MIXED the U-Net's guess, energy-optimally scaled, as
 *                         the starting point of FP_SOLVER_PCG_MIXED's FP64
 *                         refinement ("learned + mixed"); plain PCG fallback. */
enum { FP_SOLVER_PCG = 0, FP_SOLVER_PCG_MIXED = 1, FP_SOLVER_PCG_MG = 2, FP_SOLVER_PCG_LEARNED = 3,
       FP_SOLVER_PCG_LEARNED_MIXED = 4 };

/* Advection: the reference's adaptive Ralston RK3 (AdvectParticlesFunctor,
 * FluidSolver3D.cu:1241-1330) or midpoint RK2 with the same substepping. */
enum { FP_ADVECT_RK3REF = 0, FP_ADVECT_RK2 = 1 };

/* Step scheme.  FP_SCHEME_DEFAULT runs the 3D scheme of FluidSolver3D.cu on
 * any grid (a 2D grid is its depth-1 case).  FP_SCHEME_REF2D (dim = 2 only)
 * runs FluidSolver2D.cu's own step (:1302-1331): cell-centre-weighted P2G,
 * VEL_UNKNOWN faces, 1D-linear G2P, Euler advection with projection into the
 * nearest SOLID cell, and particle deletion; particles keep their order and
 * fp_num_particles shrinks as they are deleted.  Its fp_config.advection and
 * cfl are unused (the reference fixes Euler and C = 1). */
enum { FP_SCHEME_DEFAULT = 0, FP_SCHEME_REF2D = 1 };

/* Collision of advected particles with the rigid body (fp_config.collision). */
enum { FP_COLLISION_LABELS = 0, FP_COLLISION_SDF = 1 };

/* Fluid force on the rigid body.  FP_BODY_FORCES_FACE_FRACTION (default):
 * the pressure integral over SDF face fractions, an FP64 reduction.
 * FP_BODY_FORCES_REFERENCE: the reference's panel drag and lift
 * (DragLiftForceCalculator, FluidSolver3D.cu:2674-2791; Cd = Cl = 0.1) plus
 * its voxel buoyancy (applyBuoyancy, :2917-3026), summed in FP64; the
 * analytic sphere is sampled on a voxel grid of spacing dx / 2 for it. */
enum { FP_BODY_FORCES_FACE_FRACTION = 0, FP_BODY_FORCES_REFERENCE = 1 };

/* Grid selectors for fp_get_grid / fp_set_grid.  FP_GRID_RHS (read only) is
 * the dense right-hand side of the last pressure solve, zero off FLUID cells
 * (the reference's RHS, FluidSolver3D.cu:1518-1596, before compaction). */
enum { FP_GRID_U = 0, FP_GRID_V = 1, FP_GRID_W = 2, FP_GRID_U_SAVED = 3, FP_GRID_V_SAVED = 4,
       FP_GRID_W_SAVED = 5, FP_GRID_P = 6, FP_GRID_RHS = 7 };

/* Step phases for fp_run_phase, in frameStep order (FluidSolver3D.cu:3030-3098). */
enum { FP_PHASE_LABEL = 0, FP_PHASE_P2G = 1, FP_PHASE_SAVE = 2, FP_PHASE_FORCES = 3, FP_PHASE_PRESSURE = 4,
       FP_PHASE_PROJECT = 5, FP_PHASE_BODY = 6, FP_PHASE_G2P = 7, FP_PHASE_ADVECT = 8,
       FP_PHASE_CLEANUP = 9 /* FP_SCHEME_REF2D only: cleanUpParticles, FluidSolver2D.cu:1171-1204 */ };

/* Solver configuration.  Keys and defaults follow main.cpp:17-52 and the
 * member initialisers of FluidSolver3D.cuh:71-79,156-166; the fields after
 * body_mass are additions whose defaults reproduce the reference's behaviour. */
typedef struct fp_config {
    int      dim;                  /* 3 (FluidSolver3D) or 2 (FluidSolver2D)        */
    float    dx;                   /* "dx"            default 0.1                   */
    float    dt;                   /* "dt"            default 0.02                  */
    float    pic_weight;           /* "PIC_WEIGHT"    default 0.01 (alpha)          */
    int      iter_per_frame;       /* "iterPerFrame"  default 1                     */
    int      output_format;        /* "outputFormat"  FP_OUT_PLY                    */
    char     output_template[256]; /* "outputTemplate" "InputData/particles_"       */
    int      active_body;          /* "activeBody"    default 0                     */
    float    body_pos[3];          /* "body_x/y/z"    default 0.5                   */
    float    body_mass;            /* "body_mass"     default 50                    */
    /* additions */
    int      ppc;                  /* particles per cell at seeding (reference 4)  */
    uint32_t seed;                 /* mt19937 seed (the reference: random_device)  */
    int      solver;               /* FP_SOLVER_*                                   */
    int      advection;            /* FP_ADVECT_*                                   */
    float    cfl;                  /* advection C (reference 0.1)                   */
    double   tol;                  /* relative residual target (default 1e-6)      */
    int      max_iters;            /* PCG iteration cap (default 20000)            */
    float    body_radius;          /* analytic sphere SDF radius; 0 = SDF file     */
    float    body_density;         /* sphere density relative to water            */
    int      device;               /* CUDA device ordinal; -1 = current device     */
    int      scheme;               /* FP_SCHEME_* (default FP_SCHEME_DEFAULT)      */
    int      extrapolate;          /* velocity extrapolation (extrapolateGridFluidData,
                                      FluidSolver2D.cu:1207-1295), off by default:
                                      FP_SCHEME_REF2D: nonzero enables the 2D step's
                                      two commented-out calls with their depths;
                                      default scheme: this many wavefront layers into
                                      faces with no FLUID side, between G2P and
                                      advection */
    int      body_forces;          /* FP_BODY_FORCES_* (default face fractions)   */
    int      mg_sweeps;            /* FP_SOLVER_PCG_MG / _LEARNED: red-black sweep
                                      pairs before and after the coarse correction
                                      on the finest level (coarser levels: one);
                                      0 = the default, 2                           */
    int      warm_start;           /* FP_SOLVER_PCG_MG: nonzero (the default)
                                      starts each solve from the pressure of the
                                      previous step, scaled by its energy-optimal
                                      factor; the stopping test stays relative
                                      to ||b||.  0: from x = 0                  */
    int      collision;            /* particles that advection moves into the body:
                                      FP_COLLISION_LABELS (default) nudges them
                                      half a cell toward the nearest FLUID cell
                                      centre (projectParticleDevice3D,
                                      FluidSolver3D.cu:1161-1239);
                                      FP_COLLISION_SDF projects them along the
                                      body SDF's normal to phi = dx/4 (SOLID
                                      cells keep the label search)              */
    char     body_sdf[256];        /* "body_sdf": SDF file of the body that the
                                      FluidGPU driver loads when activeBody is
                                      set and body_radius is 0 (the reference's
                                      fixed InputData/ball.sdf,
                                      FluidSolver3D.cu:158)                     */
} fp_config;

/* Per-step statistics: the reference's cudaEvent phase timers
 * (FluidSolver3D.cuh:112-119) plus solver diagnostics.  Times in ms. */
typedef struct fp_step_stats {
    int64_t step;              /* steps taken so far                              */
    int64_t num_particles;
    int32_t num_fluid_cells;   /* fluidCellsAmount                                */
    int32_t pcg_iters;         /* inner PCG iterations of the last solve          */
    int32_t outer_iters;       /* refinement loops of the last solve              */
    int32_t fallback;          /* 1 if the learned preconditioner fell back       */
    int32_t solve_status;      /* FP_OK or the failure of the last solve          */
    int32_t pad_;
    double  residual;          /* final true relative residual ||b-Ax||/||b||    */
    float   t_label, t_p2g, t_forces, t_pressure, t_project, t_body, t_g2p, t_advect;
    float   t_total;
    float   guess_relres;      /* ||b - A x0|| / ||b|| of the initial guess (the
                                  learned one, or the previous pressure with
                                  warm_start), after its energy-optimal scaling;
                                  1 for solves that start from x = 0            */
    double  body_pos[3], body_vel[3], body_omega[3], body_angles[3];
    double  body_force[3], body_torque[3];
    int64_t kernel_launches;   /* kernels this library launched, cumulative     */
    float   t_pcg;             /* device time of the pressure solve, last step  */
    float   t_learned;         /* of which the learned initial guess            */
    int64_t particles_removed; /* FP_SCHEME_REF2D: deleted by the last clean-up  */
    int32_t advect_capped;     /* FP_SCHEME_REF2D: particles whose substep loop
                                  hit its bound in the last step                */
    int32_t pad2_;
} fp_step_stats;

typedef struct fp_solver fp_solver;

/* Fill *cfg with the reference defaults. */
int fp_config_default(fp_config* cfg);

/* Parse a reference config.json (keys of main.cpp:17-52 plus the additions)
 * into *cfg; missing keys keep their current values.  label_path receives
 * "inputLabelData" and frames "frameAmount" when non-null. */
int fp_config_load_json(const char* path, fp_config* cfg, char* label_path, size_t label_path_len, int* frames);

/* FluidSolver3D::FluidSolver3D (FluidSolver3D.cu:4-35).  Grid dimensions come
 * from fp_load_labels / fp_set_labels, as in the reference's init(). */
int fp_create(const fp_config* cfg, fp_solver** out);
int fp_destroy(fp_solver* s);
const char* fp_last_error(const fp_solver* s);

/* Labels: the reference file format (init, FluidSolver3D.cu:81-153; 2D reader
 * FluidSolver2D.cu:52-104) or a caller array (n = W*H*D uint8).  Sizes the
 * grids; SOLID cells stay fixed for the whole run. */
int fp_load_labels(fp_solver* s, const char* path);
int fp_set_labels(fp_solver* s, const uint8_t* labels, int W, int H, int D);

/* Labels from level sets, combined on the GPU as the reference's DistrGen
 * tools do (fluidLabels.py: SOLID where solid < 0, else FLUID where
 * fluid < 0, else AIR); host arrays of W*H*D floats in i + j*W + k*W*H order.
 * fp_read_levelset_file reads one 2D level-set file of
 * DistrGen/fluidLevelSets.py (dims = {W, H}; out may be NULL to query them). */
int fp_set_labels_from_levelsets(fp_solver* s, const float* solid, const float* fluid, int W, int H, int D);
int fp_read_levelset_file(const char* path, int* dims, float* out);

/* The large seabed scene, labelled on the GPU: SOLID walls, SOLID below
 * bed_base + bed_amp * noise(x, z) (four octaves of value noise, seeded),
 * FLUID below y = level where x >= water_xmin, AIR elsewhere.  The grid
 * spacing is fp_config.dx. */
int fp_scene_seabed(fp_solver* s, int W, int H, int D, float level, float bed_base, float bed_amp, uint32_t seed,
                    float water_xmin);
int fp_get_dims(const fp_solver* s, int* W, int* H, int* D);

/* Body SDF (RigidBody::loadSDF, utility.cuh:231-338) from a text file, or the
 * analytic sphere of fp_config.body_radius when path is NULL. */
int fp_load_sdf(fp_solver* s, const char* path);

/* Wave paddle (no reference counterpart; the large seabed scene's moving
 * boundary): the half-space x < x_p(t) = x_rest + amplitude sin(2 pi t /
 * period), t from this call, is a BODY region moving at dx_p/dt.  It takes
 * the body slot (replacing an SDF body) and sets active_body; its motion is
 * prescribed, and fp_step_stats.body_force reports the fluid's load on it. */
int fp_set_paddle(fp_solver* s, float x_rest, float amplitude, float period);

/* Particles: seeding of FLUID cells (seedParticles, FluidSolver3D.cu:213-297)
 * with a deterministic mt19937(seed); caller arrays; PLY files.  A
 * non-finite position or velocity is rejected with FP_ERR_ARG (checked on
 * the device); the solver then holds no particles.  At most 2,139,062,143
 * particles (0x7F7F7F7F); more are rejected with FP_ERR_ARG. */
int fp_seed_particles(fp_solver* s, int ppc, uint32_t seed);
int fp_set_particles(fp_solver* s, const float* pos, const float* vel, int64_t n);
int fp_load_ply(fp_solver* s, const char* path);
int fp_save_ply(fp_solver* s, const char* path, int format);
int64_t fp_num_particles(const fp_solver* s);
int fp_get_particles(fp_solver* s, float* pos, float* vel, int64_t n);

/* One full step (frameStep, FluidSolver3D.cu:3030-3098), n times.  Returns
 * when the last step has finished; fp_stats then holds that step's phase
 * timers (the earlier steps of the call are not waited for). */
int fp_step(fp_solver* s, int n);

/* run() (FluidSolver3D.cu:3100-3163): frames*iter_per_frame + 1 steps with
 * frame output every iter_per_frame steps (particles PLY/OFF, body PLY and
 * the body CSV when a body is active). */
int fp_run(fp_solver* s, int frames);

/* One phase of the step on the current state (diagnostics and parity tests). */
int fp_run_phase(fp_solver* s, int phase);

/* Grid and label copies (n must equal the grid's element count). */
int fp_get_grid(fp_solver* s, int which, float* out, int64_t n);
int fp_set_grid(fp_solver* s, int which, const float* in, int64_t n);
int fp_get_labels(fp_solver* s, uint8_t* out, int64_t n);
/* The same copies into caller DEVICE memory, ordered on the solver's stream
 * and complete on return (no host staging; used to build training sets). */
int fp_get_grid_device(fp_solver* s, int which, float* d_out, int64_t n);
int fp_get_labels_device(fp_solver* s, uint8_t* d_out, int64_t n);

/* Rigid-body kinematic state used by the RHS and projection; setting it
 * overrides the integrated state (FluidSolver3D.cu:1368-1370). */
int fp_set_body_state(fp_solver* s, const float* pos, const float* vel, const float* omega);

int fp_stats(const fp_solver* s, fp_step_stats* out);

/* The solver's CUDA stream (a cudaStream_t), for callers that record their
 * own events or order their own work after the solver's. */
void* fp_cuda_stream(const fp_solver* s);

/* Per-step log (the reference prints its phase timers at the end of run(),
 * FluidSolver3D.cu:3149-3162): with a path, every step of fp_step / fp_run
 * appends one JSON line of its fp_step_stats (step, particles, FLUID cells,
 * PCG iterations, residual and status, phase times in ms, body position and
 * velocity) to that file; each step then waits for its own end, so that its
 * times are its own.  NULL or "" closes the log. */
int fp_set_step_log(fp_solver* s, const char* path);

/* Exact-resume snapshots (no counterpart in the reference): fp_save_state
 * writes the grid dimensions, dx and dt, the step count, the SOLID map and
 * labels, u, v, w, u*, v*, w* and p, the particles (in the order given) and
 * the rigid body's full state (with its SDF); fp_load_state restores them on
 * a solver created with the same dx and dt (FP_ERR_ARG otherwise; FP_ERR_IO
 * for a missing, truncated or foreign file), re-sizing its grids.  The
 * solver's own configuration (solver, advection, ...) is kept.  A loaded
 * state steps on as the saved solver would, up to the order of P2G's
 * floating-point sums. */
int fp_save_state(fp_solver* s, const char* path);
int fp_load_state(fp_solver* s, const char* path);

/* Diagnostics (no counterpart in the reference): the number of polls after
 * which a grid-barrier wait of the persistent pressure solvers gives up and
 * the step returns FP_ERR_TIMEOUT (default 2^27, about a minute; 0 restores
 * it).  A small limit makes the timeout path run without any fault, so a
 * caller can test its error handling: after FP_ERR_TIMEOUT the particles and
 * the body are as before the step, and the next step with the default limit
 * solves normally. */
int fp_set_wait_limit(fp_solver* s, int64_t polls);

/* Pressure solve of the current labels for a caller right-hand side (dense,
 * W*H*D, zero off FLUID cells); x receives the dense solution.  Uses the
 * configured solver.  Reports iterations and the true relative residual. */
int fp_pressure_solve(fp_solver* s, const float* rhs, float* x, int64_t n, int* iters, double* relres);

/* Stand-alone SPD solve of an upper-triangle CSR matrix (the storage passed to
 * cuDSS with CUDSS_MVIEW_UPPER, FluidSolver3D.cu:1932-1945) by GPU CG with
 * FP64 vectors: the known-answer path of test.cu:223-395.  Host arrays. */
int fp_solve_csr_upper(int n, const int* offsets, const int* cols, const double* vals, const double* b, double* x,
                       double tol, int max_iters, int* iters, double* relres);

/* Allocation-free variant of fp_solve_csr_upper; it has no counterpart in the
 * reference.  Same system and algorithm, but every pointer is a DEVICE buffer
 * owned by the caller (offsets n+1, cols/vals offsets[n], b and x n doubles)
 * and the work vectors live in one fixed device array, so the call never
 * allocates.  For hosts whose own pool allocator owns the GPU, and for loops
 * that cannot pay cudaMalloc's latency and device-wide sync.
 *   - n above FP_NOALLOC_MAX_N is rejected with FP_ERR_ARG; so is a
 *     malformed matrix, checked on the device before the solve: offsets[0]
 *     must be 0, offsets must not decrease, columns must lie in [0, n);
 *   - like fp_solve_csr_upper it returns FP_OK when CG stops at max_iters or
 *     breaks down: check *relres against tol;
 *   - the call is synchronous (it reads scalars back every iteration and
 *     drains its stream before returning), so it must not be issued on a
 *     stream that is being captured;
 *   - all calls on a device share the array, so they take turns: a call
 *     holds a per-device host lock until its stream has drained, and calls
 *     from several host threads are serialised;
 *   - the first call on a device, with that device current, looks up the
 *     array's address.
 * stream may be NULL (the legacy default stream). */
#define FP_NOALLOC_MAX_N (1 << 18)
int fp_solve_csr_upper_noalloc(int n, const int* d_offsets, const int* d_cols, const double* d_vals,
                               const double* d_b, double* d_x, double tol, int max_iters, int* iters,
                               double* relres, void* stream);

/* Learned preconditioner (no counterpart in the reference).  A 3D U-Net with
 * three levels (16/32/64 channels, 3x3x3 convolutions, BF16 weights and
 * activations, FP32 accumulation) maps the cell labels and the divergence to
 * a pressure guess.  FP_SOLVER_PCG_LEARNED scales that guess by its
 * energy-optimal factor and uses it as the initial iterate of the
 * multigrid-preconditioned PCG.  If that solve stalls or misses tol, the plain
 * FP64 PCG solves again from zero (fp_step_stats.fallback = 1).
 * fp_load_learned loads a weight file written by fp_unet_save (labels must be
 * loaded first; 3D only). */
int fp_load_learned(fp_solver* s, const char* weights_path);

/* The network itself, for training and tests.  All array arguments are DEVICE
 * pointers on the real grid (labels uint8, rhs/p/x float, W*H*D each); grids
 * are padded to multiples of 4 inside, the padding counting as SOLID.  Calls
 * are complete on return, except fp_unet_train_step with loss == NULL, which
 * returns once the step is queued on the network's stream.  Weights are the
 * flat FP32 vector of fp_unet_num_params() entries: layers L0..L9 as
 * [27][COUT][CIN] (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)), then 16 head
 * weights.  The loss is sum_F (out - p/s)^2 / sum_F (p/s)^2 over FLUID cells,
 * s = the RMS of rhs over FLUID cells. */
typedef struct fp_unet fp_unet;
int64_t fp_unet_num_params(void);
int fp_unet_create(int W, int H, int D, int train, uint64_t seed, fp_unet** out);
void fp_unet_destroy(fp_unet* u);
const char* fp_unet_last_error(const fp_unet* u);
void* fp_unet_cuda_stream(const fp_unet* u);
int fp_unet_get_params(fp_unet* u, float* out, int64_t n);
int fp_unet_set_params(fp_unet* u, const float* in, int64_t n);
int fp_unet_save(fp_unet* u, const char* path);
int fp_unet_load(fp_unet* u, const char* path);
int fp_unet_forward(fp_unet* u, const uint8_t* d_labels, const float* d_rhs, float* d_x);
int fp_unet_loss_grad(fp_unet* u, const uint8_t* d_labels, const float* d_rhs, const float* d_p, double* loss,
                      float* grad);
int fp_unet_train_step(fp_unet* u, const uint8_t* d_labels, const float* d_rhs, const float* d_p, float lr,
                       double* loss);

/* Host-only readers (no GPU needed).  fp_read_label_file parses a reference
 * label file (dim 3: FluidSolver3D.cu:81-153, dim 2: FluidSolver2D.cu:52-104);
 * call with out = NULL to get dims[0..2] = W, H, D (D = 1 in 2D) first.
 * fp_read_ply_file reads ascii or binary_little_endian PLY vertices; call with
 * pos = NULL to get *n; vel may be NULL; *has_vel reports vx vy vz. */
int fp_read_label_file(const char* path, int dim, int* dims, uint8_t* out);
int fp_read_ply_file(const char* path, int64_t* n, float* pos, float* vel, int* has_vel);
/* Writes n particles (pos, and vel for FP_OUT_PLY_BINARY; vel may be NULL) in
 * a frame format: ASCII PLY / OFF of positions as save3dParticlesToPLY / OFF write
 * them (utility.cu:91-127, %g), or binary little-endian PLY. */
int fp_write_particle_file(const char* path, const float* pos, const float* vel, int64_t n, int format);

/* Library version string. */
const char* fp_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FLUIDPRJCT_H */
