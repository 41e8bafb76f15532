// solver.cu -- host runtime of the B200 PIC/FLIP solver and its C ABI.
//
// One fp_solver per scene: it owns a CUDA stream and every device buffer,
// allocated once when the labels (grid) and particles are set, so a step
// performs no allocation (the reference allocates ~15 Thrust temporaries per
// step).  The step is the reference's frameStep (FluidSolver3D.cu:3030-3098)
// with its phases fused into fewer kernels:
//   label   : bin + label/scan + scatter  (labelGrid, and the cell sort)
//   p2g     : brick-tiled P2G with normalise, u* save and gravity fused
//   pressure: fluid compaction + RHS, persistent PCG, scatter, residual check
//   project : one kernel over all faces
//   g2p+adv : one kernel per particle
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/fluidprjct.h"
#include "io.hpp"
#include "kernels.hpp"
#include "unet.hpp"

using namespace fp;

namespace {

constexpr float kGravity[3] = {0.0f, -9.81f, 0.0f};  // FluidSolver3D.cuh:78

// NVTX range over a scope (the phases of a step, as the reference's
// cudaEvent timers of frameStep, FluidSolver3D.cu:3030-3098, delimit them);
// a no-op unless a profiler is attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

template <class T>
cudaError_t dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    return cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
}
template <class T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}
cudaError_t dalloc_bytes(void** p, size_t bytes) {
    *p = nullptr;
    return cudaMalloc(p, bytes ? bytes : 1);
}

// The solve's read-back block, on the device and pinned on the host: PcgOut,
// then the true residual's two FP64 sums, then the FLUID count, so that one
// copy per step brings all three back (three small copies each took their
// own turn on the stream).
constexpr size_t kRbRed = (sizeof(PcgOut) + 7) & ~size_t(7);
constexpr size_t kRbNf = kRbRed + 2 * sizeof(double);
constexpr size_t kRbBytes = (kRbNf + sizeof(int) + 15) & ~size_t(15);
template <class Out, class Red, class Nf>
void readback_views(void* base, Out*& out, Red*& red, Nf*& nf) {
    char* b = static_cast<char*>(base);
    out = reinterpret_cast<Out*>(b);
    red = b ? reinterpret_cast<Red*>(b + kRbRed) : nullptr;
    nf = b ? reinterpret_cast<Nf*>(b + kRbNf) : nullptr;
}

}  // namespace

// Rigid body state on the host (RigidBody, utility.cuh:195-491): position,
// velocity, Euler angles (theta, psi, phi) with their rotation matrix, scalar
// inertia 0.4*m*r^2 (FluidSolver3D.cu:165-169).
struct HostBody {
    bool loaded = false;
    int kind = BODY_SPHERE;
    double pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, omega[3] = {0, 0, 0};
    double theta = 0, psi = 0, phi = 0;
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double mass = 1, inertia = 1, radius = 0;
    double force[3] = {0, 0, 0}, torque[3] = {0, 0, 0};
    // voxel SDF
    int nx = 0, ny = 0, nz = 0;
    float origin[3] = {0, 0, 0}, cell = 1, local_com[3] = {0, 0, 0};
    std::vector<float> sdf_host;  // voxel SDF values (surface-point output)
    // paddle: face at x0 + amp sin(2 pi t / period), t since fp_set_paddle
    double pad_x0 = 0, pad_amp = 0, pad_period = 1, pad_t = 0;

    void paddle_at(double t) {
        const double w = 2.0 * 3.14159265358979323846 / pad_period;
        pos[0] = pad_x0 + pad_amp * std::sin(w * t);
        vel[0] = pad_amp * w * std::cos(w * t);
        vel[1] = vel[2] = 0.0;
        omega[0] = omega[1] = omega[2] = 0.0;
    }

    // update_rotation_matrix (utility.cuh:470-484)
    void update_rotation() {
        const double ct = std::cos(theta), st = std::sin(theta), cp = std::cos(psi), sp = std::sin(psi),
                     cf = std::cos(phi), sf = std::sin(phi);
        R[0] = ct * cp; R[1] = st * sf - ct * cf * sp; R[2] = cf * st + ct * sf * sp;
        R[3] = sp;      R[4] = cf * cp;                R[5] = -cp * sf;
        R[6] = -cp * st; R[7] = ct * sf + cf * st * sp; R[8] = ct * cf - st * sf * sp;
    }
    // integrate (utility.cuh:408-467): semi-implicit Euler for the centre of
    // mass; body-frame angular acceleration tau/I; Euler-angle kinematics.
    void integrate(double dt) {
        for (int a = 0; a < 3; ++a) { vel[a] += force[a] / mass * dt; pos[a] += vel[a] * dt; }
        const double pi = 3.14159265358979323846;
        theta = std::min(std::max(theta, -pi), pi);
        update_rotation();
        const double tl[3] = {R[0] * torque[0] + R[3] * torque[1] + R[6] * torque[2],
                              R[1] * torque[0] + R[4] * torque[1] + R[7] * torque[2],
                              R[2] * torque[0] + R[5] * torque[1] + R[8] * torque[2]};
        for (int a = 0; a < 3; ++a) omega[a] += tl[a] / inertia * dt;
        const double dth = omega[1] * std::cos(phi) - omega[2] * std::sin(phi);
        const double dps = (omega[1] * std::sin(phi) + omega[2] * std::cos(phi)) / std::cos(theta);
        const double dph = omega[0] + dps * std::sin(theta);
        theta += dth * dt; psi += dps * dt; phi += dph * dt;
    }
};

struct fp_solver {
    fp_config cfg{};
    std::string err;
    int W = 0, H = 0, D = 0;
    Dims g{};
    cudaStream_t st = nullptr;
    cudaEvent_t ev[10]{};
    cudaEvent_t ev_pcg[2]{};
    int64_t launches = 0;   // kernels launched by this solver
    float pcg_ms = 0.0f;
    unsigned wait_polls = kDefaultWaitPolls;  // grid-barrier poll limit (fp_set_wait_limit)
    bool have_grid = false;

    // grids
    uint8_t *d_base = nullptr, *d_labels = nullptr, *d_bodymark = nullptr;
    float *d_u = nullptr, *d_v = nullptr, *d_w = nullptr, *d_us = nullptr, *d_vs = nullptr, *d_ws = nullptr,
          *d_p = nullptr, *d_scratch = nullptr, *d_scratch2 = nullptr;
    float2* d_acc = nullptr;  // P2G (num, den) pairs of every face; zero between steps
    int *d_counts = nullptr, *d_start = nullptr, *d_tiles = nullptr;
    // particles (cell order; pid in pos.w)
    float4 *d_pos = nullptr, *d_vel = nullptr, *d_pos2 = nullptr, *d_vel2 = nullptr;
    int *d_key = nullptr, *d_rank = nullptr;
    float* d_io = nullptr;  // n*3 staging for unsort/pack
    int64_t np = 0, cap = 0;
    bool sorted = false;
    // pressure
    PressureBufs pb{};
    int64_t padded = 0;
    // multigrid hierarchy (level 0 shares the padded layout of pb)
    MgLevel mg[MG_MAX_LEVELS]{};
    int mgL = 0;
    double *d_mgp = nullptr, *d_mgq = nullptr, *d_mgx = nullptr, *d_mgr = nullptr;
    int *d_l1list = nullptr, *d_l1n = nullptr;  // level 1's FLUID cells (multigrid)
    // learned initial guess
    fp_unet* net = nullptr;
    std::string learned_path;
    float* d_rhs_dense = nullptr;  // dense right-hand side (network input, FP_GRID_RHS)
    float* d_x0c = nullptr;        // compact initial guess
    cudaEvent_t ev_net = nullptr;
    // a PCG / MG solve whose read-back one_step has deferred (ev[9] marks it)
    bool solve_pending = false;
    bool pending_guess = false;
    // pinned result mirrors
    PcgOut* h_out = nullptr;
    double* h_red = nullptr;
    int* h_nf = nullptr;
    int* d_bad = nullptr;   // first non-finite particle of an upload
    int* h_bad = nullptr;
    // scheme ref2d: bins over (W+4)*(H+4) cells, particle lists and keep flags
    R2Scratch r2{};
    int r2_nb = 0;
    int64_t r2_cap = 0;
    int* h_r2 = nullptr;    // pinned: [0] particles kept, [1] capped substep loops
    int* d_extmark = nullptr;  // wavefront markers of the velocity extrapolation (largest face grid)
    // body
    BodyKin body{};
    HostBody hb;
    float* d_sdf = nullptr;
    double *d_bpart = nullptr, *d_bforce = nullptr, *h_bforce = nullptr;
    // stats
    fp_step_stats stats{};
    int64_t steps = 0;
    FILE* step_log = nullptr;  // one JSON line per step (fp_set_step_log)

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* where) {
        err = std::string(where) + ": " + cudaGetErrorString(e);
        return FP_ERR_CUDA;
    }
};

namespace {

void free_r2(fp_solver* s) {
    dfree(s->r2.start); dfree(s->r2.misc);
    s->r2_nb = 0;
}

void free_grid(fp_solver* s) {
    dfree(s->d_base); dfree(s->d_labels); dfree(s->d_bodymark);
    dfree(s->d_u); dfree(s->d_v); dfree(s->d_w); dfree(s->d_us); dfree(s->d_vs); dfree(s->d_ws);
    dfree(s->d_acc);
    dfree(s->d_p); dfree(s->d_scratch); dfree(s->d_scratch2);
    dfree(s->d_counts); dfree(s->d_start); dfree(s->d_tiles);
    PressureBufs& pb = s->pb;
    pb.nf = nullptr; pb.red = nullptr;  // inside the read-back block (pb.out)
    dfree(pb.fidx); dfree(pb.diag); dfree(pb.b); dfree(pb.bin);
    for (int i = 0; i < 2; ++i) { dfree(pb.R[i]); dfree(pb.Wv[i]); dfree(pb.S[i]); }
    dfree(pb.invd); dfree(pb.P); dfree(pb.X);
    dfree(pb.x64); dfree(pb.xd); dfree(pb.part); dfree(pb.bar); dfree(pb.out);
    for (int l = 0; l < s->mgL; ++l) {
        dfree(s->mg[l].lab); dfree(s->mg[l].x); dfree(s->mg[l].b); dfree(s->mg[l].code);
    }
    s->mgL = 0;
    dfree(s->d_mgp); dfree(s->d_mgq); dfree(s->d_mgx); dfree(s->d_mgr);
    dfree(s->d_l1list); dfree(s->d_l1n);
    dfree(s->d_rhs_dense); dfree(s->d_x0c);
    if (s->net) { fp_unet_destroy(s->net); s->net = nullptr; }
    free_r2(s);
    dfree(s->d_extmark);
    s->have_grid = false;
}

void free_body(fp_solver* s) {
    dfree(s->d_sdf); dfree(s->d_bpart); dfree(s->d_bforce);
    s->hb.loaded = false;
}

void free_particles(fp_solver* s) {
    dfree(s->d_pos); dfree(s->d_vel); dfree(s->d_pos2); dfree(s->d_vel2);
    dfree(s->d_key); dfree(s->d_rank); dfree(s->d_io);
    dfree(s->r2.list); dfree(s->r2.keep);
    s->np = s->cap = s->r2_cap = 0;
}


// (Re)create the inference network for the current grid from learned_path.
int load_net(fp_solver* s) {
    if (s->net) { fp_unet_destroy(s->net); s->net = nullptr; }
    if (s->cfg.dim != 3 || s->W < 4 || s->H < 4 || s->D < 4)
        return s->fail(FP_ERR_ARG, "the learned preconditioner needs a 3D grid of at least 4 cells per axis");
    int rc = fp_unet_create(s->W, s->H, s->D, 0, 0, &s->net);
    if (rc) return s->fail(rc, "network allocation failed");
    rc = fp_unet_load(s->net, s->learned_path.c_str());
    if (rc) {
        s->err = fp_unet_last_error(s->net);
        fp_unet_destroy(s->net);
        s->net = nullptr;
        return rc;
    }
    return FP_OK;
}

int alloc_grid(fp_solver* s, int W, int H, int D) {
    free_grid(s);
    s->W = W; s->H = H; s->D = D;
    s->g = Dims{W, H, D, s->cfg.dx};
    {
        // dx a power of two: its reciprocal is exact, and x * (1/dx) == x / dx
        int ex = 0;
        if (std::frexp(double(s->cfg.dx), &ex) == 0.5) s->g.idx = float(1.0 / double(s->cfg.dx));
    }
    const int64_t nc = s->g.nc();
    s->padded = int64_t(W + 2) * (H + 2) * (D + 2);
    const int ntiles = int((nc + 4095) / 4096) + 1;
    const int maxb = pcg_max_blocks();
    cudaError_t e = cudaSuccess;
    auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    ck(dalloc(&s->d_base, nc)); ck(dalloc(&s->d_labels, nc)); ck(dalloc(&s->d_bodymark, nc));
    ck(dalloc(&s->d_u, s->g.nu())); ck(dalloc(&s->d_us, s->g.nu()));
    ck(dalloc(&s->d_v, s->g.nv())); ck(dalloc(&s->d_vs, s->g.nv()));
    ck(dalloc(&s->d_w, s->g.nw())); ck(dalloc(&s->d_ws, s->g.nw()));
    ck(dalloc(&s->d_acc, s->g.nu() + s->g.nv() + s->g.nw()));
    ck(dalloc(&s->d_p, nc)); ck(dalloc(&s->d_scratch, nc)); ck(dalloc(&s->d_scratch2, nc));
    ck(dalloc(&s->d_counts, nc + 1)); ck(dalloc(&s->d_start, nc + 1)); ck(dalloc(&s->d_tiles, ntiles));
    PressureBufs& pb = s->pb;
    {
        void* rb = nullptr;
        ck(dalloc_bytes(&rb, kRbBytes));
        readback_views(rb, pb.out, pb.red, pb.nf);
    }
    ck(dalloc(&pb.fidx, nc)); ck(dalloc(&pb.diag, nc)); ck(dalloc(&pb.b, nc));
    ck(dalloc(&pb.bin, nc));
    const size_t pbytes = sizeof(double) * size_t(s->padded), cbytes = sizeof(double) * size_t(nc);
    for (int i = 0; i < 2; ++i) {
        ck(dalloc_bytes(&pb.R[i], pbytes)); ck(dalloc_bytes(&pb.Wv[i], pbytes)); ck(dalloc_bytes(&pb.S[i], pbytes));
    }
    ck(dalloc_bytes(&pb.invd, pbytes)); ck(dalloc_bytes(&pb.P, cbytes)); ck(dalloc_bytes(&pb.X, cbytes));
    ck(dalloc(&pb.x64, nc)); ck(dalloc(&pb.xd, s->padded));
    ck(dalloc(&pb.part, size_t(6) * std::max(maxb, 1024)));
    ck(dalloc(&pb.bar, 1));
    pb.tile_sums = s->d_tiles;
    ck(dalloc(&s->d_rhs_dense, nc));
    if (s->cfg.solver == FP_SOLVER_PCG_LEARNED || s->cfg.solver == FP_SOLVER_PCG_LEARNED_MIXED)
        ck(dalloc(&s->d_x0c, nc));
    if (s->cfg.solver == FP_SOLVER_PCG_MG || s->cfg.solver == FP_SOLVER_PCG_LEARNED) {
        s->mgL = mg_levels_for(W, H, D, s->mg);
        for (int l = 0; l < s->mgL && e == cudaSuccess; ++l) {
            MgLevel& L = s->mg[l];
            const size_t np_ = size_t(L.W + 2) * (L.H + 2) * (L.D + 2);
            ck(dalloc(&L.lab, np_)); ck(dalloc(&L.x, np_)); ck(dalloc(&L.b, np_)); ck(dalloc(&L.code, np_));
            if (e == cudaSuccess) {
                ck(cudaMemsetAsync(L.lab, 0, np_, s->st));  // SOLID halo
                ck(cudaMemsetAsync(L.code, 0, np_, s->st));
                ck(cudaMemsetAsync(L.x, 0, np_ * sizeof(float), s->st));
                ck(cudaMemsetAsync(L.b, 0, np_ * sizeof(float), s->st));
            }
        }
        if (s->mgL > 1) {
            ck(dalloc(&s->d_l1list, size_t(s->mg[1].W) * s->mg[1].H * s->mg[1].D));
            ck(dalloc(&s->d_l1n, 1));
        }
        ck(dalloc(&s->d_mgp, size_t(s->padded))); ck(dalloc(&s->d_mgq, size_t(s->padded)));
        ck(dalloc(&s->d_mgx, size_t(s->padded))); ck(dalloc(&s->d_mgr, size_t(s->padded)));
        for (double* a : {s->d_mgp, s->d_mgq, s->d_mgx, s->d_mgr})
            if (e == cudaSuccess) ck(cudaMemsetAsync(a, 0, sizeof(double) * size_t(s->padded), s->st));
    }
    if (e != cudaSuccess) { free_grid(s); return s->cuda_fail(e, "device allocation of the grid"); }
    for (float* a : {s->d_u, s->d_us}) ck(cudaMemsetAsync(a, 0, sizeof(float) * s->g.nu(), s->st));
    for (float* a : {s->d_v, s->d_vs}) ck(cudaMemsetAsync(a, 0, sizeof(float) * s->g.nv(), s->st));
    for (float* a : {s->d_w, s->d_ws}) ck(cudaMemsetAsync(a, 0, sizeof(float) * s->g.nw(), s->st));
    ck(cudaMemsetAsync(s->d_acc, 0, sizeof(float2) * (s->g.nu() + s->g.nv() + s->g.nw()), s->st));
    ck(cudaMemsetAsync(s->d_p, 0, sizeof(float) * nc, s->st));
    ck(cudaMemsetAsync(s->d_bodymark, 0, nc, s->st));
    for (int i = 0; i < 2; ++i) {
        ck(cudaMemsetAsync(pb.R[i], 0, pbytes, s->st)); ck(cudaMemsetAsync(pb.Wv[i], 0, pbytes, s->st));
        ck(cudaMemsetAsync(pb.S[i], 0, pbytes, s->st));
    }
    ck(cudaMemsetAsync(pb.invd, 0, pbytes, s->st));
    ck(cudaMemsetAsync(pb.xd, 0, sizeof(double) * size_t(s->padded), s->st));
    ck(cudaMemsetAsync(pb.bar, 0, sizeof(GridBar), s->st));
    // No FLUID list until the first pressure set-up: the count starts at 0, so
    // FP_GRID_RHS read before any step densifies nothing (an all-zero grid).
    ck(cudaMemsetAsync(pb.nf, 0, sizeof(int), s->st));
    if (e != cudaSuccess) { free_grid(s); return s->cuda_fail(e, "grid initialisation"); }
    s->have_grid = true;
    s->sorted = false;
    if (!s->learned_path.empty()) return load_net(s);
    return FP_OK;
}

int alloc_particles(fp_solver* s, int64_t n) {
    if (n <= s->cap) { s->np = n; return FP_OK; }
    free_particles(s);
    cudaError_t e = cudaSuccess;
    auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    ck(dalloc(&s->d_pos, n)); ck(dalloc(&s->d_vel, n)); ck(dalloc(&s->d_pos2, n)); ck(dalloc(&s->d_vel2, n));
    ck(dalloc(&s->d_key, n)); ck(dalloc(&s->d_rank, n)); ck(dalloc(&s->d_io, size_t(n) * 6));
    if (e != cudaSuccess) { free_particles(s); return s->cuda_fail(e, "device allocation of particles"); }
    s->cap = n;
    s->np = n;
    return FP_OK;
}

float3 gravity3() { return make_float3(kGravity[0], kGravity[1], kGravity[2]); }

bool body_on(const fp_solver* s) { return s->cfg.active_body && s->hb.loaded; }

BodyShape body_shape(const fp_solver* s) {
    const HostBody& h = s->hb;
    BodyShape b{};
    b.kind = h.kind;
    b.com = make_float3(float(h.pos[0]), float(h.pos[1]), float(h.pos[2]));
    b.radius = float(h.radius);
    for (int i = 0; i < 9; ++i) b.rot[i] = float(h.R[i]);
    b.local_com = make_float3(h.local_com[0], h.local_com[1], h.local_com[2]);
    b.origin = make_float3(h.origin[0], h.origin[1], h.origin[2]);
    b.cell = h.cell;
    b.nx = h.nx; b.ny = h.ny; b.nz = h.nz;
    b.sdf = s->d_sdf;
    return b;
}

// The rigid-body velocity field seen by the RHS and the projection.
BodyKin body_kin(const fp_solver* s) {
    BodyKin b{};
    b.active = 1;  // zero velocities unless a body is loaded or its state was set
    const HostBody& h = s->hb;
    b.vel = make_float3(float(h.vel[0]), float(h.vel[1]), float(h.vel[2]));
    b.omega = make_float3(float(h.omega[0]), float(h.omega[1]), float(h.omega[2]));
    b.com = make_float3(float(h.pos[0]), float(h.pos[1]), float(h.pos[2]));
    return b;
}

void fill_body_stats(fp_solver* s) {
    const HostBody& h = s->hb;
    for (int a = 0; a < 3; ++a) {
        s->stats.body_pos[a] = h.pos[a];
        s->stats.body_vel[a] = h.vel[a];
        s->stats.body_omega[a] = h.omega[a];
    }
    s->stats.body_angles[0] = h.theta; s->stats.body_angles[1] = h.psi; s->stats.body_angles[2] = h.phi;
}

// ---------------------------------------------------------------- phases
void phase_label(fp_solver* s) {
    s->launches += 5;  // bin, label tiles, tile scan, start tiles, scatter
    cudaMemsetAsync(s->d_counts, 0, sizeof(int) * (s->g.nc() + 1), s->st);
    if (body_on(s)) {
        launch_mark_body(s->d_bodymark, s->g, body_shape(s), s->st);  // MarkBodyCellsFunctor at the body's pose
        s->launches += 1;
    }
    launch_bin(s->d_pos, s->np, s->g, s->d_counts, s->d_key, s->d_rank, s->st);
    launch_label_scan(s->d_base, body_on(s) ? s->d_bodymark : nullptr, s->d_counts, s->d_labels, s->d_start,
                      s->d_tiles, s->g, s->st);
    launch_scatter(s->d_pos, s->d_vel, s->d_key, s->d_rank, s->d_start, s->np, s->d_pos2, s->d_vel2, s->st);
    std::swap(s->d_pos, s->d_pos2);
    std::swap(s->d_vel, s->d_vel2);
    s->sorted = true;
}

void phase_p2g(fp_solver* s, int fused) {
    if (!s->sorted) phase_label(s);
    s->launches += 4;
    launch_p2g(s->d_pos, s->d_vel, s->d_start, s->g, s->cfg.dt, gravity3(), s->d_acc, s->d_u, s->d_v, s->d_w,
               s->d_us, s->d_vs, s->d_ws, fused, s->st);
}

void phase_save(fp_solver* s) {
    s->launches += 3;
    launch_copy(s->d_u, s->d_us, s->g.nu(), s->st);
    launch_copy(s->d_v, s->d_vs, s->g.nv(), s->st);
    launch_copy(s->d_w, s->d_ws, s->g.nw(), s->st);
}

// Pressure solve of the system already set up in s->pb (fidx, diag, b); writes
// the dense solution to p_out and the diagnostics to s->stats.
//   FP_SOLVER_PCG       one FP64-vector PCG to tol (the FP64 path);
//   FP_SOLVER_PCG_MIXED FP64 iterative refinement: r = b - A x in FP64, an
//                       FP32-vector PCG solves A c = r loosely, x += c.
int solve_tail(fp_solver* s, int inner_total, int outer, int dev_status, float pcg_ms, float learned_ms,
               float guess_relres, int fallback);

// defer: for the plain PCG and MG solvers, queue the read-back of the solve's
// statistics behind ev[9] and return without waiting; solve_finalize then
// waits and fills them (one_step issues the projection and advection first).
int solve_system(fp_solver* s, float* p_out, bool defer = false) {
    PressureBufs& pb = s->pb;
    const double tol = s->cfg.tol;
    const int maxit = s->cfg.max_iters;
    int outer = 0, inner_total = 0;
    int dev_status = DEV_OK;
    float pcg_ms = 0.0f;
    cudaError_t ce;
    float learned_ms = 0.0f, guess_relres = 1.0f;
    int fallback = 0;
    if (s->cfg.solver == FP_SOLVER_PCG || s->cfg.solver == FP_SOLVER_PCG_MG ||
        s->cfg.solver == FP_SOLVER_PCG_LEARNED) {
        const bool learned = s->cfg.solver == FP_SOLVER_PCG_LEARNED;
        const bool mg = s->cfg.solver != FP_SOLVER_PCG;
        if (learned && !s->net) return s->fail(FP_ERR_STATE, "learned solver: no weights loaded (fp_load_learned)");
        if (mg) {
            s->launches += launch_mg_setup(s->d_labels, s->g, s->mg, s->mgL, s->d_l1list, s->d_l1n, s->st);
        }
        cudaEventRecord(s->ev_pcg[0], s->st);
        const float* x0 = nullptr;
        if (learned) {
            const unet::Lvl real{s->W, s->H, s->D};
            unet::launch_rhs_dense(pb.nf, pb.fidx, real, pb.b, s->d_rhs_dense, s->st);
            if (unet::forward_on(s->net, s->d_labels, s->d_rhs_dense, s->st))
                return s->cuda_fail(cudaGetLastError(), "U-Net forward");
            unet::launch_output_compact(pb.nf, pb.fidx, real, unet::net_level0(s->net), unet::net_out(s->net),
                                        unet::net_scal(s->net), s->d_x0c, s->st);
            s->launches += 1 + 16 + 1;  // rhs scatter, network (2 scale/input, 10 conv, 2 pool, 2 concat), guess
            cudaEventRecord(s->ev_net, s->st);
            x0 = s->d_x0c;
        }
        // A learned solve that has not converged after kLearnedMaxit iterations
        // counts as stalled and hands over to the plain PCG.
        constexpr int kLearnedMaxit = 300;
        int e = mg ? launch_pcg_mg(s->g, pb, s->mg, s->mgL, s->d_l1list, s->d_l1n, s->d_mgp, s->d_mgq, s->d_mgx,
                                   s->d_mgr, pb.b, tol, learned ? std::min(maxit, kLearnedMaxit) : maxit, s->st, x0,
                                   s->cfg.mg_sweeps > 0 ? s->cfg.mg_sweeps : 2,
                                   s->cfg.warm_start && p_out == s->d_p ? p_out : nullptr, p_out, s->wait_polls)
                   : launch_pcg(s->g, pb, pb.b, 1, tol, maxit, s->st, s->wait_polls);
        cudaEventRecord(s->ev_pcg[1], s->st);
        if (e) return s->cuda_fail(cudaError_t(e), "cooperative PCG launch");
        // FP64 solution to p, its true residual, then clear the work grids at
        // this solve's FLUID cells (the residual check leaves x in R[0]); the
        // MG kernel does all three itself
        auto finish_launch = [&](bool jacobi) {
            if (jacobi) {
                launch_scatter_p(pb, p_out, 1, s->g, s->st);
                launch_true_residual(pb, 1, s->g, s->st);
                launch_pcg_clear(pb, 1, 1, s->st);
                s->launches += 1 + 1 + 1 + 3 + 1;  // reset + pcg, scatter, residual (3), clear
            } else {
                s->launches += 1;  // the MG kernel
            }
            cudaMemcpyAsync(s->h_out, pb.out, kRbBytes, cudaMemcpyDeviceToHost, s->st);  // out, red and nf
        };
        auto finish = [&](bool jacobi) -> cudaError_t {
            finish_launch(jacobi);
            return cudaStreamSynchronize(s->st);
        };
        if (defer && !learned) {
            finish_launch(!mg);
            cudaEventRecord(s->ev[9], s->st);
            s->solve_pending = true;
            s->pending_guess = mg && s->cfg.warm_start && p_out == s->d_p;
            return FP_OK;
        }
        if (learned)
            cudaMemcpyAsync(s->h_bad, unet::net_status(s->net), sizeof(int), cudaMemcpyDeviceToHost, s->st);
        ce = finish(!mg);
        if (ce != cudaSuccess) return s->cuda_fail(ce, "pressure solve");
        if (learned && *s->h_bad) return s->fail(FP_ERR_TIMEOUT, "U-Net forward: a bounded tensor-core wait gave up");
        inner_total = s->h_out->iters;
        dev_status = s->h_out->status;
        outer = 1;
        cudaEventElapsedTime(&pcg_ms, s->ev_pcg[0], s->ev_pcg[1]);
        if (mg && (learned || (s->cfg.warm_start && p_out == s->d_p)))
            guess_relres = s->h_out->bb > 0 ? float(std::sqrt(s->h_out->rr0 / s->h_out->bb)) : 0.0f;
        if (learned) {
            cudaEventElapsedTime(&learned_ms, s->ev_pcg[0], s->ev_net);
            const double rel = s->h_red[1] > 0 ? std::sqrt(s->h_red[0] / s->h_red[1]) : 0.0;
            if (*s->h_nf > 0 && dev_status != DEV_TIMEOUT && (dev_status != DEV_OK || !(rel <= tol))) {
                // fallback: the plain FP64 PCG from x = 0
                fallback = 1;
                cudaEventRecord(s->ev_pcg[0], s->st);
                e = launch_pcg(s->g, pb, pb.b, 1, tol, maxit, s->st, s->wait_polls);
                cudaEventRecord(s->ev_pcg[1], s->st);
                if (e) return s->cuda_fail(cudaError_t(e), "cooperative PCG launch");
                ce = finish(true);
                if (ce != cudaSuccess) return s->cuda_fail(ce, "pressure solve (fallback)");
                inner_total += s->h_out->iters;
                dev_status = s->h_out->status;
                outer = 2;
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, s->ev_pcg[0], s->ev_pcg[1]);
                pcg_ms += ms;
            }
        }
    } else {
        // FP_SOLVER_PCG_MIXED, or FP_SOLVER_PCG_LEARNED_MIXED: the same
        // refinement started from the network's guess (energy-optimally scaled)
        const bool learned = s->cfg.solver == FP_SOLVER_PCG_LEARNED_MIXED;
        if (learned && !s->net) return s->fail(FP_ERR_STATE, "learned solver: no weights loaded (fp_load_learned)");
        cudaMemsetAsync(pb.x64, 0, sizeof(double) * s->g.nc(), s->st);
        if (learned) {
            cudaEventRecord(s->ev_pcg[0], s->st);
            const unet::Lvl real{s->W, s->H, s->D};
            unet::launch_rhs_dense(pb.nf, pb.fidx, real, pb.b, s->d_rhs_dense, s->st);
            if (unet::forward_on(s->net, s->d_labels, s->d_rhs_dense, s->st))
                return s->cuda_fail(cudaGetLastError(), "U-Net forward");
            unet::launch_output_compact(pb.nf, pb.fidx, real, unet::net_level0(s->net), unet::net_out(s->net),
                                        unet::net_scal(s->net), s->d_x0c, s->st);
            // x64 = xd = guess (xd is zero between solves), then scaled by (x, b) / (x, A x)
            cudaMemcpyAsync(pb.X, s->d_x0c, sizeof(float) * size_t(s->g.nc()), cudaMemcpyDeviceToDevice, s->st);
            launch_ir_update(pb, s->g, s->st);
            launch_guess_scale(pb, s->g, s->st);
            cudaEventRecord(s->ev_net, s->st);
            s->launches += 1 + 16 + 1 + 1 + 3;  // rhs scatter, network, guess, copy-in, scaling
            cudaMemcpyAsync(s->h_bad, unet::net_status(s->net), sizeof(int), cudaMemcpyDeviceToHost, s->st);
        }
        launch_ir_residual(pb, s->g, s->st);  // bin = b - A x64 (= b from x64 = 0)
        s->launches += 3;
        cudaMemcpyAsync(s->h_red, pb.red, sizeof(double) * 2, cudaMemcpyDeviceToHost, s->st);
        cudaMemcpyAsync(s->h_nf, pb.nf, sizeof(int), cudaMemcpyDeviceToHost, s->st);
        ce = cudaStreamSynchronize(s->st);
        if (ce != cudaSuccess) return s->cuda_fail(ce, "refinement residual");
        if (learned && *s->h_bad) return s->fail(FP_ERR_TIMEOUT, "U-Net forward: a bounded tensor-core wait gave up");
        if (learned) cudaEventElapsedTime(&learned_ms, s->ev_pcg[0], s->ev_net);
        const double bb = s->h_red[1];
        double relres = bb > 0 ? std::sqrt(s->h_red[0] / bb) : 0.0;
        if (learned) guess_relres = float(relres);
        while (relres > tol && outer < 12 && inner_total < maxit) {
            // Inner accuracy: enough to land below tol after this update, but
            // not below what FP32 vectors can resolve.
            const double inner_tol = std::min(0.1, std::max(2e-4, 0.5 * tol / relres));
            cudaEventRecord(s->ev_pcg[0], s->st);
            int e = launch_pcg(s->g, pb, pb.bin, 0, inner_tol, maxit - inner_total, s->st, s->wait_polls);
            cudaEventRecord(s->ev_pcg[1], s->st);
            if (e) return s->cuda_fail(cudaError_t(e), "cooperative PCG launch");
            launch_ir_update(pb, s->g, s->st);
            launch_pcg_clear(pb, 0, 0, s->st);
            launch_ir_residual(pb, s->g, s->st);
            s->launches += 2 + 1 + 1 + 2;  // reset + pcg, update, clear, residual (2)
            cudaMemcpyAsync(s->h_out, pb.out, sizeof(PcgOut), cudaMemcpyDeviceToHost, s->st);
            cudaMemcpyAsync(s->h_red, pb.red, sizeof(double) * 2, cudaMemcpyDeviceToHost, s->st);
            ce = cudaStreamSynchronize(s->st);
            if (ce != cudaSuccess) return s->cuda_fail(ce, "refinement step");
            inner_total += s->h_out->iters;
            ++outer;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, s->ev_pcg[0], s->ev_pcg[1]);
            pcg_ms += ms;
            if (s->h_out->status == DEV_TIMEOUT || s->h_out->status == DEV_NAN) { dev_status = s->h_out->status; break; }
            const double nr = bb > 0 ? std::sqrt(s->h_red[0] / bb) : 0.0;
            if (!(nr < relres)) { relres = nr; dev_status = DEV_BREAKDOWN; break; }  // refinement stalled
            relres = nr;
        }
        launch_pcg_clear(pb, 0, 1, s->st);  // 1/diag grid
        launch_scatter_p(pb, p_out, 2, s->g, s->st);
        s->launches += 2;
        s->h_red[0] = relres * relres * bb;
        s->h_red[1] = bb;
        if (relres > tol && dev_status == DEV_OK) dev_status = DEV_MAXIT;
        // xd must be zero at the start of the next solve
        cudaMemsetAsync(pb.xd, 0, sizeof(double) * size_t(s->padded), s->st);
        pcg_ms += learned_ms;
        if (learned && *s->h_nf > 0 && dev_status != DEV_TIMEOUT && dev_status != DEV_OK) {
            // the refinement from the learned guess stalled: plain FP64 PCG from zero
            fallback = 1;
            cudaEventRecord(s->ev_pcg[0], s->st);
            const int e = launch_pcg(s->g, pb, pb.b, 1, tol, maxit, s->st, s->wait_polls);
            cudaEventRecord(s->ev_pcg[1], s->st);
            if (e) return s->cuda_fail(cudaError_t(e), "cooperative PCG launch");
            launch_scatter_p(pb, p_out, 1, s->g, s->st);
            launch_true_residual(pb, 1, s->g, s->st);
            launch_pcg_clear(pb, 1, 1, s->st);
            s->launches += 1 + 1 + 1 + 3 + 1;
            cudaMemcpyAsync(s->h_out, pb.out, sizeof(PcgOut), cudaMemcpyDeviceToHost, s->st);
            cudaMemcpyAsync(s->h_red, pb.red, sizeof(double) * 2, cudaMemcpyDeviceToHost, s->st);
            ce = cudaStreamSynchronize(s->st);
            if (ce != cudaSuccess) return s->cuda_fail(ce, "pressure solve (fallback)");
            inner_total += s->h_out->iters;
            dev_status = s->h_out->status;
            ++outer;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, s->ev_pcg[0], s->ev_pcg[1]);
            pcg_ms += ms;
        }
    }
    return solve_tail(s, inner_total, outer, dev_status, pcg_ms, learned_ms, guess_relres, fallback);
}

// Waits for a deferred solve and fills its statistics and status.
int solve_finalize(fp_solver* s) {
    if (!s->solve_pending) return FP_OK;
    s->solve_pending = false;
    const cudaError_t ce = cudaEventSynchronize(s->ev[9]);
    if (ce != cudaSuccess) return s->cuda_fail(ce, "pressure solve");
    float pcg_ms = 0.0f;
    cudaEventElapsedTime(&pcg_ms, s->ev_pcg[0], s->ev_pcg[1]);
    const float guess = !s->pending_guess ? 1.0f
                        : (s->h_out->bb > 0 ? float(std::sqrt(s->h_out->rr0 / s->h_out->bb)) : 0.0f);
    return solve_tail(s, s->h_out->iters, 1, s->h_out->status, pcg_ms, 0.0f, guess, 0);
}

// The statistics and status of a finished solve (host copies of its results).
int solve_tail(fp_solver* s, int inner_total, int outer, int dev_status, float pcg_ms, float learned_ms,
               float guess_relres, int fallback) {
    s->pcg_ms = pcg_ms;
    s->stats.t_pcg = pcg_ms;
    s->stats.num_fluid_cells = *s->h_nf;
    s->stats.pcg_iters = inner_total;
    s->stats.outer_iters = outer;
    s->stats.fallback = fallback;
    s->stats.t_learned = learned_ms;
    s->stats.guess_relres = guess_relres;
    s->stats.residual = s->h_red[1] > 0 ? std::sqrt(s->h_red[0] / s->h_red[1]) : 0.0;
    int status = FP_OK;
    if (*s->h_nf == 0) status = FP_ERR_NO_FLUID;
    else if (dev_status == DEV_TIMEOUT) status = FP_ERR_TIMEOUT;
    else if (dev_status != DEV_OK) status = FP_ERR_SOLVER;
    s->stats.solve_status = status;
    if (status == FP_ERR_TIMEOUT && s->mgL > 0) {
        // a solve that gave up mid-way leaves the MG work grids and level-0
        // codes non-zero; restore the zero state the next solve relies on
        for (int l = 0; l < s->mgL; ++l) {
            const size_t np_ = size_t(s->mg[l].W + 2) * (s->mg[l].H + 2) * (s->mg[l].D + 2);
            cudaMemsetAsync(s->mg[l].x, 0, np_ * sizeof(float), s->st);
            cudaMemsetAsync(s->mg[l].b, 0, np_ * sizeof(float), s->st);
            cudaMemsetAsync(s->mg[l].code, 0, np_, s->st);
        }
        for (double* a : {s->d_mgp, s->d_mgq, s->d_mgx, s->d_mgr})
            cudaMemsetAsync(a, 0, sizeof(double) * size_t(s->padded), s->st);
    }
    if (status == FP_ERR_TIMEOUT) return s->fail(status, "PCG grid barrier timed out");
    if (dev_status == DEV_NAN) return s->fail(status, "PCG produced NaN");
    return FP_OK;  // no-fluid, breakdown and iteration cap are reported in stats; the step continues
}

int phase_pressure(fp_solver* s, bool defer = false) {
    s->launches += 3;  // fluid tiles, tile scan, fluid build
    BodyKin b = body_kin(s);
    launch_pressure_setup(s->d_labels, s->d_u, s->d_v, s->d_w, s->g, s->cfg.dt, b, nullptr, s->d_p, s->pb, s->st);
    return solve_system(s, s->d_p, defer);
}

// guarded: the kernel reads the solve's device status word and does nothing
// if that solve failed (one_step queues it before the status is known).
void phase_project(fp_solver* s, bool guarded = false) {
    BodyKin b = body_kin(s);
    s->launches += 1;
    launch_project(s->d_u, s->d_v, s->d_w, s->d_p, s->d_labels, s->g, s->cfg.dt, b, s->st,
                   guarded ? &s->pb.out->status : nullptr);
}

// updateBody (FluidSolver3D.cu:2793-2846): fluid force and torque from the
// pressure (FP64 reduction on the GPU), gravity m*g, then integrate.
// The SDF voxel grid of the body for the reference's buoyancy and surface
// points: the file's grid, or the analytic sphere sampled on a grid of
// spacing dx / 2 centred on its centre of mass (local_com = 0).
RefBuoyancy ref_voxels(const fp_solver* s) {
    const HostBody& h = s->hb;
    RefBuoyancy b{};
    b.com = make_float3(float(h.pos[0]), float(h.pos[1]), float(h.pos[2]));
    for (int i = 0; i < 9; ++i) b.rot[i] = float(h.R[i]);
    if (h.kind == BODY_SDF) {
        b.sdf = s->d_sdf;
        b.sw = h.nx; b.sh = h.ny; b.sd = h.nz;
        b.cs = h.cell;
        b.origin = make_float3(h.origin[0], h.origin[1], h.origin[2]);
        b.local_com = make_float3(h.local_com[0], h.local_com[1], h.local_com[2]);
    } else {
        b.sdf = nullptr;
        b.cs = 0.5f * s->cfg.dx;
        const int n = int(std::ceil(2.0 * (h.radius + 2.0 * b.cs) / b.cs));
        b.sw = b.sh = b.sd = n;
        const float o = -0.5f * float(n) * b.cs;
        b.origin = make_float3(o, o, o);
        b.local_com = make_float3(0.0f, 0.0f, 0.0f);
        b.radius = float(h.radius);
    }
    return b;
}

// generateSurfacePoints(0.5 dx) (utility.cuh:339-374): voxel corners with
// |sdf| < dx / 2, rotated about the local centre of mass into the world.
void body_surface_points(const fp_solver* s, std::vector<float>& pts) {
    pts.clear();
    const HostBody& h = s->hb;
    const RefBuoyancy b = ref_voxels(s);
    const float lim = 0.5f * s->cfg.dx;
    for (int k = 0; k < b.sd; ++k)
        for (int j = 0; j < b.sh; ++j)
            for (int i = 0; i < b.sw; ++i) {
                const float plx = b.origin.x + float(i) * b.cs, ply = b.origin.y + float(j) * b.cs,
                            plz = b.origin.z + float(k) * b.cs;
                const float cx = plx - b.local_com.x, cy = ply - b.local_com.y, cz = plz - b.local_com.z;
                float sdf;
                if (h.kind == BODY_SDF) sdf = h.sdf_host[size_t(i) + size_t(j) * b.sw + size_t(k) * b.sw * b.sh];
                else sdf = std::sqrt((cx * cx + cy * cy) + cz * cz) - b.radius;
                if (!(std::fabs(sdf) < lim)) continue;
                pts.push_back(b.com.x + ((b.rot[0] * cx + b.rot[1] * cy) + b.rot[2] * cz));
                pts.push_back(b.com.y + ((b.rot[3] * cx + b.rot[4] * cy) + b.rot[5] * cz));
                pts.push_back(b.com.z + ((b.rot[6] * cx + b.rot[7] * cy) + b.rot[8] * cz));
            }
}

int phase_body(fp_solver* s) {
    if (!body_on(s)) return FP_OK;
    if (s->cfg.body_forces == FP_BODY_FORCES_REFERENCE && s->hb.kind != BODY_PADDLE) {
        // updateBody (FluidSolver3D.cu:2793-2846): F = m g + panel drag/lift,
        // then applyBuoyancy adds -rho V_submerged g; the panel torque only.
        HostBody& h = s->hb;
        if (!s->sorted) phase_label(s);  // the buoyancy searches the cell-sorted particles
        const float3 cm = make_float3(float(h.pos[0]), float(h.pos[1]), float(h.pos[2]));
        const float3 bv = make_float3(float(h.vel[0]), float(h.vel[1]), float(h.vel[2]));
        launch_ref_body_forces(s->d_labels, s->d_u, s->d_v, s->d_w, s->g, cm, bv, ref_voxels(s), s->d_pos, s->d_start,
                               s->d_bpart, s->d_bforce, s->st);
        s->launches += 4;
        cudaMemcpyAsync(s->h_bforce, s->d_bforce, sizeof(double) * 8, cudaMemcpyDeviceToHost, s->st);
        cudaError_t e = cudaStreamSynchronize(s->st);
        if (e != cudaSuccess) return s->cuda_fail(e, "reference body forces");
        const double buoy = 1000.0 * s->h_bforce[7] * -double(kGravity[1]);
        for (int a = 0; a < 3; ++a) {
            h.force[a] = h.mass * double(kGravity[a]) + s->h_bforce[a] + (a == 1 ? buoy : 0.0);
            h.torque[a] = s->h_bforce[3 + a];
            s->stats.body_force[a] = h.force[a];
            s->stats.body_torque[a] = h.torque[a];
        }
        h.integrate(double(s->cfg.dt));
        fill_body_stats(s);
        return FP_OK;
    }
    launch_body_force(s->d_p, s->d_labels, s->g, body_shape(s), s->d_bpart, s->d_bforce, s->st);
    s->launches += 2;
    cudaMemcpyAsync(s->h_bforce, s->d_bforce, sizeof(double) * 6, cudaMemcpyDeviceToHost, s->st);
    cudaError_t e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "body force");
    HostBody& h = s->hb;
    for (int a = 0; a < 3; ++a) {
        h.force[a] = h.mass * double(kGravity[a]) + s->h_bforce[a];
        h.torque[a] = s->h_bforce[3 + a];
        s->stats.body_force[a] = h.force[a];
        s->stats.body_torque[a] = h.torque[a];
    }
    if (h.kind == BODY_PADDLE) {  // prescribed motion; the force is the fluid's load on the paddle
        for (int a = 0; a < 3; ++a) s->stats.body_force[a] = h.force[a] = s->h_bforce[a];
        h.pad_t += double(s->cfg.dt);
        h.paddle_at(h.pad_t);
    } else {
        h.integrate(double(s->cfg.dt));
    }
    fill_body_stats(s);
    return FP_OK;
}

void phase_g2p_advect(fp_solver* s, int do_g2p, int do_adv, bool guarded = false) {
    s->launches += 1;
    const bool sdf = s->cfg.collision == FP_COLLISION_SDF && body_on(s);
    const BodyShape b = sdf ? body_shape(s) : BodyShape{};
    launch_g2p_advect(s->d_pos, s->d_vel, s->np, s->d_u, s->d_v, s->d_w, s->d_us, s->d_vs, s->d_ws, s->d_labels, s->g,
                      s->cfg.pic_weight, s->cfg.dt, s->cfg.cfl, do_g2p, do_adv, s->cfg.advection == FP_ADVECT_RK2,
                      s->st, guarded ? &s->pb.out->status : nullptr, sdf ? &b : nullptr);
    if (do_adv) s->sorted = false;
}

// ---------------------------------------------------------------- extrapolation
int ext_alloc(fp_solver* s) {
    if (s->d_extmark) return FP_OK;
    const int64_t n = std::max({s->g.nu(), s->g.nv(), s->g.nw()});
    cudaError_t e = dalloc(&s->d_extmark, size_t(n));
    if (e != cudaSuccess) return s->cuda_fail(e, "device allocation of the extrapolation markers");
    return FP_OK;
}

// The 2D step's first commented-out call (after P2G, depth 2) or second one
// (after G2P, depth W for u and H for v).  checkNeighbors reads at stride W.
int r2_extrapolate(fp_solver* s, bool after_g2p) {
    int rc = ext_alloc(s);
    if (rc) return rc;
    s->launches += launch_extrapolate_unknown(s->d_u, s->W + 1, s->H, after_g2p ? s->W : 2, s->W, s->d_extmark, s->st);
    s->launches += launch_extrapolate_unknown(s->d_v, s->W, s->H + 1, after_g2p ? s->H : 2, s->W, s->d_extmark, s->st);
    return FP_OK;
}

// Default scheme: cfg.extrapolate layers into faces with no FLUID side.
int extrapolate_3d(fp_solver* s) {
    int rc = ext_alloc(s);
    if (rc) return rc;
    float* comp[3] = {s->d_u, s->d_v, s->d_w};
    for (int a = 0; a < (s->D > 1 ? 3 : 2); ++a)
        s->launches += launch_extrapolate_from_fluid(comp[a], a, s->d_labels, s->g, s->cfg.extrapolate, s->d_extmark,
                                                     s->st);
    return FP_OK;
}

// ---------------------------------------------------------------- scheme ref2d
// FluidSolver2D.cu's own step (kernels_ref2d.cu); particles stay in order.
bool ref2d(const fp_solver* s) { return s->cfg.scheme == FP_SCHEME_REF2D; }

int r2_alloc(fp_solver* s) {
    const int nb = (s->W + 4) * (s->H + 4);
    cudaError_t e = cudaSuccess;
    if (s->r2_nb != nb) {
        free_r2(s);
        e = dalloc(&s->r2.start, size_t(nb) + 1);
        if (e == cudaSuccess) e = dalloc(&s->r2.misc, size_t(4));
        if (e != cudaSuccess) { free_r2(s); return s->cuda_fail(e, "device allocation of the 2D bins"); }
        s->r2_nb = nb;
    }
    if (s->r2_cap < s->cap || !s->r2.list) {
        dfree(s->r2.list); dfree(s->r2.keep);
        const int64_t n = std::max<int64_t>(s->cap, 1);
        e = dalloc(&s->r2.list, size_t(n));
        if (e == cudaSuccess) e = dalloc(&s->r2.keep, size_t(n) + 1);
        if (e != cudaSuccess) return s->cuda_fail(e, "device allocation of the 2D particle lists");
        s->r2_cap = n;
    }
    s->r2.key = s->d_key;
    s->r2.rank = s->d_rank;
    return FP_OK;
}

void r2_label(fp_solver* s) {
    launch_r2_label(s->d_base, s->d_labels, s->d_pos, s->np, s->g, s->cfg.dx, s->st);
    s->launches += s->np > 0 ? 2 : 1;
}

void r2_p2g(fp_solver* s, int mode) {
    launch_r2_p2g(s->d_pos, s->d_vel, s->np, s->g, s->cfg.dx, s->cfg.dt, mode, s->r2, s->d_u, s->d_v, s->d_us, s->d_vs,
                  s->st);
    s->launches += s->np > 0 ? 5 : 3;
}

int r2_pressure(fp_solver* s) {
    // the 2D system has no w faces: keep the depth-1 w grid at zero
    cudaMemsetAsync(s->d_w, 0, sizeof(float) * s->g.nw(), s->st);
    return phase_pressure(s);
}

void r2_project(fp_solver* s) {
    launch_r2_project(s->d_u, s->d_v, s->d_p, s->d_labels, s->g, s->cfg.dx, s->cfg.dt, s->st);
    s->launches += 1;
}

void r2_particles(fp_solver* s, int flags) {
    if (s->np == 0) return;
    launch_r2_particles(s->d_pos, s->d_vel, s->np, s->d_u, s->d_v, s->d_us, s->d_vs, s->d_labels, s->g, s->cfg.dx,
                        s->cfg.dt, s->cfg.pic_weight, flags, s->r2, s->st);
    s->launches += 1;
}

// After r2_particles with the clean-up flag: drop deleted particles (order
// kept), read the new count and the capped-loop count.
int r2_compact(fp_solver* s, bool advected) {
    if (s->np == 0) return FP_OK;
    launch_r2_compact(s->d_pos, s->d_vel, s->np, s->r2, s->d_pos2, s->d_vel2, s->st);
    s->launches += 2;
    cudaMemcpyAsync(s->h_r2, s->r2.keep + s->np, sizeof(int), cudaMemcpyDeviceToHost, s->st);
    if (advected) cudaMemcpyAsync(s->h_r2 + 1, s->r2.misc + 2, sizeof(int), cudaMemcpyDeviceToHost, s->st);
    cudaError_t e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "2D particle clean-up");
    std::swap(s->d_pos, s->d_pos2);
    std::swap(s->d_vel, s->d_vel2);
    s->stats.particles_removed = s->np - s->h_r2[0];
    if (advected) s->stats.advect_capped = s->h_r2[1];
    s->np = s->h_r2[0];
    return FP_OK;
}

// frameStep, FluidSolver2D.cu:1302-1331
int one_step_ref2d(fp_solver* s) {
    int rc = r2_alloc(s);
    if (rc) return rc;
    cudaEventRecord(s->ev[0], s->st);
    r2_label(s);
    cudaEventRecord(s->ev[1], s->st);
    const bool ext = s->cfg.extrapolate != 0;
    if (ext) {  // P2G, extrapolation, save, forces
        r2_p2g(s, 0);
        rc = r2_extrapolate(s, false);
        if (rc) return rc;
        phase_save(s);
        launch_r2_forces(s->d_u, s->d_v, s->g, s->cfg.dt, s->st);
        s->launches += 1;
    } else {
        r2_p2g(s, 1);  // P2G + save + forces
    }
    cudaEventRecord(s->ev[2], s->st);
    rc = r2_pressure(s);
    cudaEventRecord(s->ev[3], s->st);
    if (rc != FP_OK) return rc;
    r2_project(s);
    cudaEventRecord(s->ev[4], s->st);
    if (ext) {  // G2P, extrapolation, then advection and clean-up
        r2_particles(s, 1);
        rc = r2_extrapolate(s, true);
        if (rc) return rc;
        r2_particles(s, 6);
    } else {
        r2_particles(s, 7);  // G2P, advection, clean-up
    }
    cudaEventRecord(s->ev[5], s->st);
    rc = r2_compact(s, true);
    if (rc != FP_OK) return rc;
    float t[5];
    for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&t[i], s->ev[i], s->ev[i + 1]);
    s->stats.t_label = t[0];
    s->stats.t_p2g = t[1];
    s->stats.t_forces = 0.0f;
    s->stats.t_pressure = t[2];
    s->stats.t_project = t[3];
    s->stats.t_body = 0.0f;
    s->stats.t_g2p = 0.0f;
    s->stats.t_advect = t[4];
    cudaEventElapsedTime(&s->stats.t_total, s->ev[0], s->ev[5]);
    ++s->steps;
    s->stats.step = s->steps;
    s->stats.num_particles = s->np;
    s->stats.kernel_launches = s->launches;
    return FP_OK;
}

int check_ready(fp_solver* s) {
    if (!s) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "labels not loaded");
    if (s->W < 2 || s->H < 2) return s->fail(FP_ERR_ARG, "grid must be at least 2 cells wide and high");
    if (s->cfg.dim == 3 && s->D < 2) return s->fail(FP_ERR_ARG, "a 3D grid needs at least 2 cells in depth");
    if (s->cfg.dim == 2 && s->D != 1) return s->fail(FP_ERR_ARG, "a 2D grid has depth 1");
    return FP_OK;
}

// finish: wait for the step and fill its phase timers.  fp_step skips that for
// all but the last of its steps, so the host goes on issuing the next step
// while the GPU completes this one (the solve's own read-back still waits).
int one_step(fp_solver* s, bool finish = true) {
    NvtxRange step_range("fp_step");
    if (ref2d(s)) return one_step_ref2d(s);
    cudaEventRecord(s->ev[0], s->st);
    { NvtxRange r("label"); phase_label(s); }
    cudaEventRecord(s->ev[1], s->st);
    { NvtxRange r("p2g+save+forces"); phase_p2g(s, 1); }  // P2G + save + forces
    cudaEventRecord(s->ev[2], s->st);
    cudaEventRecord(s->ev[3], s->st);
    // The solve's statistics are read back only after the projection and
    // advection are issued (solve_finalize), so the GPU does not idle while
    // the host reads them; a failed solve is still reported by this call.
    // The projection and G2P/advection kernels read the solve's device status
    // and do nothing if it timed out or produced NaN, so such a step leaves
    // the particles as they were; a body is integrated only after a good solve.
    int rc;
    { NvtxRange r("pressure"); rc = phase_pressure(s, true); }
    cudaEventRecord(s->ev[4], s->st);
    auto fail_after = [&](int rc0) { const int r = solve_finalize(s); return rc0 != FP_OK ? rc0 : r; };
    if (rc != FP_OK) return fail_after(rc);
    { NvtxRange r("project"); phase_project(s, true); }
    cudaEventRecord(s->ev[5], s->st);
    if (body_on(s)) {
        // the body phase waits for its own force anyway; finish the solve first
        rc = solve_finalize(s);
        if (rc != FP_OK) return rc;
    }
    { NvtxRange r("body"); rc = phase_body(s); }
    if (rc != FP_OK) return fail_after(rc);
    cudaEventRecord(s->ev[6], s->st);
    cudaEventRecord(s->ev[7], s->st);
    NvtxRange adv_range("g2p+advect");
    if (s->cfg.extrapolate > 0) {
        phase_g2p_advect(s, 1, 0, true);
        rc = extrapolate_3d(s);
        if (rc != FP_OK) return fail_after(rc);
        phase_g2p_advect(s, 0, 1, true);
    } else {
        phase_g2p_advect(s, 1, 1, true);
    }
    cudaEventRecord(s->ev[8], s->st);
    rc = solve_finalize(s);
    if (rc != FP_OK) return rc;
    ++s->steps;
    s->stats.step = s->steps;
    s->stats.num_particles = s->np;
    s->stats.kernel_launches = s->launches;
    if (!finish) return FP_OK;
    cudaError_t e = cudaEventSynchronize(s->ev[8]);
    if (e != cudaSuccess) return s->cuda_fail(e, "step");
    float t[8];
    for (int i = 0; i < 8; ++i) cudaEventElapsedTime(&t[i], s->ev[i], s->ev[i + 1]);
    s->stats.t_label = t[0];
    s->stats.t_p2g = t[1];
    s->stats.t_forces = t[2];
    s->stats.t_pressure = t[3];
    s->stats.t_project = t[4];
    s->stats.t_body = t[5] + t[6];
    s->stats.t_g2p = 0.0f;
    s->stats.t_advect = t[7];
    cudaEventElapsedTime(&s->stats.t_total, s->ev[0], s->ev[8]);
    return FP_OK;
}

// One JSON line of the last step's statistics to the step log.
void write_step_log(fp_solver* s) {
    if (!s->step_log) return;
    const fp_step_stats& t = s->stats;
    std::fprintf(s->step_log,
                 "{\"step\": %lld, \"particles\": %lld, \"fluid_cells\": %d, \"pcg_iters\": %d, \"outer_iters\": %d, "
                 "\"residual\": %.9g, \"solve_status\": %d, \"fallback\": %d, \"guess_relres\": %.6g, "
                 "\"t_label\": %.6g, \"t_p2g\": %.6g, \"t_pressure\": %.6g, \"t_pcg\": %.6g, \"t_learned\": %.6g, "
                 "\"t_project\": %.6g, \"t_body\": %.6g, \"t_advect\": %.6g, \"t_total\": %.6g, "
                 "\"body_pos\": [%.9g, %.9g, %.9g], \"body_vel\": [%.9g, %.9g, %.9g], \"kernel_launches\": %lld}\n",
                 (long long)t.step, (long long)t.num_particles, t.num_fluid_cells, t.pcg_iters, t.outer_iters,
                 t.residual, t.solve_status, t.fallback, double(t.guess_relres), double(t.t_label), double(t.t_p2g),
                 double(t.t_pressure), double(t.t_pcg), double(t.t_learned), double(t.t_project), double(t.t_body),
                 double(t.t_advect), double(t.t_total), t.body_pos[0], t.body_pos[1], t.body_pos[2], t.body_vel[0],
                 t.body_vel[1], t.body_vel[2], (long long)s->launches);
    std::fflush(s->step_log);
}

// Binary state file (fp_save_state / fp_load_state): host-order values in
// the order written; ok turns false on any short read or write.
constexpr char kStateMagic[8] = {'F', 'P', 'S', 'T', 'A', 'T', 'E', '1'};

struct StateFile {
    FILE* f = nullptr;
    bool ok = true;
    ~StateFile() { if (f) std::fclose(f); }
    template <class T>
    void put(const T* p, size_t n) { if (ok && n && std::fwrite(p, sizeof(T), n, f) != n) ok = false; }
    template <class T>
    void put(const T& v) { put(&v, 1); }
    template <class T>
    void get(T* p, size_t n) { if (ok && n && std::fread(p, sizeof(T), n, f) != n) ok = false; }
    template <class T>
    void get(T& v) { get(&v, 1); }
};

std::string frame_dir(const std::string& tmpl) {
    size_t p = tmpl.find_last_of('/');
    return p == std::string::npos ? std::string(".") : tmpl.substr(0, p);
}

}  // namespace

// ======================================================================== C ABI
extern "C" {

const char* fp_version(void) { return "fluidprjct_b200 0.1 (sm_100a)"; }

int fp_read_label_file(const char* path, int dim, int* dims, uint8_t* out) {
    if (!path || !dims || (dim != 2 && dim != 3)) return FP_ERR_ARG;
    std::vector<uint8_t> lab;
    std::string err;
    int W = 0, H = 0, D = 1;
    bool ok = dim == 2 ? io::read_labels2d(path, W, H, lab, err) : io::read_labels3d(path, W, H, D, lab, err);
    if (!ok) {
        std::fprintf(stderr, "fp_read_label_file: %s\n", err.c_str());
        return FP_ERR_IO;
    }
    dims[0] = W; dims[1] = H; dims[2] = D;
    if (out) std::memcpy(out, lab.data(), lab.size());
    return FP_OK;
}

int fp_read_levelset_file(const char* path, int* dims, float* out) {
    if (!path || !dims) return FP_ERR_ARG;
    std::vector<float> v;
    std::string err;
    char kind = 0;
    int W = 0, H = 0;
    if (!io::read_levelset2d(path, kind, W, H, v, err)) {
        std::fprintf(stderr, "fp_read_levelset_file: %s\n", err.c_str());
        return FP_ERR_IO;
    }
    dims[0] = W; dims[1] = H;
    if (out) std::memcpy(out, v.data(), sizeof(float) * v.size());
    return FP_OK;
}

int fp_write_particle_file(const char* path, const float* pos, const float* vel, int64_t n, int format) {
    if (!path || n < 0 || (n > 0 && !pos) || format < FP_OUT_PLY || format > FP_OUT_NONE) return FP_ERR_ARG;
    std::string err;
    if (!io::write_particles(path, pos, vel, n, format, err)) {
        std::fprintf(stderr, "fp_write_particle_file: %s\n", err.c_str());
        return FP_ERR_IO;
    }
    return FP_OK;
}

int fp_read_ply_file(const char* path, int64_t* n, float* pos, float* vel, int* has_vel) {
    if (!path || !n) return FP_ERR_ARG;
    std::vector<float> p, v;
    bool hv = false;
    std::string err;
    if (!io::read_ply(path, p, v, hv, err)) {
        std::fprintf(stderr, "fp_read_ply_file: %s\n", err.c_str());
        return FP_ERR_IO;
    }
    *n = int64_t(p.size() / 3);
    if (has_vel) *has_vel = hv ? 1 : 0;
    if (pos) std::memcpy(pos, p.data(), p.size() * sizeof(float));
    if (vel && hv) std::memcpy(vel, v.data(), v.size() * sizeof(float));
    return FP_OK;
}

int fp_config_default(fp_config* c) {
    if (!c) return FP_ERR_ARG;
    std::memset(c, 0, sizeof *c);
    c->dim = 3;
    c->dx = 0.1f;            // main.cpp:19
    c->dt = 0.02f;           // main.cpp:18
    c->pic_weight = 0.01f;   // main.cpp:23
    c->iter_per_frame = 1;   // main.cpp:24
    c->output_format = FP_OUT_PLY;
    std::snprintf(c->output_template, sizeof c->output_template, "%s", "InputData/particles_");  // main.cpp:33
    c->active_body = 0;
    c->body_pos[0] = c->body_pos[1] = c->body_pos[2] = 0.5f;  // main.cpp:44-46
    c->body_mass = 50.0f;    // main.cpp:48
    c->ppc = 4;              // FluidSolver3D.cuh:71
    c->seed = 0;
    c->solver = FP_SOLVER_PCG;
    c->advection = FP_ADVECT_RK3REF;
    c->cfl = 0.1f;           // FluidSolver3D.cu:3092
    c->tol = 1e-6;
    c->max_iters = 20000;
    c->body_radius = 0.0f;
    c->body_density = 0.5f;
    c->device = -1;
    c->warm_start = 1;
    c->collision = FP_COLLISION_LABELS;
    std::snprintf(c->body_sdf, sizeof c->body_sdf, "%s", "InputData/ball.sdf");  // FluidSolver3D.cu:158
    return FP_OK;
}

int fp_config_load_json(const char* path, fp_config* cfg, char* label_path, size_t label_path_len, int* frames) {
    if (!path || !cfg) return FP_ERR_ARG;
    std::string lp, err;
    if (!io::load_config_json(path, *cfg, &lp, frames, err)) {
        std::fprintf(stderr, "fp_config_load_json: %s\n", err.c_str());
        return FP_ERR_IO;
    }
    if (label_path && label_path_len) std::snprintf(label_path, label_path_len, "%s", lp.c_str());
    return FP_OK;
}

int fp_create(const fp_config* cfg, fp_solver** out) {
    if (!out) return FP_ERR_ARG;
    *out = nullptr;
    auto* s = new (std::nothrow) fp_solver();
    if (!s) return FP_ERR_ARG;
    if (cfg) s->cfg = *cfg; else fp_config_default(&s->cfg);
    if (!(s->cfg.dx > 0) || !(s->cfg.dt > 0) || (s->cfg.dim != 2 && s->cfg.dim != 3)) { delete s; return FP_ERR_ARG; }
    if (s->cfg.solver < FP_SOLVER_PCG || s->cfg.solver > FP_SOLVER_PCG_LEARNED_MIXED) {
        std::fprintf(stderr, "fp_create: solver %d is not available in this build\n", s->cfg.solver);
        delete s;
        return FP_ERR_ARG;
    }
    if (s->cfg.extrapolate < 0 ||
        (s->cfg.body_forces != FP_BODY_FORCES_FACE_FRACTION && s->cfg.body_forces != FP_BODY_FORCES_REFERENCE)) {
        delete s;
        return FP_ERR_ARG;
    }
    if (s->cfg.collision != FP_COLLISION_LABELS && s->cfg.collision != FP_COLLISION_SDF) {
        delete s;
        return FP_ERR_ARG;
    }
    if ((s->cfg.scheme != FP_SCHEME_DEFAULT && s->cfg.scheme != FP_SCHEME_REF2D) ||
        (s->cfg.scheme == FP_SCHEME_REF2D && s->cfg.dim != 2)) {
        std::fprintf(stderr, "fp_create: scheme %d with dim %d\n", s->cfg.scheme, s->cfg.dim);
        delete s;
        return FP_ERR_ARG;
    }
    cudaError_t e = cudaSuccess;
    if (s->cfg.device >= 0) e = cudaSetDevice(s->cfg.device);  // the calling thread's device from here on
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    for (auto& ev : s->ev) if (e == cudaSuccess) e = cudaEventCreate(&ev);
    for (auto& ev : s->ev_pcg) if (e == cudaSuccess) e = cudaEventCreate(&ev);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_net);
    if (e == cudaSuccess) {
        void* rb = nullptr;
        e = cudaMallocHost(&rb, kRbBytes);
        if (e == cudaSuccess) readback_views(rb, s->h_out, s->h_red, s->h_nf);
    }
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_bad, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_bad, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_bforce, sizeof(double) * 8);
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_r2, sizeof(int) * 2);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "fp_create: %s\n", cudaGetErrorString(e));
        fp_destroy(s);
        return FP_ERR_CUDA;
    }
    *out = s;
    return FP_OK;
}

int fp_destroy(fp_solver* s) {
    if (!s) return FP_OK;
    if (s->step_log) std::fclose(s->step_log);
    if (s->st) cudaStreamSynchronize(s->st);
    free_grid(s);
    free_particles(s);
    free_body(s);
    if (s->h_bforce) cudaFreeHost(s->h_bforce);
    if (s->h_r2) cudaFreeHost(s->h_r2);
    for (auto& ev : s->ev) if (ev) cudaEventDestroy(ev);
    for (auto& ev : s->ev_pcg) if (ev) cudaEventDestroy(ev);
    if (s->ev_net) cudaEventDestroy(s->ev_net);
    if (s->h_out) cudaFreeHost(s->h_out);  // h_red and h_nf lie inside it
    if (s->h_bad) cudaFreeHost(s->h_bad);
    if (s->d_bad) cudaFree(s->d_bad);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
    return FP_OK;
}

const char* fp_last_error(const fp_solver* s) { return s ? s->err.c_str() : "null solver"; }

int fp_set_labels(fp_solver* s, const uint8_t* labels, int W, int H, int D) {
    if (!s || !labels || W <= 0 || H <= 0 || D <= 0) return s ? s->fail(FP_ERR_ARG, "bad labels") : FP_ERR_ARG;
    const int64_t nc = int64_t(W) * H * D;
    for (int64_t c = 0; c < nc; ++c)
        if (labels[c] > FP_BODY) return s->fail(FP_ERR_ARG, "label value out of range at cell " + std::to_string(c));
    int rc = alloc_grid(s, W, H, D);
    if (rc) return rc;
    // The SOLID map is fixed for the run; BODY cells of an input are re-derived
    // from the body every step, other non-SOLID cells from the particles.
    std::vector<uint8_t> base(labels, labels + nc);
    for (auto& l : base) if (l == FP_BODY) l = FP_AIR;
    cudaError_t e = cudaMemcpyAsync(s->d_base, base.data(), size_t(nc), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_labels, labels, size_t(nc), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "label upload");
    return FP_OK;
}

// Labels already in s->d_labels (no BODY cells): the SOLID map becomes the base.
static int labels_from_device(fp_solver* s) {
    cudaError_t e = cudaMemcpyAsync(s->d_base, s->d_labels, size_t(s->g.nc()), cudaMemcpyDeviceToDevice, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "scene labels");
    return FP_OK;
}

int fp_set_labels_from_levelsets(fp_solver* s, const float* solid, const float* fluid, int W, int H, int D) {
    if (!s || !solid || !fluid || W <= 0 || H <= 0 || D <= 0)
        return s ? s->fail(FP_ERR_ARG, "bad level sets") : FP_ERR_ARG;
    int rc = alloc_grid(s, W, H, D);
    if (rc) return rc;
    const int64_t nc = int64_t(W) * H * D;
    float *ds = nullptr, *df = nullptr;
    cudaError_t e = dalloc(&ds, size_t(nc));
    if (e == cudaSuccess) e = dalloc(&df, size_t(nc));
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, solid, sizeof(float) * nc, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(df, fluid, sizeof(float) * nc, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) {
        launch_levelset_labels(ds, df, nc, s->d_labels, s->st);
        s->launches += 1;
        e = cudaStreamSynchronize(s->st);
    }
    dfree(ds);
    dfree(df);
    if (e != cudaSuccess) return s->cuda_fail(e, "level-set labels");
    return labels_from_device(s);
}

int fp_scene_seabed(fp_solver* s, int W, int H, int D, float level, float bed_base, float bed_amp, uint32_t seed,
                    float water_xmin) {
    if (!s || W < 3 || H < 3 || D < 3) return s ? s->fail(FP_ERR_ARG, "seabed grid too small") : FP_ERR_ARG;
    int rc = alloc_grid(s, W, H, D);
    if (rc) return rc;
    launch_seabed_labels(s->d_labels, W, H, D, double(s->cfg.dx), double(level), double(bed_base), double(bed_amp),
                         uint64_t(seed), double(water_xmin), s->st);
    s->launches += 1;
    return labels_from_device(s);
}

int fp_load_labels(fp_solver* s, const char* path) {
    if (!s || !path) return FP_ERR_ARG;
    std::vector<uint8_t> lab;
    int W, H, D = 1;
    bool ok = s->cfg.dim == 2 ? io::read_labels2d(path, W, H, lab, s->err) : io::read_labels3d(path, W, H, D, lab, s->err);
    if (!ok) return FP_ERR_IO;
    return fp_set_labels(s, lab.data(), W, H, D);
}

int fp_get_dims(const fp_solver* s, int* W, int* H, int* D) {
    if (!s) return FP_ERR_ARG;
    if (W) *W = s->W;
    if (H) *H = s->H;
    if (D) *D = s->D;
    return FP_OK;
}

int fp_load_sdf(fp_solver* s, const char* path) {
    if (!s) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "labels must be loaded before the body");
    free_body(s);
    HostBody& h = s->hb;
    h = HostBody();
    const double pi = 3.14159265358979323846;
    std::vector<float> data;
    if (!path) {
        if (!(s->cfg.body_radius > 0.0f)) return s->fail(FP_ERR_ARG, "analytic body needs body_radius > 0");
        h.kind = BODY_SPHERE;
        h.radius = s->cfg.body_radius;
        const double vol = 4.0 / 3.0 * pi * h.radius * h.radius * h.radius;
        h.mass = s->cfg.body_density > 0.0f ? double(s->cfg.body_density) * 1000.0 * vol : double(s->cfg.body_mass);
    } else {
        // RigidBody::loadSDF (utility.cuh:231-338): the SDF box is centred on
        // the initial position; local centre of mass = box centre.
        int w, hh, d;
        float org[3], cell;
        if (!io::read_sdf(path, w, hh, d, org, cell, data, s->err)) return FP_ERR_IO;
        h.kind = BODY_SDF;
        h.nx = w; h.ny = hh; h.nz = d; h.cell = cell;
        for (int a = 0; a < 3; ++a) h.origin[a] = org[a];
        const float size[3] = {w * cell, hh * cell, d * cell};
        for (int a = 0; a < 3; ++a) h.local_com[a] = org[a] + size[a] * 0.5f;
        h.radius = size[0] / 2.0;  // FluidSolver3D.cu:167
        h.mass = s->cfg.body_mass;
    }
    for (int a = 0; a < 3; ++a) h.pos[a] = s->cfg.body_pos[a];
    h.inertia = 0.4 * h.mass * h.radius * h.radius;  // FluidSolver3D.cu:168
    h.update_rotation();
    cudaError_t e = cudaSuccess;
    if (!data.empty()) {
        e = dalloc(&s->d_sdf, data.size());
        if (e == cudaSuccess) e = cudaMemcpy(s->d_sdf, data.data(), sizeof(float) * data.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = dalloc(&s->d_bpart, size_t(body_force_partials()));
    if (e == cudaSuccess) e = dalloc(&s->d_bforce, 8);
    if (e != cudaSuccess) { free_body(s); return s->cuda_fail(e, "body upload"); }
    h.sdf_host = std::move(data);
    h.loaded = true;
    s->cfg.active_body = 1;
    // init's marking before seeding (FluidSolver3D.cu:177-193)
    launch_mark_body(s->d_bodymark, s->g, body_shape(s), s->st);
    launch_apply_mark(s->d_labels, s->d_bodymark, s->g, s->st);
    e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "body marking");
    fill_body_stats(s);
    return FP_OK;
}

int fp_set_paddle(fp_solver* s, float x_rest, float amplitude, float period) {
    if (!s) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "labels must be loaded before the paddle");
    if (!(period > 0.0f) || !std::isfinite(x_rest) || !std::isfinite(amplitude))
        return s->fail(FP_ERR_ARG, "paddle needs a finite rest position and amplitude and a positive period");
    free_body(s);
    HostBody& h = s->hb;
    h = HostBody();
    h.kind = BODY_PADDLE;
    h.pad_x0 = x_rest;
    h.pad_amp = amplitude;
    h.pad_period = period;
    h.pos[1] = 0.5 * s->H * s->cfg.dx;  // torque reference: the face centre
    h.pos[2] = 0.5 * s->D * s->cfg.dx;
    h.paddle_at(0.0);
    cudaError_t e = dalloc(&s->d_bpart, size_t(body_force_partials()));
    if (e == cudaSuccess) e = dalloc(&s->d_bforce, 8);
    if (e != cudaSuccess) { free_body(s); return s->cuda_fail(e, "paddle"); }
    h.loaded = true;
    s->cfg.active_body = 1;
    launch_mark_body(s->d_bodymark, s->g, body_shape(s), s->st);
    launch_apply_mark(s->d_labels, s->d_bodymark, s->g, s->st);
    e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "paddle marking");
    fill_body_stats(s);
    return FP_OK;
}

int fp_set_particles(fp_solver* s, const float* pos, const float* vel, int64_t n) {
    if (!s || n < 0 || (n > 0 && !pos)) return s ? s->fail(FP_ERR_ARG, "bad particle arrays") : FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "labels must be set before particles");
    // Particle indices travel as int32 in the w lane, and the check below
    // reports the lowest bad index into a word preset with bytes of 0x7F, so
    // every index must stay below 0x7F7F7F7F (2,139,062,143).
    if (n > 0x7F7F7F7FLL) return s->fail(FP_ERR_ARG, "too many particles (at most 2,139,062,143)");
    int rc = alloc_particles(s, n);
    if (rc) return rc;
    s->sorted = false;
    if (n == 0) return FP_OK;
    float* dpos = s->d_io;
    float* dvel = s->d_io + 3 * n;
    cudaError_t e = cudaMemcpyAsync(dpos, pos, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess && vel) e = cudaMemcpyAsync(dvel, vel, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_bad, 0x7F, sizeof(int), s->st);  // 0x7F7F7F7F >= n > any index
    if (e != cudaSuccess) return s->cuda_fail(e, "particle upload");
    // pack into the second buffer and check every value on the device
    launch_pack(dpos, vel ? dvel : nullptr, n, s->d_pos2, s->d_vel2, s->d_bad, s->st);
    s->launches += 1;
    e = cudaMemcpyAsync(s->h_bad, s->d_bad, sizeof(int), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "particle upload");
    if (*s->h_bad < n) {
        s->np = 0;
        return s->fail(FP_ERR_ARG, "non-finite particle value at index " + std::to_string(*s->h_bad));
    }
    std::swap(s->d_pos, s->d_pos2);
    std::swap(s->d_vel, s->d_vel2);
    return FP_OK;
}

int fp_seed_particles(fp_solver* s, int ppc, uint32_t seed) {
    if (!s || ppc < 0) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "labels must be loaded before seeding");
    std::vector<uint8_t> lab(size_t(s->g.nc()));
    cudaError_t e = cudaMemcpy(lab.data(), s->d_labels, lab.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return s->cuda_fail(e, "label download");
    std::vector<float> pos;
    io::seed_particles(lab.data(), s->W, s->H, s->D, s->cfg.dx, ppc, seed, pos);
    return fp_set_particles(s, pos.data(), nullptr, int64_t(pos.size() / 3));
}

int fp_load_ply(fp_solver* s, const char* path) {
    if (!s || !path) return FP_ERR_ARG;
    std::vector<float> pos, vel;
    bool hv = false;
    if (!io::read_ply(path, pos, vel, hv, s->err)) return FP_ERR_IO;
    return fp_set_particles(s, pos.data(), hv ? vel.data() : nullptr, int64_t(pos.size() / 3));
}

int64_t fp_num_particles(const fp_solver* s) { return s ? s->np : -1; }

int fp_get_particles(fp_solver* s, float* pos, float* vel, int64_t n) {
    if (!s || n != s->np) return s ? s->fail(FP_ERR_ARG, "particle count mismatch") : FP_ERR_ARG;
    if (n == 0) return FP_OK;
    launch_unsort(s->d_pos, s->d_vel, n, s->d_io, s->d_io + 3 * n, s->st);
    cudaError_t e = cudaSuccess;
    if (pos) e = cudaMemcpyAsync(pos, s->d_io, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess && vel) e = cudaMemcpyAsync(vel, s->d_io + 3 * n, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "particle download");
    return FP_OK;
}

int fp_save_ply(fp_solver* s, const char* path, int format) {
    if (!s || !path) return FP_ERR_ARG;
    std::vector<float> pos(size_t(s->np) * 3), vel(size_t(s->np) * 3);
    int rc = fp_get_particles(s, pos.data(), vel.data(), s->np);
    if (rc) return rc;
    if (!io::write_particles(path, pos.data(), vel.data(), s->np, format, s->err)) return FP_ERR_IO;
    return FP_OK;
}

int fp_step(fp_solver* s, int n) {
    int rc = check_ready(s);
    if (rc) return rc;
    for (int i = 0; i < n; ++i) {
        // with a step log every step waits for its end, so that its phase
        // times are its own
        rc = one_step(s, i + 1 == n || s->step_log != nullptr);
        if (rc) return rc;
        write_step_log(s);
    }
    return FP_OK;
}

// Frame output of fp_run off the step's critical path: each frame's particles
// go (unsort kernel packing x y z vx vy vz records, then D2H on the solver
// stream) into one of two pinned buffers, and a writer thread writes the file
// (one write for binary PLY) once the copy's event has
// completed, while the host goes on issuing steps.  A buffer is reused only
// after its previous file is written.
struct FrameWriter {
    fp_solver* s;
    int format;
    float* h[2] = {nullptr, nullptr};  // pos | vel, 6 * cap floats each
    int64_t cap = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool busy[2] = {false, false};
    struct Job { int buf; int64_t n; std::string path; };
    std::deque<Job> jobs;
    std::mutex m;
    std::condition_variable cv;
    bool stop = false, failed = false;
    std::string err;
    std::thread th;

    FrameWriter(fp_solver* sv, int fmt) : s(sv), format(fmt) {}
    int start(int64_t n) {
        cap = std::max<int64_t>(n, 1);
        for (int b = 0; b < 2; ++b) {
            if (cudaMallocHost(&h[b], sizeof(float) * 6 * size_t(cap)) != cudaSuccess ||
                cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming) != cudaSuccess)
                return s->cuda_fail(cudaGetLastError(), "frame buffers");
        }
        th = std::thread([this] { loop(); });
        return FP_OK;
    }
    void loop() {
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(m);
                cv.wait(lk, [&] { return stop || !jobs.empty(); });
                if (jobs.empty()) return;
                j = jobs.front();
                jobs.pop_front();
            }
            std::string e;
            bool ok = cudaEventSynchronize(ev[j.buf]) == cudaSuccess &&
                      io::write_frame_records(j.path, h[j.buf], j.n, format, e);
            std::lock_guard<std::mutex> lk(m);
            if (!ok && !failed) { failed = true; err = e.empty() ? "frame copy failed" : e; }
            busy[j.buf] = false;
            cv.notify_all();
        }
    }
    // Queues frame `path` from buffer b; waits while b still holds an unwritten frame.
    int submit(int b, const std::string& path) {
        {
            std::unique_lock<std::mutex> lk(m);
            cv.wait(lk, [&] { return !busy[b] || failed; });
            if (failed) return s->fail(FP_ERR_IO, err);
        }
        const int64_t n = s->np;
        if (n > cap) return s->fail(FP_ERR_STATE, "particle count grew during fp_run");
        if (n > 0) {
            launch_unsort_records(s->d_pos, s->d_vel, n, s->d_io, s->st);
            s->launches += 1;
            cudaMemcpyAsync(h[b], s->d_io, sizeof(float) * 6 * size_t(n), cudaMemcpyDeviceToHost, s->st);
        }
        cudaEventRecord(ev[b], s->st);
        std::lock_guard<std::mutex> lk(m);
        busy[b] = true;
        jobs.push_back(Job{b, n, path});
        cv.notify_all();
        return FP_OK;
    }
    int finish() {
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
            cv.notify_all();
        }
        if (th.joinable()) th.join();
        for (int b = 0; b < 2; ++b) {
            if (h[b]) cudaFreeHost(h[b]);
            if (ev[b]) cudaEventDestroy(ev[b]);
        }
        if (failed) return s->fail(FP_ERR_IO, err);
        return FP_OK;
    }
};

int fp_run(fp_solver* s, int frames) {
    int rc = check_ready(s);
    if (rc) return rc;
    const int ipf = std::max(1, s->cfg.iter_per_frame);
    const std::string tmpl = s->cfg.output_template;
    FILE* csv = nullptr;
    if (s->cfg.active_body) {
        std::string cp = frame_dir(tmpl) + "/csvRes.csv";
        csv = std::fopen(cp.c_str(), "w");
        if (csv) std::fprintf(csv, "frame,centerX1,centerX2,centerX3,angleX1,angleX2,angleX3\n");
    }
    const bool out = s->cfg.output_format != FP_OUT_NONE;
    FrameWriter writer(s, s->cfg.output_format);
    if (out && (rc = writer.start(s->np)) != FP_OK) {
        writer.finish();
        if (csv) std::fclose(csv);
        return rc;
    }
    int64_t frame = 0;
    // FluidSolver3D::run labels once before its loop and takes frames * ipf + 1
    // steps (FluidSolver3D.cu:3110-3111); FluidSolver2D::run takes max_steps
    // steps and writes every one of them (FluidSolver2D.cu:1333-1342).
    const bool r2 = ref2d(s);
    if (!r2) phase_label(s);
    const int64_t last = r2 ? int64_t(frames) - 1 : int64_t(frames) * ipf;
    for (int64_t i = 0; i <= last; ++i) {
        rc = one_step(s);
        if (rc) break;
        write_step_log(s);
        if ((r2 || i % ipf == 0) && out) {
            const char* ext = s->cfg.output_format == FP_OUT_OFF ? ".off" : ".ply";
            rc = writer.submit(int(frame++ & 1), tmpl + std::to_string(r2 ? i : i / ipf) + ext);
            if (rc) break;
            if (body_on(s) && s->hb.kind != BODY_PADDLE) {  // body_<frame>.ply (run, :3130-3132)
                std::vector<float> pts;
                body_surface_points(s, pts);
                const std::string bp = frame_dir(tmpl) + "/body_" + std::to_string(i / ipf) + ".ply";
                if (!io::write_particles(bp, pts.data(), nullptr, int64_t(pts.size() / 3), FP_OUT_PLY, s->err)) {
                    rc = FP_ERR_IO;
                    break;
                }
            }
            if (csv) {
                std::fprintf(csv, "%lld,%g,%g,%g,%g,%g,%g\n", (long long)(i / ipf), s->stats.body_pos[0],
                             s->stats.body_pos[1], s->stats.body_pos[2], s->stats.body_angles[0],
                             s->stats.body_angles[1], s->stats.body_angles[2]);
                std::fflush(csv);
            }
        }
    }
    if (csv) std::fclose(csv);
    if (out) {
        const int wrc = writer.finish();
        if (rc == FP_OK) rc = wrc;
    }
    return rc;
}

int fp_run_phase(fp_solver* s, int phase) {
    int rc = check_ready(s);
    if (rc) return rc;
    if (ref2d(s)) {
        rc = r2_alloc(s);
        if (rc) return rc;
        switch (phase) {
            case FP_PHASE_LABEL: r2_label(s); break;
            case FP_PHASE_P2G:
                r2_p2g(s, 0);
                if (s->cfg.extrapolate) rc = r2_extrapolate(s, false);
                break;
            case FP_PHASE_SAVE: phase_save(s); break;
            case FP_PHASE_FORCES: launch_r2_forces(s->d_u, s->d_v, s->g, s->cfg.dt, s->st); s->launches += 1; break;
            case FP_PHASE_PRESSURE: rc = r2_pressure(s); break;
            case FP_PHASE_PROJECT: r2_project(s); break;
            case FP_PHASE_BODY: break;
            case FP_PHASE_G2P: r2_particles(s, 1); break;
            case FP_PHASE_ADVECT:
                if (s->cfg.extrapolate) {
                    rc = r2_extrapolate(s, true);
                    if (rc) return rc;
                }
                r2_particles(s, 2);
                if (s->np) cudaMemcpyAsync(s->h_r2 + 1, s->r2.misc + 2, sizeof(int), cudaMemcpyDeviceToHost, s->st);
                break;
            case FP_PHASE_CLEANUP: r2_particles(s, 4); rc = r2_compact(s, false); break;
            default: return s->fail(FP_ERR_ARG, "unknown phase");
        }
        cudaError_t e = cudaStreamSynchronize(s->st);
        if (e != cudaSuccess) return s->cuda_fail(e, "phase");
        if (phase == FP_PHASE_ADVECT && s->np) s->stats.advect_capped = s->h_r2[1];
        return rc;
    }
    switch (phase) {
        case FP_PHASE_LABEL: phase_label(s); break;
        case FP_PHASE_P2G: phase_p2g(s, 0); break;
        case FP_PHASE_SAVE: phase_save(s); break;
        case FP_PHASE_FORCES: launch_forces(s->d_u, s->d_v, s->d_w, s->g, s->cfg.dt, gravity3(), s->st); break;
        case FP_PHASE_PRESSURE: rc = phase_pressure(s); break;
        case FP_PHASE_PROJECT: phase_project(s); break;
        case FP_PHASE_BODY: rc = phase_body(s); break;
        case FP_PHASE_G2P: phase_g2p_advect(s, 1, 0); break;
        case FP_PHASE_ADVECT:
            if (s->cfg.extrapolate > 0) rc = extrapolate_3d(s);
            if (rc == FP_OK) phase_g2p_advect(s, 0, 1);
            break;
        default: return s->fail(FP_ERR_ARG, "unknown phase");
    }
    cudaError_t e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "phase");
    return rc;
}

static int64_t grid_len(const fp_solver* s, int which) {
    switch (which) {
        case FP_GRID_U: case FP_GRID_U_SAVED: return s->g.nu();
        case FP_GRID_V: case FP_GRID_V_SAVED: return s->g.nv();
        case FP_GRID_W: case FP_GRID_W_SAVED: return s->g.nw();
        case FP_GRID_P: case FP_GRID_RHS: return s->g.nc();
    }
    return -1;
}
static float* grid_ptr(fp_solver* s, int which) {
    if (which == FP_GRID_RHS) {  // densify the last solve's compact right-hand side
        unet::launch_rhs_dense(s->pb.nf, s->pb.fidx, unet::Lvl{s->W, s->H, s->D}, s->pb.b, s->d_rhs_dense, s->st);
        s->launches += 1;
        return s->d_rhs_dense;
    }
    float* a[7] = {s->d_u, s->d_v, s->d_w, s->d_us, s->d_vs, s->d_ws, s->d_p};
    return (which >= 0 && which < 7) ? a[which] : nullptr;
}

int fp_get_grid(fp_solver* s, int which, float* out, int64_t n) {
    if (!s || !out) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "no grid");
    if (grid_len(s, which) != n) return s->fail(FP_ERR_ARG, "grid size mismatch");
    cudaError_t e = cudaMemcpyAsync(out, grid_ptr(s, which), sizeof(float) * n, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? FP_OK : s->cuda_fail(e, "grid download");
}

int fp_get_grid_device(fp_solver* s, int which, float* d_out, int64_t n) {
    if (!s || !d_out) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "no grid");
    if (grid_len(s, which) != n) return s->fail(FP_ERR_ARG, "grid size mismatch");
    cudaError_t e = cudaMemcpyAsync(d_out, grid_ptr(s, which), sizeof(float) * n, cudaMemcpyDeviceToDevice, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? FP_OK : s->cuda_fail(e, "grid copy");
}

int fp_get_labels_device(fp_solver* s, uint8_t* d_out, int64_t n) {
    if (!s || !d_out) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "no grid");
    if (n != s->g.nc()) return s->fail(FP_ERR_ARG, "label size mismatch");
    cudaError_t e = cudaMemcpyAsync(d_out, s->d_labels, size_t(n), cudaMemcpyDeviceToDevice, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? FP_OK : s->cuda_fail(e, "label copy");
}

int fp_load_learned(fp_solver* s, const char* weights_path) {
    if (!s || !weights_path) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "labels must be loaded before the learned weights");
    s->learned_path = weights_path;
    const int rc = load_net(s);
    if (rc) s->learned_path.clear();
    return rc;
}

int fp_set_grid(fp_solver* s, int which, const float* in, int64_t n) {
    if (!s || !in) return FP_ERR_ARG;
    if (which == FP_GRID_RHS) return s->fail(FP_ERR_ARG, "the right-hand side grid is read only");
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "no grid");
    if (grid_len(s, which) != n) return s->fail(FP_ERR_ARG, "grid size mismatch");
    cudaError_t e = cudaMemcpyAsync(grid_ptr(s, which), in, sizeof(float) * n, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? FP_OK : s->cuda_fail(e, "grid upload");
}

int fp_get_labels(fp_solver* s, uint8_t* out, int64_t n) {
    if (!s || !out) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "no grid");
    if (n != s->g.nc()) return s->fail(FP_ERR_ARG, "label size mismatch");
    cudaError_t e = cudaMemcpyAsync(out, s->d_labels, size_t(n), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? FP_OK : s->cuda_fail(e, "label download");
}

int fp_set_body_state(fp_solver* s, const float* pos, const float* vel, const float* omega) {
    if (!s) return FP_ERR_ARG;
    for (int a = 0; a < 3; ++a) {
        if (pos) s->hb.pos[a] = pos[a];
        if (vel) s->hb.vel[a] = vel[a];
        if (omega) s->hb.omega[a] = omega[a];
    }
    fill_body_stats(s);
    return FP_OK;
}

int fp_stats(const fp_solver* s, fp_step_stats* out) {
    if (!s || !out) return FP_ERR_ARG;
    *out = s->stats;
    out->kernel_launches = s->launches;
    return FP_OK;
}

void* fp_cuda_stream(const fp_solver* s) { return s ? static_cast<void*>(s->st) : nullptr; }

int fp_set_step_log(fp_solver* s, const char* path) {
    if (!s) return FP_ERR_ARG;
    if (s->step_log) { std::fclose(s->step_log); s->step_log = nullptr; }
    if (!path || !path[0]) return FP_OK;
    s->step_log = std::fopen(path, "w");
    if (!s->step_log) return s->fail(FP_ERR_IO, std::string("cannot open step log ") + path);
    return FP_OK;
}

// ---------------------------------------------------------------- state snapshots

int fp_save_state(fp_solver* s, const char* path) {
    if (!s || !path) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "no state: labels not loaded");
    const size_t nc = size_t(s->g.nc()), nu = size_t(s->g.nu()), nv = size_t(s->g.nv()), nw = size_t(s->g.nw());
    std::vector<uint8_t> base(nc), lab(nc);
    std::vector<float> grids(2 * (nu + nv + nw) + nc);
    std::vector<float> pos(size_t(s->np) * 3), vel(size_t(s->np) * 3);
    cudaError_t e = cudaStreamSynchronize(s->st);
    size_t off = 0;
    for (auto [src, n] : {std::pair<const float*, size_t>{s->d_u, nu}, {s->d_v, nv}, {s->d_w, nw}, {s->d_us, nu},
                          {s->d_vs, nv}, {s->d_ws, nw}, {s->d_p, nc}}) {
        if (e == cudaSuccess) e = cudaMemcpy(grids.data() + off, src, sizeof(float) * n, cudaMemcpyDeviceToHost);
        off += n;
    }
    if (e == cudaSuccess) e = cudaMemcpy(base.data(), s->d_base, nc, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(lab.data(), s->d_labels, nc, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return s->cuda_fail(e, "state download");
    if (s->np) {
        const int rc = fp_get_particles(s, pos.data(), vel.data(), s->np);
        if (rc) return rc;
    }
    StateFile sf;
    sf.f = std::fopen(path, "wb");
    if (!sf.f) return s->fail(FP_ERR_IO, std::string("cannot write state file ") + path);
    sf.put(kStateMagic, 8);
    sf.put(int32_t(1));
    sf.put(int32_t(s->W)); sf.put(int32_t(s->H)); sf.put(int32_t(s->D));
    sf.put(s->cfg.dx); sf.put(s->cfg.dt);
    sf.put(int64_t(s->steps));
    sf.put(base.data(), nc); sf.put(lab.data(), nc);
    sf.put(grids.data(), grids.size());
    sf.put(int64_t(s->np));
    sf.put(pos.data(), pos.size()); sf.put(vel.data(), vel.size());
    const HostBody& h = s->hb;
    sf.put(int32_t(h.loaded ? 1 : 0));
    sf.put(int32_t(s->cfg.active_body));
    if (h.loaded) {
        sf.put(int32_t(h.kind));
        sf.put(h.pos, 3); sf.put(h.vel, 3); sf.put(h.omega, 3);
        sf.put(h.theta); sf.put(h.psi); sf.put(h.phi);
        sf.put(h.mass); sf.put(h.inertia); sf.put(h.radius);
        sf.put(h.force, 3); sf.put(h.torque, 3);
        sf.put(int32_t(h.nx)); sf.put(int32_t(h.ny)); sf.put(int32_t(h.nz));
        sf.put(h.origin, 3); sf.put(h.cell); sf.put(h.local_com, 3);
        sf.put(h.pad_x0); sf.put(h.pad_amp); sf.put(h.pad_period); sf.put(h.pad_t);
        sf.put(int64_t(h.sdf_host.size()));
        sf.put(h.sdf_host.data(), h.sdf_host.size());
    }
    if (!sf.ok) return s->fail(FP_ERR_IO, std::string("write error on state file ") + path);
    return FP_OK;
}

int fp_load_state(fp_solver* s, const char* path) {
    if (!s || !path) return FP_ERR_ARG;
    StateFile sf;
    sf.f = std::fopen(path, "rb");
    if (!sf.f) return s->fail(FP_ERR_IO, std::string("cannot open state file ") + path);
    char magic[8] = {};
    int32_t ver = 0, W = 0, H = 0, D = 0;
    float dx = 0, dt = 0;
    int64_t steps = 0;
    sf.get(magic, 8); sf.get(ver);
    if (!sf.ok || std::memcmp(magic, kStateMagic, 8) != 0 || ver != 1)
        return s->fail(FP_ERR_IO, std::string("not a state file: ") + path);
    sf.get(W); sf.get(H); sf.get(D); sf.get(dx); sf.get(dt); sf.get(steps);
    if (!sf.ok || W <= 0 || H <= 0 || D <= 0 || int64_t(W) * H * D > (int64_t(1) << 34))
        return s->fail(FP_ERR_IO, "state file: bad grid header");
    if (dx != s->cfg.dx || dt != s->cfg.dt) return s->fail(FP_ERR_ARG, "state file: dx or dt differ from the solver's");
    const Dims gd{W, H, D, dx};
    const size_t nc = size_t(gd.nc()), nu = size_t(gd.nu()), nv = size_t(gd.nv()), nw = size_t(gd.nw());
    std::vector<uint8_t> base(nc), lab(nc);
    std::vector<float> grids(2 * (nu + nv + nw) + nc);
    sf.get(base.data(), nc); sf.get(lab.data(), nc);
    sf.get(grids.data(), grids.size());
    int64_t np = 0;
    sf.get(np);
    if (!sf.ok || np < 0 || np > 0x7F7F7F7FLL) return s->fail(FP_ERR_IO, "state file: truncated or bad particle count");
    std::vector<float> pos(size_t(np) * 3), vel(size_t(np) * 3);
    sf.get(pos.data(), pos.size()); sf.get(vel.data(), vel.size());
    int32_t loaded = 0, active = 0;
    sf.get(loaded); sf.get(active);
    HostBody h;
    if (sf.ok && loaded) {
        int32_t kind = 0, nx = 0, ny = 0, nz = 0;
        int64_t nsdf = 0;
        sf.get(kind);
        sf.get(h.pos, 3); sf.get(h.vel, 3); sf.get(h.omega, 3);
        sf.get(h.theta); sf.get(h.psi); sf.get(h.phi);
        sf.get(h.mass); sf.get(h.inertia); sf.get(h.radius);
        sf.get(h.force, 3); sf.get(h.torque, 3);
        sf.get(nx); sf.get(ny); sf.get(nz);
        sf.get(h.origin, 3); sf.get(h.cell); sf.get(h.local_com, 3);
        sf.get(h.pad_x0); sf.get(h.pad_amp); sf.get(h.pad_period); sf.get(h.pad_t);
        sf.get(nsdf);
        if (!sf.ok || kind < BODY_SPHERE || kind > BODY_PADDLE || nsdf < 0 || nsdf != int64_t(nx) * ny * nz ||
            (kind == BODY_SDF && nsdf == 0))
            return s->fail(FP_ERR_IO, "state file: bad body record");
        h.kind = kind; h.nx = nx; h.ny = ny; h.nz = nz;
        h.sdf_host.resize(size_t(nsdf));
        sf.get(h.sdf_host.data(), h.sdf_host.size());
        h.update_rotation();
    }
    if (!sf.ok) return s->fail(FP_ERR_IO, "state file: truncated");
    // the grid, labels and fields
    int rc = alloc_grid(s, W, H, D);
    if (rc) return rc;
    cudaError_t e = cudaMemcpy(s->d_base, base.data(), nc, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->d_labels, lab.data(), nc, cudaMemcpyHostToDevice);
    size_t off = 0;
    for (auto [dst, n] : {std::pair<float*, size_t>{s->d_u, nu}, {s->d_v, nv}, {s->d_w, nw}, {s->d_us, nu},
                          {s->d_vs, nv}, {s->d_ws, nw}, {s->d_p, nc}}) {
        if (e == cudaSuccess) e = cudaMemcpy(dst, grids.data() + off, sizeof(float) * n, cudaMemcpyHostToDevice);
        off += n;
    }
    if (e != cudaSuccess) return s->cuda_fail(e, "state upload");
    // the body
    free_body(s);
    if (loaded) {
        h.loaded = false;
        s->hb = std::move(h);
        HostBody& hb = s->hb;
        if (!hb.sdf_host.empty()) {
            e = dalloc(&s->d_sdf, hb.sdf_host.size());
            if (e == cudaSuccess)
                e = cudaMemcpy(s->d_sdf, hb.sdf_host.data(), sizeof(float) * hb.sdf_host.size(), cudaMemcpyHostToDevice);
        }
        if (e == cudaSuccess) e = dalloc(&s->d_bpart, size_t(body_force_partials()));
        if (e == cudaSuccess) e = dalloc(&s->d_bforce, 8);
        if (e != cudaSuccess) { free_body(s); return s->cuda_fail(e, "state body upload"); }
        hb.loaded = true;
        fill_body_stats(s);
    }
    s->cfg.active_body = active;
    // the particles, in their saved order
    rc = fp_set_particles(s, np ? pos.data() : nullptr, np ? vel.data() : nullptr, np);
    if (rc) return rc;
    s->steps = steps;
    s->stats.step = steps;
    s->stats.num_particles = np;
    return FP_OK;
}

int fp_set_wait_limit(fp_solver* s, int64_t polls) {
    if (!s || polls < 0) return s ? s->fail(FP_ERR_ARG, "negative wait limit") : FP_ERR_ARG;
    if (polls > 0xFFFFFFFFll) return s->fail(FP_ERR_ARG, "wait limit above 2^32 - 1 polls");
    s->wait_polls = polls == 0 ? kDefaultWaitPolls : static_cast<unsigned>(polls);
    return FP_OK;
}

int fp_pressure_solve(fp_solver* s, const float* rhs, float* x, int64_t n, int* iters, double* relres) {
    if (!s || !rhs || !x) return FP_ERR_ARG;
    if (!s->have_grid) return s->fail(FP_ERR_STATE, "no grid");
    if (n != s->g.nc()) return s->fail(FP_ERR_ARG, "rhs size mismatch");
    cudaError_t e = cudaMemcpyAsync(s->d_scratch, rhs, sizeof(float) * n, cudaMemcpyHostToDevice, s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "rhs upload");
    BodyKin b{};
    // rhs in d_scratch; the dense solution goes to d_scratch2 (zeroed by the
    // setup), leaving the solver's own pressure grid untouched.
    float* xdense = s->d_scratch2;
    launch_pressure_setup(s->d_labels, s->d_u, s->d_v, s->d_w, s->g, s->cfg.dt, b, s->d_scratch, xdense, s->pb, s->st);
    int rc = solve_system(s, xdense);
    if (rc) return rc;
    if (e == cudaSuccess) e = cudaMemcpyAsync(x, xdense, sizeof(float) * n, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return s->cuda_fail(e, "solution download");
    if (iters) *iters = s->stats.pcg_iters;
    if (relres) *relres = s->stats.residual;
    return s->stats.solve_status;
}

int fp_solve_csr_upper(int n, const int* offsets, const int* cols, const double* vals, const double* b, double* x,
                       double tol, int max_iters, int* iters, double* relres) {
    if (n <= 0 || !offsets || !cols || !vals || !b || !x) return FP_ERR_ARG;
    for (int i = 0; i < n; ++i)
        if (offsets[i + 1] < offsets[i]) return FP_ERR_ARG;
    for (int e = 0; e < offsets[n]; ++e)
        if (cols[e] < 0 || cols[e] >= n) return FP_ERR_ARG;
    int rc = csr_cg_solve(n, offsets, cols, vals, b, x, tol, max_iters, iters, relres, 0);
    return rc ? FP_ERR_CUDA : FP_OK;
}

}  // extern "C"
