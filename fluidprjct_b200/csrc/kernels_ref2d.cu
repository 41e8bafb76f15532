// kernels_ref2d.cu -- FluidPrjct's own 2D step (src/FluidSim/FluidSolver2D.cu)
// on the GPU: the "ref2d" scheme of a depth-1 grid.
//
// The reference's 2D solver is not a 2D restriction of its 3D one.  Its
// P2G weights both u and v faces (i, j) by the bilinear hat about the cell
// centre ((i + 0.5) dx, (j + 0.5) dx); its projection marks faces without a
// FLUID side VEL_UNKNOWN and leaves the border faces alone; its G2P is
// 1D-linear inside the particle's cell; its advection is forward Euler that
// moves a particle entering a SOLID cell to the nearest SOLID neighbour
// centre; and its clean-up deletes particles (:1302-1331).  These kernels
// restate that step.  The pressure solve is the shared matrix-free PCG: the
// 2D system (:408-718) is the depth-1 case of the 3D operator.
//
//   k_r2_label_reset / k_r2_label_mark   labelGrid_gpu, :168-251
//   k_r2_bin_* + k_r2_p2g               particlesToGrid, :259-338 (+ save
//                                        :340-354 and forces :362-381)
//   k_r2_forces                          applyForces, :362-381
//   k_r2_project                         applyPressure, :720-757
//   k_r2_particles                       gridToParticles :822-853,
//                                        advectParticles :1122-1166,
//                                        cleanUpParticles :1171-1204
//   k_r2_compact                         the erase loop of cleanUpParticles
//
// Particles keep the caller's order (the reference sums P2G contributions
// particle by particle, and its clean-up erases in place).  P2G is a gather:
// each face centre merges the particle lists of its 3x3 neighbouring cells
// by particle index, so every face sums in the reference's order.  All
// arithmetic uses explicit round-to-nearest intrinsics (no FMA contraction),
// so the results are bit-identical to the FP32 restatement in the oracle.
// Where the reference relies on undefined behaviour the kernels fix the
// meaning the oracle fixes: a host float -> int conversion out of range or of
// NaN gives INT_MIN, a label read past the grid's flat range is "not SOLID",
// and one particle's substep loop stops after kMaxSubsteps substeps (counted).
#include <cfloat>
#include <climits>

#include "kernels.hpp"
#include "scan.cuh"

namespace fp {
namespace {

constexpr float kVelUnknown = -2147483648.0f;  // INT_MIN stored in a float grid (utility.cuh:56)
constexpr int kMaxSubsteps = 4096;
constexpr uint8_t L_SOLID = 0, L_FLUID = 1, L_AIR = 2;

// (int)t in host code (trunc toward zero; INT_MIN where C++ leaves it undefined).
__device__ __forceinline__ int host_trunc(float t) {
    if (isnan(t) || t >= 2147483648.0f || t < -2147483648.0f) return INT_MIN;
    return __float2int_rz(t);
}

__global__ void k_r2_label_reset(const uint8_t* __restrict__ base, uint8_t* __restrict__ lab, int64_t n) {
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < n; c += int64_t(gridDim.x) * blockDim.x)
        lab[c] = base[c] == L_SOLID ? L_SOLID : L_AIR;
}

// markFluidCellsKernel: (int)(pos / dx) in device code (NaN -> 0, saturating).
__global__ void k_r2_label_mark(const float4* __restrict__ pos, int64_t np, float dx, int W, int H,
                                uint8_t* __restrict__ lab) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const float4 p = pos[q];
    const int ci = __float2int_rz(__fdiv_rn(p.x, dx)), cj = __float2int_rz(__fdiv_rn(p.y, dx));
    if (ci >= 0 && ci < W && cj >= 0 && cj < H) {
        uint8_t* c = lab + ci + int64_t(cj) * W;
        if (*c == L_AIR) *c = L_FLUID;  // AIR -> FLUID only; concurrent writers store the same value
    }
}

// Bin coordinate floor(q / dx) clamped to [-2, n + 1], offset by 2; -1 for NaN.
__device__ __forceinline__ int r2_bin(float q, float dx, int n) {
    const float f = floorf(__fdiv_rn(q, dx));
    if (isnan(f)) return -1;
    return int(fminf(fmaxf(f, -2.0f), float(n + 1))) + 2;
}

__global__ void k_r2_bin_count(const float4* __restrict__ pos, const float4* __restrict__ vel, int64_t np, float dx,
                               int W, int H, int* __restrict__ counts, int* __restrict__ key, int* __restrict__ rank,
                               int* __restrict__ nonfinite) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const float4 p = pos[q], v = vel[q];
    const int bx = r2_bin(p.x, dx, W), by = r2_bin(p.y, dx, H);
    const int k = (bx < 0 || by < 0) ? -1 : bx + by * (W + 4);
    key[q] = k;
    if (k >= 0) rank[q] = atomicAdd(counts + k, 1);
    if (!isfinite(v.x)) atomicAdd(nonfinite, 1);
    if (!isfinite(v.y)) atomicAdd(nonfinite + 1, 1);
}

__global__ void k_r2_bin_place(const int* __restrict__ key, const int* __restrict__ rank, const int* __restrict__ start,
                               int64_t np, int* __restrict__ list) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const int k = key[q];
    if (k >= 0) list[start[k] + rank[q]] = int(q);
}

// Each bin's particle indices in ascending order (insertion sort; bins hold a
// few particles).
__global__ void k_r2_bin_order(const int* __restrict__ start, int nb, int* __restrict__ list) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int s = start[b], e = start[b + 1];
    for (int a = s + 1; a < e; ++a) {
        const int x = list[a];
        int c = a - 1;
        while (c >= s && list[c] > x) {
            list[c + 1] = list[c];
            --c;
        }
        list[c + 1] = x;
    }
}

// hatFunction, utility.cu:146-153 (the threshold compares a float with a double literal)
__device__ __forceinline__ float r2_hat(float r) {
    const float a = fabsf(r);
    return double(__fsub_rn(a, 1.0f)) <= 1e-8 ? __fsub_rn(1.0f, a) : 0.0f;
}

// One thread per face centre (i, j), 0 <= i <= W, 0 <= j <= H: u face (i, j)
// when j < H, v face (i, j) when i < W.  mode: 0 writes the P2G result;
// 1 also saves it to u*, v* and adds gravity to the grid copy.
__global__ void __launch_bounds__(256) k_r2_p2g(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                const int* __restrict__ start, const int* __restrict__ list,
                                                const int* __restrict__ nonfinite, int W, int H, float dx, float dt,
                                                int mode, float* __restrict__ u, float* __restrict__ v,
                                                float* __restrict__ us, float* __restrict__ vs) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(W + 1) * (H + 1)) return;
    const int i = int(t % (W + 1)), j = int(t / (W + 1));
    const int BW = W + 4;
    int cur[9], end[9], head[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        const int b = (i + 1 + c % 3) + (j + 1 + c / 3) * BW;  // bins of cells i-1..i+1, j-1..j+1
        cur[c] = start[b];
        end[c] = start[b + 1];
        head[c] = cur[c] < end[c] ? list[cur[c]] : INT_MAX;
    }
    const float cx = __fmul_rn(__fadd_rn(float(i), 0.5f), dx), cy = __fmul_rn(__fadd_rn(float(j), 0.5f), dx);
    float un = 0.0f, ud = 0.0f, vn = 0.0f, vd = 0.0f;
    int lu = 0, lv = 0;
    for (;;) {
        int m = INT_MAX, mc = -1;
#pragma unroll
        for (int c = 0; c < 9; ++c)
            if (head[c] < m) { m = head[c]; mc = c; }
        if (mc < 0) break;
#pragma unroll
        for (int c = 0; c < 9; ++c)
            if (c == mc) {
                ++cur[c];
                head[c] = cur[c] < end[c] ? list[cur[c]] : INT_MAX;
            }
        const float4 p = pos[m], w = vel[m];
        const float k = __fmul_rn(r2_hat(__fdiv_rn(__fsub_rn(p.x, cx), dx)), r2_hat(__fdiv_rn(__fsub_rn(p.y, cy), dx)));
        if (j < H) {
            un = __fadd_rn(un, __fmul_rn(w.x, k));
            ud = __fadd_rn(ud, k);
            lu += (!isfinite(w.x) && k != 0.0f);
        }
        if (i < W) {
            vn = __fadd_rn(vn, __fmul_rn(w.y, k));
            vd = __fadd_rn(vd, k);
            lv += (!isfinite(w.y) && k != 0.0f);
        }
    }
    // a non-finite velocity outside this face's support adds inf * 0 = NaN
    if (nonfinite[0] > lu) un = __int_as_float(0x7fffffff);
    if (nonfinite[1] > lv) vn = __int_as_float(0x7fffffff);
    if (j < H) {
        const float val = ud != 0.0f ? __fdiv_rn(un, ud) : 0.0f;
        const int64_t f = i + int64_t(j) * (W + 1);
        if (mode == 1) {
            us[f] = val;
            u[f] = val != kVelUnknown ? __fadd_rn(val, __fmul_rn(dt, 0.0f)) : val;
        } else {
            u[f] = val;
        }
    }
    if (i < W) {
        const float val = vd != 0.0f ? __fdiv_rn(vn, vd) : 0.0f;
        const int64_t f = i + int64_t(j) * W;
        if (mode == 1) {
            vs[f] = val;
            v[f] = val != kVelUnknown ? __fadd_rn(val, __fmul_rn(dt, -9.81f)) : val;
        } else {
            v[f] = val;
        }
    }
}

__global__ void k_r2_forces(float* __restrict__ u, float* __restrict__ v, int W, int H, float dt) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t nu = int64_t(W + 1) * H, nv = int64_t(W) * (H + 1);
    if (t < nu && u[t] != kVelUnknown) u[t] = __fadd_rn(u[t], __fmul_rn(dt, 0.0f));
    if (t < nv && v[t] != kVelUnknown) v[t] = __fadd_rn(v[t], __fmul_rn(dt, -9.81f));
}

__global__ void k_r2_project(float* __restrict__ u, float* __restrict__ v, const float* __restrict__ p,
                             const uint8_t* __restrict__ lab, int W, int H, float scale) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(W) * H) return;
    const int i = int(t % W), j = int(t / W);
    const uint8_t C = lab[t];
    if (i >= 1) {
        const uint8_t L = lab[t - 1];
        float& f = u[i + int64_t(j) * (W + 1)];
        if (L == L_FLUID || C == L_FLUID) {
            if (L == L_SOLID || C == L_SOLID) f = 0.0f;
            else f = __fsub_rn(f, __fmul_rn(scale, __fsub_rn(p[t], p[t - 1])));
        } else {
            f = kVelUnknown;
        }
    }
    if (j >= 1) {
        const uint8_t B = lab[t - W];
        float& f = v[t];
        if (B == L_FLUID || C == L_FLUID) {
            if (B == L_SOLID || C == L_SOLID) f = 0.0f;
            else f = __fsub_rn(f, __fmul_rn(scale, __fsub_rn(p[t], p[t - W])));
        } else {
            f = kVelUnknown;
        }
    }
}

struct R2Grid {
    const float *u, *v, *us, *vs;
    const uint8_t* lab;
    int W, H;
    float dx, dt, alpha;
};

// interpVel, :792-820; delta interpolates u - u*, v - v*
__device__ void r2_interp(const R2Grid& g, bool delta, float x, float y, float& ou, float& ov) {
    const int i = host_trunc(__fdiv_rn(x, g.dx)), j = host_trunc(__fdiv_rn(y, g.dx));
    if (!(i >= 0 && i < g.W && j >= 0 && j < g.H)) {
        ou = ov = kVelUnknown;
        return;
    }
    const float cx = __fmul_rn(__fadd_rn(float(i), 0.5f), g.dx), cy = __fmul_rn(__fadd_rn(float(j), 0.5f), g.dx);
    const float off = __fdiv_rn(g.dx, 2.0f);
    const float x1 = __fsub_rn(cx, off), x2 = __fadd_rn(cx, off), y1 = __fsub_rn(cy, off), y2 = __fadd_rn(cy, off);
    const int64_t fu = i + int64_t(j) * (g.W + 1), fv = i + int64_t(j) * g.W;
    float u1 = g.u[fu], u2 = g.u[fu + 1], v1 = g.v[fv], v2 = g.v[fv + g.W];
    if (delta) {
        u1 = __fsub_rn(u1, g.us[fu]); u2 = __fsub_rn(u2, g.us[fu + 1]);
        v1 = __fsub_rn(v1, g.vs[fv]); v2 = __fsub_rn(v2, g.vs[fv + g.W]);
    }
    const float wx = __fsub_rn(x2, x1), wy = __fsub_rn(y2, y1);
    ou = __fadd_rn(__fmul_rn(__fdiv_rn(__fsub_rn(x2, x), wx), u1), __fmul_rn(__fdiv_rn(__fsub_rn(x, x1), wx), u2));
    ov = __fadd_rn(__fmul_rn(__fdiv_rn(__fsub_rn(y2, y), wy), v1), __fmul_rn(__fdiv_rn(__fsub_rn(y, y1), wy), v2));
}

// projectParticle, :1072-1119: to the nearest SOLID cell centre among the
// 8 neighbours, else the nearest AIR one; false if neither exists.  Distances
// are the correctly rounded float hypot.
__device__ bool r2_project_particle(const R2Grid& g, float& x, float& y) {
    const int nbr[8][2] = {{-1, 1}, {-1, 0}, {-1, -1}, {0, 1}, {0, -1}, {1, 1}, {1, 0}, {1, -1}};
    const int ci = host_trunc(__fdiv_rn(x, g.dx)), cj = host_trunc(__fdiv_rn(y, g.dx));
    for (int pass = 0; pass < 2; ++pass) {
        const uint8_t want = pass == 0 ? L_SOLID : L_AIR;
        bool any = false;
        float best = FLT_MAX, nx = x, ny = y;
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const int64_t a = int64_t(ci) + nbr[n][0], c = int64_t(cj) + nbr[n][1];
            if (!(a >= 0 && a < g.W && c >= 0 && c < g.H) || g.lab[a + c * g.W] != want) continue;
            any = true;
            const float px = __fmul_rn(__fadd_rn(float(a), 0.5f), g.dx), py = __fmul_rn(__fadd_rn(float(c), 0.5f), g.dx);
            const double ex = double(__fsub_rn(px, x)), ey = double(__fsub_rn(py, y));
            const float dist = __double2float_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey))));
            if (dist < best) { best = dist; nx = px; ny = py; }
        }
        if (any) {
            x = __fadd_rn(x, __fmul_rn(1.0f, __fsub_rn(nx, x)));
            y = __fadd_rn(y, __fmul_rn(1.0f, __fsub_rn(ny, y)));
            return true;
        }
    }
    return false;
}

// G2P (flags & 1), advection (flags & 2) and clean-up (flags & 4) of one
// particle; they read only grids and labels, so one thread runs all three.
// keep[q] = 1 unless the clean-up deletes the particle.
__global__ void k_r2_particles(float4* __restrict__ pos, float4* __restrict__ vel, int64_t np, R2Grid g, int flags,
                               int* __restrict__ keep, int* __restrict__ capped) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    float4 P = pos[q], V = vel[q];
    float x = P.x, y = P.y;
    if (flags & 1) {
        float pu, pv, fu, fv;
        r2_interp(g, false, x, y, pu, pv);
        r2_interp(g, true, x, y, fu, fv);
        const float b = __fsub_rn(1.0f, g.alpha);
        V.x = __fadd_rn(__fmul_rn(pu, g.alpha), __fmul_rn(__fadd_rn(V.x, fu), b));
        V.y = __fadd_rn(__fmul_rn(pv, g.alpha), __fmul_rn(__fadd_rn(V.y, fv), b));
        vel[q] = V;
    }
    if (flags & 2) {
        const float C = 1.0f;  // ADVECT_MAX
        float sub = 0.0f;
        bool finished = false;
        int n = 0;
        while (!finished) {
            if (n++ == kMaxSubsteps) {
                atomicAdd(capped, 1);
                break;
            }
            float cu, cv;
            r2_interp(g, false, x, y, cu, cv);
            float dT = __fdiv_rn(__fmul_rn(C, g.dx),
                                 __fadd_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(cu, cu), __fmul_rn(cv, cv))), FLT_MIN));
            if (__fadd_rn(sub, dT) >= g.dt) {
                dT = __fsub_rn(g.dt, sub);
                finished = true;
            } else if (__fadd_rn(sub, __fmul_rn(2.0f, dT)) >= g.dt) {
                dT = __fmul_rn(0.5f, __fsub_rn(g.dt, sub));
            }
            x = __fadd_rn(x, __fmul_rn(cu, dT));
            y = __fadd_rn(y, __fmul_rn(cv, dT));
            sub = __fadd_rn(sub, dT);
            if (x < 0.0f || y < 0.0f || isnan(x) || isnan(y)) break;
            const int64_t f = int64_t(host_trunc(__fdiv_rn(x, g.dx))) + int64_t(host_trunc(__fdiv_rn(y, g.dx))) * g.W;
            const bool solid = f >= 0 && f < int64_t(g.W) * g.H && g.lab[f] == L_SOLID;
            if (solid && !r2_project_particle(g, x, y)) break;
        }
    }
    int k = 1;
    if (flags & 4) {
        const int ci = host_trunc(__fdiv_rn(x, g.dx)), cj = host_trunc(__fdiv_rn(y, g.dx));
        k = !(ci < 0 || cj < 0 || ci >= g.W || cj >= g.H || isnan(x) || isnan(y));
        if (k && g.lab[ci + int64_t(cj) * g.W] == L_SOLID) k = r2_project_particle(g, x, y);
    }
    if (flags & 6) {
        P.x = x;
        P.y = y;
        pos[q] = P;
    }
    keep[q] = k;
}

// keep[] holds the exclusive scan of the keep flags, keep[np] the count.
__global__ void k_r2_compact(const float4* __restrict__ pos, const float4* __restrict__ vel, int64_t np,
                             const int* __restrict__ keep, float4* __restrict__ pos2, float4* __restrict__ vel2) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const int d = keep[q];
    if (keep[q + 1] == d) return;
    float4 P = pos[q];
    P.w = __int_as_float(d);
    pos2[d] = P;
    vel2[d] = vel[q];
}

unsigned blocks_for(int64_t n, int t = 256) { return unsigned((n + t - 1) / t); }

}  // namespace

void launch_r2_label(const uint8_t* base, uint8_t* labels, const float4* pos, int64_t np, Dims g, float dx,
                     cudaStream_t st) {
    const int64_t nc = int64_t(g.W) * g.H;
    k_r2_label_reset<<<blocks_for(nc), 256, 0, st>>>(base, labels, nc);
    if (np > 0) k_r2_label_mark<<<blocks_for(np), 256, 0, st>>>(pos, np, dx, g.W, g.H, labels);
}

void launch_r2_p2g(const float4* pos, const float4* vel, int64_t np, Dims g, float dx, float dt, int mode,
                   R2Scratch& sc, float* u, float* v, float* us, float* vs, cudaStream_t st) {
    const int nb = (g.W + 4) * (g.H + 4);
    cudaMemsetAsync(sc.start, 0, sizeof(int) * (nb + 1), st);
    cudaMemsetAsync(sc.misc, 0, sizeof(int) * 2, st);
    if (np > 0) k_r2_bin_count<<<blocks_for(np), 256, 0, st>>>(pos, vel, np, dx, g.W, g.H, sc.start, sc.key, sc.rank,
                                                                sc.misc);
    k_scan_single_block<<<1, 1024, 0, st>>>(sc.start, nb, sc.start + nb);
    if (np > 0) k_r2_bin_place<<<blocks_for(np), 256, 0, st>>>(sc.key, sc.rank, sc.start, np, sc.list);
    k_r2_bin_order<<<blocks_for(nb), 256, 0, st>>>(sc.start, nb, sc.list);
    k_r2_p2g<<<blocks_for(int64_t(g.W + 1) * (g.H + 1)), 256, 0, st>>>(pos, vel, sc.start, sc.list, sc.misc, g.W, g.H,
                                                                         dx, dt, mode, u, v, us, vs);
}

void launch_r2_forces(float* u, float* v, Dims g, float dt, cudaStream_t st) {
    const int64_t n = int64_t(g.W + 1) * (g.H + 1);
    k_r2_forces<<<blocks_for(n), 256, 0, st>>>(u, v, g.W, g.H, dt);
}

void launch_r2_project(float* u, float* v, const float* p, const uint8_t* labels, Dims g, float dx, float dt,
                       cudaStream_t st) {
    const float scale = dt / (1000.0f * dx);  // host float arithmetic, as applyPressure :721
    k_r2_project<<<blocks_for(int64_t(g.W) * g.H), 256, 0, st>>>(u, v, p, labels, g.W, g.H, scale);
}

void launch_r2_particles(float4* pos, float4* vel, int64_t np, const float* u, const float* v, const float* us,
                         const float* vs, const uint8_t* labels, Dims g, float dx, float dt, float alpha, int flags,
                         R2Scratch& sc, cudaStream_t st) {
    if (np == 0) return;
    R2Grid a{u, v, us, vs, labels, g.W, g.H, dx, dt, alpha};
    if (flags & 2) cudaMemsetAsync(sc.misc + 2, 0, sizeof(int), st);
    k_r2_particles<<<blocks_for(np), 256, 0, st>>>(pos, vel, np, a, flags, sc.keep, sc.misc + 2);
}

void launch_r2_compact(const float4* pos, const float4* vel, int64_t np, R2Scratch& sc, float4* pos2, float4* vel2,
                       cudaStream_t st) {
    k_scan_single_block<<<1, 1024, 0, st>>>(sc.keep, int(np), sc.keep + np);
    if (np > 0) k_r2_compact<<<blocks_for(np), 256, 0, st>>>(pos, vel, np, sc.keep, pos2, vel2);
}

}  // namespace fp
