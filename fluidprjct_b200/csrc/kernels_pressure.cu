// kernels_pressure.cu -- pressure projection: RHS, matrix-free PCG, projection.
//
// Replaces pressureSolve (FluidSolver3D.cu:1815-2062) and applyPressure
// (:2072-2464).  The reference assembles an upper-triangle CSR of the unit
// 7-point Laplacian over FLUID cells (MatrixBuilder3D/MatrixFiller3D,
// :1598-1777) and hands it to cuDSS every step.  Here the operator is never
// stored: A*d at a FLUID cell is diag*d - sum of d over FLUID neighbours, with
// diag = number of in-domain FLUID or AIR neighbours (SOLID, BODY and
// out-of-domain neighbours are Neumann walls; AIR is Dirichlet p = 0).
//
// Layout: FLUID cells are compacted once per solve (fidx: padded dense index of
// the n-th FLUID cell, in i-fastest order, the reference's fluidNumbers order);
// x, r, q, b and diag are compact; the search direction dd lives on a dense
// grid with a one-cell zero halo so that the stencil needs no bounds tests.
//
// The PCG is one persistent cooperative kernel: FP32 stencil and vector
// updates, FP64 dot products reduced per CTA and then summed by every CTA in
// a fixed order (deterministic, no host round trip per iteration), and a
// bounded software grid barrier that reports a timeout instead of hanging.
#include <cstdio>

#include "device_memo.hpp"
#include "kernels.hpp"
#include "pcg_common.cuh"
#include "scan.cuh"

namespace fp {

namespace {

constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;
constexpr int PCG_THREADS = 512;

__device__ __forceinline__ int64_t padded_index(int i, int j, int k, const Dims& g) {
    return int64_t(i + 1) + int64_t(j + 1) * (g.W + 2) + int64_t(k + 1) * (g.W + 2) * (g.H + 2);
}

__device__ __forceinline__ bool solidish(uint8_t l) { return l == SOLID || l == BODY; }

// Pass 1 of the fluid compaction: tile counts of FLUID cells; zero p off the
// fluid (the solve writes every FLUID cell; until then they keep the previous
// pressure, which a warm-started MG solve reads as its guess).
__global__ void __launch_bounds__(SCAN_BLOCK) k_fluid_tiles(const uint8_t* __restrict__ labels, int64_t nc,
                                                            float* __restrict__ p, int* __restrict__ tile_sums) {
    int64_t e0 = int64_t(blockIdx.x) * SCAN_TILE + int64_t(threadIdx.x) * SCAN_ITEMS;
    int s = 0;
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; ++t) {
        int64_t e = e0 + t;
        if (e < nc) {
            const bool f = labels[e] == FLUID;
            s += f;
            if (!f) p[e] = 0.0f;
        }
    }
    int total;
    block_exclusive_scan<SCAN_BLOCK>(s, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// RHSCalculator3D::operator() (FluidSolver3D.cu:1371-1456) at FLUID cell (i,j,k).
__device__ __forceinline__ float rhs_at(const uint8_t* __restrict__ lab, const float* __restrict__ u,
                                        const float* __restrict__ v, const float* __restrict__ w, const Dims& g,
                                        int i, int j, int k, float scale, const BodyKin& body) {
    const int W = g.W, H = g.H;
    const float dx = g.dx;
    const int64_t ui = int64_t(i) + int64_t(j) * (W + 1) + int64_t(k) * (W + 1) * H;
    const int64_t vi = int64_t(i) + int64_t(j) * W + int64_t(k) * W * (H + 1);
    const int64_t wi = int64_t(i) + int64_t(j) * W + int64_t(k) * W * H;
    const float u0 = u[ui], u1 = u[ui + 1], v0 = v[vi], v1 = v[vi + W], w0 = w[wi], w1 = w[wi + int64_t(W) * H];
    float div = u1 - u0 + v1 - v0 + w1 - w0;
    float rhs = -scale * div;
    uint8_t l;
    l = label_at(lab, g, i - 1, j, k);
    if (solidish(l)) {
        float s = l == BODY ? body_vel_at(body, make_float3(float(i) * dx, (float(j) + 0.5f) * dx, (float(k) + 0.5f) * dx)).x : 0.0f;
        rhs -= scale * (u0 - s);
    }
    l = label_at(lab, g, i + 1, j, k);
    if (solidish(l)) {
        float s = l == BODY ? body_vel_at(body, make_float3(float(i + 1) * dx, (float(j) + 0.5f) * dx, (float(k) + 0.5f) * dx)).x : 0.0f;
        rhs += scale * (u1 - s);
    }
    l = label_at(lab, g, i, j - 1, k);
    if (solidish(l)) {
        float s = l == BODY ? body_vel_at(body, make_float3((float(i) + 0.5f) * dx, float(j) * dx, (float(k) + 0.5f) * dx)).y : 0.0f;
        rhs -= scale * (v0 - s);
    }
    l = label_at(lab, g, i, j + 1, k);
    if (solidish(l)) {
        float s = l == BODY ? body_vel_at(body, make_float3((float(i) + 0.5f) * dx, float(j + 1) * dx, (float(k) + 0.5f) * dx)).y : 0.0f;
        rhs += scale * (v1 - s);
    }
    l = label_at(lab, g, i, j, k - 1);
    if (solidish(l)) {
        float s = l == BODY ? body_vel_at(body, make_float3((float(i) + 0.5f) * dx, (float(j) + 0.5f) * dx, float(k) * dx)).z : 0.0f;
        rhs -= scale * (w0 - s);
    }
    l = label_at(lab, g, i, j, k + 1);
    if (solidish(l)) {
        float s = l == BODY ? body_vel_at(body, make_float3((float(i) + 0.5f) * dx, (float(j) + 0.5f) * dx, float(k + 1) * dx)).z : 0.0f;
        rhs += scale * (w1 - s);
    }
    return rhs;
}

// Pass 3: write the compact system (fidx, diag, b) of every FLUID cell.
__global__ void __launch_bounds__(SCAN_BLOCK) k_fluid_build(const uint8_t* __restrict__ labels,
                                                            const float* __restrict__ u, const float* __restrict__ v,
                                                            const float* __restrict__ w, Dims g, float scale,
                                                            BodyKin body, const float* __restrict__ rhs_dense,
                                                            const int* __restrict__ tile_off, int* __restrict__ fidx,
                                                            uint8_t* __restrict__ diag, float* __restrict__ b) {
    const int64_t nc = g.nc();
    int64_t e0 = int64_t(blockIdx.x) * SCAN_TILE + int64_t(threadIdx.x) * SCAN_ITEMS;
    uint8_t lab[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; ++t) {
        int64_t e = e0 + t;
        lab[t] = e < nc ? labels[e] : SOLID;
        s += lab[t] == FLUID;
    }
    int total;
    int n = block_exclusive_scan<SCAN_BLOCK>(s, total) + tile_off[blockIdx.x];
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; ++t) {
        if (lab[t] != FLUID) continue;
        int64_t e = e0 + t;
        // 32-bit decode: cell indices fit in an int (the padded index does too)
        const uint32_t eu = uint32_t(e), W = uint32_t(g.W), H = uint32_t(g.H);
        const uint32_t ej = eu / W;
        const int i = int(eu - ej * W), j = int(ej % H), k = int(ej / H);
        fidx[n] = int(padded_index(i, j, k, g));
        int d = 0;
        const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
#pragma unroll
        for (int o = 0; o < 6; ++o) {
            uint8_t l = label_at(labels, g, i + off[o][0], j + off[o][1], k + off[o][2]);
            d += (l == FLUID || l == AIR);
        }
        diag[n] = uint8_t(d | (((i + j + k) & 1) << 7));  // bit 7: red/black colour
        b[n] = rhs_dense ? rhs_dense[e] : rhs_at(labels, u, v, w, g, i, j, k, scale, body);
        ++n;
    }
}

__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }

template <class T>
struct PcgArgs {
    Dims g;
    const int* nf;
    const int* fidx;     // padded dense index of the n-th FLUID cell
    const uint8_t* diag; // compact diagonal
    const float* b;      // compact right-hand side
    T* R[2];             // padded dense residual r (double-buffered)
    T* Wv[2];            // padded dense w = A M^-1 r
    T* S[2];             // padded dense s = A p
    T* invd;             // padded dense 1/diag (0 off the fluid)
    T* P;                // compact search direction
    T* X;                // compact solution
    double* part;        // [2 parities][3][nblocks]
    GridBar* bar;
    int* status;
    PcgOut* out;
    double tol;
    int maxit;
};

// Jacobi-preconditioned conjugate gradients in the Chronopoulos-Gear form
// (one reduction phase per iteration):
//   s_i = w_i + b_i s_{i-1}; p_i = u_i + b_i p_{i-1}; x += a_i p_i;
//   r_{i+1} = r_i - a_i s_i; u = M^-1 r; w_{i+1} = A u_{i+1};
//   g = (r,u), d = (w,u); b = g_new/g; a = g_new/(d - b g_new/a_old).
// The stencil of w_{i+1} needs u_{i+1} at the six neighbours; each thread
// recomputes those from the neighbours' r_i, w_i, s_{i-1} of the previous
// iteration (double-buffered, fused multiply-adds pinned with __fma_rn so the
// owner and its neighbours produce the same bits), so a single grid barrier
// per iteration both publishes the vectors and completes the reductions.
template <class T>
__global__ void __launch_bounds__(PCG_THREADS) k_pcg_cg(PcgArgs<T> a) {
    const int nf = *a.nf;
    const int nb = int(gridDim.x);
    // Blocked distribution: block b owns the contiguous fluid range
    // [n0, n1), so the x and y neighbours of its cells mostly lie in the
    // same block (L1 hits); threads stride by blockDim (coalesced).
    const int chunk = (nf + nb - 1) / nb;
    const int n0 = min(nf, int(blockIdx.x) * chunk), n1 = min(nf, n0 + chunk);
    const int sy = a.g.W + 2, sz = (a.g.W + 2) * (a.g.H + 2);
    const int offs[6] = {1, -1, sy, -sy, sz, -sz};

    // Init 1: r0 = b, 1/diag, s_{-1} = p_{-1} = x0 = 0.
    for (int n = n0 + threadIdx.x; n < n1; n += PCG_THREADS) {
        const int c = a.fidx[n];
        const uint8_t d = a.diag[n] & 0x7F;
        a.invd[c] = d > 0 ? T(1) / T(d) : T(0);
        a.R[0][c] = T(a.b[n]);
        a.S[0][c] = T(0);
        a.P[n] = T(0);
        a.X[n] = T(0);
    }
    if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
    // Init 2: u0 = M^-1 r0, w0 = A u0; partials (r,u), (w,u), (r,r).
    {
        double g_l = 0.0, d_l = 0.0, rr_l = 0.0;
        const T* __restrict__ R0 = a.R[0];
        const T* __restrict__ iv = a.invd;
        for (int n = n0 + threadIdx.x; n < n1; n += PCG_THREADS) {
            const int c = a.fidx[n];
            const T r = R0[c];
            const T u = r * iv[c];
            T nbs = T(0);
#pragma unroll
            for (int o = 0; o < 6; ++o) nbs += R0[c + offs[o]] * iv[c + offs[o]];
            const T w = T(a.diag[n] & 0x7F) * u - nbs;
            a.Wv[0][c] = w;
            g_l += double(r) * double(u);
            d_l += double(w) * double(u);
            rr_l += double(r) * double(r);
        }
        double3 bs = block_sum3(g_l, d_l, rr_l);
        double* pp = a.part + 3 * nb;  // parity 1
        if (threadIdx.x == 0) { pp[blockIdx.x] = bs.x; pp[nb + blockIdx.x] = bs.y; pp[2 * nb + blockIdx.x] = bs.z; }
    }
    if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
    double3 tot = grid_sum3(a.part + 3 * nb, nb);
    double gam = tot.x, del = tot.y, rr = tot.z;
    const double bb = tot.z;
    const double thr = a.tol * a.tol * bb;
    double alpha = del > 0.0 ? gam / del : 0.0, beta = 0.0;
    int it = 0;
    int st = DEV_OK;
    if (bb > 0.0 && !(del > 0.0)) st = isnan(del) ? DEV_NAN : DEV_BREAKDOWN;
    while (st == DEV_OK && rr > thr && bb > 0.0) {
        if (it >= a.maxit) { st = DEV_MAXIT; break; }
        const int cur = it & 1, nxt = cur ^ 1;
        const T al = T(alpha), be = T(beta);
        const T* __restrict__ Rc = a.R[cur];
        const T* __restrict__ Wc = a.Wv[cur];
        const T* __restrict__ Sc = a.S[cur];
        const T* __restrict__ iv = a.invd;
        T* __restrict__ Rn = a.R[nxt];
        T* __restrict__ Wn = a.Wv[nxt];
        T* __restrict__ Sn = a.S[nxt];
        double g_l = 0.0, d_l = 0.0, rr_l = 0.0;
        for (int n = n0 + threadIdx.x; n < n1; n += PCG_THREADS) {
            const int c = a.fidx[n];
            const T id = iv[c];
            const T r = Rc[c];
            const T s = fmaT(be, Sc[c], Wc[c]);        // s_i
            const T p = fmaT(be, a.P[n], r * id);      // p_i
            a.X[n] = fmaT(al, p, a.X[n]);
            const T rn = fmaT(-al, s, r);              // r_{i+1}
            const T un = rn * id;
            T nbs = T(0);
#pragma unroll
            for (int o = 0; o < 6; ++o) {
                const int q = c + offs[o];
                const T sq = fmaT(be, Sc[q], Wc[q]);
                nbs += fmaT(-al, sq, Rc[q]) * iv[q];
            }
            const T wn = T(a.diag[n] & 0x7F) * un - nbs;
            Rn[c] = rn;
            Wn[c] = wn;
            Sn[c] = s;
            a.P[n] = p;
            g_l += double(rn) * double(un);
            d_l += double(wn) * double(un);
            rr_l += double(rn) * double(rn);
        }
        double3 bs = block_sum3(g_l, d_l, rr_l);
        double* pp = a.part + (it & 1) * 3 * nb;
        if (threadIdx.x == 0) { pp[blockIdx.x] = bs.x; pp[nb + blockIdx.x] = bs.y; pp[2 * nb + blockIdx.x] = bs.z; }
        if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
        tot = grid_sum3(pp, nb);
        ++it;
        if (isnan(tot.x) || isnan(tot.y) || isnan(tot.z)) { st = DEV_NAN; rr = tot.z; break; }
        const double gn = tot.x, dn = tot.y;
        rr = tot.z;
        if (rr <= thr) break;
        beta = gn / gam;
        const double den = dn - beta * gn / alpha;
        if (!(den > 0.0) || !(gn > 0.0)) { st = DEV_BREAKDOWN; break; }
        alpha = gn / den;
        gam = gn;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out->iters = it;
        atomicCAS(a.status, DEV_OK, st);  // never masks a timeout recorded by another CTA
        a.out->rr = rr;
        a.out->bb = bb;
        a.out->rz = gam;
    }
}

__global__ void k_reset_pcg(GridBar* bar, int* status, unsigned limit) {
    bar->count = 0;
    bar->limit = limit;
    *status = DEV_OK;
}

// Zero the FLUID entries of the padded work grids after a solve, so that every
// solve starts from all-zero grids whatever cells were fluid before.
template <class T>
__global__ void k_clear_padded(const int* __restrict__ nf_p, const int* __restrict__ fidx, T* r0, T* r1, T* w0, T* w1,
                               T* s0, T* s1, T* invd) {
    const int nf = *nf_p;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) {
        const int c = fidx[n];
        r0[c] = T(0); r1[c] = T(0); w0[c] = T(0); w1[c] = T(0); s0[c] = T(0); s1[c] = T(0);
        if (invd) invd[c] = T(0);
    }
}

// Compact T vector -> padded dense grid.
template <class T>
__global__ void k_to_dense(const int* __restrict__ nf_p, const int* __restrict__ fidx, const T* __restrict__ x,
                           T* __restrict__ dst) {
    const int nf = *nf_p;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) dst[fidx[n]] = x[n];
}

template <class T>
__global__ void k_scatter_p(const int* __restrict__ nf_p, const int* __restrict__ fidx, const T* __restrict__ x, Dims g,
                            float* __restrict__ p) {
    const int nf = *nf_p;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) {
        int cp = fidx[n];
        int i = cp % (g.W + 2) - 1, j = (cp / (g.W + 2)) % (g.H + 2) - 1, k = cp / ((g.W + 2) * (g.H + 2)) - 1;
        p[int64_t(i) + int64_t(j) * g.W + int64_t(k) * g.W * g.H] = float(x[n]);
    }
}

// Partials of ||b - A x||^2 and ||b||^2 over the padded dense x (float or double).
template <class T>
__global__ void __launch_bounds__(256) k_residual(const int* __restrict__ nf_p, const int* __restrict__ fidx,
                                                  const uint8_t* __restrict__ diag, const float* __restrict__ b,
                                                  const T* __restrict__ xd, Dims g, double2* __restrict__ part,
                                                  float* __restrict__ r_out, double* __restrict__ r64_out) {
    const int nf = *nf_p;
    const int sx = 1, sy = g.W + 2, sz = (g.W + 2) * (g.H + 2);
    double e2 = 0.0, b2 = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) {
        const T* x = xd + fidx[n];
        double ax = double(diag[n] & 0x7F) * double(x[0]) -
                    (double(x[sx]) + double(x[-sx]) + double(x[sy]) + double(x[-sy]) + double(x[sz]) + double(x[-sz]));
        double e = double(b[n]) - ax;
        if (r_out) r_out[n] = float(e);
        if (r64_out) r64_out[n] = e;
        e2 += e * e;
        b2 += double(b[n]) * double(b[n]);
    }
    double2 s = block_sum2(e2, b2);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_sum_partials(const double2* __restrict__ part, int nb, double* __restrict__ out) {
    double2 s = grid_sum2(part, nb);
    if (threadIdx.x == 0) { out[0] = s.x; out[1] = s.y; }
}

// Partials of (x, b) and (x, A x) over the padded dense guess xd (FP64).
__global__ void __launch_bounds__(256) k_guess_dots(const int* __restrict__ nf_p, const int* __restrict__ fidx,
                                                    const uint8_t* __restrict__ diag, const float* __restrict__ b,
                                                    const double* __restrict__ xd, Dims g, double2* __restrict__ part) {
    const int nf = *nf_p;
    const int sy = g.W + 2, sz = (g.W + 2) * (g.H + 2);
    double xb = 0.0, xax = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) {
        const double* x = xd + fidx[n];
        const double ax = double(diag[n] & 0x7F) * x[0] - ((x[1] + x[-1]) + (x[sy] + x[-sy]) + (x[sz] + x[-sz]));
        xb += x[0] * double(b[n]);
        xax += x[0] * ax;
    }
    double2 s = block_sum2(xb, xax);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// x64 and its padded copy xd scaled by alpha = (x, b) / (x, A x) (red[0..1]),
// 0 when (x, A x) is not positive: the A-norm error of alpha x is never above
// that of x = 0.
__global__ void k_scale_guess(const int* __restrict__ nf_p, const int* __restrict__ fidx, const double* __restrict__ red,
                              double* __restrict__ x64, double* __restrict__ xd) {
    const int nf = *nf_p;
    const double d = red[1];
    const double alpha = (d > 0.0 && isfinite(red[0] / d)) ? red[0] / d : 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) {
        const double v = x64[n] * alpha;
        x64[n] = v;
        xd[fidx[n]] = v;
    }
}

__global__ void k_ir_update(const int* __restrict__ nf_p, const int* __restrict__ fidx, const float* __restrict__ c,
                            double* __restrict__ x64, double* __restrict__ xd) {
    const int nf = *nf_p;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) {
        double v = x64[n] + double(c[n]);
        x64[n] = v;
        xd[fidx[n]] = v;
    }
}

// ---------------------------------------------------------------- projection
// UFunctor/VFunctor/WFunctor (FluidSolver3D.cu:2072-2336) for one face between
// cells L and R: a SOLID/BODY side gets a ghost pressure that makes the face
// velocity equal to the wall velocity (0 or the rigid-body velocity).
__device__ __forceinline__ float project_face(float vel, uint8_t lL, uint8_t lR, float pL, float pR, float vb,
                                              float scale, float inv) {
    const bool fL = (lL == FLUID || lL == AIR), fR = (lR == FLUID || lR == AIR);
    float p0, p1;
    if (fL && fR) { p0 = pL; p1 = pR; }
    else if (solidish(lL)) { float s = lL == BODY ? vb : 0.0f; p0 = pR - inv * (vel - s); p1 = pR; }
    else if (solidish(lR)) { float s = lR == BODY ? vb : 0.0f; p0 = pL; p1 = pL + inv * (vel - s); }
    else { p0 = pL; p1 = pR; }
    return vel - scale * (p1 - p0);
}

__device__ __forceinline__ float p_at(const float* __restrict__ p, const Dims& g, int i, int j, int k) {
    if (i < 0 || i >= g.W || j < 0 || j >= g.H || k < 0 || k >= g.D) return 0.0f;
    return p[i + j * g.W + k * g.W * g.H];
}

__global__ void k_project(float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
                          const float* __restrict__ p, const uint8_t* __restrict__ lab, Dims g, float scale, float inv,
                          BodyKin body, const int* __restrict__ guard) {
    if (solve_failed(guard)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int W = g.W, H = g.H, D = g.D;
    if (i > W || j > H || k > D) return;
    const float dx = g.dx;
    const uint8_t lc = label_at(lab, g, i, j, k);
    // A face between two AIR cells keeps its velocity exactly (the pressure is
    // zero off the fluid: vel - scale * (0 - 0) is vel), so it is neither read
    // nor written; in a dam break most faces are such.
    const uint8_t lx = label_at(lab, g, i - 1, j, k), ly = label_at(lab, g, i, j - 1, k),
                  lz = label_at(lab, g, i, j, k - 1);
    const bool air = lc == AIR;
    const float pc = p_at(p, g, i, j, k);
    if (j < H && k < D && !(air && lx == AIR)) {
        int64_t id = int64_t(i) + int64_t(j) * (W + 1) + int64_t(k) * (W + 1) * H;
        float vb = body.active ? body_vel_at(body, make_float3(float(i) * dx, (float(j) + 0.5f) * dx, (float(k) + 0.5f) * dx)).x : 0.0f;
        u[id] = project_face(u[id], lx, lc, p_at(p, g, i - 1, j, k), pc, vb, scale, inv);
    }
    if (i < W && k < D && !(air && ly == AIR)) {
        int64_t id = int64_t(i) + int64_t(j) * W + int64_t(k) * W * (H + 1);
        float vb = body.active ? body_vel_at(body, make_float3((float(i) + 0.5f) * dx, float(j) * dx, (float(k) + 0.5f) * dx)).y : 0.0f;
        v[id] = project_face(v[id], ly, lc, p_at(p, g, i, j - 1, k), pc, vb, scale, inv);
    }
    if (i < W && j < H && !(air && lz == AIR)) {
        int64_t id = int64_t(i) + int64_t(j) * W + int64_t(k) * W * H;
        float vb = body.active ? body_vel_at(body, make_float3((float(i) + 0.5f) * dx, (float(j) + 0.5f) * dx, float(k) * dx)).z : 0.0f;
        w[id] = project_face(w[id], lz, lc, p_at(p, g, i, j, k - 1), pc, vb, scale, inv);
    }
}

// ---------------------------------------------------------------- CSR CG (FP64)
// Symmetric matrix from its upper triangle: y = U x + U^T x - diag(U) x.
__global__ void k_csr_sym_spmv(int n, const int* __restrict__ off, const int* __restrict__ cols,
                               const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int e = off[i]; e < off[i + 1]; ++e) {
        int c = cols[e];
        s += vals[e] * x[c];
        if (c != i) atomicAdd(&y[c], vals[e] * x[i]);
    }
    atomicAdd(&y[i], s);
}
__global__ void k_csr_diag(int n, const int* __restrict__ off, const int* __restrict__ cols,
                           const double* __restrict__ vals, double* __restrict__ dg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 1.0;
    for (int e = off[i]; e < off[i + 1]; ++e) if (cols[e] == i) d = vals[e];
    dg[i] = d;
}
__global__ void k_dot(int n, const double* __restrict__ a, const double* __restrict__ b, double2* part) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
    double2 r = block_sum2(s, 0.0);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}
__global__ void k_axpy2(int n, double alpha, const double* __restrict__ d, const double* __restrict__ q,
                        double* __restrict__ x, double* __restrict__ r, const double* __restrict__ dg,
                        double* __restrict__ z) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] += alpha * d[i];
    r[i] -= alpha * q[i];
    z[i] = r[i] / dg[i];
}
__global__ void k_xpby(int n, const double* __restrict__ z, double beta, double* __restrict__ d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = z[i] + beta * d[i];
}

}  // namespace

// ---------------------------------------------------------------- launchers

void launch_pressure_setup(const uint8_t* labels, const float* u, const float* v, const float* w, Dims g, float dt,
                           BodyKin body, const float* rhs_dense, float* p, PressureBufs& pb, cudaStream_t st) {
    const int64_t nc = g.nc();
    const int ntiles = int((nc + SCAN_TILE - 1) / SCAN_TILE);
    const float scale = (1000.0f * g.dx) / dt;  // rho*dx/dt, FluidSolver3D.cu:1520
    k_fluid_tiles<<<ntiles, SCAN_BLOCK, 0, st>>>(labels, nc, p, pb.tile_sums);
    k_scan_single_block<<<1, 1024, 0, st>>>(pb.tile_sums, ntiles, pb.nf);
    k_fluid_build<<<ntiles, SCAN_BLOCK, 0, st>>>(labels, u, v, w, g, scale, body, rhs_dense, pb.tile_sums, pb.fidx,
                                                 pb.diag, pb.b);
}

int pcg_max_blocks() {
    static DeviceMemo memo;
    return memo.get([](int dev) {
        int sms = 0, pf = 0, pd = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pf, k_pcg_cg<float>, PCG_THREADS, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pd, k_pcg_cg<double>, PCG_THREADS, 0);
        return sms * std::max(1, std::min(pf, pd));
    });
}

template <class T>
static int launch_pcg_t(Dims g, PressureBufs& pb, const float* rhs, double tol, int maxit, cudaStream_t st,
                        unsigned wait_polls) {
    // One block per four cells per thread, at most the resident maximum: a
    // small grid waits at cheaper barriers (one block: __syncthreads).
    const int64_t want = (g.nc() + int64_t(PCG_THREADS) * 4 - 1) / (int64_t(PCG_THREADS) * 4);
    const int nb = int(std::max<int64_t>(1, std::min<int64_t>(pcg_max_blocks(), want)));
    int* status = &pb.out->status;
    k_reset_pcg<<<1, 1, 0, st>>>(pb.bar, status, wait_polls);
    PcgArgs<T> a;
    a.g = g; a.nf = pb.nf; a.fidx = pb.fidx; a.diag = pb.diag; a.b = rhs;
    for (int i = 0; i < 2; ++i) {
        a.R[i] = static_cast<T*>(pb.R[i]);
        a.Wv[i] = static_cast<T*>(pb.Wv[i]);
        a.S[i] = static_cast<T*>(pb.S[i]);
    }
    a.invd = static_cast<T*>(pb.invd);
    a.P = static_cast<T*>(pb.P);
    a.X = static_cast<T*>(pb.X);
    a.part = pb.part; a.bar = pb.bar; a.status = status; a.out = pb.out;
    a.tol = tol; a.maxit = maxit;
    void* args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_pcg_cg<T>, dim3(nb), dim3(PCG_THREADS), args, 0, st);
    return e == cudaSuccess ? 0 : int(e);
}

void launch_reset_barrier(GridBar* bar, int* status, unsigned wait_polls, cudaStream_t st) {
    k_reset_pcg<<<1, 1, 0, st>>>(bar, status, wait_polls);
}

int launch_pcg(Dims g, PressureBufs& pb, const float* rhs, int fp64, double tol, int maxit, cudaStream_t st,
               unsigned wait_polls) {
    return fp64 ? launch_pcg_t<double>(g, pb, rhs, tol, maxit, st, wait_polls)
                : launch_pcg_t<float>(g, pb, rhs, tol, maxit, st, wait_polls);
}

void launch_pcg_clear(PressureBufs& pb, int fp64, int with_invd, cudaStream_t st) {
    if (fp64) {
        auto c = [&](void* p) { return static_cast<double*>(p); };
        k_clear_padded<double><<<592, 256, 0, st>>>(pb.nf, pb.fidx, c(pb.R[0]), c(pb.R[1]), c(pb.Wv[0]), c(pb.Wv[1]),
                                                    c(pb.S[0]), c(pb.S[1]), with_invd ? c(pb.invd) : nullptr);
    } else {
        auto c = [&](void* p) { return static_cast<float*>(p); };
        k_clear_padded<float><<<592, 256, 0, st>>>(pb.nf, pb.fidx, c(pb.R[0]), c(pb.R[1]), c(pb.Wv[0]), c(pb.Wv[1]),
                                                   c(pb.S[0]), c(pb.S[1]), with_invd ? c(pb.invd) : nullptr);
    }
}

void launch_scatter_p(const PressureBufs& pb, float* p, int src, Dims g, cudaStream_t st) {
    if (src == 0) k_scatter_p<float><<<592, 256, 0, st>>>(pb.nf, pb.fidx, static_cast<const float*>(pb.X), g, p);
    else if (src == 1) k_scatter_p<double><<<592, 256, 0, st>>>(pb.nf, pb.fidx, static_cast<const double*>(pb.X), g, p);
    else k_scatter_p<double><<<592, 256, 0, st>>>(pb.nf, pb.fidx, pb.x64, g, p);
}

void launch_true_residual(PressureBufs& pb, int fp64, Dims g, cudaStream_t st) {
    // The compact solution goes to the padded R[0] grid (free after a solve).
    const int nb = 592;
    auto* part = reinterpret_cast<double2*>(pb.part);
    if (fp64) {
        k_to_dense<double><<<592, 256, 0, st>>>(pb.nf, pb.fidx, static_cast<const double*>(pb.X), static_cast<double*>(pb.R[0]));
        k_residual<double><<<nb, 256, 0, st>>>(pb.nf, pb.fidx, pb.diag, pb.b, static_cast<const double*>(pb.R[0]), g, part,
                                               nullptr, nullptr);
    } else {
        k_to_dense<float><<<592, 256, 0, st>>>(pb.nf, pb.fidx, static_cast<const float*>(pb.X), static_cast<float*>(pb.R[0]));
        k_residual<float><<<nb, 256, 0, st>>>(pb.nf, pb.fidx, pb.diag, pb.b, static_cast<const float*>(pb.R[0]), g, part,
                                              nullptr, nullptr);
    }
    k_sum_partials<<<1, 32, 0, st>>>(part, nb, pb.red);
}

void launch_ir_residual(PressureBufs& pb, Dims g, cudaStream_t st) {
    // r = b - A x64 in FP64 over the padded x64 grid xd; bin = r rounded to FP32.
    const int nb = 592;
    auto* part = reinterpret_cast<double2*>(pb.part);
    k_residual<double><<<nb, 256, 0, st>>>(pb.nf, pb.fidx, pb.diag, pb.b, pb.xd, g, part, pb.bin, nullptr);
    k_sum_partials<<<1, 32, 0, st>>>(part, nb, pb.red);
}

void launch_guess_scale(PressureBufs& pb, Dims g, cudaStream_t st) {
    const int nb = 592;
    auto* part = reinterpret_cast<double2*>(pb.part);
    k_guess_dots<<<nb, 256, 0, st>>>(pb.nf, pb.fidx, pb.diag, pb.b, pb.xd, g, part);
    k_sum_partials<<<1, 32, 0, st>>>(part, nb, pb.red);
    k_scale_guess<<<592, 256, 0, st>>>(pb.nf, pb.fidx, pb.red, pb.x64, pb.xd);
}

void launch_ir_update(PressureBufs& pb, Dims g, cudaStream_t st) {
    k_ir_update<<<592, 256, 0, st>>>(pb.nf, pb.fidx, static_cast<const float*>(pb.X), pb.x64, pb.xd);
    (void)g;
}

void launch_project(float* u, float* v, float* w, const float* p, const uint8_t* labels, Dims g, float dt, BodyKin b,
                    cudaStream_t st, const int* guard) {
    const float scale = dt / (1000.0f * g.dx);  // dt/(rho*dx), FluidSolver3D.cu:2341
    const float inv = 1.0f / scale;
    dim3 blk(32, 8, 1);
    dim3 grd((g.W + 1 + 31) / 32, (g.H + 1 + 7) / 8, g.D + 1);
    k_project<<<grd, blk, 0, st>>>(u, v, w, p, labels, g, scale, inv, b, guard);
}

int csr_cg_solve(int n, const int* offsets, const int* cols, const double* vals, const double* b, double* x, double tol,
                 int maxit, int* iters, double* relres, cudaStream_t st) {
    if (n <= 0) return -1;
    int nnz = offsets[n];
    int *d_off = nullptr, *d_cols = nullptr;
    double *d_vals = nullptr, *d_x = nullptr, *d_r = nullptr, *d_d = nullptr, *d_q = nullptr, *d_z = nullptr,
           *d_dg = nullptr;
    double2* d_part = nullptr;
    cudaError_t e = cudaSuccess;
    auto ck = [&](cudaError_t r) { if (r != cudaSuccess && e == cudaSuccess) e = r; };
    ck(cudaMalloc(&d_off, sizeof(int) * (n + 1)));
    ck(cudaMalloc(&d_cols, sizeof(int) * nnz));
    ck(cudaMalloc(&d_vals, sizeof(double) * nnz));
    for (double** p : {&d_x, &d_r, &d_d, &d_q, &d_z, &d_dg}) ck(cudaMalloc(p, sizeof(double) * n));
    ck(cudaMalloc(&d_part, sizeof(double2) * 65));
    if (e != cudaSuccess) goto done;
    ck(cudaMemcpyAsync(d_off, offsets, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(d_cols, cols, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(d_vals, vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(d_r, b, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    ck(cudaMemsetAsync(d_x, 0, sizeof(double) * n, st));
    {
        const int blk = 128, grd = (n + blk - 1) / blk;
        k_csr_diag<<<grd, blk, 0, st>>>(n, d_off, d_cols, d_vals, d_dg);
        auto dot = [&](const double* a, const double* bb) {
            double h[2];
            k_dot<<<64, 128, 0, st>>>(n, a, bb, d_part);
            k_sum_partials<<<1, 32, 0, st>>>(d_part, 64, reinterpret_cast<double*>(d_part + 64));
            cudaMemcpyAsync(h, reinterpret_cast<double*>(d_part + 64), sizeof(double) * 2, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            return h[0];
        };
        // z = r/diag, d = z
        k_axpy2<<<grd, blk, 0, st>>>(n, 0.0, d_d, d_d, d_x, d_r, d_dg, d_z);
        ck(cudaMemcpyAsync(d_d, d_z, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        const double bb = dot(d_r, d_r);
        double rz = dot(d_r, d_z), rr = bb;
        int it = 0;
        while (bb > 0 && rr > tol * tol * bb && it < maxit) {
            ck(cudaMemsetAsync(d_q, 0, sizeof(double) * n, st));
            k_csr_sym_spmv<<<grd, blk, 0, st>>>(n, d_off, d_cols, d_vals, d_d, d_q);
            double dq = dot(d_d, d_q);
            if (!(dq > 0)) break;
            double alpha = rz / dq;
            k_axpy2<<<grd, blk, 0, st>>>(n, alpha, d_d, d_q, d_x, d_r, d_dg, d_z);
            double rz2 = dot(d_r, d_z);
            rr = dot(d_r, d_r);
            k_xpby<<<grd, blk, 0, st>>>(n, d_z, rz2 / rz, d_d);
            rz = rz2;
            ++it;
        }
        if (iters) *iters = it;
        if (relres) *relres = bb > 0 ? sqrt(rr / bb) : 0.0;
        ck(cudaMemcpyAsync(x, d_x, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        ck(cudaStreamSynchronize(st));
    }
done:
    cudaFree(d_off); cudaFree(d_cols); cudaFree(d_vals);
    for (double* p : {d_x, d_r, d_d, d_q, d_z, d_dg}) cudaFree(p);
    cudaFree(d_part);
    return e == cudaSuccess ? 0 : int(e);
}

}  // namespace fp
