// kernels_p2g.cu -- particle-to-grid transfer on the MAC grid.
//
// Restates particlesToGrid (FluidSolver3D.cu:438-685): per particle, 8
// trilinear weights per velocity component (base index floor(r - offset),
// clamped; fractions clamped to [0,1]; faces outside the grid skipped), then
// u = num/den where den > 1e-8, else 0.  The epilogue also performs
// saveVelocities (:399-415, u* = u before gravity) and applyForces
// (:700-761, gravity on every face with the x > (float)INT_MIN test).
//
// B200 design: particles are sorted by cell, so each CTA owns a brick of
// BX x BY x BZ cells and the faces of those cells.  One thread per cell of
// the brick plus a one-cell halo walks that cell's (contiguous) particles and
// sums their contributions to the 2x3x3 faces the cell can reach in
// registers; it then adds the faces owned by the brick into shared-memory
// accumulators (one atomic per face and cell instead of one per particle and
// corner), and the CTA writes each owned face once: no global atomics and no
// accumulator arrays in HBM.  Halo cells are read by up to 8 CTAs (from L2).
#include "kernels.hpp"

namespace fp {

namespace {

// Slot weights along one axis: slot m is face s0 + m; the particle's two
// corners are faces base (weight 1 - f) and base + 1 (weight f).
template <int NS>
__device__ __forceinline__ void axis_weights(int s0, int base, float f, float (&w)[NS]) {
#pragma unroll
    for (int m = 0; m < NS; ++m) {
        const int face = s0 + m;
        w[m] = face == base ? 1.0f - f : (face == base + 1 ? f : 0.0f);
    }
}

// Accumulates one velocity component of the particles [q0, q1) of cell
// (ci, cj, ck) over the faces that cell can reach -- NX x NY x NZ slots whose
// first face is (sx0, sy0, sz0) -- and adds the owned ones into shared memory.
// COMP selects the component and its base-index rules (AccumulateVelocities,
// FluidSolver3D.cu:465-574); weights are (wx*wy)*wz and contributions
// vel*wgt, rounded as in the reference.
template <int COMP, int NX, int NY, int NZ>
__device__ __forceinline__ void splat_cell(const float4* __restrict__ pos, const float4* __restrict__ vel, int q0,
                                           int q1, int ci, int cj, int ck, const Dims& g, float* s_num, float* s_den,
                                           int fx0, int fx1, int fy0, int fy1, int fz0, int fz1, int lsx, int lsy) {
    const int W = g.W, H = g.H, D = g.D;
    const int sx0 = COMP == 0 ? ci : ci - 1, sy0 = COMP == 1 ? cj : cj - 1, sz0 = COMP == 2 ? ck : ck - 1;
    float an[NX * NY * NZ], ad[NX * NY * NZ];
#pragma unroll
    for (int m = 0; m < NX * NY * NZ; ++m) { an[m] = 0.0f; ad[m] = 0.0f; }
    const float dx = g.dx;
    for (int q = q0; q < q1; ++q) {
        const float4 P = pos[q];
        const float4 V = vel[q];
        const float rx = P.x / dx, ry = P.y / dx, rz = P.z / dx;
        int bi, bj, bk;
        float fx, fy, fz, vc;
        if (COMP == 0) {
            bi = clampi(int(floorf(rx)), 0, W); bj = clampi(int(floorf(ry - 0.5f)), 0, H - 1);
            bk = clampi(int(floorf(rz - 0.5f)), 0, D - 1);
            fx = clamp01(rx - float(bi)); fy = clamp01((ry - 0.5f) - float(bj)); fz = clamp01((rz - 0.5f) - float(bk));
            vc = V.x;
        } else if (COMP == 1) {
            bi = clampi(int(floorf(rx - 0.5f)), 0, W - 1); bj = clampi(int(floorf(ry)), 0, H);
            bk = clampi(int(floorf(rz - 0.5f)), 0, D - 1);
            fx = clamp01((rx - 0.5f) - float(bi)); fy = clamp01(ry - float(bj)); fz = clamp01((rz - 0.5f) - float(bk));
            vc = V.y;
        } else {
            bi = clampi(int(floorf(rx - 0.5f)), 0, W - 1); bj = clampi(int(floorf(ry - 0.5f)), 0, H - 1);
            bk = clampi(int(floorf(rz)), 0, D);
            fx = clamp01((rx - 0.5f) - float(bi)); fy = clamp01((ry - 0.5f) - float(bj)); fz = clamp01(rz - float(bk));
            vc = V.z;
        }
        float wx[NX], wy[NY], wz[NZ];
        axis_weights<NX>(sx0, bi, fx, wx);
        axis_weights<NY>(sy0, bj, fy, wy);
        axis_weights<NZ>(sz0, bk, fz, wz);
#pragma unroll
        for (int c = 0; c < NZ; ++c)
#pragma unroll
            for (int b = 0; b < NY; ++b)
#pragma unroll
                for (int a = 0; a < NX; ++a) {
                    const float wgt = wx[a] * wy[b] * wz[c];
                    const int m = a + NX * (b + NY * c);
                    an[m] += __fmul_rn(vc, wgt);
                    ad[m] += wgt;
                }
    }
#pragma unroll
    for (int c = 0; c < NZ; ++c)
#pragma unroll
        for (int b = 0; b < NY; ++b)
#pragma unroll
            for (int a = 0; a < NX; ++a) {
                const int m = a + NX * (b + NY * c);
                const int fi = sx0 + a, fj = sy0 + b, fk = sz0 + c;
                if (ad[m] == 0.0f || fi < fx0 || fi > fx1 || fj < fy0 || fj > fy1 || fk < fz0 || fk > fz1) continue;
                const int sidx = (fi - fx0) + lsx * ((fj - fy0) + lsy * (fk - fz0));
                atomicAdd(&s_num[sidx], an[m]);
                atomicAdd(&s_den[sidx], ad[m]);
            }
}

// Three CTAs per SM: 80 registers and no spills, against 126 registers and
// two CTAs unbounded; the walk over a cell's particles is latency-bound.
template <int BX, int BY, int BZ, int NT>
__global__ void __launch_bounds__(NT, 3) k_p2g(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                            const int* __restrict__ start, Dims g, float dt, float3 grav,
                                            float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
                                            float* __restrict__ us, float* __restrict__ vs, float* __restrict__ ws,
                                            int fused) {
    constexpr int NU = (BX + 1) * BY * BZ, NV = BX * (BY + 1) * BZ, NW = BX * BY * (BZ + 1);
    __shared__ float s_num[NU + NV + NW];
    __shared__ float s_den[NU + NV + NW];

    const int W = g.W, H = g.H, D = g.D;
    const int nbx = (W + BX - 1) / BX, nby = (H + BY - 1) / BY;
    const int bid = blockIdx.x;
    const int i0 = (bid % nbx) * BX, j0 = ((bid / nbx) % nby) * BY, k0 = (bid / (nbx * nby)) * BZ;

    for (int t = threadIdx.x; t < NU + NV + NW; t += NT) { s_num[t] = 0.0f; s_den[t] = 0.0f; }

    // Owned face ranges (inclusive); the last brick on an axis also owns the
    // far boundary face of that axis' component.
    const int ie = min(i0 + BX, W) - 1, je = min(j0 + BY, H) - 1, ke = min(k0 + BZ, D) - 1;
    const int iue = (i0 + BX >= W) ? W : ie;
    const int jve = (j0 + BY >= H) ? H : je;
    const int kwe = (k0 + BZ >= D) ? D : ke;
    __syncthreads();

    // Cells whose particles reach an owned face: the brick plus one halo cell.
    const int ilo = max(i0 - 1, 0), ihi = min(i0 + BX, W - 1);
    const int jlo = max(j0 - 1, 0), jhi = min(j0 + BY, H - 1);
    const int klo = max(k0 - 1, 0), khi = min(k0 + BZ, D - 1);
    const int ni = ihi - ilo + 1, nj = jhi - jlo + 1, ncell = ni * nj * (khi - klo + 1);
    for (int t = threadIdx.x; t < ncell; t += NT) {
        const int ci = ilo + t % ni, cj = jlo + (t / ni) % nj, ck = klo + t / (ni * nj);
        const int c = ci + cj * W + ck * W * H;
        const int q0 = start[c], q1 = start[c + 1];
        if (q0 == q1) continue;
        splat_cell<0, 2, 3, 3>(pos, vel, q0, q1, ci, cj, ck, g, s_num, s_den, i0, iue, j0, je, k0, ke, BX + 1, BY);
        splat_cell<1, 3, 2, 3>(pos, vel, q0, q1, ci, cj, ck, g, s_num + NU, s_den + NU, i0, ie, j0, jve, k0, ke, BX,
                               BY + 1);
        splat_cell<2, 3, 3, 2>(pos, vel, q0, q1, ci, cj, ck, g, s_num + NU + NV, s_den + NU + NV, i0, ie, j0, je, k0,
                               kwe, BX, BY);
    }
    __syncthreads();

    // Epilogue: num/den (ComputeVelocityFunc :598-605), u* <- u, u += dt*g.
    const float lim = -2147483648.0f;
    auto finish = [&](float num, float den, float gcomp, float* dst, float* sav, int64_t idx) {
        float val = (den > 1e-8f) ? num / den : 0.0f;
        if (fused) {
            sav[idx] = val;
            dst[idx] = (val > lim) ? val + dt * gcomp : val;
        } else {
            dst[idx] = val;
        }
    };
    {
        const int ni2 = iue - i0 + 1, nj2 = je - j0 + 1, nk2 = ke - k0 + 1;
        for (int t = threadIdx.x; t < ni2 * nj2 * nk2; t += NT) {
            int li = t % ni2, lj = (t / ni2) % nj2, lk = t / (ni2 * nj2);
            int sidx = li + (BX + 1) * (lj + BY * lk);
            int64_t idx = int64_t(i0 + li) + int64_t(j0 + lj) * (W + 1) + int64_t(k0 + lk) * (W + 1) * H;
            finish(s_num[sidx], s_den[sidx], grav.x, u, us, idx);
        }
    }
    {
        const int ni2 = ie - i0 + 1, nj2 = jve - j0 + 1, nk2 = ke - k0 + 1;
        for (int t = threadIdx.x; t < ni2 * nj2 * nk2; t += NT) {
            int li = t % ni2, lj = (t / ni2) % nj2, lk = t / (ni2 * nj2);
            int sidx = NU + li + BX * (lj + (BY + 1) * lk);
            int64_t idx = int64_t(i0 + li) + int64_t(j0 + lj) * W + int64_t(k0 + lk) * W * (H + 1);
            finish(s_num[sidx], s_den[sidx], grav.y, v, vs, idx);
        }
    }
    {
        const int ni2 = ie - i0 + 1, nj2 = je - j0 + 1, nk2 = kwe - k0 + 1;
        for (int t = threadIdx.x; t < ni2 * nj2 * nk2; t += NT) {
            int li = t % ni2, lj = (t / ni2) % nj2, lk = t / (ni2 * nj2);
            int sidx = NU + NV + li + BX * (lj + BY * lk);
            int64_t idx = int64_t(i0 + li) + int64_t(j0 + lj) * W + int64_t(k0 + lk) * W * H;
            finish(s_num[sidx], s_den[sidx], grav.z, w, ws, idx);
        }
    }
}

// applyForces alone (phase-by-phase mode): x > (float)INT_MIN ? x + dt*a : x.
__global__ void k_forces(float* __restrict__ a, int64_t n, float dt, float acc) {
    int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    float x = a[t];
    a[t] = (x > -2147483648.0f) ? x + dt * acc : x;
}

__global__ void k_copy(const float* __restrict__ s, float* __restrict__ d, int64_t n) {
    int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n) d[t] = s[t];
}

}  // namespace

constexpr int P2G_BX = 16, P2G_BY = 8, P2G_BZ = 8, P2G_NT = 256;

void launch_p2g(const float4* pos, const float4* vel, const int* start, Dims g, float dt, float3 gravity, float* u,
                float* v, float* w, float* us, float* vs, float* ws, int fused_forces, cudaStream_t st) {
    int nb = ((g.W + P2G_BX - 1) / P2G_BX) * ((g.H + P2G_BY - 1) / P2G_BY) * ((g.D + P2G_BZ - 1) / P2G_BZ);
    k_p2g<P2G_BX, P2G_BY, P2G_BZ, P2G_NT>
        <<<nb, P2G_NT, 0, st>>>(pos, vel, start, g, dt, gravity, u, v, w, us, vs, ws, fused_forces);
}

void launch_forces(float* u, float* v, float* w, Dims g, float dt, float3 gravity, cudaStream_t st) {
    k_forces<<<unsigned((g.nu() + 255) / 256), 256, 0, st>>>(u, g.nu(), dt, gravity.x);
    k_forces<<<unsigned((g.nv() + 255) / 256), 256, 0, st>>>(v, g.nv(), dt, gravity.y);
    k_forces<<<unsigned((g.nw() + 255) / 256), 256, 0, st>>>(w, g.nw(), dt, gravity.z);
}

void launch_copy(const float* src, float* dst, int64_t n, cudaStream_t st) {
    if (n > 0) k_copy<<<unsigned((n + 255) / 256), 256, 0, st>>>(src, dst, n);
}

}  // namespace fp
