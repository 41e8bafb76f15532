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
// BX x BY x BZ cells and the faces of those cells.  It reads the particles of
// the brick plus a one-cell halo (contiguous runs per (j,k) row of cells),
// splats them into shared-memory accumulators, and writes each owned face
// once: no global atomics, no accumulator arrays in HBM, coalesced particle
// loads.  Halo particles are read by up to 8 CTAs (from L2).
#include "kernels.hpp"

namespace fp {

namespace {

template <int BX, int BY, int BZ, int NT>
__global__ void __launch_bounds__(NT) k_p2g(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                            const int* __restrict__ start, Dims g, float dt, float3 grav,
                                            float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
                                            float* __restrict__ us, float* __restrict__ vs, float* __restrict__ ws,
                                            int fused) {
    constexpr int NU = (BX + 1) * BY * BZ, NV = BX * (BY + 1) * BZ, NW = BX * BY * (BZ + 1);
    constexpr int MAXROWS = (BY + 2) * (BZ + 2);
    __shared__ float s_num[NU + NV + NW];
    __shared__ float s_den[NU + NV + NW];
    __shared__ int s_row_begin[MAXROWS];
    __shared__ int s_row_pref[MAXROWS + 1];

    const int W = g.W, H = g.H, D = g.D;
    const int nbx = (W + BX - 1) / BX, nby = (H + BY - 1) / BY;
    const int bid = blockIdx.x;
    const int i0 = (bid % nbx) * BX, j0 = ((bid / nbx) % nby) * BY, k0 = (bid / (nbx * nby)) * BZ;

    for (int t = threadIdx.x; t < NU + NV + NW; t += NT) { s_num[t] = 0.0f; s_den[t] = 0.0f; }

    // Particle rows of the halo region [i0-1, i0+BX] x [j0-1, j0+BY] x [k0-1, k0+BZ].
    const int ilo = max(i0 - 1, 0), ihi = min(i0 + BX, W - 1);
    const int jlo = max(j0 - 1, 0), jhi = min(j0 + BY, H - 1);
    const int klo = max(k0 - 1, 0), khi = min(k0 + BZ, D - 1);
    const int nrj = jhi - jlo + 1, nrows = nrj * (khi - klo + 1);
    for (int r = threadIdx.x; r < nrows; r += NT) {
        int rj = jlo + r % nrj, rk = klo + r / nrj;
        int c0 = ilo + rj * W + rk * W * H, c1 = ihi + rj * W + rk * W * H;
        int b0 = start[c0];
        s_row_begin[r] = b0;
        s_row_pref[r + 1] = start[c1 + 1] - b0;
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // inclusive scan of the row lengths by one warp
        int carry = 0;
        for (int base = 0; base < nrows; base += 32) {
            int r = base + threadIdx.x;
            int x = r < nrows ? s_row_pref[r + 1] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, o);
                if ((threadIdx.x & 31) >= o) x += y;
            }
            if (r < nrows) s_row_pref[r + 1] = carry + x;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (threadIdx.x == 0) s_row_pref[0] = 0;
    }
    __syncthreads();

    // Owned face ranges (inclusive upper bounds); the last brick on an axis
    // also owns the far boundary face of that axis' component.
    const int ie = min(i0 + BX, W) - 1, je = min(j0 + BY, H) - 1, ke = min(k0 + BZ, D) - 1;
    const int iue = (i0 + BX >= W) ? W : ie;
    const int jve = (j0 + BY >= H) ? H : je;
    const int kwe = (k0 + BZ >= D) ? D : ke;

    const int total = s_row_pref[nrows];
    const float dx = g.dx;
    for (int t = threadIdx.x; t < total; t += NT) {
        int lo = 0, hi = nrows - 1;  // last row with pref <= t
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (s_row_pref[mid] <= t) lo = mid; else hi = mid - 1;
        }
        const int q = s_row_begin[lo] + (t - s_row_pref[lo]);
        const float4 P = pos[q];
        const float4 V = vel[q];
        const float rx = P.x / dx, ry = P.y / dx, rz = P.z / dx;
        // U component (AccumulateVelocities, FluidSolver3D.cu:465-498)
        {
            int iU = clampi(int(floorf(rx)), 0, W), jU = clampi(int(floorf(ry - 0.5f)), 0, H - 1),
                kU = clampi(int(floorf(rz - 0.5f)), 0, D - 1);
            float fx = clamp01(rx - float(iU)), fy = clamp01((ry - 0.5f) - float(jU)), fz = clamp01((rz - 0.5f) - float(kU));
#pragma unroll
            for (int dz = 0; dz < 2; ++dz) {
                int k = kU + dz;
                if (k >= D || k < k0 || k > ke) continue;
#pragma unroll
                for (int dy = 0; dy < 2; ++dy) {
                    int j = jU + dy;
                    if (j >= H || j < j0 || j > je) continue;
#pragma unroll
                    for (int dxx = 0; dxx < 2; ++dxx) {
                        int i = iU + dxx;
                        if (i > W || i < i0 || i > iue) continue;
                        float wx = dxx == 0 ? 1.0f - fx : fx, wy = dy == 0 ? 1.0f - fy : fy, wz = dz == 0 ? 1.0f - fz : fz;
                        float wgt = wx * wy * wz;
                        int s = (i - i0) + (BX + 1) * ((j - j0) + BY * (k - k0));
                        atomicAdd(&s_num[s], __fmul_rn(V.x, wgt));
                        atomicAdd(&s_den[s], wgt);
                    }
                }
            }
        }
        // V component (:503-536)
        {
            int iV = clampi(int(floorf(rx - 0.5f)), 0, W - 1), jV = clampi(int(floorf(ry)), 0, H),
                kV = clampi(int(floorf(rz - 0.5f)), 0, D - 1);
            float fx = clamp01((rx - 0.5f) - float(iV)), fy = clamp01(ry - float(jV)), fz = clamp01((rz - 0.5f) - float(kV));
#pragma unroll
            for (int dz = 0; dz < 2; ++dz) {
                int k = kV + dz;
                if (k >= D || k < k0 || k > ke) continue;
#pragma unroll
                for (int dy = 0; dy < 2; ++dy) {
                    int j = jV + dy;
                    if (j > H || j < j0 || j > jve) continue;
#pragma unroll
                    for (int dxx = 0; dxx < 2; ++dxx) {
                        int i = iV + dxx;
                        if (i >= W || i < i0 || i > ie) continue;
                        float wx = dxx == 0 ? 1.0f - fx : fx, wy = dy == 0 ? 1.0f - fy : fy, wz = dz == 0 ? 1.0f - fz : fz;
                        float wgt = wx * wy * wz;
                        int s = NU + (i - i0) + BX * ((j - j0) + (BY + 1) * (k - k0));
                        atomicAdd(&s_num[s], __fmul_rn(V.y, wgt));
                        atomicAdd(&s_den[s], wgt);
                    }
                }
            }
        }
        // W component (:541-574)
        {
            int iW = clampi(int(floorf(rx - 0.5f)), 0, W - 1), jW = clampi(int(floorf(ry - 0.5f)), 0, H - 1),
                kW = clampi(int(floorf(rz)), 0, D);
            float fx = clamp01((rx - 0.5f) - float(iW)), fy = clamp01((ry - 0.5f) - float(jW)), fz = clamp01(rz - float(kW));
#pragma unroll
            for (int dz = 0; dz < 2; ++dz) {
                int k = kW + dz;
                if (k > D || k < k0 || k > kwe) continue;
#pragma unroll
                for (int dy = 0; dy < 2; ++dy) {
                    int j = jW + dy;
                    if (j >= H || j < j0 || j > je) continue;
#pragma unroll
                    for (int dxx = 0; dxx < 2; ++dxx) {
                        int i = iW + dxx;
                        if (i >= W || i < i0 || i > ie) continue;
                        float wx = dxx == 0 ? 1.0f - fx : fx, wy = dy == 0 ? 1.0f - fy : fy, wz = dz == 0 ? 1.0f - fz : fz;
                        float wgt = wx * wy * wz;
                        int s = NU + NV + (i - i0) + BX * ((j - j0) + BY * (k - k0));
                        atomicAdd(&s_num[s], __fmul_rn(V.z, wgt));
                        atomicAdd(&s_den[s], wgt);
                    }
                }
            }
        }
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
        const int ni = iue - i0 + 1, nj = je - j0 + 1, nk = ke - k0 + 1;
        for (int t = threadIdx.x; t < ni * nj * nk; t += NT) {
            int li = t % ni, lj = (t / ni) % nj, lk = t / (ni * nj);
            int s = li + (BX + 1) * (lj + BY * lk);
            int64_t idx = int64_t(i0 + li) + int64_t(j0 + lj) * (W + 1) + int64_t(k0 + lk) * (W + 1) * H;
            finish(s_num[s], s_den[s], grav.x, u, us, idx);
        }
    }
    {
        const int ni = ie - i0 + 1, nj = jve - j0 + 1, nk = ke - k0 + 1;
        for (int t = threadIdx.x; t < ni * nj * nk; t += NT) {
            int li = t % ni, lj = (t / ni) % nj, lk = t / (ni * nj);
            int s = NU + li + BX * (lj + (BY + 1) * lk);
            int64_t idx = int64_t(i0 + li) + int64_t(j0 + lj) * W + int64_t(k0 + lk) * W * (H + 1);
            finish(s_num[s], s_den[s], grav.y, v, vs, idx);
        }
    }
    {
        const int ni = ie - i0 + 1, nj = je - j0 + 1, nk = kwe - k0 + 1;
        for (int t = threadIdx.x; t < ni * nj * nk; t += NT) {
            int li = t % ni, lj = (t / ni) % nj, lk = t / (ni * nj);
            int s = NU + NV + li + BX * (lj + BY * lk);
            int64_t idx = int64_t(i0 + li) + int64_t(j0 + lj) * W + int64_t(k0 + lk) * W * H;
            finish(s_num[s], s_den[s], grav.z, w, ws, idx);
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

constexpr int P2G_BX = 16, P2G_BY = 8, P2G_BZ = 8, P2G_NT = 512;

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
