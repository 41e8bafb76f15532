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

// Packed FP32 pairs (sm_100's f32x2 FMA/mul/add): two lanes of one 64-bit
// register, each an IEEE FP32 operation rounded to nearest.
__device__ __forceinline__ float2 f2_fma(float2 a, float2 b, float2 c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;"
        : "=l"(d)
        : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)),
          "l"(*reinterpret_cast<unsigned long long*>(&c)));
    return *reinterpret_cast<float2*>(&d);
}
__device__ __forceinline__ float2 f2_mul(float2 a, float2 b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;"
        : "=l"(d)
        : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)));
    return *reinterpret_cast<float2*>(&d);
}
__device__ __forceinline__ float2 f2_add(float2 a, float2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;"
        : "=l"(d)
        : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)));
    return *reinterpret_cast<float2*>(&d);
}

// Weights of the three face slots s0, s0+1, s0+2 along a non-staggered axis:
// the particle's corners are faces base (1 - f) and base + 1 (f), with base
// s0 or s0 + 1.
__device__ __forceinline__ void axis3(int s0, int base, float f, float (&w)[3]) {
    const bool lo = base == s0;
    w[0] = lo ? 1.0f - f : 0.0f;
    w[1] = lo ? f : 1.0f - f;
    w[2] = lo ? 0.0f : f;
}

// Accumulates one velocity component of the particles [q0, q1) of cell
// (ci, cj, ck) over the 2 x 3 x 3 faces that cell can reach (2 along the
// component's own axis, whose base face is always the cell's), and adds the
// owned ones into shared memory.  COMP selects the component and its
// base-index rules (AccumulateVelocities, FluidSolver3D.cu:465-574).  Weights
// are (wx*wy)*wz as in the reference; the two faces along the component's
// axis are one packed pair, so each particle costs 12 packed multiplies and
// 9 packed FMAs and adds per component.  num accumulates vel*wgt with one
// fused multiply-add (the reference rounds the product first; its float
// atomics already leave the last bits of the sums order-dependent).
template <int COMP>
__device__ __forceinline__ void splat_cell(const float4* __restrict__ pos, const float4* __restrict__ vel, int q0,
                                           int q1, int ci, int cj, int ck, const Dims& g, float* s_num, float* s_den,
                                           int fx0, int fx1, int fy0, int fy1, int fz0, int fz1, int lsx, int lsy) {
    const int W = g.W, H = g.H, D = g.D;
    // first face of each axis' slot range: the cell's own face on the
    // component's axis, the face below the cell on the other two
    const int sx0 = COMP == 0 ? ci : ci - 1, sy0 = COMP == 1 ? cj : cj - 1, sz0 = COMP == 2 ? ck : ck - 1;
    float2 an[9], ad[9];  // pair = the component axis' two faces; index = the other two axes' slots
#pragma unroll
    for (int m = 0; m < 9; ++m) { an[m] = make_float2(0.0f, 0.0f); ad[m] = make_float2(0.0f, 0.0f); }
    // (unrolling this walk by 2 or 4 measured slower: 0.463 and 0.586 ms
    // against 0.401, the larger code missing in the instruction cache)
    for (int q = q0; q < q1; ++q) {
        const float4 P = pos[q];
        const float rx = over_dx(P.x, g), ry = over_dx(P.y, g), rz = over_dx(P.z, g);
        int bi, bj, bk;
        float fx, fy, fz, vc;
        if (COMP == 0) {
            bi = clampi(int(floorf(rx)), 0, W); bj = clampi(int(floorf(ry - 0.5f)), 0, H - 1);
            bk = clampi(int(floorf(rz - 0.5f)), 0, D - 1);
            fx = clamp01(rx - float(bi)); fy = clamp01((ry - 0.5f) - float(bj)); fz = clamp01((rz - 0.5f) - float(bk));
            vc = vel[q].x;
        } else if (COMP == 1) {
            bi = clampi(int(floorf(rx - 0.5f)), 0, W - 1); bj = clampi(int(floorf(ry)), 0, H);
            bk = clampi(int(floorf(rz - 0.5f)), 0, D - 1);
            fx = clamp01((rx - 0.5f) - float(bi)); fy = clamp01(ry - float(bj)); fz = clamp01((rz - 0.5f) - float(bk));
            vc = vel[q].y;
        } else {
            bi = clampi(int(floorf(rx - 0.5f)), 0, W - 1); bj = clampi(int(floorf(ry - 0.5f)), 0, H - 1);
            bk = clampi(int(floorf(rz)), 0, D);
            fx = clamp01((rx - 0.5f) - float(bi)); fy = clamp01((ry - 0.5f) - float(bj)); fz = clamp01(rz - float(bk));
            vc = vel[q].z;
        }
        const float2 vv = make_float2(vc, vc);
        if (COMP == 0) {
            // faces along the component's axis: the base is the cell's own face,
            // or the next one for a particle beyond the grid's far edge (whose
            // cell key is clamped); the other two axes' bases are always the
            // face below the cell or the cell's own (axis3)
            const float2 wa = bi == sx0 ? make_float2(1.0f - fx, fx) : make_float2(0.0f, 1.0f - fx);
            float wy[3], wz[3];
            axis3(sy0, bj, fy, wy);
            axis3(sz0, bk, fz, wz);
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const float2 wab = f2_mul(wa, make_float2(wy[b], wy[b]));
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float2 wgt = f2_mul(wab, make_float2(wz[c], wz[c]));
                    an[b + 3 * c] = f2_fma(vv, wgt, an[b + 3 * c]);
                    ad[b + 3 * c] = f2_add(ad[b + 3 * c], wgt);
                }
            }
        } else if (COMP == 1) {
            const float2 wb = bj == sy0 ? make_float2(1.0f - fy, fy) : make_float2(0.0f, 1.0f - fy);
            float wx[3], wz[3];
            axis3(sx0, bi, fx, wx);
            axis3(sz0, bk, fz, wz);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float2 wab = f2_mul(make_float2(wx[a], wx[a]), wb);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float2 wgt = f2_mul(wab, make_float2(wz[c], wz[c]));
                    an[a + 3 * c] = f2_fma(vv, wgt, an[a + 3 * c]);
                    ad[a + 3 * c] = f2_add(ad[a + 3 * c], wgt);
                }
            }
        } else {
            const float2 wc = bk == sz0 ? make_float2(1.0f - fz, fz) : make_float2(0.0f, 1.0f - fz);
            float wx[3], wy[3];
            axis3(sx0, bi, fx, wx);
            axis3(sy0, bj, fy, wy);
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const float wab = wx[a] * wy[b];
                    const float2 wgt = f2_mul(make_float2(wab, wab), wc);
                    an[a + 3 * b] = f2_fma(vv, wgt, an[a + 3 * b]);
                    ad[a + 3 * b] = f2_add(ad[a + 3 * b], wgt);
                }
        }
    }
    // owned faces into shared memory: slot m of the pair is face +0 / +1 along
    // the component's axis
#pragma unroll
    for (int m = 0; m < 9; ++m)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int o1 = m % 3, o2 = m / 3;
            const float num = e ? an[m].y : an[m].x, den = e ? ad[m].y : ad[m].x;
            const int fi = COMP == 0 ? sx0 + e : sx0 + o1;
            const int fj = COMP == 1 ? sy0 + e : sy0 + (COMP == 0 ? o1 : o2);
            const int fk = COMP == 2 ? sz0 + e : sz0 + o2;
            if (den == 0.0f || fi < fx0 || fi > fx1 || fj < fy0 || fj > fy1 || fk < fz0 || fk > fz1) continue;
            const int sidx = (fi - fx0) + lsx * ((fj - fy0) + lsy * (fk - fz0));
            atomicAdd(&s_num[sidx], num);
            atomicAdd(&s_den[sidx], den);
        }
}

// Owned face ranges of a brick (inclusive): cells [i0, ie] x [j0, je] x
// [k0, ke]; the staggered component of an axis also owns the far boundary
// face in the last brick of that axis (iue, jve, kwe).
struct Owned {
    int i0, ie, iue, j0, je, jve, k0, ke, kwe;
};

// All three components of one cell's particles.
template <int BX, int BY, int BZ>
__device__ __forceinline__ void splat_all(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                             const int* __restrict__ start, int ci, int cj, int ck, const Dims& g,
                                             float* s_num, float* s_den, const Owned& o) {
    constexpr int NU = (BX + 1) * BY * BZ, NV = BX * (BY + 1) * BZ;
    const int c = ci + cj * g.W + ck * g.W * g.H;
    const int q0 = start[c], q1 = start[c + 1];
    if (q0 == q1) return;
    splat_cell<0>(pos, vel, q0, q1, ci, cj, ck, g, s_num, s_den, o.i0, o.iue, o.j0, o.je, o.k0, o.ke, BX + 1, BY);
    splat_cell<1>(pos, vel, q0, q1, ci, cj, ck, g, s_num + NU, s_den + NU, o.i0, o.ie, o.j0, o.jve, o.k0, o.ke, BX,
                  BY + 1);
    splat_cell<2>(pos, vel, q0, q1, ci, cj, ck, g, s_num + NU + NV, s_den + NU + NV, o.i0, o.ie, o.j0, o.je, o.k0,
                  o.kwe, BX, BY);
}

// CTAs per SM that the register budget must allow (P2G_MIN_BLOCKS, a build
// tunable): 3 gives 80 registers, 2 gives up to 128; the walk over a cell's
// particles is latency-bound, so occupancy and spills trade against each other.
#ifndef P2G_MIN_BLOCKS
#define P2G_MIN_BLOCKS 3
#endif

template <int BX, int BY, int BZ, int NT>
__global__ void __launch_bounds__(NT, P2G_MIN_BLOCKS) k_p2g(const float4* __restrict__ pos, const float4* __restrict__ vel,
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

    // Cells whose particles reach an owned face: the brick plus one halo
    // cell, each with its full 2 x 3 x 3 window per component.  (Splats
    // specialised to the few slots a halo cell reaches, one per face of the
    // halo shell, made the kernel 2.7x larger and slower: instruction-cache
    // misses became its largest stall.)
    const Owned own{i0, ie, iue, j0, je, jve, k0, ke, kwe};
    const int ilo = max(i0 - 1, 0), ihi = min(ie + 1, W - 1);
    const int jlo = max(j0 - 1, 0), jhi = min(je + 1, H - 1);
    const int klo = max(k0 - 1, 0), khi = min(ke + 1, D - 1);
    const int ni = ihi - ilo + 1, nj = jhi - jlo + 1;
    for (int t = threadIdx.x; t < ni * nj * (khi - klo + 1); t += NT)
        splat_all<BX, BY, BZ>(pos, vel, start, ilo + t % ni, jlo + (t / ni) % nj, klo + t / (ni * nj), g, s_num, s_den,
                              own);
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
