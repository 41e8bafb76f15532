// kernels_p2g.cu -- particle-to-grid transfer on the MAC grid.
//
// Restates particlesToGrid (FluidSolver3D.cu:438-685): per particle, 8
// trilinear weights per velocity component (base index floor(r - offset),
// clamped; fractions clamped to [0,1]; faces outside the grid skipped), then
// u = num/den where den > 1e-8, else 0.  The epilogue also performs
// saveVelocities (:399-415, u* = u before gravity) and applyForces
// (:700-761, gravity on every face with the x > (float)INT_MIN test).
//
// B200 design: particles are sorted by cell, and each CTA owns a brick of
// BX x BY x BZ cells.  One thread per cell walks that cell's (contiguous)
// particles once and sums their contributions to the 2 x 3 x 3 faces the cell
// can reach in registers; it then adds them into shared-memory accumulators
// covering the faces the brick's cells reach (one atomic per face and cell
// instead of one per particle and corner).  Each brick adds its accumulated
// (num, den) pairs into a global FP32 pair array with one vector reduction
// per face, so every particle is walked once (a brick that instead re-walks
// a one-cell halo to own its faces outright walks each particle 1.76 times
// on average for 16 x 8 x 8 bricks); empty bricks return at once.  Small
// bricks balance the SMs: the dam break's ~640 full 16 x 8 x 8 bricks filled
// 1.4 waves of three CTAs per SM (0.232 ms for the phase at 128^3, 0.198 with
// 8 x 8 x 8).  The default is 8 x 8 x 4 cells, one per thread of a 128-thread
// CTA, eight CTAs per SM (0.180 ms; 8 x 8 x 8 with 256 threads at four per SM
// 0.186, 8 x 4 x 4 0.182).  A second,
// elementwise kernel divides, saves and adds gravity, and zeroes the pair
// array for the next step.
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
// component's own axis, whose base face is always the cell's), and adds them
// into the brick's shared-memory accumulators, whose face (ex0, ey0, ez0) is
// slot 0 (strides lsx, lsy).  COMP selects the component and its base-index
// rules (AccumulateVelocities::operator(), FluidSolver3D.cu:469-574).  Weights are
// (wx*wy)*wz as in the reference; the two faces along the component's axis
// are one packed pair, so each particle costs 12 packed multiplies and 9
// packed FMAs and adds per component.  num accumulates vel*wgt with one fused
// multiply-add (the reference rounds the product first; its float atomics
// already leave the last bits of the sums order-dependent).
// The particle's velocity component COMP.
template <int COMP>
__device__ __forceinline__ float comp_of(const float4& v) { return COMP == 0 ? v.x : (COMP == 1 ? v.y : v.z); }

template <int COMP, bool P2>
__device__ __forceinline__ void splat_cell(const float4* __restrict__ pos, const float4* __restrict__ vel, int q0,
                                           int q1, int ci, int cj, int ck, const Dims& g, float* s_num, float* s_den,
                                           int ex0, int ey0, int ez0, int lsx, int lsy) {
    const int W = g.W, H = g.H, D = g.D;
    // first face of each axis' slot range: the cell's own face on the
    // component's axis, the face below the cell on the other two
    const int sx0 = COMP == 0 ? ci : ci - 1, sy0 = COMP == 1 ? cj : cj - 1, sz0 = COMP == 2 ? ck : ck - 1;
    float2 an[9], ad[9];  // pair = the component axis' two faces; index = the other two axes' slots
#pragma unroll
    for (int m = 0; m < 9; ++m) { an[m] = make_float2(0.0f, 0.0f); ad[m] = make_float2(0.0f, 0.0f); }
    // (unrolling this walk by 2 or 4 measured slower: the larger code missed
    // in the instruction cache; prefetching the next particle gained 1 us)
    for (int q = q0; q < q1; ++q) {
        const float4 P = pos[q];
        const float vc = comp_of<COMP>(vel[q]);
        const float rx = to_grid<P2>(P.x, g), ry = to_grid<P2>(P.y, g), rz = to_grid<P2>(P.z, g);
        int bi, bj, bk;
        float fx, fy, fz;
        if (COMP == 0) {
            bi = clampi(int(floorf(rx)), 0, W); bj = clampi(int(floorf(ry - 0.5f)), 0, H - 1);
            bk = clampi(int(floorf(rz - 0.5f)), 0, D - 1);
            fx = clamp01(rx - float(bi)); fy = clamp01((ry - 0.5f) - float(bj)); fz = clamp01((rz - 0.5f) - float(bk));
        } else if (COMP == 1) {
            bi = clampi(int(floorf(rx - 0.5f)), 0, W - 1); bj = clampi(int(floorf(ry)), 0, H);
            bk = clampi(int(floorf(rz - 0.5f)), 0, D - 1);
            fx = clamp01((rx - 0.5f) - float(bi)); fy = clamp01(ry - float(bj)); fz = clamp01((rz - 0.5f) - float(bk));
        } else {
            bi = clampi(int(floorf(rx - 0.5f)), 0, W - 1); bj = clampi(int(floorf(ry - 0.5f)), 0, H - 1);
            bk = clampi(int(floorf(rz)), 0, D);
            fx = clamp01((rx - 0.5f) - float(bi)); fy = clamp01((ry - 0.5f) - float(bj)); fz = clamp01(rz - float(bk));
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
    // into shared memory: slot m of the pair is face +0 / +1 along the
    // component's axis; every slot lies inside the brick's reach region
#pragma unroll
    for (int m = 0; m < 9; ++m)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int o1 = m % 3, o2 = m / 3;
            const float num = e ? an[m].y : an[m].x, den = e ? ad[m].y : ad[m].x;
            if (den == 0.0f) continue;
            const int fi = COMP == 0 ? sx0 + e : sx0 + o1;
            const int fj = COMP == 1 ? sy0 + e : sy0 + (COMP == 0 ? o1 : o2);
            const int fk = COMP == 2 ? sz0 + e : sz0 + o2;
            const int sidx = (fi - ex0) + lsx * ((fj - ey0) + lsy * (fk - ez0));
            atomicAdd(&s_num[sidx], num);
            atomicAdd(&s_den[sidx], den);
        }
}

// The faces the cells of a brick [i0, i0+BX) x [j0, j0+BY) x [k0, k0+BZ)
// reach, per component: along the component's own axis the brick's faces
// and the far one (N+1), along the other two one more on each side (N+2).
template <int BX, int BY, int BZ>
struct Reach {
    static constexpr int UX = BX + 1, UY = BY + 2, UZ = BZ + 2;
    static constexpr int VX = BX + 2, VY = BY + 1, VZ = BZ + 2;
    static constexpr int WX = BX + 2, WY = BY + 2, WZ = BZ + 1;
    static constexpr int NU = UX * UY * UZ, NV = VX * VY * VZ, NW = WX * WY * WZ, N = NU + NV + NW;
};

// CTAs per SM that the register budget must allow (P2G_MIN_BLOCKS, a build
// tunable): the walk over a cell's particles is latency-bound, so occupancy
// and spills trade against each other.  With 256-thread 8 x 8 x 8 bricks at
// 128^3, four per SM (64 registers, a 12-byte spill) took the phase to 0.186
// ms; three (78 registers) gave 0.202, two 0.220, and five and six spilled
// (0.30, 0.49 ms).  The default is 64 registers for the 128-thread CTAs.
#ifndef P2G_MIN_BLOCKS
#define P2G_MIN_BLOCKS 8
#endif

// Pass 1: one CTA per brick.  acc holds (num, den) pairs for the u, v and w
// faces back to back ([nu | nv | nw]); it is zero on entry except for what
// other bricks of this launch add.
template <int BX, int BY, int BZ, int NT, bool P2>
__global__ void __launch_bounds__(NT, P2G_MIN_BLOCKS) k_p2g_accum(const float4* __restrict__ pos,
                                                                  const float4* __restrict__ vel,
                                                                  const int* __restrict__ start, Dims g,
                                                                  float2* __restrict__ acc) {
    using R = Reach<BX, BY, BZ>;
    __shared__ float s_num[R::N];
    __shared__ float s_den[R::N];

    const int W = g.W, H = g.H, D = g.D;
    const int nbx = (W + BX - 1) / BX, nby = (H + BY - 1) / BY;
    const int bid = blockIdx.x;
    const int i0 = (bid % nbx) * BX, j0 = ((bid / nbx) % nby) * BY, k0 = (bid / (nbx * nby)) * BZ;
    const int ni = min(BX, W - i0), nj = min(BY, H - j0), nk = min(BZ, D - k0);

    bool any = false;
    for (int t = threadIdx.x; t < ni * nj * nk; t += NT) {
        const int c = (i0 + t % ni) + (j0 + (t / ni) % nj) * W + (k0 + t / (ni * nj)) * W * H;
        any |= start[c + 1] > start[c];
    }
    if (!__syncthreads_or(any)) return;  // no particle: nothing to add
    for (int t = threadIdx.x; t < R::N; t += NT) { s_num[t] = 0.0f; s_den[t] = 0.0f; }
    __syncthreads();

    for (int t = threadIdx.x; t < ni * nj * nk; t += NT) {
        const int ci = i0 + t % ni, cj = j0 + (t / ni) % nj, ck = k0 + t / (ni * nj);
        const int c = ci + cj * W + ck * W * H;
        const int q0 = start[c], q1 = start[c + 1];
        if (q0 == q1) continue;
        splat_cell<0, P2>(pos, vel, q0, q1, ci, cj, ck, g, s_num, s_den, i0, j0 - 1, k0 - 1, R::UX, R::UY);
        splat_cell<1, P2>(pos, vel, q0, q1, ci, cj, ck, g, s_num + R::NU, s_den + R::NU, i0 - 1, j0, k0 - 1, R::VX,
                      R::VY);
        splat_cell<2, P2>(pos, vel, q0, q1, ci, cj, ck, g, s_num + R::NU + R::NV, s_den + R::NU + R::NV, i0 - 1, j0 - 1,
                      k0, R::WX, R::WY);
    }
    __syncthreads();

    // Add the reached faces inside the grid into acc (one 8-byte vector
    // reduction per face); faces outside the grid are dropped, as the
    // reference skips them.
    const int64_t nu = g.nu(), nv = g.nv();
    for (int t = threadIdx.x; t < R::N; t += NT) {
        const float den = s_den[t];
        if (den == 0.0f) continue;
        int fi, fj, fk;
        int64_t idx;
        if (t < R::NU) {
            fi = i0 + t % R::UX; fj = j0 - 1 + (t / R::UX) % R::UY; fk = k0 - 1 + t / (R::UX * R::UY);
            if (fi > W || fj < 0 || fj >= H || fk < 0 || fk >= D) continue;
            idx = int64_t(fi) + int64_t(fj) * (W + 1) + int64_t(fk) * (W + 1) * H;
        } else if (t < R::NU + R::NV) {
            const int r = t - R::NU;
            fi = i0 - 1 + r % R::VX; fj = j0 + (r / R::VX) % R::VY; fk = k0 - 1 + r / (R::VX * R::VY);
            if (fi < 0 || fi >= W || fj > H || fk < 0 || fk >= D) continue;
            idx = nu + int64_t(fi) + int64_t(fj) * W + int64_t(fk) * W * (H + 1);
        } else {
            const int r = t - R::NU - R::NV;
            fi = i0 - 1 + r % R::WX; fj = j0 - 1 + (r / R::WX) % R::WY; fk = k0 + r / (R::WX * R::WY);
            if (fi < 0 || fi >= W || fj < 0 || fj >= H || fk > D) continue;
            idx = nu + nv + int64_t(fi) + int64_t(fj) * W + int64_t(fk) * W * H;
        }
        atomicAdd(&acc[idx], make_float2(s_num[t], den));
    }
}

// +0 computed from x (min(|x|, 0) is +0 for every x, NaN and infinities
// included).  A store of a constant to an address whose load is still in
// flight in the same thread waits on that load in the memory pipeline (on B200
// a read-then-clear pass over 50 MB ran at 0.2 ms against 0.03 ms); a value
// computed from the load is stored only after the load has returned.
__device__ __forceinline__ float dep_zero(float x) { return fminf(fabsf(x), 0.0f); }

// Pass 2, over every face of one component: num/den (ComputeVelocityFunc
// :598-605), u* <- u, u += dt*g (the x > (float)INT_MIN test of applyForces),
// and acc <- 0.
template <bool FUSED>
__global__ void k_p2g_finish(float2* __restrict__ acc, int64_t n, float dt, float gc, float* __restrict__ dst,
                             float* __restrict__ sav) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float2 a = acc[t];
    acc[t] = make_float2(dep_zero(a.x), dep_zero(a.y));
    float val = 0.0f;
    if (a.y > 1e-8f) val = a.x / a.y;
    if (FUSED) {
        sav[t] = val;
        dst[t] = (val > -2147483648.0f) ? val + dt * gc : val;
    } else {
        dst[t] = val;
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

// Brick shape and CTA size (build tunables).
#ifndef P2G_BRICK_X
#define P2G_BRICK_X 8
#define P2G_BRICK_Y 8
#define P2G_BRICK_Z 4
#define P2G_THREADS 128
#endif
constexpr int P2G_BX = P2G_BRICK_X, P2G_BY = P2G_BRICK_Y, P2G_BZ = P2G_BRICK_Z, P2G_NT = P2G_THREADS;

void launch_p2g(const float4* pos, const float4* vel, const int* start, Dims g, float dt, float3 gravity,
                float2* acc, float* u, float* v, float* w, float* us, float* vs, float* ws, int fused_forces,
                cudaStream_t st) {
    const int nb = ((g.W + P2G_BX - 1) / P2G_BX) * ((g.H + P2G_BY - 1) / P2G_BY) * ((g.D + P2G_BZ - 1) / P2G_BZ);
    if (g.idx != 0.0f) k_p2g_accum<P2G_BX, P2G_BY, P2G_BZ, P2G_NT, true><<<nb, P2G_NT, 0, st>>>(pos, vel, start, g, acc);
    else k_p2g_accum<P2G_BX, P2G_BY, P2G_BZ, P2G_NT, false><<<nb, P2G_NT, 0, st>>>(pos, vel, start, g, acc);
    const int64_t n3[3] = {g.nu(), g.nv(), g.nw()};
    float* dst[3] = {u, v, w};
    float* sav[3] = {us, vs, ws};
    const float gc[3] = {gravity.x, gravity.y, gravity.z};
    float2* a = acc;
    for (int c = 0; c < 3; ++c) {
        const unsigned nb2 = unsigned((n3[c] + 255) / 256);
        if (fused_forces) k_p2g_finish<true><<<nb2, 256, 0, st>>>(a, n3[c], dt, gc[c], dst[c], sav[c]);
        else k_p2g_finish<false><<<nb2, 256, 0, st>>>(a, n3[c], dt, gc[c], dst[c], sav[c]);
        a += n3[c];
    }
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
