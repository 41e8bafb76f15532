// kernels_advect.cu -- fused grid-to-particle transfer and advection.
//
// One thread per particle, particles in cell order (so the 48 + 72*substeps
// grid gathers of neighbouring threads hit the same L1/L2 lines):
//   G2P  (GridToParticleFunctor, FluidSolver3D.cu:803-980):
//        v = alpha*I(u) + (1-alpha)*(v + I(u - u*)), the FLIP delta sampled
//        corner by corner from u and u* instead of a materialised delta grid
//        (:983-1012 allocates three per step);
//   advection (AdvectParticlesFunctor, :1241-1330): adaptive substeps
//        dT = C*dx/(|v| + 1e-37 + sqrt(5*dx*9.8)), halved when within 2*dT of
//        the end; Ralston RK3 (weights 2/9, 3/9, 4/9) or midpoint RK2; clamp to
//        [0, (N-1)*dx]; a particle that lands in SOLID/BODY is nudged half a
//        cell toward the nearest FLUID cell centre among 34 offsets
//        (projectParticleDevice3D, :1161-1239); at most 1000 substeps.
//        With SDF collision (fp_config.collision) a particle whose body SDF
//        is below eps = 0.25 dx is first projected along the SDF normal to
//        phi = eps (sdf_push_out), and the label search is kept for SOLID
//        cells only.
#include "kernels.hpp"

namespace fp {

namespace {

// Offsets searched by projectParticleDevice3D (:1164-1181); entry 9 is the
// reference's {-1,-1} which value-initialises to {-1,-1,0}.
__constant__ signed char c_off[34][3] = {
    {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
    {1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0},
    {1, 0, 1}, {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1},
    {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1},
    {1, 1, 1}, {-1, 1, 1}, {1, -1, 1}, {1, 1, -1},
    {-1, -1, 1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, -1},
    {-2, -1, 0}, {0, -1, -2}, {-2, -2, 0}, {0, -2, -2},
    {-2, -2, -2}, {-2, 0, -2}, {2, -1, 0}, {0, -1, 2}};

template <bool P2>
__device__ __forceinline__ bool project_particle(float3& pos, const uint8_t* __restrict__ lab, const Dims& g) {
    const float dx = g.dx;
    const int cx = int(floorf(to_grid<P2>(pos.x, g))), cy = int(floorf(to_grid<P2>(pos.y, g))),
              cz = int(floorf(to_grid<P2>(pos.z, g)));
    float best = 1e10f;
    int bn = -1;
#pragma unroll 2
    for (int n = 0; n < 34; ++n) {
        const int nx = cx + c_off[n][0], ny = cy + c_off[n][1], nz = cz + c_off[n][2];
        if (nx < 0 || nx >= g.W || ny < 0 || ny >= g.H || nz < 0 || nz >= g.D) continue;
        if (__ldg(lab + nx + ny * g.W + nz * g.W * g.H) != FLUID) continue;
        const float ccx = (float(nx) + 0.5f) * dx, ccy = (float(ny) + 0.5f) * dx, ccz = (float(nz) + 0.5f) * dx;
        const float d = (ccx - pos.x) * (ccx - pos.x) + (ccy - pos.y) * (ccy - pos.y) + (ccz - pos.z) * (ccz - pos.z);
        if (d < best) { best = d; bn = n; }
    }
    if (bn < 0) return false;
    pos.x = pos.x + (float(c_off[bn][0]) * 0.5f) * dx;
    pos.y = pos.y + (float(c_off[bn][1]) * 0.5f) * dx;
    pos.z = pos.z + (float(c_off[bn][2]) * 0.5f) * dx;
    return true;
}

// Face-grid sampler of the per-particle update: the six face grids through
// L1 (trilinear corners as scalar loads; particles in cell order make
// neighbouring threads share lines).  A variant that staged each 8^3 brick's
// faces in shared memory measured slower (0.355 against 0.294 ms at 128^3):
// its index arithmetic and bank conflicts cost more than the L1 loads.
struct GlobalSampler {
    const float *u, *v, *w, *us, *vs, *ws;
    Dims g;
    // PIC sample I(u) and FLIP delta I(u - u*) of each component at r = x/dx
    __device__ __forceinline__ void g2p(float rx, float ry, float rz, float3& pic, float3& dlt) const {
        const Stencil su = stencil_u(rx, ry, rz, g), sv = stencil_v(rx, ry, rz, g), sw = stencil_w(rx, ry, rz, g);
        const int sxu = g.W + 1, sxyu = sxy_u(g), sxv = g.W, sxyv = sxy_v(g), sxw = g.W, sxyw = g.W * g.H;
        pic = make_float3(sample(u, su, sxu, sxyu), sample(v, sv, sxv, sxyv), sample(w, sw, sxw, sxyw));
        dlt = make_float3(sample_delta(u, us, su, sxu, sxyu), sample_delta(v, vs, sv, sxv, sxyv),
                          sample_delta(w, ws, sw, sxw, sxyw));
    }
    template <bool P2>
    __device__ __forceinline__ float3 vel(float3 p) const { return interp_vel<P2>(u, v, w, g, p); }
};

// Packed FP32 pairs (sm_100's f32x2 FMA/mul): two lanes of one 64-bit
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

// The eight trilinear corners of one face grid at one stencil base, kept in
// registers across one particle's samples, as z pairs: z0 = (c000, c001),
// z1 = (c100, c101), z2 = (c010, c011), z3 = (c110, c111), the first index
// along x, the second along y (row stride sx), the third along z (slice
// stride sxy).
struct Corners {
    int base;
    float2 z0, z1, z2, z3;
};
__device__ __forceinline__ void load_corners(const float* __restrict__ f, int base, int sx, int sxy, Corners& k) {
    const float* b = f + base;
    k.z0 = make_float2(__ldg(b), __ldg(b + sxy));
    k.z1 = make_float2(__ldg(b + 1), __ldg(b + 1 + sxy));
    k.z2 = make_float2(__ldg(b + sx), __ldg(b + sx + sxy));
    k.z3 = make_float2(__ldg(b + 1 + sx), __ldg(b + 1 + sx + sxy));
    k.base = base;
}
// trilinearInterpolation (FluidSolver3D.cu:783-801) on z pairs: the four x
// lerps as two packed ones, the two y lerps as one, then the z lerp.
__device__ __forceinline__ float trilin_pairs(float xd, float yd, float zd, float2 z0, float2 z1, float2 z2,
                                              float2 z3) {
    const float2 ox = make_float2(1.0f - xd, 1.0f - xd), wx = make_float2(xd, xd);
    const float2 y0 = f2_fma(z1, wx, f2_mul(z0, ox));  // (c00, c01)
    const float2 y1 = f2_fma(z3, wx, f2_mul(z2, ox));  // (c10, c11)
    const float2 oy = make_float2(1.0f - yd, 1.0f - yd), wy = make_float2(yd, yd);
    const float2 c = f2_fma(y1, wy, f2_mul(y0, oy));   // (c0, c1)
    return c.x * (1.0f - zd) + c.y * zd;
}
__device__ __forceinline__ float trilin_k(const Stencil& s, const Corners& k) {
    return trilin_pairs(s.fx, s.fy, s.fz, k.z0, k.z1, k.z2, k.z3);
}
// Sample of f at stencil s, loading the corners only when the base moved.
__device__ __forceinline__ float sample_cached(const float* __restrict__ f, const Stencil& s, int sx, int sxy,
                                               Corners& k) {
    if (s.base != k.base) load_corners(f, s.base, sx, sxy, k);
    return trilin_k(s, k);
}
// FLIP delta sample from the u corners already loaded in k and u*: each
// corner is u* * (-1) + u in one fused step, which rounds as u - u* does.
__device__ __forceinline__ float delta_k(const float* __restrict__ g, const Stencil& s, int sx, int sxy,
                                         const Corners& k) {
    const float* b = g + s.base;
    const float2 m1 = make_float2(-1.0f, -1.0f);
    const float2 d0 = f2_fma(make_float2(__ldg(b), __ldg(b + sxy)), m1, k.z0);
    const float2 d1 = f2_fma(make_float2(__ldg(b + 1), __ldg(b + 1 + sxy)), m1, k.z1);
    const float2 d2 = f2_fma(make_float2(__ldg(b + sx), __ldg(b + sx + sxy)), m1, k.z2);
    const float2 d3 = f2_fma(make_float2(__ldg(b + 1 + sx), __ldg(b + 1 + sx + sxy)), m1, k.z3);
    return trilin_pairs(s.fx, s.fy, s.fz, d0, d1, d2, d3);
}

// The same samples with each face grid's eight corners cached per particle:
// a particle moves a small fraction of a cell per substep (C = 0.1), so its
// G2P sample and most of its advection samples share stencil bases, and the
// corners are loaded again only when a base changes.  The interpolation is
// the packed form of GlobalSampler's: the same products, the x and y lerps
// two lanes at a time, each lerp one multiply and one fused multiply-add.
struct CachedSampler {
    GlobalSampler s;
    Corners cu, cv, cw;
    __device__ __forceinline__ explicit CachedSampler(const GlobalSampler& g) : s(g) {
        cu.base = cv.base = cw.base = -1;
    }
    __device__ __forceinline__ void g2p(float rx, float ry, float rz, float3& pic, float3& dlt) {
        const Dims& g = s.g;
        const Stencil su = stencil_u(rx, ry, rz, g), sv = stencil_v(rx, ry, rz, g), sw = stencil_w(rx, ry, rz, g);
        const int sxu = g.W + 1, sxyu = sxy_u(g), sxv = g.W, sxyv = sxy_v(g), sxw = g.W, sxyw = g.W * g.H;
        load_corners(s.u, su.base, sxu, sxyu, cu);
        load_corners(s.v, sv.base, sxv, sxyv, cv);
        load_corners(s.w, sw.base, sxw, sxyw, cw);
        pic = make_float3(trilin_k(su, cu), trilin_k(sv, cv), trilin_k(sw, cw));
        dlt = make_float3(delta_k(s.us, su, sxu, sxyu, cu), delta_k(s.vs, sv, sxv, sxyv, cv),
                          delta_k(s.ws, sw, sxw, sxyw, cw));
    }
    template <bool P2>
    __device__ __forceinline__ float3 vel(float3 p) {
        const Dims& g = s.g;
        const float rx = to_grid<P2>(p.x, g), ry = to_grid<P2>(p.y, g), rz = to_grid<P2>(p.z, g);
        return make_float3(sample_cached(s.u, stencil_u(rx, ry, rz, g), g.W + 1, sxy_u(g), cu),
                           sample_cached(s.v, stencil_v(rx, ry, rz, g), g.W, sxy_v(g), cv),
                           sample_cached(s.w, stencil_w(rx, ry, rz, g), g.W, g.W * g.H, cw));
    }
};

struct AdvectParams {
    float alpha, dt, C;
    int do_g2p, do_advect, rk2, sdf_collide;
    BodyShape body;
};

// G2P and advection of particle q (GridToParticleFunctor :803-980,
// AdvectParticlesFunctor :1241-1330), with face samples from S; P2: dx is a
// power of two (to_grid).
template <class S, bool P2>
__device__ __forceinline__ void particle_update(S& smp, float4* __restrict__ pos, float4* __restrict__ vel,
                                                int64_t q, const uint8_t* __restrict__ lab, const Dims& g,
                                                const AdvectParams& a) {
    const float4 P = pos[q];
    float3 p = make_float3(P.x, P.y, P.z);
    const float dx = g.dx;
    if (a.do_g2p) {
        const float4 V = vel[q];
        float3 pic, dlt;
        smp.g2p(to_grid<P2>(p.x, g), to_grid<P2>(p.y, g), to_grid<P2>(p.z, g), pic, dlt);
        const float alpha = a.alpha;
        float4 out;
        out.x = alpha * pic.x + (1.0f - alpha) * (V.x + dlt.x);
        out.y = alpha * pic.y + (1.0f - alpha) * (V.y + dlt.y);
        out.z = alpha * pic.z + (1.0f - alpha) * (V.z + dlt.z);
        out.w = V.w;
        vel[q] = out;
    }
    if (!a.do_advect) return;
    const float dt = a.dt;
    float subT = 0.0f;
    bool finished = false;
    int iter = 0;
    const float floor_speed = sqrtf((5.0f * dx) * 9.8f);
    const float xmax = float(g.W - 1) * dx, ymax = float(g.H - 1) * dx, zmax = float(g.D - 1) * dx;
    while (!finished && iter++ < 1000) {
        const float3 vel0 = smp.template vel<P2>(p);
        const float speed = sqrtf(vel0.x * vel0.x + vel0.y * vel0.y + vel0.z * vel0.z) + 1e-37f + floor_speed;
        float dT = (a.C * dx) / speed;
        if (subT + dT >= dt) { dT = dt - subT; finished = true; }
        else if (subT + 2.0f * dT >= dt) { dT *= 0.5f; }
        if (a.rk2) {
            const float3 mid = make_float3(p.x + (vel0.x * 0.5f) * dT, p.y + (vel0.y * 0.5f) * dT, p.z + (vel0.z * 0.5f) * dT);
            const float3 k2 = smp.template vel<P2>(mid);
            p = make_float3(p.x + k2.x * dT, p.y + k2.y * dT, p.z + k2.z * dT);
        } else {
            const float3 k1 = vel0;
            const float3 k2 = smp.template vel<P2>(make_float3(p.x + (k1.x * 0.5f) * dT, p.y + (k1.y * 0.5f) * dT,
                                                  p.z + (k1.z * 0.5f) * dT));
            const float3 k3 = smp.template vel<P2>(make_float3(p.x + (k2.x * 0.75f) * dT, p.y + (k2.y * 0.75f) * dT,
                                                  p.z + (k2.z * 0.75f) * dT));
            const float a1 = (2.0f / 9.0f) * dT, a2 = (3.0f / 9.0f) * dT, a3 = (4.0f / 9.0f) * dT;
            p = make_float3(p.x + k1.x * a1 + k2.x * a2 + k3.x * a3, p.y + k1.y * a1 + k2.y * a2 + k3.y * a3,
                            p.z + k1.z * a1 + k2.z * a2 + k3.z * a3);
        }
        subT += dT;
        p.x = fminf(fmaxf(p.x, 0.0f), xmax);
        p.y = fminf(fmaxf(p.y, 0.0f), ymax);
        p.z = fminf(fmaxf(p.z, 0.0f), zmax);
        if (a.sdf_collide) {
            if (!sdf_push_out(a.body, p, __fmul_rn(0.25f, dx))) break;
            p.x = fminf(fmaxf(p.x, 0.0f), xmax);
            p.y = fminf(fmaxf(p.y, 0.0f), ymax);
            p.z = fminf(fmaxf(p.z, 0.0f), zmax);
        }
        const int cx = int(floorf(to_grid<P2>(p.x, g))), cy = int(floorf(to_grid<P2>(p.y, g))),
                  cz = int(floorf(to_grid<P2>(p.z, g)));
        if (cx >= 0 && cx < g.W && cy >= 0 && cy < g.H && cz >= 0 && cz < g.D) {
            const uint8_t l = __ldg(lab + cx + cy * g.W + cz * g.W * g.H);
            if (l == SOLID || (l == BODY && !a.sdf_collide)) {
                if (!project_particle<P2>(p, lab, g)) break;
            }
        }
        if (p.x < 0.0f || p.y < 0.0f || p.z < 0.0f || isnan(p.x) || isnan(p.y) || isnan(p.z)) break;
    }
    pos[q] = make_float4(p.x, p.y, p.z, P.w);
}

// One thread per particle, any particle order (also 2D grids).  G2P_THREADS
// and G2P_MIN_BLOCKS (build tunables) set the CTA size and bound registers
// for that many CTAs per SM.
// Per-particle corner cache of the face samples (a build tunable).
#ifndef G2P_CORNER_CACHE
#define G2P_CORNER_CACHE 1
#endif
#ifndef G2P_THREADS
#define G2P_THREADS 128
#endif
#ifdef G2P_MIN_BLOCKS
#define G2P_BOUNDS __launch_bounds__(G2P_THREADS, G2P_MIN_BLOCKS)
#else
#define G2P_BOUNDS __launch_bounds__(G2P_THREADS)
#endif
template <bool P2>
__global__ void G2P_BOUNDS k_g2p_advect(float4* __restrict__ pos, float4* __restrict__ vel, int64_t np,
                                                    GlobalSampler smp, const uint8_t* __restrict__ lab,
                                                    AdvectParams a, const int* __restrict__ guard) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np || solve_failed(guard)) return;
#if G2P_CORNER_CACHE
    CachedSampler cs(smp);
    particle_update<CachedSampler, P2>(cs, pos, vel, q, lab, smp.g, a);
#else
    GlobalSampler gs = smp;
    particle_update<GlobalSampler, P2>(gs, pos, vel, q, lab, smp.g, a);
#endif
}

__global__ void k_unsort(const float4* __restrict__ pos, const float4* __restrict__ vel, int64_t np,
                         float* __restrict__ pos_out, float* __restrict__ vel_out) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const float4 P = pos[q];
    const int64_t id = __float_as_int(P.w);
    if (pos_out) { pos_out[3 * id] = P.x; pos_out[3 * id + 1] = P.y; pos_out[3 * id + 2] = P.z; }
    if (vel_out) { const float4 V = vel[q]; vel_out[3 * id] = V.x; vel_out[3 * id + 1] = V.y; vel_out[3 * id + 2] = V.z; }
}

// Frame records x y z vx vy vz in the original order (the binary PLY layout).
__global__ void k_unsort_records(const float4* __restrict__ pos, const float4* __restrict__ vel, int64_t np,
                                 float* __restrict__ rec) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const float4 P = pos[q], V = vel[q];
    float* r = rec + 6 * int64_t(__float_as_int(P.w));
    r[0] = P.x; r[1] = P.y; r[2] = P.z; r[3] = V.x; r[4] = V.y; r[5] = V.z;
}

// AoS (x y z) arrays to float4 pos (w = original index) and vel.  The
// lowest index of a particle with a non-finite value goes to *bad (the
// caller sets it to INT_MAX first).
__global__ void k_pack(const float* __restrict__ pos, const float* __restrict__ vel, int64_t np, float4* __restrict__ p4,
                       float4* __restrict__ v4, int* __restrict__ bad) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const float4 p = make_float4(pos[3 * q], pos[3 * q + 1], pos[3 * q + 2], __int_as_float(int(q)));
    const float4 v = vel ? make_float4(vel[3 * q], vel[3 * q + 1], vel[3 * q + 2], 0.0f) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    p4[q] = p;
    v4[q] = v;
    if (bad && !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z)))
        atomicMin(bad, int(q));
}

}  // namespace

void launch_g2p_advect(float4* pos, float4* vel, int64_t np, const float* u, const float* v, const float* w,
                       const float* us, const float* vs, const float* ws, const uint8_t* labels, Dims g, float alpha,
                       float dt, float cfl, int do_g2p, int do_advect, int rk2, cudaStream_t st, const int* guard,
                       const BodyShape* collide) {
    if (np == 0) return;
    AdvectParams a{};
    a.alpha = alpha; a.dt = dt; a.C = cfl;
    a.do_g2p = do_g2p; a.do_advect = do_advect; a.rk2 = rk2; a.sdf_collide = collide ? 1 : 0;
    if (collide) a.body = *collide;
    const GlobalSampler G{u, v, w, us, vs, ws, g};
    const unsigned nb = unsigned((np + G2P_THREADS - 1) / G2P_THREADS);
    if (g.idx != 0.0f) k_g2p_advect<true><<<nb, G2P_THREADS, 0, st>>>(pos, vel, np, G, labels, a, guard);
    else k_g2p_advect<false><<<nb, G2P_THREADS, 0, st>>>(pos, vel, np, G, labels, a, guard);
}

void launch_unsort(const float4* pos, const float4* vel, int64_t np, float* pos_out, float* vel_out, cudaStream_t st) {
    if (np == 0) return;
    k_unsort<<<unsigned((np + 255) / 256), 256, 0, st>>>(pos, vel, np, pos_out, vel_out);
}

void launch_unsort_records(const float4* pos, const float4* vel, int64_t np, float* rec, cudaStream_t st) {
    if (np == 0) return;
    k_unsort_records<<<unsigned((np + 255) / 256), 256, 0, st>>>(pos, vel, np, rec);
}

void launch_pack(const float* pos, const float* vel, int64_t np, float4* pos4, float4* vel4, int* bad,
                 cudaStream_t st) {
    if (np == 0) return;
    k_pack<<<unsigned((np + 255) / 256), 256, 0, st>>>(pos, vel, np, pos4, vel4, bad);
}

}  // namespace fp
