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
#include "device_memo.hpp"
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

__device__ __forceinline__ bool project_particle(float3& pos, const uint8_t* __restrict__ lab, const Dims& g) {
    const float dx = g.dx;
    const int cx = int(floorf(over_dx(pos.x, g))), cy = int(floorf(over_dx(pos.y, g))), cz = int(floorf(over_dx(pos.z, g)));
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

// Face-grid samplers for the per-particle update.  GlobalSampler reads the
// six face grids through L1 (trilinear corners as scalar loads).
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
    __device__ __forceinline__ float3 vel(float3 p) const { return interp_vel(u, v, w, g, p); }
};

// Base corner (i, j, k) and fractions of component COMP's stencil: the same
// clamps and arithmetic as stencil_u / stencil_v / stencil_w.
struct Corner {
    int i, j, k;
    float fx, fy, fz;
};
template <int COMP>
__device__ __forceinline__ Corner corner(float rx, float ry, float rz, const Dims& g) {
    Corner c;
    if (COMP == 0) {
        c.i = clampi(int(floorf(rx)), 0, g.W - 1); c.j = clampi(int(floorf(ry - 0.5f)), 0, g.H - 2);
        c.k = clampi(int(floorf(rz - 0.5f)), 0, max(g.D - 2, 0));
        c.fx = clamp01(rx - float(c.i)); c.fy = clamp01((ry - 0.5f) - float(c.j)); c.fz = clamp01((rz - 0.5f) - float(c.k));
    } else if (COMP == 1) {
        c.i = clampi(int(floorf(rx - 0.5f)), 0, g.W - 2); c.j = clampi(int(floorf(ry)), 0, g.H - 1);
        c.k = clampi(int(floorf(rz - 0.5f)), 0, max(g.D - 2, 0));
        c.fx = clamp01((rx - 0.5f) - float(c.i)); c.fy = clamp01(ry - float(c.j)); c.fz = clamp01((rz - 0.5f) - float(c.k));
    } else {
        c.i = clampi(int(floorf(rx - 0.5f)), 0, g.W - 2); c.j = clampi(int(floorf(ry - 0.5f)), 0, g.H - 2);
        c.k = clampi(int(floorf(rz)), 0, g.D - 1);
        c.fx = clamp01((rx - 0.5f) - float(c.i)); c.fy = clamp01((ry - 0.5f) - float(c.j)); c.fz = clamp01(rz - float(c.k));
    }
    return c;
}

// Shared-memory tile of one brick of BX x BY x BZ cells and HL halo cells:
// for each face grid f (u, v, w) an array of entries (f[i], f[i+1], f*[i],
// f*[i+1]) over the stencil bases that particles inside the brick and halo
// can have, so that one 16-byte load gives both x corners of f and f*.
// Tile extents and origins (in face indices) per component:
//   u: x BX+2HL from i0-HL, y BY+2HL+2 from j0-HL-1, z BZ+2HL+2 from k0-HL-1
//   v: x BX+2HL+1 from i0-HL-1, y BY+2HL+1 from j0-HL, z as u
//   w: x as v, y as u, z BZ+2HL+1 from k0-HL
template <int BX, int BY, int BZ, int HL>
struct Tile {
    static __host__ __device__ constexpr int nx(int comp) { return comp == 0 ? BX + 2 * HL : BX + 2 * HL + 1; }
    static __host__ __device__ constexpr int ny(int comp) { return comp == 1 ? BY + 2 * HL + 1 : BY + 2 * HL + 2; }
    static __host__ __device__ constexpr int nz(int comp) { return comp == 2 ? BZ + 2 * HL + 1 : BZ + 2 * HL + 2; }
    static __host__ __device__ constexpr int n(int comp) { return nx(comp) * ny(comp) * nz(comp); }
    static constexpr int TOTAL = n(0) + n(1) + n(2);
    static __host__ __device__ constexpr int offset(int comp) { return comp == 0 ? 0 : (comp == 1 ? n(0) : n(0) + n(1)); }
    // origin of component comp's tile for the brick at (i0, j0, k0)
    static __device__ __forceinline__ int ox(int comp, int i0) { return comp == 0 ? i0 - HL : i0 - HL - 1; }
    static __device__ __forceinline__ int oy(int comp, int j0) { return comp == 1 ? j0 - HL : j0 - HL - 1; }
    static __device__ __forceinline__ int oz(int comp, int k0) { return comp == 2 ? k0 - HL : k0 - HL - 1; }
};

// TileSampler reads the staged tile when the whole stencil lies in it, and
// the global grids otherwise (particles that left the brick and its halo).
// The values and the arithmetic are the same either way, so the result does
// not depend on which path a sample takes.
template <int BX, int BY, int BZ, int HL>
struct TileSampler {
    using T = Tile<BX, BY, BZ, HL>;
    GlobalSampler G;
    const float4* t;  // the staged tile (shared memory)
    int i0, j0, k0;   // brick origin

    template <int COMP>
    __device__ __forceinline__ int entry(const Corner& c) const {
        const int li = c.i - T::ox(COMP, i0), lj = c.j - T::oy(COMP, j0), lk = c.k - T::oz(COMP, k0);
        if (unsigned(li) >= unsigned(T::nx(COMP)) || unsigned(lj) >= unsigned(T::ny(COMP) - 1) ||
            unsigned(lk) >= unsigned(T::nz(COMP) - 1))
            return -1;
        return T::offset(COMP) + li + T::nx(COMP) * (lj + T::ny(COMP) * lk);
    }
    // PIC and FLIP samples of component COMP from entry e (4 tile loads)
    template <int COMP>
    __device__ __forceinline__ void both(int e, const Corner& c, float& pic, float& dlt) const {
        const int sy = T::nx(COMP), sz = T::nx(COMP) * T::ny(COMP);
        const float4 a = t[e], b = t[e + sy], d = t[e + sz], f = t[e + sy + sz];  // (y,z): a 00, b 10, d 01, f 11
        pic = trilin(c.fx, c.fy, c.fz, a.x, a.y, d.x, d.y, b.x, b.y, f.x, f.y);
        dlt = trilin(c.fx, c.fy, c.fz, a.x - a.z, a.y - a.w, d.x - d.z, d.y - d.w, b.x - b.z, b.y - b.w, f.x - f.z,
                     f.y - f.w);
    }
    template <int COMP>
    __device__ __forceinline__ float one(int e, const Corner& c) const {
        const int sy = T::nx(COMP), sz = T::nx(COMP) * T::ny(COMP);
        const float2* t2 = reinterpret_cast<const float2*>(t);  // the (f[i], f[i+1]) half of each entry
        const float2 a = t2[2 * e], b = t2[2 * (e + sy)], d = t2[2 * (e + sz)], f = t2[2 * (e + sy + sz)];
        return trilin(c.fx, c.fy, c.fz, a.x, a.y, d.x, d.y, b.x, b.y, f.x, f.y);
    }
    __device__ __forceinline__ void g2p(float rx, float ry, float rz, float3& pic, float3& dlt) const {
        const Corner cu = corner<0>(rx, ry, rz, G.g), cv = corner<1>(rx, ry, rz, G.g), cw = corner<2>(rx, ry, rz, G.g);
        const int eu = entry<0>(cu), ev = entry<1>(cv), ew = entry<2>(cw);
        if (eu < 0 || ev < 0 || ew < 0) { G.g2p(rx, ry, rz, pic, dlt); return; }
        both<0>(eu, cu, pic.x, dlt.x);
        both<1>(ev, cv, pic.y, dlt.y);
        both<2>(ew, cw, pic.z, dlt.z);
    }
    __device__ __forceinline__ float3 vel(float3 p) const {
        const float rx = over_dx(p.x, G.g), ry = over_dx(p.y, G.g), rz = over_dx(p.z, G.g);
        const Corner cu = corner<0>(rx, ry, rz, G.g), cv = corner<1>(rx, ry, rz, G.g), cw = corner<2>(rx, ry, rz, G.g);
        const int eu = entry<0>(cu), ev = entry<1>(cv), ew = entry<2>(cw);
        if (eu < 0 || ev < 0 || ew < 0) return G.vel(p);
        return make_float3(one<0>(eu, cu), one<1>(ev, cv), one<2>(ew, cw));
    }
};

struct AdvectParams {
    float alpha, dt, C;
    int do_g2p, do_advect, rk2, sdf_collide;
    BodyShape body;
};

// G2P and advection of particle q (GridToParticleFunctor :803-980,
// AdvectParticlesFunctor :1241-1330), with face samples from S.
template <class S>
__device__ __forceinline__ void particle_update(const S& smp, float4* __restrict__ pos, float4* __restrict__ vel,
                                                int64_t q, const uint8_t* __restrict__ lab, const Dims& g,
                                                const AdvectParams& a) {
    const float4 P = pos[q];
    float3 p = make_float3(P.x, P.y, P.z);
    const float dx = g.dx;
    if (a.do_g2p) {
        const float4 V = vel[q];
        float3 pic, dlt;
        smp.g2p(over_dx(p.x, g), over_dx(p.y, g), over_dx(p.z, g), pic, dlt);
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
        const float3 vel0 = smp.vel(p);
        const float speed = sqrtf(vel0.x * vel0.x + vel0.y * vel0.y + vel0.z * vel0.z) + 1e-37f + floor_speed;
        float dT = (a.C * dx) / speed;
        if (subT + dT >= dt) { dT = dt - subT; finished = true; }
        else if (subT + 2.0f * dT >= dt) { dT *= 0.5f; }
        if (a.rk2) {
            const float3 mid = make_float3(p.x + (vel0.x * 0.5f) * dT, p.y + (vel0.y * 0.5f) * dT, p.z + (vel0.z * 0.5f) * dT);
            const float3 k2 = smp.vel(mid);
            p = make_float3(p.x + k2.x * dT, p.y + k2.y * dT, p.z + k2.z * dT);
        } else {
            const float3 k1 = vel0;
            const float3 k2 = smp.vel(make_float3(p.x + (k1.x * 0.5f) * dT, p.y + (k1.y * 0.5f) * dT,
                                                  p.z + (k1.z * 0.5f) * dT));
            const float3 k3 = smp.vel(make_float3(p.x + (k2.x * 0.75f) * dT, p.y + (k2.y * 0.75f) * dT,
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
        const int cx = int(floorf(over_dx(p.x, g))), cy = int(floorf(over_dx(p.y, g))), cz = int(floorf(over_dx(p.z, g)));
        if (cx >= 0 && cx < g.W && cy >= 0 && cy < g.H && cz >= 0 && cz < g.D) {
            const uint8_t l = __ldg(lab + cx + cy * g.W + cz * g.W * g.H);
            if (l == SOLID || (l == BODY && !a.sdf_collide)) {
                if (!project_particle(p, lab, g)) break;
            }
        }
        if (p.x < 0.0f || p.y < 0.0f || p.z < 0.0f || isnan(p.x) || isnan(p.y) || isnan(p.z)) break;
    }
    pos[q] = make_float4(p.x, p.y, p.z, P.w);
}

// One thread per particle, any particle order (also 2D grids).
__global__ void __launch_bounds__(256) k_g2p_advect(float4* __restrict__ pos, float4* __restrict__ vel, int64_t np,
                                                    GlobalSampler smp, const uint8_t* __restrict__ lab,
                                                    AdvectParams a, const int* __restrict__ guard) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np || solve_failed(guard)) return;
    particle_update(smp, pos, vel, q, lab, smp.g, a);
}

// Cell-sorted particles, one CTA per brick of cells (3D grids): the CTA
// stages the brick's six face grids with a one-cell halo in shared memory
// (Tile), then its threads update the brick's particles, which are BY*BZ
// contiguous ranges (one per row of cells along x) of the cell-sorted order.
// Bricks without particles return before staging.
// G2P_TILED (a build tunable, default 1) selects this kernel for sorted 3D
// particles; 0 keeps the particle-parallel kernel everywhere.
#ifndef G2P_TILED
#define G2P_TILED 1
#endif
constexpr int G2P_BX = 8, G2P_BY = 8, G2P_BZ = 8, G2P_HL = 1, G2P_NT = 256;
using G2PTile = Tile<G2P_BX, G2P_BY, G2P_BZ, G2P_HL>;

__global__ void __launch_bounds__(G2P_NT) k_g2p_advect_tiled(float4* __restrict__ pos, float4* __restrict__ vel,
                                                            const int* __restrict__ start, GlobalSampler G,
                                                            const uint8_t* __restrict__ lab, AdvectParams a,
                                                            const int* __restrict__ guard) {
    extern __shared__ float4 s_tile[];
    constexpr int NR = G2P_BY * G2P_BZ;
    __shared__ int s_row0[NR + 1];  // prefix of the rows' particle counts
    __shared__ int s_q0[NR];        // first particle of each row
    const Dims& g = G.g;
    const int W = g.W, H = g.H, D = g.D;
    const int nbx = (W + G2P_BX - 1) / G2P_BX, nby = (H + G2P_BY - 1) / G2P_BY;
    const int bid = blockIdx.x;
    const int i0 = (bid % nbx) * G2P_BX, j0 = ((bid / nbx) % nby) * G2P_BY, k0 = (bid / (nbx * nby)) * G2P_BZ;
    const int bxe = min(G2P_BX, W - i0), bye = min(G2P_BY, H - j0), bze = min(G2P_BZ, D - k0);
    if (threadIdx.x < NR) {
        const int r = threadIdx.x, j = j0 + r % G2P_BY, k = k0 + r / G2P_BY;
        int q0 = 0, n = 0;
        if (r % G2P_BY < bye && r / G2P_BY < bze) {
            const int c0 = i0 + j * W + k * W * H;
            q0 = start[c0];
            n = start[c0 + bxe] - q0;
        }
        s_q0[r] = q0;
        s_row0[r + 1] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        s_row0[0] = 0;
        for (int r = 1; r <= NR; ++r) { acc += s_row0[r]; s_row0[r] = acc; }
    }
    __syncthreads();
    const int total = s_row0[NR];
    if (total == 0 || solve_failed(guard)) return;
    // stage the three tiles: entry (li, lj, lk) of component f holds
    // f[i], f[i+1], f*[i], f*[i+1] at face (i, j, k) = origin + (li, lj, lk),
    // zero outside the face grid
    for (int e = threadIdx.x; e < G2PTile::TOTAL; e += G2P_NT) {
        int comp = e < G2PTile::n(0) ? 0 : (e < G2PTile::n(0) + G2PTile::n(1) ? 1 : 2);
        const int le = e - G2PTile::offset(comp);
        const int nx = G2PTile::nx(comp), ny = G2PTile::ny(comp);
        const int i = G2PTile::ox(comp, i0) + le % nx, j = G2PTile::oy(comp, j0) + (le / nx) % ny,
                  k = G2PTile::oz(comp, k0) + le / (nx * ny);
        const int fw = W + (comp == 0), fh = H + (comp == 1), fd = D + (comp == 2);
        const float* f = comp == 0 ? G.u : (comp == 1 ? G.v : G.w);
        const float* fs = comp == 0 ? G.us : (comp == 1 ? G.vs : G.ws);
        float4 val = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (j >= 0 && j < fh && k >= 0 && k < fd) {
            const int64_t row = (int64_t(k) * fh + j) * fw;
            if (i >= 0 && i < fw) { val.x = __ldg(f + row + i); val.z = __ldg(fs + row + i); }
            if (i + 1 >= 0 && i + 1 < fw) { val.y = __ldg(f + row + i + 1); val.w = __ldg(fs + row + i + 1); }
        }
        s_tile[e] = val;
    }
    __syncthreads();
    TileSampler<G2P_BX, G2P_BY, G2P_BZ, G2P_HL> smp{G, s_tile, i0, j0, k0};
    for (int t = threadIdx.x; t < total; t += G2P_NT) {
        // the row holding the t-th particle of the brick
        int lo = 0, hi = NR - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_row0[mid] <= t) lo = mid; else hi = mid - 1;
        }
        const int64_t q = int64_t(s_q0[lo]) + (t - s_row0[lo]);
        particle_update(smp, pos, vel, q, lab, g, a);
    }
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
                       const BodyShape* collide, const int* cell_start) {
    if (np == 0) return;
    AdvectParams a{};
    a.alpha = alpha; a.dt = dt; a.C = cfl;
    a.do_g2p = do_g2p; a.do_advect = do_advect; a.rk2 = rk2; a.sdf_collide = collide ? 1 : 0;
    if (collide) a.body = *collide;
    const GlobalSampler G{u, v, w, us, vs, ws, g};
    if (G2P_TILED && cell_start && g.D > 1) {
        static DeviceMemo memo;
        constexpr int smem = int(sizeof(float4)) * G2PTile::TOTAL;
        memo.get([](int) {
            cudaFuncSetAttribute(k_g2p_advect_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            return 1;
        });
        const int nb = ((g.W + G2P_BX - 1) / G2P_BX) * ((g.H + G2P_BY - 1) / G2P_BY) * ((g.D + G2P_BZ - 1) / G2P_BZ);
        k_g2p_advect_tiled<<<nb, G2P_NT, smem, st>>>(pos, vel, cell_start, G, labels, a, guard);
        return;
    }
    k_g2p_advect<<<unsigned((np + 255) / 256), 256, 0, st>>>(pos, vel, np, G, labels, a, guard);
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
