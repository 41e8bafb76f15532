// common.cuh -- shared device helpers of the PIC/FLIP kernels (sm_100a).
//
// Arithmetic follows the reference functors of src/FluidSim/FluidSolver3D.cu
// expression by expression (IEEE division, no fast-math), so that integer
// results (cell keys, labels) are bit-identical and floating-point ones agree
// to rounding.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fp {

constexpr uint8_t SOLID = 0, FLUID = 1, AIR = 2, BODY = 3;

// Grid geometry passed by value to every kernel.  idx = 1/dx when dx is a
// power of two (then x * idx is exactly x / dx, so the cheap multiply gives
// the reference's quotient bit for bit), else 0 (divide).
struct Dims {
    int W, H, D;
    float dx;
    float idx = 0.0f;
    __host__ __device__ int64_t nc() const { return int64_t(W) * H * D; }
    __host__ __device__ int64_t nu() const { return int64_t(W + 1) * H * D; }
    __host__ __device__ int64_t nv() const { return int64_t(W) * (H + 1) * D; }
    __host__ __device__ int64_t nw() const { return int64_t(W) * H * (D + 1); }
};

// Rigid-body kinematics seen by the RHS and the projection
// (RHSCalculator3D / UFunctor members, FluidSolver3D.cu:1368-1370, 2081-2083).
struct BodyKin {
    float3 vel, omega, com;
    int active;
};

// x / dx, by the exact reciprocal multiply when dx is a power of two.
__device__ __forceinline__ float over_dx(float x, const Dims& g) { return g.idx != 0.0f ? x * g.idx : x / g.dx; }
// The same with the choice made at compile time (P2: dx is a power of two and
// Dims.idx = 1/dx).  Hot kernels take P2 as a template argument: a run-time
// choice lets the compiler evaluate the division on every path.
template <bool P2>
__device__ __forceinline__ float to_grid(float x, const Dims& g) { return P2 ? x * g.idx : x / g.dx; }

__device__ __forceinline__ int clampi(int a, int lo, int hi) { return min(max(a, lo), hi); }
__device__ __forceinline__ float clamp01(float f) { return fminf(fmaxf(f, 0.0f), 1.0f); }

// Cell of a particle: floorf(p/dx) clamped to the grid (MarkFluidCellsFunctor,
// FluidSolver3D.cu:316-331).
template <bool P2>
__device__ __forceinline__ int cell_key(float x, float y, float z, const Dims& g) {
    int i = int(floorf(to_grid<P2>(x, g))), j = int(floorf(to_grid<P2>(y, g))), k = int(floorf(to_grid<P2>(z, g)));
    i = clampi(i, 0, g.W - 1);
    j = clampi(j, 0, g.H - 1);
    k = clampi(k, 0, g.D - 1);
    return i + j * g.W + k * g.W * g.H;
}

__device__ __forceinline__ float3 body_vel_at(const BodyKin& b, float3 pos) {
    float3 r = make_float3(pos.x - b.com.x, pos.y - b.com.y, pos.z - b.com.z);
    return make_float3(b.vel.x + b.omega.y * r.z - b.omega.z * r.y,
                       b.vel.y + b.omega.z * r.x - b.omega.x * r.z,
                       b.vel.z + b.omega.x * r.y - b.omega.y * r.x);
}

// trilinearInterpolation (FluidSolver3D.cu:783-801).
__device__ __forceinline__ float trilin(float xd, float yd, float zd, float c000, float c100, float c001, float c101,
                                        float c010, float c110, float c011, float c111) {
    float c00 = c000 * (1.0f - xd) + c100 * xd;
    float c01 = c001 * (1.0f - xd) + c101 * xd;
    float c10 = c010 * (1.0f - xd) + c110 * xd;
    float c11 = c011 * (1.0f - xd) + c111 * xd;
    float c0 = c00 * (1.0f - yd) + c10 * yd;
    float c1 = c01 * (1.0f - yd) + c11 * yd;
    return c0 * (1.0f - zd) + c1 * zd;
}

// MAC sample stencil: base corner index and fractions.  Base indices are
// clamped so that base+1 stays inside the face grid; for positions inside
// [0, (N-1)*dx] (where advection keeps particles) these are the reference's
// clamps of interpVelDevice3D (FluidSolver3D.cu:1052-1157).  A 2D grid is a
// grid with D = 1: its z corner pairs collapse onto one slice (slice stride 0
// in sample()) with weight 0 on the duplicate, which is exact bilinear
// interpolation.
struct Stencil {
    int base;
    float fx, fy, fz;
};
__device__ __forceinline__ Stencil stencil_u(float rx, float ry, float rz, const Dims& g) {
    int i = int(floorf(rx)), j = int(floorf(ry - 0.5f)), k = int(floorf(rz - 0.5f));
    i = clampi(i, 0, g.W - 1); j = clampi(j, 0, g.H - 2); k = clampi(k, 0, max(g.D - 2, 0));
    Stencil s;
    s.fx = clamp01(rx - float(i)); s.fy = clamp01((ry - 0.5f) - float(j)); s.fz = clamp01((rz - 0.5f) - float(k));
    s.base = i + j * (g.W + 1) + k * (g.W + 1) * g.H;
    return s;
}
__device__ __forceinline__ Stencil stencil_v(float rx, float ry, float rz, const Dims& g) {
    int i = int(floorf(rx - 0.5f)), j = int(floorf(ry)), k = int(floorf(rz - 0.5f));
    i = clampi(i, 0, g.W - 2); j = clampi(j, 0, g.H - 1); k = clampi(k, 0, max(g.D - 2, 0));
    Stencil s;
    s.fx = clamp01((rx - 0.5f) - float(i)); s.fy = clamp01(ry - float(j)); s.fz = clamp01((rz - 0.5f) - float(k));
    s.base = i + j * g.W + k * g.W * (g.H + 1);
    return s;
}
__device__ __forceinline__ Stencil stencil_w(float rx, float ry, float rz, const Dims& g) {
    int i = int(floorf(rx - 0.5f)), j = int(floorf(ry - 0.5f)), k = int(floorf(rz));
    i = clampi(i, 0, g.W - 2); j = clampi(j, 0, g.H - 2); k = clampi(k, 0, g.D - 1);
    Stencil s;
    s.fx = clamp01((rx - 0.5f) - float(i)); s.fy = clamp01((ry - 0.5f) - float(j)); s.fz = clamp01(rz - float(k));
    s.base = i + j * g.W + k * g.W * g.H;
    return s;
}

__device__ __forceinline__ float sample(const float* __restrict__ f, const Stencil& s, int sx, int sxy) {
    const float* b = f + s.base;
    return trilin(s.fx, s.fy, s.fz, __ldg(b), __ldg(b + 1), __ldg(b + sxy), __ldg(b + 1 + sxy), __ldg(b + sx),
                  __ldg(b + 1 + sx), __ldg(b + sx + sxy), __ldg(b + 1 + sx + sxy));
}
// Sample of (f - g) per corner, the FLIP delta grid of gridToParticles
// (FluidSolver3D.cu:995-1012) without materialising it.
__device__ __forceinline__ float sample_delta(const float* __restrict__ f, const float* __restrict__ g, const Stencil& s,
                                              int sx, int sxy) {
    const float* a = f + s.base;
    const float* b = g + s.base;
    auto d = [&](int o) { return __ldg(a + o) - __ldg(b + o); };
    return trilin(s.fx, s.fy, s.fz, d(0), d(1), d(sxy), d(1 + sxy), d(sx), d(1 + sx), d(sx + sxy), d(1 + sx + sxy));
}

// Slice strides of the u and v face grids for sample() (0 on a 2D grid).
__device__ __forceinline__ int sxy_u(const Dims& g) { return g.D > 1 ? (g.W + 1) * g.H : 0; }
__device__ __forceinline__ int sxy_v(const Dims& g) { return g.D > 1 ? g.W * (g.H + 1) : 0; }

template <bool P2>
__device__ __forceinline__ float3 interp_vel(const float* __restrict__ u, const float* __restrict__ v,
                                             const float* __restrict__ w, const Dims& g, float3 pos) {
    const float rx = to_grid<P2>(pos.x, g), ry = to_grid<P2>(pos.y, g), rz = to_grid<P2>(pos.z, g);
    return make_float3(sample(u, stencil_u(rx, ry, rz, g), g.W + 1, sxy_u(g)),
                       sample(v, stencil_v(rx, ry, rz, g), g.W, sxy_v(g)),
                       sample(w, stencil_w(rx, ry, rz, g), g.W, g.W * g.H));
}

// Rigid-body geometry for marking and the force integral: an analytic
// sphere, or the reference's voxel SDF (RigidBody, utility.cuh:195-491) with
// its rotation (row-major, world = R * local) and local centre of mass.
// Body shapes: analytic sphere, the reference's voxel SDF, and a wave paddle
// (the half-space x < com.x, moved by a prescribed law, not by the fluid).
enum : int { BODY_SPHERE = 0, BODY_SDF = 1, BODY_PADDLE = 2 };
struct BodyShape {
    int kind;
    float3 com;          // body position (centre of mass) in world space
    float radius;        // sphere radius
    float rot[9];        // rotation matrix, row-major
    float3 local_com;    // centre of mass in SDF-file coordinates
    float3 origin;       // SDF file origin
    float cell;          // SDF voxel size
    int nx, ny, nz;      // SDF dimensions
    const float* sdf;    // device SDF values, i fastest
};

// Voxel of the SDF grid that holds world point x (nearest-lower voxel in body
// coordinates: local = R^T (x - pos) + local_com, voxel (local - origin) /
// cell); false outside the SDF box.
__device__ __forceinline__ bool body_voxel(const BodyShape& b, float3 x, int& i, int& j, int& k) {
    const float3 d = make_float3(x.x - b.com.x, x.y - b.com.y, x.z - b.com.z);
    const float lx = b.rot[0] * d.x + b.rot[3] * d.y + b.rot[6] * d.z + b.local_com.x;
    const float ly = b.rot[1] * d.x + b.rot[4] * d.y + b.rot[7] * d.z + b.local_com.y;
    const float lz = b.rot[2] * d.x + b.rot[5] * d.y + b.rot[8] * d.z + b.local_com.z;
    const float sx = (lx - b.origin.x) / b.cell, sy = (ly - b.origin.y) / b.cell, sz = (lz - b.origin.z) / b.cell;
    if (sx < 0.0f || sx >= float(b.nx) || sy < 0.0f || sy >= float(b.ny) || sz < 0.0f || sz >= float(b.nz))
        return false;
    i = min(int(sx), b.nx - 1); j = min(int(sy), b.ny - 1); k = min(int(sz), b.nz - 1);
    return true;
}

// Signed distance of world point x to the body (negative inside): the
// analytic sphere |x - c| - r, the paddle's x - x_p, or the voxel SDF
// (Utility::contains, utility.cu:163-206; 1e30 outside its box).  The sphere
// is explicitly rounded (no contraction) so BODY marks match a CPU
// evaluation bit for bit.
__device__ __forceinline__ float body_sdf(const BodyShape& b, float3 x) {
    const float3 d = make_float3(x.x - b.com.x, x.y - b.com.y, x.z - b.com.z);
    if (b.kind == BODY_SPHERE)
        return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(d.x, d.x), __fmul_rn(d.y, d.y)), __fmul_rn(d.z, d.z))) - b.radius;
    if (b.kind == BODY_PADDLE) return d.x;  // signed distance to the paddle face x = com.x
    int i, j, k;
    if (!body_voxel(b, x, i, j, k)) return 1e30f;
    return __ldg(b.sdf + i + j * b.nx + k * b.nx * b.ny);
}

// SDF collision projection: a point with phi(x) < eps is moved along the
// outward normal to phi = eps.  Sphere: radially to r + eps from the centre
// (straight up if it sits at the centre); paddle: to x_p + eps; voxel SDF:
// x += (eps - phi) n with n the normalised central-difference gradient of the
// voxel values, rotated into the world, repeated up to four times because
// the nearest-voxel SDF is piecewise constant.  Returns false if the point
// was inside and could not be moved (a voxel with zero gradient).
__device__ __forceinline__ bool sdf_push_out(const BodyShape& b, float3& x, float eps) {
    if (b.kind == BODY_SPHERE) {
        const float3 d = make_float3(__fsub_rn(x.x, b.com.x), __fsub_rn(x.y, b.com.y), __fsub_rn(x.z, b.com.z));
        const float r = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(d.x, d.x), __fmul_rn(d.y, d.y)), __fmul_rn(d.z, d.z)));
        const float target = __fadd_rn(b.radius, eps);
        if (!(__fsub_rn(r, b.radius) < eps)) return true;
        if (r > 0.0f) {
            const float sc = __fdiv_rn(target, r);
            x = make_float3(__fadd_rn(b.com.x, __fmul_rn(d.x, sc)), __fadd_rn(b.com.y, __fmul_rn(d.y, sc)),
                            __fadd_rn(b.com.z, __fmul_rn(d.z, sc)));
        } else {
            x = make_float3(b.com.x, __fadd_rn(b.com.y, target), b.com.z);
        }
        return true;
    }
    if (b.kind == BODY_PADDLE) {
        if (__fsub_rn(x.x, b.com.x) < eps) x.x = __fadd_rn(b.com.x, eps);
        return true;
    }
    for (int it = 0; it < 4; ++it) {
        int i, j, k;
        if (!body_voxel(b, x, i, j, k)) return true;
        const float* s = b.sdf;
        const int sx = 1, sy = b.nx, sz = b.nx * b.ny;
        const int c = i + j * sy + k * sz;
        const float phi = __ldg(s + c);
        if (!(phi < eps)) return true;
        // central differences (one-sided at the box faces), in voxel units
        const int i0 = max(i - 1, 0), i1 = min(i + 1, b.nx - 1), j0 = max(j - 1, 0), j1 = min(j + 1, b.ny - 1),
                  k0 = max(k - 1, 0), k1 = min(k + 1, b.nz - 1);
        const float gx = i1 > i0 ? (__ldg(s + c + (i1 - i) * sx) - __ldg(s + c + (i0 - i) * sx)) / float(i1 - i0) : 0.0f;
        const float gy = j1 > j0 ? (__ldg(s + c + (j1 - j) * sy) - __ldg(s + c + (j0 - j) * sy)) / float(j1 - j0) : 0.0f;
        const float gz = k1 > k0 ? (__ldg(s + c + (k1 - k) * sz) - __ldg(s + c + (k0 - k) * sz)) / float(k1 - k0) : 0.0f;
        const float gn = sqrtf(gx * gx + gy * gy + gz * gz);
        if (!(gn > 0.0f)) return false;
        const float lx = gx / gn, ly = gy / gn, lz = gz / gn;  // local normal
        const float step = eps - phi;
        x.x += step * (b.rot[0] * lx + b.rot[1] * ly + b.rot[2] * lz);
        x.y += step * (b.rot[3] * lx + b.rot[4] * ly + b.rot[5] * lz);
        x.z += step * (b.rot[6] * lx + b.rot[7] * ly + b.rot[8] * lz);
    }
    return true;
}

// Labels with out-of-domain cells reading as SOLID.
__device__ __forceinline__ uint8_t label_at(const uint8_t* __restrict__ lab, const Dims& g, int i, int j, int k) {
    if (i < 0 || i >= g.W || j < 0 || j >= g.H || k < 0 || k >= g.D) return SOLID;
    return lab[i + j * g.W + k * g.W * g.H];
}

// Device status word written by kernels that can fail without trapping.
enum : int { DEV_OK = 0, DEV_TIMEOUT = 1, DEV_NAN = 2, DEV_BREAKDOWN = 3, DEV_MAXIT = 4 };

// True when the pressure solve whose status word is *status failed in a way
// that makes the step return an error (a grid barrier gave up, or NaN).  The
// kernels queued after the solve then leave the face velocities and the
// particles as they are, so a failed step changes no particle.  A null
// pointer means "no guard".
__device__ __forceinline__ bool solve_failed(const int* status) {
    if (!status) return false;
    const int s = *status;
    return s == DEV_TIMEOUT || s == DEV_NAN;
}

}  // namespace fp
