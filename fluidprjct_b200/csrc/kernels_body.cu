// kernels_body.cu -- SDF rigid body: cell marking and fluid force/torque.
//
// Marking restates MarkBodyCellsFunctor + Utility::contains
// (FluidSolver3D.cu:45-78, utility.cu:163-206): a cell whose centre lies
// inside the body (SDF <= 0) and is not SOLID becomes BODY.  The SDF is either
// the reference's voxel grid (nearest-lower voxel in body coordinates, rotated
// about the centre of mass) or an analytic sphere |x - c| - r.
//
// The fluid force replaces the reference's panel drag/lift plus host
// buoyancy loop (DragLiftForceCalculator :2674-2791, applyBuoyancy
// :2917-3026) by the pressure integral over the body written with SDF face
// fractions:  F = - sum_faces theta_f (p_R - p_L) dx^2 e_axis,
// tau = sum_faces (x_f - c) x dF, where theta_f = clamp(1/2 - phi(x_f)/dx, 0, 1)
// is the body fraction of face f and p is extended one cell into the body
// (BODY cells take the mean of their FLUID/AIR neighbours).  Along every grid
// line through the body the sum telescopes to the pressure difference across
// the body surface, so buoyancy and dynamic pressure forces both follow, and
// the force varies smoothly as the body moves by sub-cell amounts.  Each block
// reduces its faces in FP64 in a fixed order; a second kernel sums the block
// partials in a fixed order.
#include "kernels.hpp"

namespace fp {

namespace {

__global__ void k_mark_body(uint8_t* __restrict__ mark, Dims g, BodyShape b) {
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= g.nc()) return;
    const int i = int(c % g.W), j = int((c / g.W) % g.H), k = int(c / (int64_t(g.W) * g.H));
    const float3 x = make_float3((float(i) + 0.5f) * g.dx, (float(j) + 0.5f) * g.dx, (float(k) + 0.5f) * g.dx);
    mark[c] = body_sdf(b, x) <= 0.0f ? 1 : 0;
}

// Pressure with BODY cells extended by the mean of their FLUID/AIR neighbours
// (0 when they have none); SOLID and out-of-domain cells are invalid.
__device__ __forceinline__ bool p_ext(const float* __restrict__ p, const uint8_t* __restrict__ lab, const Dims& g,
                                      int i, int j, int k, float& out) {
    const uint8_t l = label_at(lab, g, i, j, k);
    if (l == SOLID) return false;
    if (l != BODY) { out = p[i + j * g.W + k * g.W * g.H]; return true; }
    const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    float s = 0.0f;
    int n = 0;
#pragma unroll
    for (int o = 0; o < 6; ++o) {
        const int a = i + off[o][0], b = j + off[o][1], e = k + off[o][2];
        const uint8_t ln = label_at(lab, g, a, b, e);
        if (ln == FLUID || ln == AIR) { s += p[a + b * g.W + e * g.W * g.H]; ++n; }
    }
    out = n ? s / float(n) : 0.0f;
    return true;
}

constexpr int FORCE_THREADS = 256;

__global__ void __launch_bounds__(FORCE_THREADS) k_body_force(const float* __restrict__ p,
                                                              const uint8_t* __restrict__ lab, Dims g, BodyShape b,
                                                              double* __restrict__ part) {
    const int64_t nc1 = int64_t(g.W + 1) * (g.H + 1) * (g.D + 1);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const float dx = g.dx;
    const double area = double(dx) * double(dx);
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nc1; t += int64_t(gridDim.x) * blockDim.x) {
        const int i = int(t % (g.W + 1)), j = int((t / (g.W + 1)) % (g.H + 1)), k = int(t / (int64_t(g.W + 1) * (g.H + 1)));
        for (int ax = 0; ax < 3; ++ax) {
            // face of axis ax at the low side of cell (i,j,k)
            if (ax == 0 && (j >= g.H || k >= g.D)) continue;
            if (ax == 1 && (i >= g.W || k >= g.D)) continue;
            if (ax == 2 && (i >= g.W || j >= g.H)) continue;
            const float3 xf = make_float3(ax == 0 ? float(i) * dx : (float(i) + 0.5f) * dx,
                                          ax == 1 ? float(j) * dx : (float(j) + 0.5f) * dx,
                                          ax == 2 ? float(k) * dx : (float(k) + 0.5f) * dx);
            const float theta = clamp01(0.5f - body_sdf(b, xf) / dx);
            if (theta <= 0.0f) continue;
            float pl, pr;
            const int li = i - (ax == 0), lj = j - (ax == 1), lk = k - (ax == 2);
            if (!p_ext(p, lab, g, li, lj, lk, pl) || !p_ext(p, lab, g, i, j, k, pr)) continue;
            const double dF = -double(theta) * (double(pr) - double(pl)) * area;
            const double rx = double(xf.x) - double(b.com.x), ry = double(xf.y) - double(b.com.y),
                         rz = double(xf.z) - double(b.com.z);
            const double fx = ax == 0 ? dF : 0.0, fy = ax == 1 ? dF : 0.0, fz = ax == 2 ? dF : 0.0;
            acc[0] += fx; acc[1] += fy; acc[2] += fz;
            acc[3] += ry * fz - rz * fy;
            acc[4] += rz * fx - rx * fz;
            acc[5] += rx * fy - ry * fx;
        }
    }
    __shared__ double sh[6][FORCE_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        double v = acc[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[m][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0.0;
        for (int w = 0; w < FORCE_THREADS / 32; ++w) v += sh[threadIdx.x][w];
        part[blockIdx.x * 6 + threadIdx.x] = v;
    }
}

__global__ void k_body_force_sum(const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x < 6) {
        double v = 0.0;
        for (int b = 0; b < nb; ++b) v += part[b * 6 + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

// ---------------------------------------------------------------- reference forces
// fp_config.body_forces = FP_BODY_FORCES_REFERENCE restates the reference's
// panel drag/lift (DragLiftForceCalculator, FluidSolver3D.cu:2674-2791) and
// its buoyancy (applyBuoyancy, :2917-3026).  Each panel and voxel is computed
// in FP32 in the reference's expression order (explicit round-to-nearest, no
// contraction); the sums are FP64 with a fixed order, where the reference adds
// FP32 values with atomics or in a host loop.
__device__ __forceinline__ float3 add3(float3 a, float3 b) {
    return make_float3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z));
}
__device__ __forceinline__ float3 sub3(float3 a, float3 b) {
    return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
__device__ __forceinline__ float3 mul3(float3 a, float s) {
    return make_float3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s));
}
__device__ __forceinline__ float dot3(float3 a, float3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
                       __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
                       __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// Force and torque of the panel between BODY cell (i, j, k) and its FLUID
// neighbour in direction dir (+x, -x, +y, -y, +z, -z), :2697-2783.
__device__ void ref_panel(int i, int j, int k, int dir, const float* u, const float* v, const float* w, const Dims& g,
                          float3 cm, float3 bvel, float3& F, float3& T) {
    const float dx = g.dx, rho = 1000.0f;
    const float3 cc = make_float3(__fmul_rn(__fadd_rn(float(i), 0.5f), dx), __fmul_rn(__fadd_rn(float(j), 0.5f), dx),
                                  __fmul_rn(__fadd_rn(float(k), 0.5f), dx));
    const float area = __fmul_rn(dx, dx);
    const int ax = dir >> 1;
    const float sgn = (dir & 1) ? -1.0f : 1.0f;
    const float3 nrm = make_float3(ax == 0 ? sgn : 0.0f, ax == 1 ? sgn : 0.0f, ax == 2 ? sgn : 0.0f);
    const float3 off = mul3(nrm, 0.5f);  // face offset (+-0.5 along the normal)
    const float3 fc = add3(cc, mul3(off, dx));
    const float3 r = sub3(fc, cm);
    const float3 up = interp_vel<false>(u, v, w, g, fc);
    const float3 ur = sub3(bvel, up);
    const float ua = __fsqrt_rn(dot3(ur, ur));
    const float alpha_s = 0.5f;
    float A = 0.0f;
    const float nu = dot3(nrm, ur);
    if (nu > 0.0f) A = __fmul_rn(__fadd_rn(__fmul_rn(__fdiv_rn(nu, ua), alpha_s), __fsub_rn(1.0f, alpha_s)), area);
    // drag: the scalar -0.5 * rho * Cd * A * |u_rel| is evaluated in double (the literal -0.5)
    const float Cd = 0.1f;
    const float sd = float(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(-0.5, double(rho)), double(Cd)), double(A)), double(ua)));
    const float3 Fd = mul3(ur, sd);
    // lift: -0.5f * rho * Cl * A * |u_rel| * (u_rel x (n x u_rel) / |n x u_rel|)
    const float Cl = 0.1f;
    const float3 nx = cross3(nrm, ur);
    const float nxa = __fsqrt_rn(dot3(nx, nx));
    const float3 dirv = make_float3(__fdiv_rn(nx.x, nxa), __fdiv_rn(nx.y, nxa), __fdiv_rn(nx.z, nxa));
    const float sl = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(-0.5f, rho), Cl), A), ua);
    const float3 Fl = mul3(cross3(ur, dirv), sl);
    F = add3(Fd, Fl);
    T = add3(cross3(r, Fd), cross3(r, Fl));
}

template <int N>
__device__ __forceinline__ void block_partials(double (&acc)[N], double* __restrict__ part) {
    __shared__ double sh[N][FORCE_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < N; ++m) {
        double v = acc[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[m][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < N) {
        double v = 0.0;
        for (int w = 0; w < FORCE_THREADS / 32; ++w) v += sh[threadIdx.x][w];
        part[blockIdx.x * N + threadIdx.x] = v;
    }
}

__global__ void __launch_bounds__(FORCE_THREADS) k_ref_drag_lift(const uint8_t* __restrict__ lab,
                                                                 const float* __restrict__ u,
                                                                 const float* __restrict__ v,
                                                                 const float* __restrict__ w, Dims g, float3 cm,
                                                                 float3 bvel, double* __restrict__ part) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < g.nc(); c += int64_t(gridDim.x) * blockDim.x) {
        if (lab[c] != BODY) continue;
        const int i = int(c % g.W), j = int((c / g.W) % g.H), k = int(c / (int64_t(g.W) * g.H));
        for (int dir = 0; dir < 6; ++dir) {
            const int ax = dir >> 1, sg = (dir & 1) ? -1 : 1;
            const int ni = i + (ax == 0) * sg, nj = j + (ax == 1) * sg, nk = k + (ax == 2) * sg;
            if (ni < 0 || ni >= g.W || nj < 0 || nj >= g.H || nk < 0 || nk >= g.D) continue;
            if (lab[ni + int64_t(nj) * g.W + int64_t(nk) * g.W * g.H] != FLUID) continue;
            float3 F, T;
            ref_panel(i, j, k, dir, u, v, w, g, cm, bvel, F, T);
            acc[0] += F.x; acc[1] += F.y; acc[2] += F.z;
            acc[3] += T.x; acc[4] += T.y; acc[5] += T.z;
        }
    }
    block_partials<6>(acc, part);
}

// Buoyancy: every SDF voxel with sdf <= 0 (corner origin + (i, j, k) cs,
// rotated about the local centre of mass into the world), weighted by its
// volume fraction, counts as submerged when its grid cell is FLUID or holds a
// particle within 2 dx (the particles are cell-sorted: start[c]..start[c+1]).
// part gets (total volume, submerged volume) per block.
__global__ void __launch_bounds__(FORCE_THREADS) k_ref_buoyancy(RefBuoyancy b, const uint8_t* __restrict__ lab, Dims g,
                                                                const float4* __restrict__ pos,
                                                                const int* __restrict__ start,
                                                                double* __restrict__ part) {
    double acc[2] = {0.0, 0.0};
    const int64_t nv = int64_t(b.sw) * b.sh * b.sd;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nv; t += int64_t(gridDim.x) * blockDim.x) {
        const int i = int(t % b.sw), j = int((t / b.sw) % b.sh), k = int(t / (int64_t(b.sw) * b.sh));
        const float3 pl = make_float3(__fadd_rn(b.origin.x, __fmul_rn(float(i), b.cs)),
                                      __fadd_rn(b.origin.y, __fmul_rn(float(j), b.cs)),
                                      __fadd_rn(b.origin.z, __fmul_rn(float(k), b.cs)));
        float sdf;
        if (b.sdf) {
            sdf = b.sdf[t];
        } else {  // analytic sphere sampled at the voxel corner
            const float3 d = sub3(pl, b.local_com);
            sdf = __fsub_rn(__fsqrt_rn(dot3(d, d)), b.radius);
        }
        if (sdf > 0.0f) continue;
        const float3 pc = sub3(pl, b.local_com);
        const float3 pr = make_float3(__fadd_rn(__fadd_rn(__fmul_rn(b.rot[0], pc.x), __fmul_rn(b.rot[1], pc.y)), __fmul_rn(b.rot[2], pc.z)),
                                      __fadd_rn(__fadd_rn(__fmul_rn(b.rot[3], pc.x), __fmul_rn(b.rot[4], pc.y)), __fmul_rn(b.rot[5], pc.z)),
                                      __fadd_rn(__fadd_rn(__fmul_rn(b.rot[6], pc.x), __fmul_rn(b.rot[7], pc.y)), __fmul_rn(b.rot[8], pc.z)));
        const float3 vc = add3(b.com, pr);
        float vol = __fmul_rn(__fmul_rn(b.cs, b.cs), b.cs);
        if (sdf > -b.cs) vol = __fmul_rn(vol, __fsub_rn(0.5f, __fdiv_rn(__fmul_rn(0.5f, sdf), b.cs)));
        acc[0] += vol;
        const int ii = min(max(__float2int_rz(__fdiv_rn(vc.x, g.dx)), 0), g.W - 1);
        const int jj = min(max(__float2int_rz(__fdiv_rn(vc.y, g.dx)), 0), g.H - 1);
        const int kk = min(max(__float2int_rz(__fdiv_rn(vc.z, g.dx)), 0), g.D - 1);
        const int64_t c = ii + int64_t(jj) * g.W + int64_t(kk) * g.W * g.H;
        bool sub = lab[c] == FLUID;
        const float rad = __fmul_rn(2.0f, g.dx);
        for (int q = start[c]; !sub && q < start[c + 1]; ++q) {
            const float4 P = pos[q];
            const float3 d = sub3(make_float3(P.x, P.y, P.z), vc);
            sub = __fsqrt_rn(dot3(d, d)) < rad;
        }
        if (sub) acc[1] += vol;
    }
    block_partials<2>(acc, part);
}

__global__ void k_sum_partials(const double* __restrict__ part, int nb, int n, double* __restrict__ out) {
    if (threadIdx.x < n) {
        double v = 0.0;
        for (int b = 0; b < nb; ++b) v += part[b * n + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

}  // namespace

namespace {
__global__ void k_apply_mark(uint8_t* __restrict__ labels, const uint8_t* __restrict__ mark, int64_t nc) {
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c < nc && mark[c] && labels[c] != SOLID) labels[c] = BODY;
}
}  // namespace

void launch_apply_mark(uint8_t* labels, const uint8_t* mark, Dims g, cudaStream_t st) {
    k_apply_mark<<<unsigned((g.nc() + 255) / 256), 256, 0, st>>>(labels, mark, g.nc());
}

void launch_mark_body(uint8_t* mark, Dims g, const BodyShape& b, cudaStream_t st) {
    k_mark_body<<<unsigned((g.nc() + 255) / 256), 256, 0, st>>>(mark, g, b);
}

constexpr int FORCE_BLOCKS = 592;

void launch_ref_body_forces(const uint8_t* labels, const float* u, const float* v, const float* w, Dims g, float3 cm,
                            float3 bvel, const RefBuoyancy& b, const float4* pos, const int* start, double* part,
                            double* out, cudaStream_t st) {
    k_ref_drag_lift<<<FORCE_BLOCKS, FORCE_THREADS, 0, st>>>(labels, u, v, w, g, cm, bvel, part);
    k_sum_partials<<<1, 32, 0, st>>>(part, FORCE_BLOCKS, 6, out);
    k_ref_buoyancy<<<FORCE_BLOCKS, FORCE_THREADS, 0, st>>>(b, labels, g, pos, start, part);
    k_sum_partials<<<1, 32, 0, st>>>(part, FORCE_BLOCKS, 2, out + 6);
}

void launch_body_force(const float* p, const uint8_t* labels, Dims g, const BodyShape& b, double* part, double* out,
                       cudaStream_t st) {
    k_body_force<<<FORCE_BLOCKS, FORCE_THREADS, 0, st>>>(p, labels, g, b, part);
    k_body_force_sum<<<1, 32, 0, st>>>(part, FORCE_BLOCKS, out);
}

int body_force_partials() { return FORCE_BLOCKS * 6; }

}  // namespace fp
