// fluid_oracle.cpp -- CPU oracle for the FluidPrjct PIC/FLIP step.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the CPU, the algorithm of
// Ship-Vano/FluidPrjct's 3D solver (src/FluidSim/FluidSolver3D.cu) so that the
// CUDA path can be checked against it.  Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline / reference arm may load it; the product library
// never links or calls it.
//
// Two arithmetic modes share one template:
//   Real = float : the reference's FP32 operation order (same expressions as the
//                  Thrust functors, evaluated left to right, no FMA contraction);
//   Real = double: the same algorithm in FP64 ("error vs FP64 oracle").
// The pressure system is always solved in FP64 (Jacobi-preconditioned CG to a
// caller-chosen relative residual), standing in for the reference's cuDSS
// direct factorisation (FluidSolver3D.cu:1930-2008): the SPD system has one
// solution, so the exact solve is the arbiter.
//
// Out-of-domain neighbours are treated as SOLID walls everywhere.  The
// reference reads wrapped or out-of-range memory at the domain border
// (FluidSolver3D.cu:1406,1427,1448,2109-2110); for every scene with a 1-cell
// SOLID border (all reference fixtures and all benchmark scenes) the two
// agree exactly.
//
// Parity pins (see tests/): particles_-1.ply binning (44,144 particles in
// 11,036 cells x 4 at dx = 0.02), the labels_simple3d.txt Poisson system and
// the 5x5 SPD known-answer system of src/FluidSim/test.cu:261-290,378-383.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <random>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Cell labels, utility.cuh:65-68.
constexpr uint8_t SOLID = 0, FLUID = 1, AIR = 2, BODY = 3;

template <class R> struct V3 { R x, y, z; };
template <class R> inline V3<R> mk(R x, R y, R z) { return {x, y, z}; }
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }

// Rigid body state used by the RHS and projection (FluidSolver3D.cu:1368-1370,
// 2081-2083): linear velocity, angular velocity and centre of mass.
template <class R> struct BodyKin { V3<R> vel{0, 0, 0}, omega{0, 0, 0}, com{0, 0, 0}; };

// trilinearInterpolation, FluidSolver3D.cu:783-801.
template <class R>
inline R trilin(R xd, R yd, R zd, R c000, R c100, R c001, R c101, R c010, R c110, R c011, R c111) {
    const R one = R(1);
    R c00 = c000 * (one - xd) + c100 * xd;
    R c01 = c001 * (one - xd) + c101 * xd;
    R c10 = c010 * (one - xd) + c110 * xd;
    R c11 = c011 * (one - xd) + c111 * xd;
    R c0 = c00 * (one - yd) + c10 * yd;
    R c1 = c01 * (one - yd) + c11 * yd;
    return c0 * (one - zd) + c1 * zd;
}

template <class R> inline R clamp01(R f) { return std::min(std::max(f, R(0)), R(1)); }

// Rigid body (RigidBody, utility.cuh:195-491) with an analytic sphere SDF.
struct OBody {
    bool loaded = false;
    bool paddle = false;  // half-space x < pos[0] with prescribed motion (fp_set_paddle)
    double pad_x0 = 0, pad_amp = 0, pad_period = 1, pad_t = 0;
    void paddle_at(double t) {
        const double w = 2.0 * 3.14159265358979323846 / pad_period;
        pos[0] = pad_x0 + pad_amp * std::sin(w * t);
        vel[0] = pad_amp * w * std::cos(w * t);
        vel[1] = vel[2] = 0.0;
        omega[0] = omega[1] = omega[2] = 0.0;
    }
    double pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, omega[3] = {0, 0, 0};
    double theta = 0, psi = 0, phi = 0, Rm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double mass = 1, inertia = 1, radius = 0;
    double force[3] = {0, 0, 0}, torque[3] = {0, 0, 0};
    void update_rotation() {  // utility.cuh:470-484
        const double ct = std::cos(theta), st = std::sin(theta), cp = std::cos(psi), sp = std::sin(psi),
                     cf = std::cos(phi), sf = std::sin(phi);
        Rm[0] = ct * cp; Rm[1] = st * sf - ct * cf * sp; Rm[2] = cf * st + ct * sf * sp;
        Rm[3] = sp;      Rm[4] = cf * cp;                Rm[5] = -cp * sf;
        Rm[6] = -cp * st; Rm[7] = ct * sf + cf * st * sp; Rm[8] = ct * cf - st * sf * sp;
    }
    void integrate(double dt) {  // utility.cuh:408-467
        for (int a = 0; a < 3; ++a) { vel[a] += force[a] / mass * dt; pos[a] += vel[a] * dt; }
        const double pi = 3.14159265358979323846;
        theta = std::min(std::max(theta, -pi), pi);
        update_rotation();
        const double tl[3] = {Rm[0] * torque[0] + Rm[3] * torque[1] + Rm[6] * torque[2],
                              Rm[1] * torque[0] + Rm[4] * torque[1] + Rm[7] * torque[2],
                              Rm[2] * torque[0] + Rm[5] * torque[1] + Rm[8] * torque[2]};
        for (int a = 0; a < 3; ++a) omega[a] += tl[a] / inertia * dt;
        const double dth = omega[1] * std::cos(phi) - omega[2] * std::sin(phi);
        const double dps = (omega[1] * std::sin(phi) + omega[2] * std::cos(phi)) / std::cos(theta);
        const double dph = omega[0] + dps * std::sin(theta);
        theta += dth * dt; psi += dps * dt; phi += dph * dt;
    }
};

template <class R> struct Sim3 {
    int W = 0, H = 0, D = 0;
    R dx = 0, dt = 0;
    R alpha = R(0.05);      // PIC_WEIGHT
    R cfl = R(0.1);         // advectParticles(0.1), FluidSolver3D.cu:3092
    int rk2 = 0;            // 1: midpoint RK2 in place of the reference's RK3
    int sdf_collide = 0;    // 1: SDF collision projection against the body (not the reference's)
    double tol = 1e-12;     // relative residual of the FP64 solve
    int maxit = 100000;
    BodyKin<R> body;
    OBody ob;
    std::vector<uint8_t> labels;
    std::vector<R> u, v, w, us, vs, ws, p;
    std::vector<R> px, py, pz, vx, vy, vz;
    int extrap = 0;  // layers of velocity extrapolation between G2P and advection
    int ref_forces = 0;  // 1: the reference's panel drag/lift and voxel buoyancy
    double ref_out[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // last reference force, torque, volumes
    int last_iters = 0;
    double last_res = 0.0;
    int last_nf = 0;

    size_t nc() const { return size_t(W) * H * D; }
    size_t nu() const { return size_t(W + 1) * H * D; }
    size_t nv() const { return size_t(W) * (H + 1) * D; }
    size_t nw() const { return size_t(W) * H * (D + 1); }
    size_t np() const { return px.size(); }

    void alloc() {
        labels.assign(nc(), AIR);
        u.assign(nu(), 0); us.assign(nu(), 0);
        v.assign(nv(), 0); vs.assign(nv(), 0);
        w.assign(nw(), 0); ws.assign(nw(), 0);
        p.assign(nc(), 0);
    }
    inline size_t cidx(int i, int j, int k) const { return size_t(i) + size_t(j) * W + size_t(k) * W * H; }
    inline uint8_t lab(int i, int j, int k) const {
        if (i < 0 || i >= W || j < 0 || j >= H || k < 0 || k >= D) return SOLID;
        return labels[cidx(i, j, k)];
    }
    inline size_t uidx(int i, int j, int k) const { return size_t(i) + size_t(j) * (W + 1) + size_t(k) * (W + 1) * H; }
    inline size_t vidx(int i, int j, int k) const { return size_t(i) + size_t(j) * W + size_t(k) * W * (H + 1); }
    inline size_t widx(int i, int j, int k) const { return size_t(i) + size_t(j) * W + size_t(k) * W * H; }

    // ---- labelGrid, FluidSolver3D.cu:340-397 (K1, K3; K2 needs a body SDF) ----
    // Cell key of a particle: floorf(p/dx) clamped to [0, N-1] (:323-331).
    inline void cell_of(R x, R y, R z, int& i, int& j, int& k) const {
        i = int(std::floor(x / dx)); j = int(std::floor(y / dx)); k = int(std::floor(z / dx));
        i = std::min(std::max(i, 0), W - 1);
        j = std::min(std::max(j, 0), H - 1);
        k = std::min(std::max(k, 0), D - 1);
    }
    // Body SDF in FP32 (the GPU's explicitly rounded float evaluation): the
    // sphere, or the paddle's signed distance x - x_p.
    float sphere_sdf(float x, float y, float z) const {
        if (ob.paddle) return x - float(ob.pos[0]);
        const float cx = float(ob.pos[0]), cy = float(ob.pos[1]), cz = float(ob.pos[2]);
        const float dxp = x - cx, dyp = y - cy, dzp = z - cz;
        const float s2 = (dxp * dxp + dyp * dyp) + dzp * dzp;
        return std::sqrt(s2) - float(ob.radius);
    }
    void label_grid() {
        for (auto& l : labels) l = (l == SOLID) ? SOLID : AIR;  // ClearNonSolidFunctor
        if (ob.loaded) {  // MarkBodyCellsFunctor (:45-78) with the analytic sphere
            const float fdx = float(dx);
            for (int k = 0; k < D; ++k) for (int j = 0; j < H; ++j) for (int i = 0; i < W; ++i) {
                uint8_t& l = labels[cidx(i, j, k)];
                if (l != SOLID && sphere_sdf((float(i) + 0.5f) * fdx, (float(j) + 0.5f) * fdx, (float(k) + 0.5f) * fdx) <= 0.0f)
                    l = BODY;
            }
        }
        for (size_t q = 0; q < np(); ++q) {
            int i, j, k;
            cell_of(px[q], py[q], pz[q], i, j, k);
            uint8_t& l = labels[cidx(i, j, k)];
            if (l != SOLID && l != BODY) l = FLUID;
        }
    }

    // ---- particlesToGrid, FluidSolver3D.cu:438-685 ----
    void p2g() {
        std::vector<R> un(nu(), 0), ud(nu(), 0), vn(nv(), 0), vd(nv(), 0), wn(nw(), 0), wd(nw(), 0);
        const R half = R(0.5);
        for (size_t q = 0; q < np(); ++q) {
            R rx = px[q] / dx, ry = py[q] / dx, rz = pz[q] / dx;
            // U component (:465-498)
            {
                int i0 = int(std::floor(rx)), j0 = int(std::floor(ry - half)), k0 = int(std::floor(rz - half));
                i0 = std::min(std::max(i0, 0), W); j0 = std::min(std::max(j0, 0), H - 1); k0 = std::min(std::max(k0, 0), D - 1);
                R f[3] = {clamp01(rx - R(i0)), clamp01((ry - half) - R(j0)), clamp01((rz - half) - R(k0))};
                for (int dz = 0; dz < 2; ++dz) { int k = k0 + dz; if (k < 0 || k >= D) continue;
                for (int dy = 0; dy < 2; ++dy) { int j = j0 + dy; if (j < 0 || j >= H) continue;
                for (int dxx = 0; dxx < 2; ++dxx) { int i = i0 + dxx; if (i < 0 || i > W) continue;
                    R wx = dxx == 0 ? R(1) - f[0] : f[0], wy = dy == 0 ? R(1) - f[1] : f[1], wz = dz == 0 ? R(1) - f[2] : f[2];
                    R wgt = wx * wy * wz;
                    size_t id = uidx(i, j, k); un[id] += vx[q] * wgt; ud[id] += wgt; } } }
            }
            // V component (:503-536)
            {
                int i0 = int(std::floor(rx - half)), j0 = int(std::floor(ry)), k0 = int(std::floor(rz - half));
                i0 = std::min(std::max(i0, 0), W - 1); j0 = std::min(std::max(j0, 0), H); k0 = std::min(std::max(k0, 0), D - 1);
                R f[3] = {clamp01((rx - half) - R(i0)), clamp01(ry - R(j0)), clamp01((rz - half) - R(k0))};
                for (int dz = 0; dz < 2; ++dz) { int k = k0 + dz; if (k < 0 || k >= D) continue;
                for (int dy = 0; dy < 2; ++dy) { int j = j0 + dy; if (j < 0 || j > H) continue;
                for (int dxx = 0; dxx < 2; ++dxx) { int i = i0 + dxx; if (i < 0 || i >= W) continue;
                    R wx = dxx == 0 ? R(1) - f[0] : f[0], wy = dy == 0 ? R(1) - f[1] : f[1], wz = dz == 0 ? R(1) - f[2] : f[2];
                    R wgt = wx * wy * wz;
                    size_t id = vidx(i, j, k); vn[id] += vy[q] * wgt; vd[id] += wgt; } } }
            }
            // W component (:541-574)
            {
                int i0 = int(std::floor(rx - half)), j0 = int(std::floor(ry - half)), k0 = int(std::floor(rz));
                i0 = std::min(std::max(i0, 0), W - 1); j0 = std::min(std::max(j0, 0), H - 1); k0 = std::min(std::max(k0, 0), D);
                R f[3] = {clamp01((rx - half) - R(i0)), clamp01((ry - half) - R(j0)), clamp01(rz - R(k0))};
                for (int dz = 0; dz < 2; ++dz) { int k = k0 + dz; if (k < 0 || k > D) continue;
                for (int dy = 0; dy < 2; ++dy) { int j = j0 + dy; if (j < 0 || j >= H) continue;
                for (int dxx = 0; dxx < 2; ++dxx) { int i = i0 + dxx; if (i < 0 || i >= W) continue;
                    R wx = dxx == 0 ? R(1) - f[0] : f[0], wy = dy == 0 ? R(1) - f[1] : f[1], wz = dz == 0 ? R(1) - f[2] : f[2];
                    R wgt = wx * wy * wz;
                    size_t id = widx(i, j, k); wn[id] += vz[q] * wgt; wd[id] += wgt; } } }
            }
        }
        // ComputeVelocityFunc (:598-605): den > 1e-8 ? num/den : 0
        const R eps = R(1e-8f);
        for (size_t i = 0; i < nu(); ++i) u[i] = ud[i] > eps ? un[i] / ud[i] : R(0);
        for (size_t i = 0; i < nv(); ++i) v[i] = vd[i] > eps ? vn[i] / vd[i] : R(0);
        for (size_t i = 0; i < nw(); ++i) w[i] = wd[i] > eps ? wn[i] / wd[i] : R(0);
    }

    // ---- saveVelocities (:399-415) and applyForces (:700-761) ----
    void save() { us = u; vs = v; ws = w; }
    void forces() {
        // ApplyScalarForce: x > (float)INT_MIN ? x + dt*a : x; gravity (0,-9.81,0) (:78,:687-698)
        const R lim = R(-2147483648.0f);
        const R ax = R(0.0f), ay = R(-9.81f), az = R(0.0f);
        for (auto& x : u) x = (x > lim) ? x + dt * ax : x;
        for (auto& x : v) x = (x > lim) ? x + dt * ay : x;
        for (auto& x : w) x = (x > lim) ? x + dt * az : x;
    }

    inline V3<R> body_vel_at(V3<R> pos) const {
        V3<R> r = pos - body.com;
        return {body.vel.x + body.omega.y * r.z - body.omega.z * r.y,
                body.vel.y + body.omega.z * r.x - body.omega.x * r.z,
                body.vel.z + body.omega.x * r.y - body.omega.y * r.x};
    }
    static inline bool solidish(uint8_t l) { return l == SOLID || l == BODY; }

    // ---- RHSCalculator3D, FluidSolver3D.cu:1360-1474, scale = rho*dx/dt (:1520) ----
    R rhs_at(int i, int j, int k) const {
        const R scale = (R(1000.0f) * dx) / dt;
        R div = u[uidx(i + 1, j, k)] - u[uidx(i, j, k)] + v[vidx(i, j + 1, k)] - v[vidx(i, j, k)] +
                w[widx(i, j, k + 1)] - w[widx(i, j, k)];
        R rhs = -scale * div;
        const R h = R(0.5f);
        uint8_t l;
        if ((l = lab(i - 1, j, k)), solidish(l)) {
            R us_ = l == BODY ? body_vel_at(mk(R(i) * dx, (R(j) + h) * dx, (R(k) + h) * dx)).x : R(0);
            rhs -= scale * (u[uidx(i, j, k)] - us_);
        }
        if ((l = lab(i + 1, j, k)), solidish(l)) {
            R us_ = l == BODY ? body_vel_at(mk(R(i + 1) * dx, (R(j) + h) * dx, (R(k) + h) * dx)).x : R(0);
            rhs += scale * (u[uidx(i + 1, j, k)] - us_);
        }
        if ((l = lab(i, j - 1, k)), solidish(l)) {
            R vs_ = l == BODY ? body_vel_at(mk((R(i) + h) * dx, R(j) * dx, (R(k) + h) * dx)).y : R(0);
            rhs -= scale * (v[vidx(i, j, k)] - vs_);
        }
        if ((l = lab(i, j + 1, k)), solidish(l)) {
            R vs_ = l == BODY ? body_vel_at(mk((R(i) + h) * dx, R(j + 1) * dx, (R(k) + h) * dx)).y : R(0);
            rhs += scale * (v[vidx(i, j + 1, k)] - vs_);
        }
        if ((l = lab(i, j, k - 1)), solidish(l)) {
            R ws_ = l == BODY ? body_vel_at(mk((R(i) + h) * dx, (R(j) + h) * dx, R(k) * dx)).z : R(0);
            rhs -= scale * (w[widx(i, j, k)] - ws_);
        }
        if ((l = lab(i, j, k + 1)), solidish(l)) {
            R ws_ = l == BODY ? body_vel_at(mk((R(i) + h) * dx, (R(j) + h) * dx, R(k + 1) * dx)).z : R(0);
            rhs += scale * (w[widx(i, j, k + 1)] - ws_);
        }
        return rhs;
    }

    // Unit 7-point operator of MatrixBuilder3D/MatrixFiller3D (:1598-1777):
    // diag = # in-domain FLUID or AIR neighbours, off-diagonal -1 to FLUID ones.
    inline int diag_at(int i, int j, int k) const {
        int d = 0;
        const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        for (auto& o : off) { uint8_t l = lab(i + o[0], j + o[1], k + o[2]); if (l == FLUID || l == AIR) ++d; }
        return d;
    }

    // FP64 Jacobi-PCG on the dense grid (non-fluid entries held at zero).
    // Returns the iteration count; x holds the solution on FLUID cells.
    int solve(const std::vector<double>& b, std::vector<double>& x) {
        const size_t n = nc();
        std::vector<double> r(n, 0.0), z(n, 0.0), d(n, 0.0), q(n, 0.0), dg(n, 0.0);
        std::vector<uint8_t> fl(n, 0);
        const long long WH = (long long)W * H;
        #pragma omp parallel for schedule(static)
        for (long long c = 0; c < (long long)n; ++c) {
            int i = int(c % W), j = int((c / W) % H), k = int(c / WH);
            fl[c] = labels[c] == FLUID;
            dg[c] = fl[c] ? double(diag_at(i, j, k)) : 0.0;
        }
        auto apply = [&](const std::vector<double>& in, std::vector<double>& out) {
            #pragma omp parallel for schedule(static)
            for (long long c = 0; c < (long long)n; ++c) {
                if (!fl[c]) { out[c] = 0.0; continue; }
                int i = int(c % W), j = int((c / W) % H), k = int(c / WH);
                double s = dg[c] * in[c];
                if (i + 1 < W && fl[c + 1]) s -= in[c + 1];
                if (i - 1 >= 0 && fl[c - 1]) s -= in[c - 1];
                if (j + 1 < H && fl[c + W]) s -= in[c + W];
                if (j - 1 >= 0 && fl[c - W]) s -= in[c - W];
                if (k + 1 < D && fl[c + WH]) s -= in[c + WH];
                if (k - 1 >= 0 && fl[c - WH]) s -= in[c - WH];
                out[c] = s;
            }
        };
        auto dot = [&](const std::vector<double>& a, const std::vector<double>& bb) {
            double s = 0.0;
            #pragma omp parallel for reduction(+ : s) schedule(static)
            for (long long c = 0; c < (long long)n; ++c) s += a[c] * bb[c];
            return s;
        };
        x.assign(n, 0.0);
        apply(x, q);
        #pragma omp parallel for schedule(static)
        for (long long c = 0; c < (long long)n; ++c) r[c] = fl[c] ? b[c] - q[c] : 0.0;
        double bn = std::sqrt(dot(b, b));
        if (bn == 0.0) { last_res = 0.0; return 0; }
        #pragma omp parallel for schedule(static)
        for (long long c = 0; c < (long long)n; ++c) { z[c] = fl[c] && dg[c] > 0 ? r[c] / dg[c] : 0.0; d[c] = z[c]; }
        double rz = dot(r, z);
        int it = 0;
        double rn = std::sqrt(dot(r, r));
        while (rn / bn > tol && it < maxit) {
            apply(d, q);
            double dq = dot(d, q);
            if (dq == 0.0) break;
            double a = rz / dq;
            #pragma omp parallel for schedule(static)
            for (long long c = 0; c < (long long)n; ++c) {
                x[c] += a * d[c]; r[c] -= a * q[c];
                z[c] = fl[c] && dg[c] > 0 ? r[c] / dg[c] : 0.0;
            }
            double rz2 = dot(r, z);
            double be = rz2 / rz; rz = rz2;
            #pragma omp parallel for schedule(static)
            for (long long c = 0; c < (long long)n; ++c) d[c] = z[c] + be * d[c];
            rn = std::sqrt(dot(r, r));
            ++it;
        }
        // True residual of the returned solution.
        apply(x, q);
        double s = 0.0;
        #pragma omp parallel for reduction(+ : s) schedule(static)
        for (long long c = 0; c < (long long)n; ++c) if (fl[c]) { double e = b[c] - q[c]; s += e * e; }
        last_res = std::sqrt(s) / bn;
        return it;
    }

    // ---- pressureSolve (:1815-2062): rhs, unit operator, solve, scatter to dense p ----
    int pressure() {
        const size_t n = nc();
        std::vector<double> b(n, 0.0), x;
        int nf = 0;
        for (int k = 0; k < D; ++k) for (int j = 0; j < H; ++j) for (int i = 0; i < W; ++i) {
            size_t c = cidx(i, j, k);
            if (labels[c] == FLUID) { b[c] = double(rhs_at(i, j, k)); ++nf; }
        }
        last_nf = nf;
        std::fill(p.begin(), p.end(), R(0));
        if (nf == 0) { last_iters = 0; last_res = 0; return -1; }  // :1875-1878
        last_iters = solve(b, x);
        for (size_t c = 0; c < n; ++c) p[c] = labels[c] == FLUID ? R(x[c]) : R(0);
        return 0;
    }

    // ---- applyPressure, UFunctor/VFunctor/WFunctor (:2072-2464), scale = dt/(rho*dx) ----
    // One face between cells L and Rc, both possibly out of domain (=SOLID).
    inline R project_face(R vel, uint8_t lL, uint8_t lR, R pL, R pR, R vb, R scale, R inv) const {
        auto fa = [](uint8_t l) { return l == FLUID || l == AIR; };
        R p0, p1;
        if (fa(lL) && fa(lR)) { p0 = pL; p1 = pR; }
        else if (solidish(lL)) { R s = lL == BODY ? vb : R(0); p0 = pR - inv * (vel - s); p1 = pR; }
        else if (solidish(lR)) { R s = lR == BODY ? vb : R(0); p0 = pL; p1 = pL + inv * (vel - s); }
        else { p0 = pL; p1 = pR; }
        return vel - scale * (p1 - p0);
    }
    inline R pat(int i, int j, int k) const {
        if (i < 0 || i >= W || j < 0 || j >= H || k < 0 || k >= D) return R(0);
        return p[cidx(i, j, k)];
    }
    void project() {
        const R scale = dt / (R(1000.0f) * dx);
        const R inv = R(1) / scale;
        const R h = R(0.5f);
        for (int k = 0; k < D; ++k) for (int j = 0; j < H; ++j) for (int i = 0; i <= W; ++i) {
            V3<R> vb = body_vel_at(mk(R(i) * dx, (R(j) + h) * dx, (R(k) + h) * dx));
            size_t id = uidx(i, j, k);
            u[id] = project_face(u[id], lab(i - 1, j, k), lab(i, j, k), pat(i - 1, j, k), pat(i, j, k), vb.x, scale, inv);
        }
        for (int k = 0; k < D; ++k) for (int j = 0; j <= H; ++j) for (int i = 0; i < W; ++i) {
            V3<R> vb = body_vel_at(mk((R(i) + h) * dx, R(j) * dx, (R(k) + h) * dx));
            size_t id = vidx(i, j, k);
            v[id] = project_face(v[id], lab(i, j - 1, k), lab(i, j, k), pat(i, j - 1, k), pat(i, j, k), vb.y, scale, inv);
        }
        for (int k = 0; k <= D; ++k) for (int j = 0; j < H; ++j) for (int i = 0; i < W; ++i) {
            V3<R> vb = body_vel_at(mk((R(i) + h) * dx, (R(j) + h) * dx, R(k) * dx));
            size_t id = widx(i, j, k);
            w[id] = project_face(w[id], lab(i, j, k - 1), lab(i, j, k), pat(i, j, k - 1), pat(i, j, k), vb.z, scale, inv);
        }
    }

    // ---- MAC trilinear sample (interpVelDevice3D :1051-1157, GridToParticleFunctor :803-980) ----
    // Base indices are clamped so that base+1 stays inside the face grid; for
    // positions inside [0, (N-1)*dx] (where advection keeps particles) this is
    // the reference's clamp exactly.
    struct Stencil { int i, j, k; R fx, fy, fz; };
    inline Stencil st_u(R rx, R ry, R rz) const {
        const R h = R(0.5f);
        int i = int(std::floor(rx)), j = int(std::floor(ry - h)), k = int(std::floor(rz - h));
        i = std::min(std::max(i, 0), W - 1); j = std::min(std::max(j, 0), H - 2); k = std::min(std::max(k, 0), std::max(D - 2, 0));
        return {i, j, k, clamp01(rx - R(i)), clamp01((ry - h) - R(j)), clamp01((rz - h) - R(k))};
    }
    inline Stencil st_v(R rx, R ry, R rz) const {
        const R h = R(0.5f);
        int i = int(std::floor(rx - h)), j = int(std::floor(ry)), k = int(std::floor(rz - h));
        i = std::min(std::max(i, 0), W - 2); j = std::min(std::max(j, 0), H - 1); k = std::min(std::max(k, 0), std::max(D - 2, 0));
        return {i, j, k, clamp01((rx - h) - R(i)), clamp01(ry - R(j)), clamp01((rz - h) - R(k))};
    }
    inline Stencil st_w(R rx, R ry, R rz) const {
        const R h = R(0.5f);
        int i = int(std::floor(rx - h)), j = int(std::floor(ry - h)), k = int(std::floor(rz));
        i = std::min(std::max(i, 0), W - 2); j = std::min(std::max(j, 0), H - 2); k = std::min(std::max(k, 0), D - 1);
        return {i, j, k, clamp01((rx - h) - R(i)), clamp01((ry - h) - R(j)), clamp01(rz - R(k))};
    }
    // Sample f (or f - g when g is given) over one face grid with row stride sx, slice stride sxy.
    inline R sample(const std::vector<R>& f, const std::vector<R>* g, const Stencil& s, size_t sx, size_t sxy) const {
        size_t b = size_t(s.i) + size_t(s.j) * sx + size_t(s.k) * sxy;
        auto val = [&](size_t o) { return g ? f[b + o] - (*g)[b + o] : f[b + o]; };
        return trilin(s.fx, s.fy, s.fz, val(0), val(1), val(sxy), val(1 + sxy), val(sx), val(1 + sx), val(sx + sxy), val(1 + sx + sxy));
    }
    // Slice strides of u and v for sample(); a 2D grid (D = 1) uses 0, so the
    // duplicate z corners carry weight 0 (exact bilinear interpolation).
    size_t sxy_u() const { return D > 1 ? size_t(W + 1) * H : 0; }
    size_t sxy_v() const { return D > 1 ? size_t(W) * (H + 1) : 0; }
    inline V3<R> interp_vel(V3<R> pos) const {
        R rx = pos.x / dx, ry = pos.y / dx, rz = pos.z / dx;
        return {sample(u, nullptr, st_u(rx, ry, rz), size_t(W + 1), sxy_u()),
                sample(v, nullptr, st_v(rx, ry, rz), size_t(W), sxy_v()),
                sample(w, nullptr, st_w(rx, ry, rz), size_t(W), size_t(W) * H)};
    }

    // ---- gridToParticles (:983-1039): v = a*PIC + (1-a)*(v + FLIP delta) ----
    void g2p() {
        #pragma omp parallel for schedule(static)
        for (long long q = 0; q < (long long)np(); ++q) {
            R rx = px[q] / dx, ry = py[q] / dx, rz = pz[q] / dx;
            Stencil su = st_u(rx, ry, rz), sv = st_v(rx, ry, rz), sw = st_w(rx, ry, rz);
            size_t sxu = W + 1, sxyu = sxy_u(), sxv = W, sxyv = sxy_v(), sxw = W, sxyw = size_t(W) * H;
            R uP = sample(u, nullptr, su, sxu, sxyu), dU = sample(u, &us, su, sxu, sxyu);
            R vP = sample(v, nullptr, sv, sxv, sxyv), dV = sample(v, &vs, sv, sxv, sxyv);
            R wP = sample(w, nullptr, sw, sxw, sxyw), dW = sample(w, &ws, sw, sxw, sxyw);
            const R one = R(1);
            vx[q] = alpha * uP + (one - alpha) * (vx[q] + dU);
            vy[q] = alpha * vP + (one - alpha) * (vy[q] + dV);
            vz[q] = alpha * wP + (one - alpha) * (vz[q] + dW);
        }
    }

    // ---- projectParticleDevice3D (:1161-1239): nudge toward the nearest FLUID
    // cell centre among 34 offsets (entry 9 is {-1,-1,0}). ----
    bool project_particle(V3<R>& pos) const {
        static const int off[34][3] = {
            {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
            {1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0},
            {1, 0, 1}, {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1},
            {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1},
            {1, 1, 1}, {-1, 1, 1}, {1, -1, 1}, {1, 1, -1},
            {-1, -1, 1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, -1},
            {-2, -1, 0}, {0, -1, -2}, {-2, -2, 0}, {0, -2, -2},
            {-2, -2, -2}, {-2, 0, -2}, {2, -1, 0}, {0, -1, 2}};
        int cx = int(std::floor(pos.x / dx)), cy = int(std::floor(pos.y / dx)), cz = int(std::floor(pos.z / dx));
        R best = R(1e10f);
        int bn = -1;
        const R h = R(0.5f);
        for (int n = 0; n < 34; ++n) {
            int nx = cx + off[n][0], ny = cy + off[n][1], nz = cz + off[n][2];
            if (nx < 0 || nx >= W || ny < 0 || ny >= H || nz < 0 || nz >= D) continue;
            if (labels[cidx(nx, ny, nz)] != FLUID) continue;
            R ccx = (R(nx) + h) * dx, ccy = (R(ny) + h) * dx, ccz = (R(nz) + h) * dx;
            R d = (ccx - pos.x) * (ccx - pos.x) + (ccy - pos.y) * (ccy - pos.y) + (ccz - pos.z) * (ccz - pos.z);
            if (d < best) { best = d; bn = n; }
        }
        if (bn < 0) return false;
        pos = pos + mk((R(off[bn][0]) * h) * dx, (R(off[bn][1]) * h) * dx, (R(off[bn][2]) * h) * dx);
        return true;
    }

    // ---- SDF collision projection (an addition beside projectParticleDevice3D,
    // the same arithmetic as the GPU's sdf_push_out): a point whose body SDF is
    // below eps moves along the SDF normal to phi = eps -- radially to r + eps
    // for the sphere, to x_p + eps for the paddle. ----
    void sdf_push_out(V3<R>& x, R eps) const {
        if (ob.paddle) {
            const R xp = R(float(ob.pos[0]));
            if (x.x - xp < eps) x.x = xp + eps;
            return;
        }
        const R cx = R(float(ob.pos[0])), cy = R(float(ob.pos[1])), cz = R(float(ob.pos[2]));
        const R rad = R(float(ob.radius));
        const R ex = x.x - cx, ey = x.y - cy, ez = x.z - cz;
        const R r = std::sqrt((ex * ex + ey * ey) + ez * ez);
        if (!(r - rad < eps)) return;
        const R target = rad + eps;
        if (r > R(0)) {
            const R sc = target / r;
            x = mk(cx + ex * sc, cy + ey * sc, cz + ez * sc);
        } else {
            x = mk(cx, cy + target, cz);
        }
    }

    // ---- AdvectParticlesFunctor (:1241-1330): adaptive substeps, Ralston RK3 ----
    void advect_one(R& x, R& y, R& z) const {
        V3<R> pos = mk(x, y, z);
        R subT = R(0);
        bool finished = false;
        int iter = 0;
        const R floor_speed = std::sqrt((R(5.0f) * dx) * R(9.8f));
        const R xmax = R(W - 1) * dx, ymax = R(H - 1) * dx, zmax = R(D - 1) * dx;
        while (!finished && iter++ < 1000) {
            V3<R> vel = interp_vel(pos);
            R speed = std::sqrt(vel.x * vel.x + vel.y * vel.y + vel.z * vel.z) + R(1e-37f) + floor_speed;
            R dT = (cfl * dx) / speed;
            if (subT + dT >= dt) { dT = dt - subT; finished = true; }
            else if (subT + R(2) * dT >= dt) { dT *= R(0.5f); }
            if (rk2) {  // the commented-out RK2 of FluidSolver3D.cu:1293-1296
                V3<R> k2 = interp_vel(pos + (vel * R(0.5f)) * dT);
                pos = pos + k2 * dT;
            } else {
                V3<R> k1 = vel;
                V3<R> k2 = interp_vel(pos + (k1 * R(0.5f)) * dT);
                V3<R> k3 = interp_vel(pos + (k2 * R(0.75f)) * dT);
                const R a1 = (R(2.0f) / R(9.0f)) * dT, a2 = (R(3.0f) / R(9.0f)) * dT, a3 = (R(4.0f) / R(9.0f)) * dT;
                pos = pos + k1 * a1 + k2 * a2 + k3 * a3;
            }
            subT += dT;
            pos.x = std::min(std::max(pos.x, R(0)), xmax);
            pos.y = std::min(std::max(pos.y, R(0)), ymax);
            pos.z = std::min(std::max(pos.z, R(0)), zmax);
            const bool sdf = sdf_collide && ob.loaded;
            if (sdf) {
                sdf_push_out(pos, R(0.25f) * dx);
                pos.x = std::min(std::max(pos.x, R(0)), xmax);
                pos.y = std::min(std::max(pos.y, R(0)), ymax);
                pos.z = std::min(std::max(pos.z, R(0)), zmax);
            }
            int cx = int(std::floor(pos.x / dx)), cy = int(std::floor(pos.y / dx)), cz = int(std::floor(pos.z / dx));
            if (cx >= 0 && cx < W && cy >= 0 && cy < H && cz >= 0 && cz < D) {
                uint8_t l = labels[cidx(cx, cy, cz)];
                if (l == SOLID || (l == BODY && !sdf)) {
                    if (!project_particle(pos)) break;  // the reference retries once, then stops (:1313-1317)
                }
            }
            if (pos.x < R(0) || pos.y < R(0) || pos.z < R(0) || std::isnan(pos.x) || std::isnan(pos.y) || std::isnan(pos.z)) break;
        }
        x = pos.x; y = pos.y; z = pos.z;
    }
    void advect() {
        #pragma omp parallel for schedule(dynamic, 4096)
        for (long long q = 0; q < (long long)np(); ++q) advect_one(px[q], py[q], pz[q]);
    }

    // Fluid force and torque on the body: -sum_f theta_f (p_R - p_L) dx^2 e_axis
    // over faces with body fraction theta_f = clamp(1/2 - phi(x_f)/dx, 0, 1);
    // BODY cells take the mean pressure of their FLUID/AIR neighbours; faces
    // touching SOLID or the outside are skipped.  FP64 accumulation.
    bool p_ext(int i, int j, int k, double& out) const {
        const uint8_t l = lab(i, j, k);
        if (l == SOLID) return false;
        if (l != BODY) { out = double(p[cidx(i, j, k)]); return true; }
        const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        float acc = 0.0f;
        int n = 0;
        for (auto& o : off) {
            const uint8_t ln = lab(i + o[0], j + o[1], k + o[2]);
            if (ln == FLUID || ln == AIR) { acc += float(p[cidx(i + o[0], j + o[1], k + o[2])]); ++n; }
        }
        out = n ? double(acc / float(n)) : 0.0;
        return true;
    }
    void body_force(double out[6]) const {
        for (int m = 0; m < 6; ++m) out[m] = 0.0;
        const float fdx = float(dx);
        const double area = double(fdx) * double(fdx);
        for (int k = 0; k <= D; ++k) for (int j = 0; j <= H; ++j) for (int i = 0; i <= W; ++i)
            for (int ax = 0; ax < 3; ++ax) {
                if (ax == 0 && (j >= H || k >= D)) continue;
                if (ax == 1 && (i >= W || k >= D)) continue;
                if (ax == 2 && (i >= W || j >= H)) continue;
                const float xf = ax == 0 ? float(i) * fdx : (float(i) + 0.5f) * fdx;
                const float yf = ax == 1 ? float(j) * fdx : (float(j) + 0.5f) * fdx;
                const float zf = ax == 2 ? float(k) * fdx : (float(k) + 0.5f) * fdx;
                const float th = std::min(std::max(0.5f - sphere_sdf(xf, yf, zf) / fdx, 0.0f), 1.0f);
                if (th <= 0.0f) continue;
                double pl, pr;
                if (!p_ext(i - (ax == 0), j - (ax == 1), k - (ax == 2), pl) || !p_ext(i, j, k, pr)) continue;
                const double dF = -double(th) * (pr - pl) * area;
                const double rx = double(xf) - double(float(ob.pos[0])), ry = double(yf) - double(float(ob.pos[1])),
                             rz = double(zf) - double(float(ob.pos[2]));
                const double fx = ax == 0 ? dF : 0.0, fy = ax == 1 ? dF : 0.0, fz = ax == 2 ? dF : 0.0;
                out[0] += fx; out[1] += fy; out[2] += fz;
                out[3] += ry * fz - rz * fy; out[4] += rz * fx - rx * fz; out[5] += rx * fy - ry * fx;
            }
    }
    // The reference's body forces (FP32 panels and voxels, FP64 sums):
    // DragLiftForceCalculator (:2674-2791) over BODY cells' FLUID faces, and
    // applyBuoyancy (:2917-3026) over the sphere sampled on a dx/2 voxel grid.
    void ref_body_forces(double out[8]) const {
        for (int m = 0; m < 8; ++m) out[m] = 0.0;
        const float fdx = float(dx), rho = 1000.0f;
        const float cmx = float(ob.pos[0]), cmy = float(ob.pos[1]), cmz = float(ob.pos[2]);
        const float bvx = float(ob.vel[0]), bvy = float(ob.vel[1]), bvz = float(ob.vel[2]);
        auto cross = [](float ax, float ay, float az, float bx, float by, float bz, float& cx, float& cy, float& cz) {
            cx = ay * bz - az * by; cy = az * bx - ax * bz; cz = ax * by - ay * bx;
        };
        for (int k = 0; k < D; ++k) for (int j = 0; j < H; ++j) for (int i = 0; i < W; ++i) {
            if (labels[cidx(i, j, k)] != BODY) continue;
            for (int dir = 0; dir < 6; ++dir) {
                const int ax = dir >> 1, sg = (dir & 1) ? -1 : 1;
                const int ni = i + (ax == 0) * sg, nj = j + (ax == 1) * sg, nk = k + (ax == 2) * sg;
                if (ni < 0 || ni >= W || nj < 0 || nj >= H || nk < 0 || nk >= D) continue;
                if (labels[cidx(ni, nj, nk)] != FLUID) continue;
                const float nx = ax == 0 ? float(sg) : 0.0f, ny = ax == 1 ? float(sg) : 0.0f, nz = ax == 2 ? float(sg) : 0.0f;
                const float fcx = (float(i) + 0.5f) * fdx + (nx * 0.5f) * fdx;
                const float fcy = (float(j) + 0.5f) * fdx + (ny * 0.5f) * fdx;
                const float fcz = (float(k) + 0.5f) * fdx + (nz * 0.5f) * fdx;
                const float rx = fcx - cmx, ry = fcy - cmy, rz = fcz - cmz;
                const V3<R> up = interp_vel(mk(R(fcx), R(fcy), R(fcz)));
                const float urx = bvx - float(up.x), ury = bvy - float(up.y), urz = bvz - float(up.z);
                const float ua = std::sqrt((urx * urx + ury * ury) + urz * urz);
                const float area = fdx * fdx;
                float A = 0.0f;
                const float nu = (nx * urx + ny * ury) + nz * urz;
                if (nu > 0.0f) A = (nu / ua * 0.5f + (1.0f - 0.5f)) * area;
                const float sd = float(-0.5 * double(rho) * double(0.1f) * double(A) * double(ua));
                const float fdx_ = urx * sd, fdy = ury * sd, fdz = urz * sd;
                float cx, cy, cz;
                cross(nx, ny, nz, urx, ury, urz, cx, cy, cz);
                const float cxa = std::sqrt((cx * cx + cy * cy) + cz * cz);
                float lx, ly, lz;
                cross(urx, ury, urz, cx / cxa, cy / cxa, cz / cxa, lx, ly, lz);
                const float sl = (((-0.5f * rho) * 0.1f) * A) * ua;
                const float flx = lx * sl, fly = ly * sl, flz = lz * sl;
                float t1x, t1y, t1z, t2x, t2y, t2z;
                cross(rx, ry, rz, fdx_, fdy, fdz, t1x, t1y, t1z);
                cross(rx, ry, rz, flx, fly, flz, t2x, t2y, t2z);
                out[0] += double(fdx_ + flx); out[1] += double(fdy + fly); out[2] += double(fdz + flz);
                out[3] += double(t1x + t2x); out[4] += double(t1y + t2y); out[5] += double(t1z + t2z);
            }
        }
        // buoyancy voxels: sphere on a grid of spacing dx/2 centred on the centre of mass
        const float cs = 0.5f * fdx;
        const int n = int(std::ceil(2.0 * (ob.radius + 2.0 * cs) / cs));
        const float o = -0.5f * float(n) * cs, r = float(ob.radius);
        float Rf[9];
        for (int m = 0; m < 9; ++m) Rf[m] = float(ob.Rm[m]);
        std::vector<std::vector<int>> bins(nc());
        for (size_t q = 0; q < np(); ++q) {
            int i, j, k;
            cell_of(px[q], py[q], pz[q], i, j, k);
            bins[cidx(i, j, k)].push_back(int(q));
        }
        const float rad = 2.0f * fdx;
        for (int k = 0; k < n; ++k) for (int j = 0; j < n; ++j) for (int i = 0; i < n; ++i) {
            const float plx = o + float(i) * cs, ply = o + float(j) * cs, plz = o + float(k) * cs;
            const float sdf = std::sqrt((plx * plx + ply * ply) + plz * plz) - r;
            if (sdf > 0.0f) continue;
            const float vx = cmx + ((Rf[0] * plx + Rf[1] * ply) + Rf[2] * plz);
            const float vy = cmy + ((Rf[3] * plx + Rf[4] * ply) + Rf[5] * plz);
            const float vz = cmz + ((Rf[6] * plx + Rf[7] * ply) + Rf[8] * plz);
            float vol = (cs * cs) * cs;
            if (sdf > -cs) vol = vol * (0.5f - (0.5f * sdf) / cs);
            out[6] += double(vol);
            const int ii = std::min(std::max(int(vx / fdx), 0), W - 1), jj = std::min(std::max(int(vy / fdx), 0), H - 1),
                      kk = std::min(std::max(int(vz / fdx), 0), D - 1);
            bool sub = labels[cidx(ii, jj, kk)] == FLUID;
            for (int q : bins[cidx(ii, jj, kk)]) {
                if (sub) break;
                const float ex = float(px[q]) - vx, ey = float(py[q]) - vy, ez = float(pz[q]) - vz;
                sub = std::sqrt((ex * ex + ey * ey) + ez * ez) < rad;
            }
            if (sub) out[7] += double(vol);
        }
    }

    // updateBody (:2793-2846) with the pressure-integral force.
    void body_phase() {
        if (!ob.loaded) return;
        if (ref_forces && !ob.paddle) {
            ref_body_forces(ref_out);
            const double g[3] = {0.0, double(-9.81f), 0.0};
            const double buoy = 1000.0 * ref_out[7] * double(9.81f);
            for (int a = 0; a < 3; ++a) {
                ob.force[a] = ob.mass * g[a] + ref_out[a] + (a == 1 ? buoy : 0.0);
                ob.torque[a] = ref_out[3 + a];
            }
            ob.integrate(double(float(dt)));
            sync_body_kin();
            return;
        }
        double f[6];
        body_force(f);
        const double g[3] = {0.0, double(-9.81f), 0.0};
        for (int a = 0; a < 3; ++a) { ob.force[a] = ob.mass * g[a] + f[a]; ob.torque[a] = f[3 + a]; }
        if (ob.paddle) {
            for (int a = 0; a < 3; ++a) ob.force[a] = f[a];
            ob.pad_t += double(float(dt));
            ob.paddle_at(ob.pad_t);
        } else {
            ob.integrate(double(float(dt)));
        }
        sync_body_kin();
    }
    void sync_body_kin() {
        body.vel = {R(float(ob.vel[0])), R(float(ob.vel[1])), R(float(ob.vel[2]))};
        body.omega = {R(float(ob.omega[0])), R(float(ob.omega[1])), R(float(ob.omega[2]))};
        body.com = {R(float(ob.pos[0])), R(float(ob.pos[1])), R(float(ob.pos[2]))};
    }

    // Velocity extrapolation into faces with no FLUID side (the wavefront
    // scheme of FluidSolver2D.cu:1207-1295 on the 26-neighbourhood), extrap layers.
    void extrapolate(std::vector<R>& g, int axis) const {
        const int nx = W + (axis == 0), ny = H + (axis == 1), nz = D + (axis == 2);
        auto id = [&](int i, int j, int k) { return size_t(i) + size_t(j) * nx + size_t(k) * nx * ny; };
        auto lab_or_solid = [&](int i, int j, int k) -> uint8_t {
            return (i < 0 || i >= W || j < 0 || j >= H || k < 0 || k >= D) ? SOLID : labels[cidx(i, j, k)];
        };
        std::vector<int> d(size_t(nx) * ny * nz);
        for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
            const uint8_t a = lab_or_solid(i, j, k);
            const uint8_t b = lab_or_solid(i - (axis == 0), j - (axis == 1), k - (axis == 2));
            d[id(i, j, k)] = (a == FLUID || b == FLUID) ? 0 : INT32_MAX;
        }
        auto for_nb = [&](int i, int j, int k, auto f) {
            for (int ox = -1; ox <= 1; ++ox) for (int oy = 1; oy >= -1; --oy) for (int oz = -1; oz <= 1; ++oz) {
                if (ox == 0 && oy == 0 && oz == 0) continue;
                const int a = i + ox, b = j + oy, e = k + oz;
                if (a < 0 || a >= nx || b < 0 || b >= ny || e < 0 || e >= nz) continue;
                f(a, b, e);
            }
        };
        for (int wave = 1; wave <= extrap; ++wave) {
            std::vector<size_t> front;
            for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
                if (d[id(i, j, k)] != INT32_MAX) continue;
                bool adj = false;
                for_nb(i, j, k, [&](int a, int b, int e) { adj = adj || d[id(a, b, e)] == wave - 1; });
                if (adj) front.push_back(id(i, j, k));
            }
            for (size_t c : front) d[c] = wave;
            for (size_t c : front) {
                const int i = int(c % nx), j = int((c / nx) % ny), k = int(c / (size_t(nx) * ny));
                R avg = R(0);
                int used = 0;
                for_nb(i, j, k, [&](int a, int b, int e) {
                    if (d[id(a, b, e)] < wave) { avg = R(avg + g[id(a, b, e)]); ++used; }
                });
                g[c] = R(avg / R(used));
            }
        }
    }

    // frameStep (:3030-3098).
    int phase(int ph) {
        switch (ph) {
            case 0: label_grid(); return 0;
            case 1: p2g(); return 0;
            case 2: save(); return 0;
            case 3: forces(); return 0;
            case 4: return pressure();
            case 5: project(); return 0;
            case 6: body_phase(); return 0;
            case 7: g2p(); return 0;
            case 8:
                if (extrap > 0) { extrapolate(u, 0); extrapolate(v, 1); if (D > 1) extrapolate(w, 2); }
                advect();
                return 0;
        }
        return -99;
    }
    int step() {
        int rc = 0;
        for (int ph = 0; ph <= 8; ++ph) { int r = phase(ph); if (ph == 4) rc = r; }
        return rc;
    }
};

struct Handle {
    int fp64;
    Sim3<float> s32;
    Sim3<double> s64;
};

template <class F> auto with(Handle* h, F f) { return h->fp64 ? f(h->s64) : f(h->s32); }

}  // namespace

extern "C" {

// ---------------------------------------------------------------- label files
// 3D reader (FluidSolver3D.cu:81-153): header "W H D", then W*H*D S/F/A chars in
// fully reversed order (k = D-1..0, j = H-1..0, i = W-1..0).
int or_read_labels3d(const char* path, int* dims, uint8_t* out) {
    std::ifstream f(path);
    if (!f) return -1;
    int W, H, D;
    if (!(f >> W >> H >> D) || W <= 0 || H <= 0 || D <= 0) return -2;
    dims[0] = W; dims[1] = H; dims[2] = D;
    if (!out) return 0;
    for (int k = D - 1; k >= 0; --k) for (int j = H - 1; j >= 0; --j) for (int i = W - 1; i >= 0; --i) {
        char c;
        if (!(f >> c)) return -3;
        uint8_t l = c == 'S' ? SOLID : c == 'F' ? FLUID : c == 'A' ? AIR : 255;
        if (l == 255) return -4;
        out[size_t(i) + size_t(j) * W + size_t(k) * W * H] = l;
    }
    return 0;
}

// 2D reader (FluidSolver2D.cu:52-104): "W H", then rows from top (j = H-1) to
// bottom, columns ascending.
int or_read_labels2d(const char* path, int* dims, uint8_t* out) {
    std::ifstream f(path);
    if (!f) return -1;
    int W, H;
    if (!(f >> W >> H) || W <= 0 || H <= 0) return -2;
    dims[0] = W; dims[1] = H;
    if (!out) return 0;
    for (int j = H - 1; j >= 0; --j) for (int i = 0; i < W; ++i) {
        char c;
        if (!(f >> c)) return -3;
        uint8_t l = c == 'S' ? SOLID : c == 'F' ? FLUID : c == 'A' ? AIR : 255;
        if (l == 255) return -4;
        out[size_t(i) + size_t(j) * W] = l;
    }
    return 0;
}

// ---------------------------------------------------------------- seeding
// seedParticles (FluidSolver3D.cu:213-297) with a caller-chosen mt19937 seed in
// place of std::random_device.  Returns the particle count; pos may be null.
int64_t or_seed3d(const uint8_t* labels, int W, int H, int D, float dx, int ppc, uint32_t seed, float* pos) {
    std::mt19937 gen(seed);
    std::uniform_int_distribution<> sub(0, 7);
    std::uniform_real_distribution<> jit(-0.24f, 0.24f);
    int64_t n = 0;
    for (int k = 0; k < D; ++k) for (int j = 0; j < H; ++j) for (int i = 0; i < W; ++i) {
        if (labels[size_t(i) + size_t(j) * W + size_t(k) * W * H] != FLUID) continue;
        float cx = (i + 0.5f) * dx, cy = (j + 0.5f) * dx, cz = (k + 0.5f) * dx;
        const float o = 0.25f * dx;
        for (int q = 0; q < ppc; ++q) {
            int s = sub(gen);
            float jx = float(jit(gen) * dx), jy = float(jit(gen) * dx), jz = float(jit(gen) * dx);
            float x = (cx + ((s & 1) ? o : -o)) + jx;
            float y = (cy + ((s & 2) ? o : -o)) + jy;
            float z = (cz + ((s & 4) ? o : -o)) + jz;
            x = std::clamp(x, i * dx, (i + 1) * dx);
            y = std::clamp(y, j * dx, (j + 1) * dx);
            z = std::clamp(z, k * dx, (k + 1) * dx);
            if (pos) { pos[3 * n] = x; pos[3 * n + 1] = y; pos[3 * n + 2] = z; }
            ++n;
        }
    }
    return n;
}

// 2D seeding (FluidSolver2D.cu:114-158): quadrant centres (top-left,
// top-right, bottom-right, bottom-left), jitter U(-0.24, 0.24)*dx, clamped to
// the cell; z = 0.  pos (n x 3) may be null.
int64_t or_seed2d(const uint8_t* labels, int W, int H, float dx, int ppc, uint32_t seed, float* pos) {
    std::mt19937 gen(seed);
    std::uniform_int_distribution<> sub(0, 3);
    std::uniform_real_distribution<> jit(-0.24f, 0.24f);
    int64_t n = 0;
    for (int j = 0; j < H; ++j) for (int i = 0; i < W; ++i) {
        if (labels[size_t(i) + size_t(j) * W] != FLUID) continue;
        const float cx = (i + 0.5f) * dx, cy = (j + 0.5f) * dx;
        const float sc[4][2] = {{cx - 0.25f * dx, cy + 0.25f * dx}, {cx + 0.25f * dx, cy + 0.25f * dx},
                                {cx + 0.25f * dx, cy - 0.25f * dx}, {cx - 0.25f * dx, cy - 0.25f * dx}};
        for (int q = 0; q < ppc; ++q) {
            const int s = sub(gen);
            const float jx = float(jit(gen) * dx), jy = float(jit(gen) * dx);
            float x = sc[s][0] + jx, y = sc[s][1] + jy;
            if (pos) {
                pos[3 * n] = std::clamp(x, cx - 0.5f * dx, cx + 0.5f * dx);
                pos[3 * n + 1] = std::clamp(y, cy - 0.5f * dx, cy + 0.5f * dx);
                pos[3 * n + 2] = 0.0f;
            }
            ++n;
        }
    }
    return n;
}

// ---------------------------------------------------------------- binning
// Cell key of every particle (MarkFluidCellsFunctor, :316-331) and the per-cell
// counts; the integer results the GPU sort must reproduce bit for bit.
void or_bin3d(const float* pos, int64_t n, int W, int H, int D, float dx, int32_t* keys, int32_t* counts) {
    if (counts) std::memset(counts, 0, sizeof(int32_t) * size_t(W) * H * D);
    for (int64_t q = 0; q < n; ++q) {
        int i = int(std::floor(pos[3 * q] / dx)), j = int(std::floor(pos[3 * q + 1] / dx)), k = int(std::floor(pos[3 * q + 2] / dx));
        i = std::min(std::max(i, 0), W - 1); j = std::min(std::max(j, 0), H - 1); k = std::min(std::max(k, 0), D - 1);
        int32_t key = int32_t(i + j * W + k * W * H);
        if (keys) keys[q] = key;
        if (counts) counts[key]++;
    }
}

// ---------------------------------------------------------------- CSR operator
// MatrixBuilder3D + exclusive scan + MatrixFiller3D (:1598-1777), upper triangle
// with fluid renumbering by exclusive scan (:1820-1853).  Two-call pattern:
// first with null outputs to get n and nnz.
int or_build_csr_upper(const uint8_t* labels, int W, int H, int D, int* n_out, int* nnz_out,
                       int* offsets, int* cols, float* vals) {
    size_t nc = size_t(W) * H * D;
    std::vector<int> num(nc, -1);
    int nf = 0;
    for (size_t c = 0; c < nc; ++c) if (labels[c] == FLUID) num[c] = nf++;
    const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    int nnz = 0;
    for (int k = 0; k < D; ++k) for (int j = 0; j < H; ++j) for (int i = 0; i < W; ++i) {
        size_t c = size_t(i) + size_t(j) * W + size_t(k) * W * H;
        if (labels[c] != FLUID) continue;
        int row = num[c];
        if (offsets) offsets[row] = nnz;
        int pos = nnz++;
        float diag = 0.0f;
        if (cols) cols[pos] = row;
        for (auto& o : off) {
            int a = i + o[0], b = j + o[1], e = k + o[2];
            if (a < 0 || a >= W || b < 0 || b >= H || e < 0 || e >= D) continue;
            size_t nb = size_t(a) + size_t(b) * W + size_t(e) * W * H;
            if (labels[nb] == FLUID) {
                if (num[nb] > row) { if (cols) { cols[nnz] = num[nb]; vals[nnz] = -1.0f; } ++nnz; }
                diag += 1.0f;
            } else if (labels[nb] == AIR) diag += 1.0f;
        }
        if (vals) vals[pos] = diag;
    }
    if (offsets) offsets[nf] = nnz;
    *n_out = nf; *nnz_out = nnz;
    return 0;
}

// FP64 CG on a symmetric matrix given by its upper-triangle CSR (the storage of
// CUDSS_MVIEW_UPPER, :1932-1945).  Returns iterations; x in/out (zero start).
int or_cg_csr_upper(int n, const int* offsets, const int* cols, const double* vals, const double* b, double* x,
                    double tol, int maxit, double* relres) {
    std::vector<double> r(n), d(n), q(n), dg(n, 1.0);
    auto apply = [&](const double* in, double* out) {
        for (int i = 0; i < n; ++i) out[i] = 0.0;
        for (int i = 0; i < n; ++i)
            for (int e = offsets[i]; e < offsets[i + 1]; ++e) {
                int c = cols[e];
                out[i] += vals[e] * in[c];
                if (c != i) out[c] += vals[e] * in[i];
            }
    };
    for (int i = 0; i < n; ++i)
        for (int e = offsets[i]; e < offsets[i + 1]; ++e) if (cols[e] == i) dg[i] = vals[e];
    for (int i = 0; i < n; ++i) x[i] = 0.0;
    double bn = 0; for (int i = 0; i < n; ++i) bn += b[i] * b[i];
    bn = std::sqrt(bn);
    for (int i = 0; i < n; ++i) { r[i] = b[i]; d[i] = r[i] / dg[i]; }
    double rz = 0; for (int i = 0; i < n; ++i) rz += r[i] * r[i] / dg[i];
    int it = 0;
    double rn = bn;
    while (bn > 0 && rn / bn > tol && it < maxit) {
        apply(d.data(), q.data());
        double dq = 0; for (int i = 0; i < n; ++i) dq += d[i] * q[i];
        double a = rz / dq;
        for (int i = 0; i < n; ++i) { x[i] += a * d[i]; r[i] -= a * q[i]; }
        double rz2 = 0; for (int i = 0; i < n; ++i) rz2 += r[i] * r[i] / dg[i];
        double be = rz2 / rz; rz = rz2;
        for (int i = 0; i < n; ++i) d[i] = r[i] / dg[i] + be * d[i];
        rn = 0; for (int i = 0; i < n; ++i) rn += r[i] * r[i];
        rn = std::sqrt(rn);
        ++it;
    }
    if (relres) *relres = bn > 0 ? rn / bn : 0.0;
    return it;
}

// ---------------------------------------------------------------- 3D simulation
void* or3_create(int W, int H, int D, double dx, double dt, int fp64) {
    auto* h = new Handle();
    h->fp64 = fp64;
    auto init = [&](auto& s) {
        using R = std::decay_t<decltype(s.dx)>;
        s.W = W; s.H = H; s.D = D; s.dx = R(float(dx)); s.dt = R(float(dt));
        s.alloc();
        return 0;
    };
    with(h, init);
    return h;
}
void or3_destroy(void* p) { delete static_cast<Handle*>(p); }

void or3_set_params(void* p, double pic_weight, double cfl, double tol, int maxit) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        using R = std::decay_t<decltype(s.dx)>;
        s.alpha = R(float(pic_weight)); s.cfl = R(float(cfl)); s.tol = tol; s.maxit = maxit; return 0;
    });
}
void or3_set_ref_forces(void* p, int on) {
    with(static_cast<Handle*>(p), [&](auto& s) { s.ref_forces = on; return 0; });
}
void or3_ref_forces(void* p, double* out) {  // out[8]: of the last body phase
    with(static_cast<Handle*>(p), [&](auto& s) { for (int m = 0; m < 8; ++m) out[m] = s.ref_out[m]; return 0; });
}
void or3_set_extrap(void* p, int layers) {
    with(static_cast<Handle*>(p), [&](auto& s) { s.extrap = layers; return 0; });
}
void or3_set_rk2(void* p, int rk2) {
    with(static_cast<Handle*>(p), [&](auto& s) { s.rk2 = rk2; return 0; });
}
void or3_set_collision(void* p, int sdf) {
    with(static_cast<Handle*>(p), [&](auto& s) { s.sdf_collide = sdf; return 0; });
}
void or3_set_body(void* p, const double* vel, const double* omega, const double* com) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        using R = std::decay_t<decltype(s.dx)>;
        s.body.vel = {R(float(vel[0])), R(float(vel[1])), R(float(vel[2]))};
        s.body.omega = {R(float(omega[0])), R(float(omega[1])), R(float(omega[2]))};
        s.body.com = {R(float(com[0])), R(float(com[1])), R(float(com[2]))};
        if (s.ob.loaded)  // the loaded body's own state too (fp_set_body_state)
            for (int a = 0; a < 3; ++a) { s.ob.vel[a] = vel[a]; s.ob.omega[a] = omega[a]; s.ob.pos[a] = com[a]; }
        return 0;
    });
}
void or3_set_labels(void* p, const uint8_t* l) {
    with(static_cast<Handle*>(p), [&](auto& s) { std::memcpy(s.labels.data(), l, s.nc()); return 0; });
}
void or3_get_labels(void* p, uint8_t* l) {
    with(static_cast<Handle*>(p), [&](auto& s) { std::memcpy(l, s.labels.data(), s.nc()); return 0; });
}
void or3_set_particles(void* p, int64_t n, const float* pos, const float* vel) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        s.px.resize(n); s.py.resize(n); s.pz.resize(n); s.vx.resize(n); s.vy.resize(n); s.vz.resize(n);
        for (int64_t q = 0; q < n; ++q) {
            s.px[q] = pos[3 * q]; s.py[q] = pos[3 * q + 1]; s.pz[q] = pos[3 * q + 2];
            s.vx[q] = vel ? vel[3 * q] : 0; s.vy[q] = vel ? vel[3 * q + 1] : 0; s.vz[q] = vel ? vel[3 * q + 2] : 0;
        }
        return 0;
    });
}
int64_t or3_num_particles(void* p) {
    return with(static_cast<Handle*>(p), [&](auto& s) { return int64_t(s.np()); });
}
void or3_get_particles(void* p, double* pos, double* vel) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        for (size_t q = 0; q < s.np(); ++q) {
            if (pos) { pos[3 * q] = s.px[q]; pos[3 * q + 1] = s.py[q]; pos[3 * q + 2] = s.pz[q]; }
            if (vel) { vel[3 * q] = s.vx[q]; vel[3 * q + 1] = s.vy[q]; vel[3 * q + 2] = s.vz[q]; }
        }
        return 0;
    });
}
// which: 0 u, 1 v, 2 w, 3 u*, 4 v*, 5 w*, 6 p
static int64_t grid_len(int which, int W, int H, int D) {
    switch (which) {
        case 0: case 3: return int64_t(W + 1) * H * D;
        case 1: case 4: return int64_t(W) * (H + 1) * D;
        case 2: case 5: return int64_t(W) * H * (D + 1);
        case 6: return int64_t(W) * H * D;
    }
    return -1;
}
int64_t or3_grid_len(void* p, int which) {
    return with(static_cast<Handle*>(p), [&](auto& s) { return grid_len(which, s.W, s.H, s.D); });
}
int or3_grid_io(void* p, int which, double* buf, int set) {
    return with(static_cast<Handle*>(p), [&](auto& s) {
        using R = std::decay_t<decltype(s.dx)>;
        std::vector<R>* g[7] = {&s.u, &s.v, &s.w, &s.us, &s.vs, &s.ws, &s.p};
        if (which < 0 || which > 6) return -1;
        auto& a = *g[which];
        for (size_t i = 0; i < a.size(); ++i) { if (set) a[i] = R(buf[i]); else buf[i] = double(a[i]); }
        return 0;
    });
}
// Analytic sphere body (radius r, mass m) at pos, at rest.
void or3_set_sphere(void* p, const double* pos, double r, double m) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        s.ob = OBody();
        s.ob.loaded = true;
        for (int a = 0; a < 3; ++a) s.ob.pos[a] = pos[a];
        s.ob.radius = r; s.ob.mass = m; s.ob.inertia = 0.4 * m * r * r;
        s.ob.update_rotation();
        s.sync_body_kin();
        return 0;
    });
}
// Wave paddle (fp_set_paddle): BODY where x < x0 + amp sin(2 pi t / period).
void or3_set_paddle(void* p, double x0, double amp, double period) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        s.ob = OBody();
        s.ob.loaded = true;
        s.ob.paddle = true;
        s.ob.pad_x0 = double(float(x0)); s.ob.pad_amp = double(float(amp)); s.ob.pad_period = double(float(period));
        s.ob.pos[1] = 0.5 * s.H * double(float(s.dx)); s.ob.pos[2] = 0.5 * s.D * double(float(s.dx));
        s.ob.paddle_at(0.0);
        s.sync_body_kin();
        return 0;
    });
}
// out: pos[3] vel[3] omega[3] angles[3] force[3] torque[3]
void or3_body_state(void* p, double* out) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        const OBody& b = s.ob;
        for (int a = 0; a < 3; ++a) {
            out[a] = b.pos[a]; out[3 + a] = b.vel[a]; out[6 + a] = b.omega[a];
            out[12 + a] = b.force[a]; out[15 + a] = b.torque[a];
        }
        out[9] = b.theta; out[10] = b.psi; out[11] = b.phi;
        return 0;
    });
}
void or3_body_force(void* p, double* out) {
    with(static_cast<Handle*>(p), [&](auto& s) { s.body_force(out); return 0; });
}

int or3_phase(void* p, int ph) { return with(static_cast<Handle*>(p), [&](auto& s) { return s.phase(ph); }); }
int or3_step(void* p, int n) {
    return with(static_cast<Handle*>(p), [&](auto& s) { int rc = 0; for (int i = 0; i < n; ++i) rc = s.step(); return rc; });
}
// RHS of the pressure system on the dense grid (0 at non-fluid cells).
void or3_rhs(void* p, double* out) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        for (int k = 0; k < s.D; ++k) for (int j = 0; j < s.H; ++j) for (int i = 0; i < s.W; ++i) {
            size_t c = s.cidx(i, j, k);
            out[c] = s.labels[c] == FLUID ? double(s.rhs_at(i, j, k)) : 0.0;
        }
        return 0;
    });
}
// Solve the unit Poisson operator of the current labels for a dense rhs.
int or3_solve(void* p, const double* b, double* x) {
    return with(static_cast<Handle*>(p), [&](auto& s) {
        std::vector<double> bb(b, b + s.nc()), xx;
        int it = s.solve(bb, xx);
        std::memcpy(x, xx.data(), sizeof(double) * s.nc());
        s.last_iters = it;
        return it;
    });
}
// Apply the unit Poisson operator (FP64) to a dense vector.
void or3_apply(void* p, const double* in, double* out) {
    with(static_cast<Handle*>(p), [&](auto& s) {
        const int W = s.W, H = s.H, D = s.D;
        for (int k = 0; k < D; ++k) for (int j = 0; j < H; ++j) for (int i = 0; i < W; ++i) {
            size_t c = s.cidx(i, j, k);
            if (s.labels[c] != FLUID) { out[c] = 0; continue; }
            double acc = double(s.diag_at(i, j, k)) * in[c];
            const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
            for (auto& o : off) {
                int a = i + o[0], b2 = j + o[1], e = k + o[2];
                if (s.lab(a, b2, e) == FLUID) acc -= in[s.cidx(a, b2, e)];
            }
            out[c] = acc;
        }
        return 0;
    });
}
void or3_stats(void* p, double* out) {
    with(static_cast<Handle*>(p), [&](auto& s) { out[0] = s.last_iters; out[1] = s.last_res; out[2] = s.last_nf; return 0; });
}
int or_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
