// ref2d_oracle.cpp -- CPU oracle of FluidPrjct's own 2D step (FluidSolver2D).
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the CPU, the step of
// Ship-Vano/FluidPrjct's src/FluidSim/FluidSolver2D.cu so that the CUDA
// "ref2d" scheme can be checked against it.  Only tests/ may load it; the
// product library never links or calls it.
//
// The 2D reference differs from the 3D one (not a depth-1 3D step):
//   label    non-SOLID cells reset to AIR, then AIR -> FLUID under every
//            particle, cell = (int)(pos / dx) in device semantics
//            (clearLabelsKernel / markFluidCellsKernel, :168-195, :217-251);
//   P2G      u and v faces (i, j) are both weighted by the bilinear hat about
//            the CELL CENTRE ((i + 0.5) dx, (j + 0.5) dx), summed particle by
//            particle in particle order; a face with zero weight becomes 0
//            (accumulateDenAndNum / applyNumDen / particlesToGrid, :259-338);
//   save     u* = u (:340-354);
//   forces   gravity on every face not equal to VEL_UNKNOWN (:362-381);
//   pressure the 5-point system of FLUID cells (diagonal = FLUID or AIR
//            neighbours, -1 to FLUID neighbours; RHS = -(rho dx / dt) div u
//            with u_solid = 0 on SOLID neighbour faces), solved exactly
//            (cuDSS, :408-718) -- here FP64 CG to a relative residual tol;
//   project  faces 1..W-1 (u) and 1..H-1 (v): a FLUID side and a SOLID side
//            give 0, a FLUID side gives u -= dt/(rho dx) (p_R - p_L), no
//            FLUID side gives VEL_UNKNOWN; border faces keep their value
//            (applyPressure, :720-757);
//   G2P      1D-linear interpolation of u along x and v along y inside the
//            particle's cell (trunc(pos / dx)), VEL_UNKNOWN outside the grid;
//            v = alpha * I(u) + (v + I(u - u*)) (1 - alpha) (:792-853);
//   advect   forward Euler, substep C dx / (|v| + FLT_MIN) with C =
//            ADVECT_MAX = 1, halved near the end of dt; stop on a negative or
//            NaN position; a particle in a SOLID cell moves to the nearest
//            SOLID neighbour centre (8-neighbourhood, else AIR), or stops if
//            there is none (advectParticles / projectParticle, :1072-1166);
//   cleanup  particles outside the grid or NaN are deleted; particles in a
//            SOLID cell are projected as above or deleted; order is kept
//            (cleanUpParticles, :1171-1204).
//
// Arithmetic: FP32 in the reference's expression order, no FMA contraction
// (the Makefile passes -ffp-contract=off), IEEE division and square root; the
// FP64 mode runs the same algorithm in double.  Where the reference relies on
// undefined behaviour the restatement fixes one meaning, shared with the
// CUDA kernels:
//   - host float -> int conversion of NaN or of values outside int range
//     gives INT_MIN (the x86 result);
//   - a label read at a flat index outside the grid (advection of a particle
//     past the right or top border) reads as "not SOLID";
//   - the substep loop of one particle stops after kMaxSubsteps substeps
//     (the reference loop has no bound); such particles are counted.
// std::hypot(float, float) is taken as the correctly rounded float of the
// exact distance, (float)sqrt((double)a * a + (double)b * b).

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr uint8_t SOLID = 0, FLUID = 1, AIR = 2;
constexpr int kMaxSubsteps = 4096;
constexpr float kVelUnknown = float(INT_MIN);  // utility.cuh:56, stored in float grids

// (int)x on the host (trunc toward zero; INT_MIN when undefined).
inline int host_trunc(double t) {
    if (std::isnan(t) || t >= 2147483648.0 || t < -2147483648.0) return INT_MIN;
    return int(t);
}
// (int)x on the device (cvt.rzi.s32: NaN -> 0, saturating).
inline int dev_trunc(double t) {
    if (std::isnan(t)) return 0;
    if (t >= 2147483647.0) return INT_MAX;
    if (t <= -2147483648.0) return INT_MIN;
    return int(t);
}

template <class R>
struct Ref2D {
    int W = 0, H = 0;
    R dx = 0, dt = 0, alpha = R(0.5f);
    double tol = 1e-12;
    int maxit = 100000;
    std::vector<uint8_t> labels;
    std::vector<R> u, v, us, vs, p;
    std::vector<R> px, py, vx, vy;
    int nf = 0, cg_iters = 0, capped = 0;
    bool extrap = false;  // the step's commented-out extrapolateGridFluidData calls (:1309-1310, :1325-1326)
    int64_t removed = 0;

    int64_t nu() const { return int64_t(W + 1) * H; }
    int64_t nv() const { return int64_t(W) * (H + 1); }
    size_t np() const { return px.size(); }

    void alloc() {
        labels.assign(size_t(W) * H, AIR);
        u.assign(nu(), R(kVelUnknown)); us = u;
        v.assign(nv(), R(kVelUnknown)); vs = v;
        p.assign(size_t(W) * H, R(0));
    }
    uint8_t lab(int i, int j) const { return labels[size_t(i) + size_t(j) * W]; }
    // label at the reference's flat index i + j * W, "not SOLID" outside the array
    bool solid_flat(int i, int j) const {
        const int64_t f = int64_t(i) + int64_t(j) * W;
        return f >= 0 && f < int64_t(W) * H && labels[size_t(f)] == SOLID;
    }

    // ---- labelGrid_gpu, :217-251
    void label() {
        for (auto& l : labels) if (l != SOLID) l = AIR;
        for (size_t q = 0; q < np(); ++q) {
            const int ci = dev_trunc(double(R(px[q] / dx))), cj = dev_trunc(double(R(py[q] / dx)));
            if (ci >= 0 && ci < W && cj >= 0 && cj < H && lab(ci, cj) == AIR) labels[size_t(ci) + size_t(cj) * W] = FLUID;
        }
    }

    // ---- hatFunction / bilinearHatKernel, utility.cu:142-153
    static R hat(R r) {
        const R a = std::fabs(r);
        return double(R(a - R(1))) <= 1e-8 ? R(R(1) - a) : R(0);
    }
    // ---- particlesToGrid, :290-338.  Every particle is added to every face in
    // particle order, as the reference's one-launch-per-particle loop does.
    void p2g() {
        std::vector<R> un(nu(), R(0)), ud(nu(), R(0)), vn(nv(), R(0)), vd(nv(), R(0));
        for (size_t q = 0; q < np(); ++q) {
            const R x = px[q], y = py[q];
            // faces whose cell-centre hat can be nonzero: |x - c| < dx
            const int i0 = std::isfinite(double(x)) ? int(std::floor(double(x / dx))) - 1 : 0;
            const int j0 = std::isfinite(double(y)) ? int(std::floor(double(y / dx))) - 1 : 0;
            const bool fin = std::isfinite(double(x)) && std::isfinite(double(y));
            auto add = [&](int i, int j) {
                const R cx = R(R(R(i) + R(0.5f)) * dx), cy = R(R(R(j) + R(0.5f)) * dx);
                const R k = R(hat(R(R(x - cx) / dx)) * hat(R(R(y - cy) / dx)));
                if (i >= 0 && i <= W && j >= 0 && j < H) {
                    const size_t f = size_t(i) + size_t(j) * (W + 1);
                    un[f] = R(un[f] + R(vx[q] * k)); ud[f] = R(ud[f] + k);
                }
                if (i >= 0 && i < W && j >= 0 && j <= H) {
                    const size_t f = size_t(i) + size_t(j) * W;
                    vn[f] = R(vn[f] + R(vy[q] * k)); vd[f] = R(vd[f] + k);
                }
            };
            if (fin && std::isfinite(double(vx[q])) && std::isfinite(double(vy[q]))) {
                // a finite particle adds +-0 (no change) outside its 3x3 face block
                for (int j = j0; j <= j0 + 2; ++j)
                    for (int i = i0; i <= i0 + 2; ++i) add(i, j);
            } else {
                for (int j = 0; j <= H; ++j)
                    for (int i = 0; i <= W; ++i) add(i, j);
            }
        }
        for (int64_t f = 0; f < nu(); ++f) u[f] = ud[f] != R(0) ? R(un[f] / ud[f]) : R(0);
        for (int64_t f = 0; f < nv(); ++f) v[f] = vd[f] != R(0) ? R(vn[f] / vd[f]) : R(0);
    }
    // extrapolateGridFluidData, :1207-1295, in the reference's sequential form.
    // Its initial front reads neighbour markers at stride W (checkNeighbors,
    // :1049-1066) whatever the grid's own width x.
    void extrapolate(std::vector<R>& g, int x, int y, int depth) const {
        std::vector<int> d(size_t(x) * y);
        for (int j = 0; j < y; ++j)
            for (int i = 0; i < x; ++i) d[size_t(i) + size_t(j) * x] = g[size_t(i) + size_t(j) * x] != R(kVelUnknown) ? 0 : INT_MAX;
        static const int nb[8][2] = {{-1, 1}, {-1, 0}, {-1, -1}, {0, 1}, {0, -1}, {1, 1}, {1, 0}, {1, -1}};
        std::vector<std::vector<std::pair<int, int>>> fronts(1);
        for (int i = 0; i < x; ++i)
            for (int j = 0; j < y; ++j) {
                if (d[size_t(i) + size_t(j) * x] == 0) continue;
                bool known_nb = false;
                for (auto& n : nb) {
                    const int a = i + n[0], b = j + n[1];
                    if (a >= 0 && a < x && b >= 0 && b < y && d[size_t(a) + size_t(b) * W] == 0) { known_nb = true; break; }
                }
                if (known_nb) { d[size_t(i) + size_t(j) * x] = 1; fronts[0].push_back({i, j}); }
            }
        for (int cur = 0; cur < depth; ++cur) {
            std::vector<std::pair<int, int>> next;
            for (auto [i, j] : fronts[size_t(cur)]) {
                const int dc = d[size_t(i) + size_t(j) * x];
                R avg = R(0);
                int used = 0;
                for (auto& n : nb) {
                    const int a = i + n[0], b = j + n[1];
                    if (!(a >= 0 && a < x && b >= 0 && b < y)) continue;
                    int& dn = d[size_t(a) + size_t(b) * x];
                    if (dn < dc) { avg = R(avg + g[size_t(a) + size_t(b) * x]); ++used; }
                    else if (dn == INT_MAX) { dn = dc + 1; next.push_back({a, b}); }
                }
                g[size_t(i) + size_t(j) * x] = R(avg / R(used));
            }
            fronts.push_back(next);
        }
    }
    void save() { us = u; vs = v; }
    void forces() {
        const R gx = R(dt * R(0.0f)), gy = R(dt * R(-9.81f));
        for (auto& x : u) if (x != R(kVelUnknown)) x = R(x + gx);
        for (auto& x : v) if (x != R(kVelUnknown)) x = R(x + gy);
    }

    // ---- pressureSolve, :566-718 (constructRHS :408-453, constructA :460-542).
    // Out-of-grid neighbours count as SOLID (the reference reads wrapped
    // memory there; scenes with a SOLID border never reach it).
    uint8_t nb(int i, int j) const { return (i < 0 || i >= W || j < 0 || j >= H) ? SOLID : lab(i, j); }
    int pressure() {
        const R scale = R(R(R(1000.0f) * dx) / dt);
        std::vector<int> num(size_t(W) * H, -1);
        std::vector<double> b, diag;
        std::vector<int> cell;
        for (int j = 0; j < H; ++j)
            for (int i = 0; i < W; ++i) {
                if (lab(i, j) != FLUID) continue;
                num[size_t(i) + size_t(j) * W] = int(b.size());
                cell.push_back(i + j * W);
                const R u0 = u[size_t(i) + size_t(j) * (W + 1)], u1 = u[size_t(i + 1) + size_t(j) * (W + 1)];
                const R v0 = v[size_t(i) + size_t(j) * W], v1 = v[size_t(i) + size_t(j + 1) * W];
                R r = R(-scale * R(R(R(u1 - u0) + v1) - v0));
                if (nb(i - 1, j) == SOLID) r = R(r - R(scale * R(u0 - R(0.0f))));
                if (nb(i + 1, j) == SOLID) r = R(r + R(scale * R(u1 - R(0.0f))));
                if (nb(i, j - 1) == SOLID) r = R(r - R(scale * R(v0 - R(0.0f))));
                if (nb(i, j + 1) == SOLID) r = R(r + R(scale * R(v1 - R(0.0f))));
                b.push_back(double(r));
                int d = 0;
                const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
                for (auto& o : off) { const uint8_t l = nb(i + o[0], j + o[1]); d += (l == FLUID || l == AIR); }
                diag.push_back(double(d));
            }
        nf = int(b.size());
        std::fill(p.begin(), p.end(), R(0));
        cg_iters = 0;
        if (nf == 0) return -5;
        auto apply = [&](const std::vector<double>& x, std::vector<double>& y) {
            for (int n = 0; n < nf; ++n) {
                const int i = cell[n] % W, j = cell[n] / W;
                double s = diag[n] * x[n];
                const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
                for (auto& o : off) {
                    const int a = i + o[0], c = j + o[1];
                    if (a >= 0 && a < W && c >= 0 && c < H) {
                        const int m = num[size_t(a) + size_t(c) * W];
                        if (m >= 0) s -= x[m];
                    }
                }
                y[n] = s;
            }
        };
        std::vector<double> x(nf, 0.0), r(b), z(nf), d(nf), q(nf);
        double bb = 0;
        for (double t : b) bb += t * t;
        if (bb == 0) return 0;
        for (int n = 0; n < nf; ++n) z[n] = r[n] / diag[n];
        d = z;
        double rz = 0;
        for (int n = 0; n < nf; ++n) rz += r[n] * z[n];
        for (int it = 0; it < maxit; ++it) {
            apply(d, q);
            double dq = 0;
            for (int n = 0; n < nf; ++n) dq += d[n] * q[n];
            const double a = rz / dq;
            double rr = 0;
            for (int n = 0; n < nf; ++n) { x[n] += a * d[n]; r[n] -= a * q[n]; rr += r[n] * r[n]; }
            cg_iters = it + 1;
            if (rr <= tol * tol * bb) break;
            double rz2 = 0;
            for (int n = 0; n < nf; ++n) { z[n] = r[n] / diag[n]; rz2 += r[n] * z[n]; }
            const double beta = rz2 / rz;
            rz = rz2;
            for (int n = 0; n < nf; ++n) d[n] = z[n] + beta * d[n];
        }
        for (int n = 0; n < nf; ++n) p[size_t(cell[n])] = R(x[n]);
        return 0;
    }

    // ---- applyPressure, :720-757
    void project() {
        const R scale = R(dt / R(R(1000.0f) * dx));
        for (int j = 0; j < H; ++j)
            for (int i = 0; i < W; ++i) {
                if (i >= 1) {
                    const uint8_t L = lab(i - 1, j), Rr = lab(i, j);
                    R& f = u[size_t(i) + size_t(j) * (W + 1)];
                    if (L == FLUID || Rr == FLUID) {
                        if (L == SOLID || Rr == SOLID) f = R(0.0f);
                        else f = R(f - R(scale * R(p[size_t(i) + size_t(j) * W] - p[size_t(i - 1) + size_t(j) * W])));
                    } else {
                        f = R(kVelUnknown);
                    }
                }
                if (j >= 1) {
                    const uint8_t B = lab(i, j - 1), T = lab(i, j);
                    R& f = v[size_t(i) + size_t(j) * W];
                    if (B == FLUID || T == FLUID) {
                        if (B == SOLID || T == SOLID) f = R(0.0f);
                        else f = R(f - R(scale * R(p[size_t(i) + size_t(j) * W] - p[size_t(i) + size_t(j - 1) * W])));
                    } else {
                        f = R(kVelUnknown);
                    }
                }
            }
    }

    // ---- interpVel, :792-820; delta = 1 interpolates u - u*, v - v*
    void interp(R x, R y, bool delta, R& ou, R& ov) const {
        const int i = host_trunc(double(R(x / dx))), j = host_trunc(double(R(y / dx)));
        if (!(i >= 0 && i < W && j >= 0 && j < H)) { ou = ov = R(kVelUnknown); return; }
        const R cx = R(R(R(i) + R(0.5f)) * dx), cy = R(R(R(j) + R(0.5f)) * dx);
        const R off = R(dx / R(2.0f));
        const R x1 = R(cx - off), x2 = R(cx + off), y1 = R(cy - off), y2 = R(cy + off);
        auto U = [&](size_t f) { return delta ? R(u[f] - us[f]) : u[f]; };
        auto Vv = [&](size_t f) { return delta ? R(v[f] - vs[f]) : v[f]; };
        const R u1 = U(size_t(i) + size_t(j) * (W + 1)), u2 = U(size_t(i + 1) + size_t(j) * (W + 1));
        const R v1 = Vv(size_t(i) + size_t(j) * W), v2 = Vv(size_t(i) + size_t(j + 1) * W);
        ou = R(R(R(R(x2 - x) / R(x2 - x1)) * u1) + R(R(R(x - x1) / R(x2 - x1)) * u2));
        ov = R(R(R(R(y2 - y) / R(y2 - y1)) * v1) + R(R(R(y - y1) / R(y2 - y1)) * v2));
    }
    void g2p() {
        const R a = alpha, b = R(R(1.0f) - alpha);
        for (size_t q = 0; q < np(); ++q) {
            R pu, pv, fu, fv;
            interp(px[q], py[q], false, pu, pv);
            interp(px[q], py[q], true, fu, fv);
            vx[q] = R(R(pu * a) + R(R(vx[q] + fu) * b));
            vy[q] = R(R(pv * a) + R(R(vy[q] + fv) * b));
        }
    }

    // ---- projectParticle, :1072-1119
    bool project_particle(R& x, R& y) const {
        static const int nbr[8][2] = {{-1, 1}, {-1, 0}, {-1, -1}, {0, 1}, {0, -1}, {1, 1}, {1, 0}, {1, -1}};
        const int ci = host_trunc(double(R(x / dx))), cj = host_trunc(double(R(y / dx)));
        for (int pass = 0; pass < 2; ++pass) {
            const uint8_t want = pass == 0 ? SOLID : AIR;
            bool any = false;
            R best = R(FLT_MAX), nx = x, ny = y;
            for (auto& n : nbr) {
                const int64_t a = int64_t(ci) + n[0], c = int64_t(cj) + n[1];
                if (!(a >= 0 && a < W && c >= 0 && c < H) || lab(int(a), int(c)) != want) continue;
                any = true;
                const R cx = R(R(R(float(a)) + R(0.5f)) * dx), cy = R(R(R(float(c)) + R(0.5f)) * dx);
                const R ex = R(cx - x), ey = R(cy - y);
                const R dist = R(float(std::sqrt(double(ex) * double(ex) + double(ey) * double(ey))));
                if (dist < best) { best = dist; nx = cx; ny = cy; }
            }
            if (any) {
                x = R(x + R(R(1.0f) * R(nx - x)));
                y = R(y + R(R(1.0f) * R(ny - y)));
                return true;
            }
        }
        return false;
    }

    // ---- advectParticles(ADVECT_MAX = 1), :1122-1166
    void advect() {
        capped = 0;
        const R C = R(1.0f);
        for (size_t q = 0; q < np(); ++q) {
            R x = px[q], y = py[q], sub = R(0.0f);
            bool finished = false;
            int n = 0;
            while (!finished) {
                if (n++ == kMaxSubsteps) { ++capped; break; }
                R cu, cv;
                interp(x, y, false, cu, cv);
                R dT = R(R(C * dx) / R(R(std::sqrt(R(R(cu * cu) + R(cv * cv)))) + R(FLT_MIN)));
                if (R(sub + dT) >= dt) { dT = R(dt - sub); finished = true; }
                else if (R(sub + R(R(2.0f) * dT)) >= dt) dT = R(R(0.5f) * R(dt - sub));
                x = R(x + R(cu * dT));
                y = R(y + R(cv * dT));
                sub = R(sub + dT);
                if (x < R(0) || y < R(0) || std::isnan(double(x)) || std::isnan(double(y))) break;
                const int ci = host_trunc(double(R(x / dx))), cj = host_trunc(double(R(y / dx)));
                if (solid_flat(ci, cj) && !project_particle(x, y)) break;
            }
            px[q] = x; py[q] = y;
        }
    }

    // ---- cleanUpParticles, :1171-1204
    void cleanup() {
        size_t k = 0;
        for (size_t q = 0; q < np(); ++q) {
            R x = px[q], y = py[q];
            const int ci = host_trunc(double(R(x / dx))), cj = host_trunc(double(R(y / dx)));
            bool keep = !(ci < 0 || cj < 0 || ci >= W || cj >= H || std::isnan(double(x)) || std::isnan(double(y)));
            if (keep && lab(ci, cj) == SOLID) keep = project_particle(x, y);
            if (!keep) continue;
            px[k] = x; py[k] = y; vx[k] = vx[q]; vy[k] = vy[q];
            ++k;
        }
        removed = int64_t(np() - k);
        px.resize(k); py.resize(k); vx.resize(k); vy.resize(k);
    }

    // frameStep, :1302-1331 (phase numbers follow the 3D solver's; 6 is a no-op)
    int phase(int ph) {
        switch (ph) {
            case 0: label(); return 0;
            case 1:
                p2g();
                if (extrap) { extrapolate(u, W + 1, H, 2); extrapolate(v, W, H + 1, 2); }
                return 0;
            case 2: save(); return 0;
            case 3: forces(); return 0;
            case 4: return pressure();
            case 5: project(); return 0;
            case 6: return 0;
            case 7: g2p(); return 0;
            case 8:
                if (extrap) { extrapolate(u, W + 1, H, W); extrapolate(v, W, H + 1, H); }
                advect();
                return 0;
            case 9: cleanup(); return 0;
        }
        return -99;
    }
};

struct Handle2 {
    int fp64;
    Ref2D<float> s32;
    Ref2D<double> s64;
};
template <class F> auto with2(Handle2* h, F f) { return h->fp64 ? f(h->s64) : f(h->s32); }

}  // namespace

extern "C" {

void* or2r_create(int W, int H, double dx, double dt, int fp64) {
    auto* h = new Handle2();
    h->fp64 = fp64;
    with2(h, [&](auto& s) {
        using R = std::decay_t<decltype(s.dx)>;
        s.W = W; s.H = H; s.dx = R(float(dx)); s.dt = R(float(dt));
        s.alloc();
        return 0;
    });
    return h;
}
void or2r_destroy(void* p) { delete static_cast<Handle2*>(p); }
void or2r_set_params(void* p, double alpha, double tol, int maxit) {
    with2(static_cast<Handle2*>(p), [&](auto& s) {
        using R = std::decay_t<decltype(s.dx)>;
        s.alpha = R(float(alpha)); s.tol = tol; s.maxit = maxit; return 0;
    });
}
void or2r_set_extrap(void* p, int on) {
    with2(static_cast<Handle2*>(p), [&](auto& s) { s.extrap = on != 0; return 0; });
}
void or2r_set_labels(void* p, const uint8_t* l) {
    with2(static_cast<Handle2*>(p), [&](auto& s) { std::memcpy(s.labels.data(), l, s.labels.size()); return 0; });
}
void or2r_get_labels(void* p, uint8_t* l) {
    with2(static_cast<Handle2*>(p), [&](auto& s) { std::memcpy(l, s.labels.data(), s.labels.size()); return 0; });
}
// pos, vel: n x 3 (z ignored)
void or2r_set_particles(void* p, int64_t n, const float* pos, const float* vel) {
    with2(static_cast<Handle2*>(p), [&](auto& s) {
        s.px.resize(n); s.py.resize(n); s.vx.resize(n); s.vy.resize(n);
        for (int64_t q = 0; q < n; ++q) {
            s.px[q] = pos[3 * q]; s.py[q] = pos[3 * q + 1];
            s.vx[q] = vel ? vel[3 * q] : 0; s.vy[q] = vel ? vel[3 * q + 1] : 0;
        }
        return 0;
    });
}
int64_t or2r_num_particles(void* p) {
    return with2(static_cast<Handle2*>(p), [&](auto& s) { return int64_t(s.np()); });
}
void or2r_get_particles(void* p, double* pos, double* vel) {
    with2(static_cast<Handle2*>(p), [&](auto& s) {
        for (size_t q = 0; q < s.np(); ++q) {
            pos[3 * q] = double(s.px[q]); pos[3 * q + 1] = double(s.py[q]); pos[3 * q + 2] = 0.0;
            vel[3 * q] = double(s.vx[q]); vel[3 * q + 1] = double(s.vy[q]); vel[3 * q + 2] = 0.0;
        }
        return 0;
    });
}
// which: 0 u, 1 v, 3 u*, 4 v*, 6 p (the 3D solver's grid numbers)
int64_t or2r_grid_len(void* p, int which) {
    return with2(static_cast<Handle2*>(p), [&](auto& s) -> int64_t {
        switch (which) {
            case 0: case 3: return s.nu();
            case 1: case 4: return s.nv();
            case 6: return int64_t(s.W) * s.H;
        }
        return -1;
    });
}
int or2r_grid_io(void* p, int which, double* buf, int set) {
    return with2(static_cast<Handle2*>(p), [&](auto& s) {
        using R = std::decay_t<decltype(s.dx)>;
        std::vector<R>* g = which == 0 ? &s.u : which == 1 ? &s.v : which == 3 ? &s.us : which == 4 ? &s.vs
                          : which == 6 ? &s.p : nullptr;
        if (!g) return -1;
        for (size_t k = 0; k < g->size(); ++k) {
            if (set) (*g)[k] = R(buf[k]);
            else buf[k] = double((*g)[k]);
        }
        return 0;
    });
}
int or2r_phase(void* p, int ph) { return with2(static_cast<Handle2*>(p), [&](auto& s) { return s.phase(ph); }); }
int or2r_step(void* p, int n) {
    return with2(static_cast<Handle2*>(p), [&](auto& s) {
        int rc = 0;
        for (int k = 0; k < n; ++k)
            for (int ph = 0; ph <= 9; ++ph) { const int r = s.phase(ph); if (ph == 4 && r) rc = r; }
        return rc;
    });
}
// fluid cells, CG iterations, particles removed by the last cleanup, capped particles of the last advection
void or2r_stats(void* p, int64_t* out) {
    with2(static_cast<Handle2*>(p), [&](auto& s) {
        out[0] = s.nf; out[1] = s.cg_iters; out[2] = s.removed; out[3] = s.capped;
        return 0;
    });
}

}  // extern "C"
