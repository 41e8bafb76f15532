// kernels_mg.cu -- multigrid-preconditioned conjugate gradients for the
// pressure Poisson system (FP_SOLVER_PCG_MG).
//
// Same system as the reference's cuDSS solve (FluidSolver3D.cu:1815-2062):
// unit 7-point operator over FLUID cells, AIR = Dirichlet 0, SOLID/BODY and
// out-of-domain = Neumann.  Preconditioner: one geometric multigrid V-cycle.
//   * Levels coarsen by 2 per axis; a coarse cell is AIR if any child is AIR,
//     else FLUID if any child is FLUID, else SOLID (Dirichlet priority), and
//     carries the rediscretised unit operator of its labels.
//   * Restriction sums the FLUID children's residuals and scales by 1/4 (3D)
//     or 1/2 (2D); prolongation adds the coarse value to every FLUID child.
//     With these transfers R*A*P equals the coarse unit operator, and P is a
//     multiple of R^T.
//   * Smoother: red-black Gauss-Seidel over-relaxed by MG_SOR, red then black
//     going down, black then red coming up (two pairs on the finest level by
//     default, one on the other grid-wide levels, two on the block levels);
//     the coarsest level does the same symmetric sweeps.  The V-cycle is therefore a symmetric positive definite
//     preconditioner.  After the black sweep only red cells carry a residual,
//     so restriction sums the red children.  The coarse correction is scaled
//     by omega.  Level 0 works on the compact FLUID list.
// Levels with more than MG_BLOCK_CELLS cells are swept by the whole grid with a
// grid barrier between sweeps; every block then does the remaining coarse
// levels on its own shared-memory copy with __syncthreads only (labels
// coarsened there at kernel start; the first block level's b and x copied in
// per cycle) and prolongs from that copy, so the stage costs no grid barrier
// of its own (one block alone, with a copy-out and a barrier, was 1.5 us per
// iteration slower at 128^3).  Block levels take MG_NU_BLOCK sweep pairs:
// two instead of one took the 128^3 dam break from 10.85 to 10.1 iterations
// per warm-started solve (1.030 to 0.985 ms); two pairs on the grid-wide
// levels as well reached 8.9 iterations, but their extra grid barriers made
// the solve slower (1.067 ms).  The whole PCG (flexible, in the Chronopoulos-Gear
// form, optionally started from a guess) runs in one persistent cooperative
// launch with the bounded grid barrier.  Precision split: the V-cycle works in FP32; the
// Krylov vectors (x, r, p, s) and all dot products are FP64, so the
// recurrence residual tracks the true residual down to the 1e-6 target
// without restarts.  Loops over the FLUID list take several cells per thread
// per trip with all loads issued before use, the first four cached in shared
// memory (the solve is latency bound: the 128^3 working set lives in L2).
#include "device_memo.hpp"
#include "kernels.hpp"
#include "pcg_common.cuh"

namespace fp {

namespace {

constexpr int MG_THREADS = 1024;
// Red-black sweep pairs before and after the coarse correction on the
// grid-wide levels below the finest (MG_NU_GRID) and on the block levels
// above the coarsest (MG_NU_BLOCK); build tunables.
#ifndef MG_NU_GRID
#define MG_NU_GRID 1
#endif
#ifndef MG_NU_BLOCK
#define MG_NU_BLOCK 2
#endif
// Symmetric sweep pairs on the coarsest level (build tunable).
#ifndef MG_NU_COARSE
#define MG_NU_COARSE 2
#endif
// Scale of the coarse-grid correction (build tunable).
#ifndef MG_OMEGA
#define MG_OMEGA 1.7f
#endif
// Over-relaxation of every red-black Gauss-Seidel update (pre- and
// post-smoothing alike, so the cycle stays symmetric): x <- x + w (y - x),
// y = (b + neighbours) / d.  1 is plain Gauss-Seidel.  With two sweep pairs
// on the block levels, 1.2 (and a coarse correction scaled by 1.7) took the
// 128^3 dam break from 10.83 to 10.35 iterations per warm-started solve and
// from 12.9 to 12.1 from x = 0 (mean of 40 steps), against 1.1 and 1.8; 1.15
// gave 10.48 and 12.5, 1.25 (with 1.8) 11.1.
#ifndef MG_SOR_VALUE
#define MG_SOR_VALUE 1.2f
#endif
constexpr float MG_SOR = MG_SOR_VALUE;
__device__ __forceinline__ float sor(float x, float y) { return MG_SOR == 1.0f ? y : x + MG_SOR * (y - x); }
// The same on the coarser levels (build tunable MG_SOR_COARSE_VALUE).
#ifndef MG_SOR_COARSE_VALUE
#define MG_SOR_COARSE_VALUE MG_SOR_VALUE
#endif
constexpr float MG_SORC = MG_SOR_COARSE_VALUE;
__device__ __forceinline__ float sorc(float x, float y) { return MG_SORC == 1.0f ? y : x + MG_SORC * (y - x); }

struct MgArgs {
    int L, G;                    // levels; levels [0, G) are grid-wide
    int smem;                    // bytes of the shared-memory copies of levels [G, L); 0: none
    float rscale;                // restriction scale (1/4 in 3D, 1/2 in 2D)
    float omega;                 // over-relaxation of the coarse-grid correction
    int nu_coarse;               // symmetric sweep pairs on the coarsest level
    int nu0;                     // red-black sweep pairs before and after on level 0
    int nu_grid;                 // ... on the other grid-wide levels
    int nu_block;                // ... on the block levels above the coarsest
    MgLevel lv[MG_MAX_LEVELS];
    double* p;                   // level-0 padded dense Krylov vectors (FP64)
    double* q;
    double* xs;
    double* r;
    const float* rhs;            // compact right-hand side
    const float* x0;             // compact initial guess, or null
    const float* pprev;          // dense W x H x D guess (the previous pressure) when x0 is null, or null
    const int* fidx;             // compact FLUID list (level-0 padded index)
    const uint8_t* diag;         // compact diagonal, bit 7 = red/black colour
    const int* nf;
    const int* l1list;           // level 1's FLUID cells (padded indices, any order), or null
    const int* l1n;              // their number
    double* X;                   // compact solution out (FP64)
    float* pout;                 // dense W x H x D pressure out (zero off the fluid already), or null
    double* red;                 // [2] out: ||rhs - A x||^2 and ||rhs||^2 of the solution, in FP64
    double* part;
    GridBar* bar;
    int* status;
    PcgOut* out;
    double tol;
    int maxit;
};

__device__ __forceinline__ int lv_diag(const MgLevel& L, int c) {
    const uint8_t* l = L.lab;
    const int o[6] = {1, -1, L.sy, -L.sy, L.sz, -L.sz};
    int d = 0;
#pragma unroll
    for (int m = 0; m < 6; ++m) { const uint8_t v = l[c + o[m]]; d += (v == FLUID || v == AIR); }
    return d;
}
__device__ __forceinline__ float lv_nbsum(const MgLevel& L, int c) {
    const float* x = L.x;
    return (x[c + 1] + x[c - 1]) + (x[c + L.sy] + x[c - L.sy]) + (x[c + L.sz] + x[c - L.sz]);
}
__device__ __forceinline__ int lv_cell(const MgLevel& L, int t, int& i, int& j, int& k) {
    i = t % L.W; j = (t / L.W) % L.H; k = t / (L.W * L.H);
    return (i + 1) + (j + 1) * L.sy + (k + 1) * L.sz;
}

// ---- level-0 operations over the compact FLUID list (colour and diagonal
// precomputed in the diag byte), four cells per thread per trip ----
constexpr int UNR = 4;
template <int N = UNR>
struct Cells {
    int c[N];
    uint8_t db[N];
    bool ok[N];
};
// A thread's cells are n = t0 + q * stride for trips q = 0, 1, ...  Its first
// UNR cells (q < UNR) are cached for the whole solve in shared memory, in its
// own column (only the thread itself reads them): padded index and diag byte,
// or `safe` and 0 past the end of the list.  `safe` is the padded index of
// interior cell (0,0,0): it and its six stencil neighbours lie inside every
// level-0 grid, so the unconditional loads of an idle lane stay in bounds (its
// result is dropped).
__shared__ int s_fc[UNR * MG_THREADS];
__shared__ uint8_t s_fd[UNR * MG_THREADS];
__device__ __forceinline__ void cache_cells(const int* fidx, const uint8_t* dg, int nf, int t0, int stride, int safe) {
#pragma unroll
    for (int q = 0; q < UNR; ++q) {
        const int n = t0 + q * stride;
        s_fc[q * MG_THREADS + threadIdx.x] = n < nf ? fidx[n] : safe;
        s_fd[q * MG_THREADS + threadIdx.x] = n < nf ? dg[n] : 0;
    }
}
// Cells of trips q0 .. q0 + N - 1 (base = t0 + q0 * stride).
template <int N>
__device__ __forceinline__ void load_cells(Cells<N>& k, const int* fidx, const uint8_t* dg, int nf, int base, int q0,
                                           int stride, int safe) {
#pragma unroll
    for (int u = 0; u < N; ++u) {
        const int n = base + u * stride, q = q0 + u;
        k.ok[u] = n < nf;
        if (q < UNR) {
            k.c[u] = s_fc[q * MG_THREADS + threadIdx.x];
            k.db[u] = s_fd[q * MG_THREADS + threadIdx.x];
        } else {
            k.c[u] = k.ok[u] ? fidx[n] : safe;
            k.db[u] = k.ok[u] ? dg[n] : 0;
        }
    }
}
__device__ void op0_sweep(const MgLevel& L, const int* fidx, const uint8_t* dg, int nf, int color, int t0, int stride) {
    for (int base = t0, q0 = 0; base < nf; base += UNR * stride, q0 += UNR) {
        Cells<> k;
        load_cells(k, fidx, dg, nf, base, q0, stride, 1 + L.sy + L.sz);
        float b[UNR], nb[UNR], xo[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            b[u] = L.b[k.c[u]];
            nb[u] = lv_nbsum(L, k.c[u]);
            xo[u] = MG_SOR == 1.0f ? 0.0f : L.x[k.c[u]];
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int d = k.db[u] & 0x7F;
            if (k.ok[u] && (k.db[u] >> 7) == color) L.x[k.c[u]] = d > 0 ? sor(xo[u], (b[u] + nb[u]) / float(d)) : 0.0f;
        }
    }
}
// ---- level operations over a (t0, stride) share of the work ----
// They read the level's code (FLUID: 1 + diagonal, else 0) instead of labels,
// and issue a cell's loads together, masked by the code afterwards: every
// load is of an interior cell or its halo, so it stays in bounds.
// Gauss-Seidel update of one FLUID cell (code dc > 0).
__device__ __forceinline__ void gs_update(const MgLevel& L, int c) {
    const int dc = L.code[c];
    const float bv = L.b[c], nb = lv_nbsum(L, c), xo = MG_SORC == 1.0f ? 0.0f : L.x[c];
    if (dc > 0) L.x[c] = dc > 1 ? sorc(xo, (bv + nb) / float(dc - 1)) : 0.0f;
}
// Gauss-Seidel update of the FLUID cells of one colour.  With an even width
// the work items are the cells of that colour only: cell i2 of a row is
// i = 2 i2 + ((j + k + colour) & 1).
__device__ void op_sweep(const MgLevel& L, int color, int t0, int stride) {
    if ((L.W & 1) == 0) {
        const int hw = L.W >> 1, n = hw * L.H * L.D;
        for (int t = t0; t < n; t += stride) {
            const int i2 = t % hw, r = t / hw, j = r % L.H, k = r / L.H;
            const int i = 2 * i2 + ((j + k + color) & 1);
            gs_update(L, (i + 1) + (j + 1) * L.sy + (k + 1) * L.sz);
        }
        return;
    }
    const int n = L.W * L.H * L.D;
    for (int t = t0; t < n; t += stride) {
        int i, j, k;
        const int c = lv_cell(L, t, i, j, k);
        if (((i + j + k) & 1) == color) gs_update(L, c);
    }
}
// Residual b - A x of fine cell c if it is FLUID, else 0.
__device__ __forceinline__ float fine_residual(const MgLevel& F, int c) {
    const int dc = F.code[c];
    const float bv = F.b[c], xv = F.x[c], nb = lv_nbsum(F, c);
    return dc > 0 ? bv - (float(dc - 1) * xv - nb) : 0.0f;
}
// Restriction to the next level fused with that level's first sweep:
// b_coarse = scale * sum over the red FLUID children of (b - A x), then
// x_coarse = b/d on red FLUID cells, 0 elsewhere.  After the black sweep the
// black residuals vanish, so only the red children (offsets with an even
// coordinate sum) are read, in k, j, i order.  A child beyond
// an odd-sized fine level (every 2D level in z) is skipped: its stencil would
// leave the padded grid.
__device__ void op_restrict_first(const MgLevel& F, const MgLevel& Cl, float scale, int t0, int stride) {
    const int n = Cl.W * Cl.H * Cl.D;
    for (int t = t0; t < n; t += stride) {
        int I, J, K;
        const int cc = lv_cell(Cl, t, I, J, K);
        const int dc = Cl.code[cc];
        float s = 0.0f, xv = 0.0f;
        if (dc > 0) {
            const bool ii = 2 * I + 1 < F.W, jj = 2 * J + 1 < F.H, kk = 2 * K + 1 < F.D;
            const int c0 = (2 * I + 1) + (2 * J + 1) * F.sy + (2 * K + 1) * F.sz;
            s += fine_residual(F, c0);
            if (ii && jj) s += fine_residual(F, c0 + 1 + F.sy);
            if (ii && kk) s += fine_residual(F, c0 + 1 + F.sz);
            if (jj && kk) s += fine_residual(F, c0 + F.sy + F.sz);
            s *= scale;
            if (((I + J + K) & 1) == 0) xv = dc > 1 ? sorc(0.0f, s / float(dc - 1)) : 0.0f;
        }
        Cl.b[cc] = s;
        Cl.x[cc] = xv;
    }
}
// The last (red) sweep of a coarse level fused with the prolongation of its
// result: every FLUID fine cell with a FLUID parent adds omega * (parent's
// value), where a red parent's value is its Gauss-Seidel update (recomputed
// by each of its children from the final black neighbours, with the same
// arithmetic, so all eight see the same bits) and a black parent's is final.
// The coarse x is not needed after this, so it is not written back.
__device__ __forceinline__ void prolong_one(const MgLevel& F, int c, const MgLevel& Cl, float omega, int i, int j,
                                            int k) {
    const int I = i >> 1, J = j >> 1, K = k >> 1;
    const int cc = (I + 1) + (J + 1) * Cl.sy + (K + 1) * Cl.sz;
    const int dc = Cl.code[cc];
    const float xc = Cl.x[cc], bc = Cl.b[cc], nb = lv_nbsum(Cl, cc), xf = F.x[c];
    if (dc == 0) return;
    const float v = ((I + J + K) & 1) != 0 ? xc : (dc > 1 ? sorc(xc, (bc + nb) / float(dc - 1)) : 0.0f);
    F.x[c] = xf + omega * v;
}
// ... over every cell of the fine level F (dense levels)
__device__ void op_prolong_red(const MgLevel& F, const MgLevel& Cl, float omega, int t0, int stride) {
    const int n = F.W * F.H * F.D;
    for (int t = t0; t < n; t += stride) {
        int i, j, k;
        const int c = lv_cell(F, t, i, j, k);
        if (F.code[c] != 0) prolong_one(F, c, Cl, omega, i, j, k);
    }
}
// The same two operations over a list of the coarse (restriction) or fine
// (prolongation) level's FLUID cells: the cells whose results the dense forms
// compute, with the same arithmetic.  A thread's loads do not wait on the
// cell's code, and one trip covers a level whose FLUID cells are fewer than
// the grid's threads (at 128^3, level 1 has about 60 K of 262 K).  The other
// cells' x and b stay zero: only FLUID cells are written, and the solve
// clears them at its end.
__device__ void op_restrict_first_list(const MgLevel& F, const MgLevel& Cl, float scale, const int* list, int n,
                                       int t0, int stride) {
    for (int t = t0; t < n; t += stride) {
        const int cc = list[t];
        const int I = cc % Cl.sy - 1, J = (cc / Cl.sy) % (Cl.H + 2) - 1, K = cc / Cl.sz - 1;
        const int dc = Cl.code[cc];
        const bool ii = 2 * I + 1 < F.W, jj = 2 * J + 1 < F.H, kk = 2 * K + 1 < F.D;
        const int c0 = (2 * I + 1) + (2 * J + 1) * F.sy + (2 * K + 1) * F.sz;
        float s = fine_residual(F, c0);
        if (ii && jj) s += fine_residual(F, c0 + 1 + F.sy);
        if (ii && kk) s += fine_residual(F, c0 + 1 + F.sz);
        if (jj && kk) s += fine_residual(F, c0 + F.sy + F.sz);
        s *= scale;
        Cl.b[cc] = s;
        Cl.x[cc] = ((I + J + K) & 1) == 0 && dc > 1 ? sorc(0.0f, s / float(dc - 1)) : 0.0f;
    }
}
__device__ void op_prolong_red_list(const MgLevel& F, const MgLevel& Cl, float omega, const int* list, int n, int t0,
                                    int stride) {
    for (int t = t0; t < n; t += stride) {
        const int c = list[t];
        const int i = c % F.sy - 1, j = (c / F.sy) % (F.H + 2) - 1, k = c / F.sz - 1;
        prolong_one(F, c, Cl, omega, i, j, k);
    }
}
// ... over the level-0 FLUID list
__device__ void op0_prolong_red(const MgLevel& F, const MgLevel& Cl, float omega, const int* fidx, int nf, int t0,
                                int stride) {
    for (int n = t0, q = 0; n < nf; n += stride, ++q) {
        const int c = q < UNR ? s_fc[q * MG_THREADS + threadIdx.x] : fidx[n];
        const int i = c % F.sy - 1, j = (c / F.sy) % (F.H + 2) - 1, k = c / F.sz - 1;
        prolong_one(F, c, Cl, omega, i, j, k);
    }
}
// Codes of the interior cells of a dense level from its labels.
__device__ void op_codes(const MgLevel& L, int t0, int stride) {
    const int n = L.W * L.H * L.D;
    for (int t = t0; t < n; t += stride) {
        int i, j, k;
        const int c = lv_cell(L, t, i, j, k);
        L.code[c] = L.lab[c] == FLUID ? uint8_t(1 + lv_diag(L, c)) : uint8_t(0);
    }
}

// Coarse label of cell t of level Cl, with Dirichlet priority: AIR if any
// child is AIR, else FLUID if any child is FLUID, else SOLID.
__device__ __forceinline__ void coarsen_cell(const MgLevel& F, const MgLevel& Cl, int t) {
    int I, J, K;
    const int cc = lv_cell(Cl, t, I, J, K);
    bool air = false, fluid = false;
    for (int c3 = 0; c3 < 2; ++c3)
        for (int b3 = 0; b3 < 2; ++b3)
            for (int a3 = 0; a3 < 2; ++a3) {
                const int i = 2 * I + a3, j = 2 * J + b3, k = 2 * K + c3;
                if (i >= F.W || j >= F.H || k >= F.D) continue;
                const uint8_t l = F.lab[(i + 1) + (j + 1) * F.sy + (k + 1) * F.sz];
                air |= l == AIR;
                fluid |= l == FLUID;
            }
    Cl.lab[cc] = air ? AIR : (fluid ? FLUID : SOLID);
}

// ---- the block stage: levels [G, L) solved by each block on its own copy ----
// Shared-memory form.  Per level: x, b and rs (the red cells' residuals) as
// FP32 padded grids; lab (labels, used while setting up) and code (FLUID:
// 1 + diagonal, else 0) as bytes; ent, the level's FLUID cells (red ones from
// the front, black ones from the back; padded index | parent's padded index
// on the next level << 16) and kid (first child's padded index on the level
// above).  Built once per solve at kernel start; afterwards each operation
// walks a FLUID list (no index decoding, no label tests).  Only FLUID cells are
// written, so every other cell stays zero.
struct BlkLevel {
    MgLevel m;            // dims, strides and the x, b, lab pointers
    float* rs;
    uint8_t* code;
    uint32_t* ent;
    uint32_t* kid;
    int cells;            // interior cells
    int nred, nblack;     // FLUID cells of each colour
};

__host__ __device__ __forceinline__ int mg_npad(const MgLevel& L) { return (L.W + 2) * (L.H + 2) * (L.D + 2); }
__host__ __device__ __forceinline__ int mg_cells(const MgLevel& L) { return L.W * L.H * L.D; }
// Bytes of the block levels [G, L): every level's three FP32 grids (padded
// cells rounded up to 4), then the two entry arrays (cells rounded up to 4),
// then the two byte grids (padded cells rounded up to 16).  The same walk
// sizes the launch and places the arrays (block_levels_init).
__host__ __device__ __forceinline__ int mg_smem_bytes(const MgLevel* lv, int G, int L) {
    int f = 0, e = 0, by = 0;
    for (int l = G; l < L; ++l) {
        f += 3 * ((mg_npad(lv[l]) + 3) & ~3);
        e += 2 * ((mg_cells(lv[l]) + 3) & ~3);
        by += 2 * ((mg_npad(lv[l]) + 15) & ~15);
    }
    return 4 * f + 4 * e + by;
}

extern __shared__ __align__(16) unsigned char mg_smem[];

// Each block at kernel start.  Returns the number of levels that carry FLUID
// cells (at least G + 1): the deepest of them is the cycle's coarsest level.
__device__ int block_levels_init(const MgArgs& a, BlkLevel* S) {
    const int G = a.G, L = a.L, t0 = threadIdx.x, st = blockDim.x;
    __shared__ int s_levels;
    if (t0 == 0) {
        float* f = reinterpret_cast<float*>(mg_smem);
        for (int l = G; l < L; ++l) {
            const int n4 = (mg_npad(a.lv[l]) + 3) & ~3;
            S[l].m = a.lv[l];
            S[l].m.x = f; f += n4;
            S[l].m.b = f; f += n4;
            S[l].rs = f; f += n4;
        }
        uint32_t* e = reinterpret_cast<uint32_t*>(f);
        for (int l = G; l < L; ++l) {
            const int c4 = (mg_cells(a.lv[l]) + 3) & ~3;
            S[l].ent = e; e += c4;
            S[l].kid = e; e += c4;
        }
        uint8_t* by = reinterpret_cast<uint8_t*>(e);
        for (int l = G; l < L; ++l) {
            const int n16 = (mg_npad(a.lv[l]) + 15) & ~15;
            S[l].m.lab = by; by += n16;
            S[l].code = by; by += n16;
            S[l].cells = mg_cells(a.lv[l]);
            S[l].nred = S[l].nblack = 0;
        }
    }
    uint4* z = reinterpret_cast<uint4*>(mg_smem);
    for (int i = t0; i < a.smem / 16; i += st) z[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    for (int c = t0; c < mg_npad(a.lv[G]); c += st) S[G].m.lab[c] = a.lv[G].lab[c];
    __syncthreads();
    for (int l = G + 1; l < L; ++l) {
        for (int t = t0; t < S[l].cells; t += st) coarsen_cell(S[l - 1].m, S[l].m, t);
        __syncthreads();
    }
    for (int l = G; l < L; ++l) {
        BlkLevel& B = S[l];
        for (int t = t0; t < B.cells; t += st) {
            int i, j, k;
            const int c = lv_cell(B.m, t, i, j, k);
            if (B.m.lab[c] != FLUID) continue;
            B.code[c] = uint8_t(1 + lv_diag(B.m, c));
            const int slot = ((i + j + k) & 1) == 0 ? atomicAdd(&B.nred, 1) : B.cells - 1 - atomicAdd(&B.nblack, 1);
            const int pc = l + 1 < L ? ((i >> 1) + 1) + ((j >> 1) + 1) * S[l + 1].m.sy + ((k >> 1) + 1) * S[l + 1].m.sz : 0;
            B.ent[slot] = uint32_t(c) | (uint32_t(pc) << 16);
            if (l > G) B.kid[slot] = uint32_t((2 * i + 1) + (2 * j + 1) * S[l - 1].m.sy + (2 * k + 1) * S[l - 1].m.sz);
        }
    }
    __syncthreads();
    if (t0 == 0) {
        int n = G + 1;
        for (int l = G; l < L; ++l)
            if (S[l].nred + S[l].nblack > 0) n = l + 1;
        s_levels = n;
    }
    __syncthreads();
    return s_levels;
}

// Slot of the t-th FLUID cell of level B (red ones first).
__device__ __forceinline__ int bl_slot(const BlkLevel& B, int t) {
    return t < B.nred ? t : B.cells - B.nblack + (t - B.nred);
}
// Gauss-Seidel update of the FLUID cells of one colour.
__device__ void bl_sweep(const BlkLevel& B, int color, int t0, int st) {
    const int n = color == 0 ? B.nred : B.nblack;
    const uint32_t* e = color == 0 ? B.ent : B.ent + (B.cells - B.nblack);
    for (int t = t0; t < n; t += st) {
        const int c = int(e[t] & 0xFFFFu);
        const int d = B.code[c] - 1;
        B.m.x[c] = d > 0 ? sorc(B.m.x[c], (B.m.b[c] + lv_nbsum(B.m, c)) / float(d)) : 0.0f;
    }
}
// rs = b - A x on the red FLUID cells (after a black sweep the black ones vanish).
__device__ void bl_residual(const BlkLevel& B, int t0, int st) {
    for (int t = t0; t < B.nred; t += st) {
        const int c = int(B.ent[t] & 0xFFFFu);
        B.rs[c] = B.m.b[c] - (float(B.code[c] - 1) * B.m.x[c] - lv_nbsum(B.m, c));
    }
}
// Restriction into C fused with C's first sweep: b = scale * (sum of the
// children's rs, in the dense restriction's order; black, non-FLUID and
// out-of-grid children read zero), x = b/d on red cells, 0 on black ones.
__device__ void bl_restrict(const BlkLevel& F, const BlkLevel& C, float scale, int t0, int st) {
    const int n = C.nred + C.nblack, sy = F.m.sy, sz = F.m.sz;
    for (int t = t0; t < n; t += st) {
        const int slot = bl_slot(C, t);
        const int cc = int(C.ent[slot] & 0xFFFFu);
        const float* r = F.rs + C.kid[slot];
        float s = 0.0f;
        s += r[0]; s += r[1]; s += r[sy]; s += r[sy + 1];
        s += r[sz]; s += r[sz + 1]; s += r[sz + sy]; s += r[sz + sy + 1];
        s *= scale;
        C.m.b[cc] = s;
        const int d = C.code[cc] - 1;
        C.m.x[cc] = (t < C.nred && d > 0) ? sorc(0.0f, s / float(d)) : 0.0f;
    }
}
// Prolongation: every FLUID cell of F adds omega * its parent's x when the
// parent is FLUID (the parent level's red cells are already swept).
__device__ void bl_prolong(const BlkLevel& F, const BlkLevel& C, float omega, int t0, int st) {
    const int n = F.nred + F.nblack;
    for (int t = t0; t < n; t += st) {
        const uint32_t e = F.ent[bl_slot(F, t)];
        const int c = int(e & 0xFFFFu), pc = int(e >> 16);
        if (C.code[pc] > 0) F.m.x[c] += omega * C.m.x[pc];
    }
}

// V-cycle over the shared-memory levels [l0, nl) by one block (nl from
// block_levels_init).  Level l0's first sweep is already done: the grid-wide
// restriction wrote its b and x, which are copied in.  The stage stops after
// level l0's last black sweep: the final red sweep of level l0 is the
// grid-wide prolongation into level l0 - 1, which recomputes it from this
// block's copy.
__device__ void block_vcycle_smem(const MgArgs& a, int l0, int nl, const BlkLevel* S) {
    const int t0 = threadIdx.x, st = blockDim.x;
    const BlkLevel& B0 = S[l0];
    const MgLevel& G0 = a.lv[l0];
    for (int t = t0; t < B0.nred + B0.nblack; t += st) {
        const int c = int(B0.ent[bl_slot(B0, t)] & 0xFFFFu);
        B0.m.b[c] = G0.b[c];
        B0.m.x[c] = G0.x[c];
    }
    __syncthreads();
    const int lc = nl - 1;
    for (int l = l0; l < lc; ++l) {
        bl_sweep(S[l], 1, t0, st); __syncthreads();
        for (int e = 1; e < a.nu_block; ++e) {
            bl_sweep(S[l], 0, t0, st); __syncthreads();
            bl_sweep(S[l], 1, t0, st); __syncthreads();
        }
        bl_residual(S[l], t0, st); __syncthreads();
        bl_restrict(S[l], S[l + 1], a.rscale, t0, st); __syncthreads();
    }
    const BlkLevel& C = S[lc];
    bl_sweep(C, 1, t0, st); __syncthreads();
    for (int it = 1; it < a.nu_coarse; ++it) {
        bl_sweep(C, 0, t0, st); __syncthreads();
        bl_sweep(C, 1, t0, st); __syncthreads();
    }
    for (int it = 0; it < a.nu_coarse; ++it) {
        bl_sweep(C, 1, t0, st); __syncthreads();
        if (it + 1 < a.nu_coarse) {
            bl_sweep(C, 0, t0, st); __syncthreads();
        } else if (lc > l0) {
            bl_sweep(C, 0, t0, st); __syncthreads();
            bl_prolong(S[lc - 1], C, a.omega, t0, st); __syncthreads();
        }
    }
    for (int l = lc - 1; l >= l0; --l) {
        for (int e = 1; e < a.nu_block; ++e) {
            bl_sweep(S[l], 1, t0, st); __syncthreads();
            bl_sweep(S[l], 0, t0, st); __syncthreads();
        }
        bl_sweep(S[l], 1, t0, st); __syncthreads();
        if (l > l0) {
            bl_sweep(S[l], 0, t0, st); __syncthreads();
            bl_prolong(S[l - 1], S[l], a.omega, t0, st); __syncthreads();
        }
    }
    // the prolongation that follows reads level l0 from this block's copy
}

// Global-memory form (the block levels do not fit in shared memory, or the
// hierarchy has one level): V-cycle over levels [l0, L) of a.lv by block 0.
// Level l0's first sweep is already done (fused into the step that wrote its
// right-hand side).  With l0 > 0 the stage stops after level l0's last black
// sweep: the final red sweep of level l0 is the grid-wide prolongation into
// level l0 - 1, which recomputes it.  With l0 == 0 it finishes level 0 itself.
__device__ void block_vcycle_global(const MgArgs& a, int l0) {
    const int t0 = threadIdx.x, st = blockDim.x;
    for (int l = l0; l < a.L - 1; ++l) {
        op_sweep(a.lv[l], 1, t0, st); __syncthreads();
        for (int e = 1; e < (l == 0 ? a.nu0 : a.nu_block); ++e) {
            op_sweep(a.lv[l], 0, t0, st); __syncthreads();
            op_sweep(a.lv[l], 1, t0, st); __syncthreads();
        }
        op_restrict_first(a.lv[l], a.lv[l + 1], a.rscale, t0, st); __syncthreads();
    }
    const int lc = a.L - 1;
    const MgLevel& C = a.lv[lc];
    op_sweep(C, 1, t0, st); __syncthreads();
    for (int it = 1; it < a.nu_coarse; ++it) {
        op_sweep(C, 0, t0, st); __syncthreads();
        op_sweep(C, 1, t0, st); __syncthreads();
    }
    for (int it = 0; it < a.nu_coarse; ++it) {
        op_sweep(C, 1, t0, st); __syncthreads();
        if (it + 1 < a.nu_coarse || lc == 0) {
            op_sweep(C, 0, t0, st); __syncthreads();
        } else if (lc > l0) {
            op_prolong_red(a.lv[lc - 1], C, a.omega, t0, st); __syncthreads();
        }
    }
    for (int l = lc - 1; l >= l0; --l) {
        for (int e = 1; e < (l == 0 ? a.nu0 : a.nu_block); ++e) {
            op_sweep(a.lv[l], 1, t0, st); __syncthreads();
            op_sweep(a.lv[l], 0, t0, st); __syncthreads();
        }
        op_sweep(a.lv[l], 1, t0, st); __syncthreads();
        if (l == 0) {
            op_sweep(a.lv[0], 0, t0, st); __syncthreads();
        } else if (l > l0) {
            op_prolong_red(a.lv[l - 1], a.lv[l], a.omega, t0, st); __syncthreads();
        }
    }
}

// z = V-cycle(r) with r = lv[0].b, z = lv[0].x.  The caller has already done
// the first (red) sweep of level 0 (z = w b/d on red FLUID cells, 0 on black
// ones) and a grid barrier since.  Ends with a grid barrier; returns false if
// a barrier timed out.  Grid-wide levels take four barriers each with one
// sweep pair (level 0 two more per extra pair): black sweep, restriction (with
// the next level's first sweep), black sweep, red sweep (with the
// prolongation into the finer level).  nl: the levels that hold FLUID cells.
// n1: the number of level 1's listed FLUID cells (a.l1list), or -1 for none.
__device__ bool vcycle(const MgArgs& a, const BlkLevel* S, int nl, int n1) {
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    const unsigned nb = gridDim.x;
    const int G = min(a.G, a.L - 1);
    const int nf = *a.nf;
    // restriction from level l and prolongation into level lf >= 1, level 1
    // over its FLUID list when there is one
    auto restrict_first = [&](int l) {
        if (l == 0 && n1 >= 0) op_restrict_first_list(a.lv[0], a.lv[1], a.rscale, a.l1list, n1, t0, st);
        else op_restrict_first(a.lv[l], a.lv[l + 1], a.rscale, t0, st);
    };
    auto prolong_into = [&](int lf, const MgLevel& Cl) {
        if (lf == 1 && n1 >= 0) op_prolong_red_list(a.lv[1], Cl, a.omega, a.l1list, n1, t0, st);
        else op_prolong_red(a.lv[lf], Cl, a.omega, t0, st);
    };
    // one grid-wide sweep of level l (colour 0 red, 1 black) and a barrier
    auto sweep = [&](int l, int color) {
        if (l == 0) op0_sweep(a.lv[0], a.fidx, a.diag, nf, color, t0, st);
        else op_sweep(a.lv[l], color, t0, st);
        return grid_barrier(a.bar, nb, a.status);
    };
    for (int l = 0; l < G; ++l) {
        // pre-smoothing (red, black)^nu (nu = nu0 on level 0, else nu_grid); the
        // first red sweep is fused upstream
        if (!sweep(l, 1)) return false;
        for (int e = 1; e < (l == 0 ? a.nu0 : a.nu_grid); ++e)
            if (!sweep(l, 0) || !sweep(l, 1)) return false;
        restrict_first(l);
        if (!grid_barrier(a.bar, nb, a.status)) return false;
    }
    if (a.smem) {
        // Every block runs the block levels on its own shared-memory copy (the
        // same arithmetic, so the same bits) and prolongs from that copy: no
        // grid barrier and no copy-out between the stage and the prolongation.
        block_vcycle_smem(a, G, nl, S);
        MgLevel cg = S[G].m;  // level G in this block's shared memory
        cg.code = S[G].code;
        if (G == 1) op0_prolong_red(a.lv[0], cg, a.omega, a.fidx, nf, t0, st);
        else prolong_into(G - 1, cg);
        if (!grid_barrier(a.bar, nb, a.status)) return false;
    } else {
        if (blockIdx.x == 0) block_vcycle_global(a, G);
        if (!grid_barrier(a.bar, nb, a.status)) return false;
        if (G > 0) {  // level G's last red sweep, fused with its prolongation into level G - 1
            if (G == 1) op0_prolong_red(a.lv[0], a.lv[1], a.omega, a.fidx, nf, t0, st);
            else prolong_into(G - 1, a.lv[G]);
            if (!grid_barrier(a.bar, nb, a.status)) return false;
        }
    }
    for (int l = G - 1; l >= 0; --l) {
        // post-smoothing (black, red)^nu, the reverse of the pre-smoothing; the
        // first red sweep was fused with the prolongation, the last red sweep
        // with the next prolongation
        if (!sweep(l, 1)) return false;
        for (int e = 1; e < (l == 0 ? a.nu0 : a.nu_grid); ++e)
            if (!sweep(l, 0) || !sweep(l, 1)) return false;
        if (l == 0) op0_sweep(a.lv[0], a.fidx, a.diag, nf, 0, t0, st);
        else if (l == 1) op0_prolong_red(a.lv[0], a.lv[1], a.omega, a.fidx, nf, t0, st);
        else prolong_into(l - 1, a.lv[l]);
        if (!grid_barrier(a.bar, nb, a.status)) return false;
    }
    return true;
}

// Level-0 first sweep value of one FLUID cell: b/d on red cells, 0 on black.
__device__ __forceinline__ float first_red0(float b, uint8_t db) {
    const int d = db & 0x7F;
    return ((db >> 7) == 0 && d > 0) ? sor(0.0f, b / float(d)) : 0.0f;
}

__global__ void __launch_bounds__(MG_THREADS) k_pcg_mg(MgArgs a) {
    const int nf = *a.nf;
    const int nb = int(gridDim.x);
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, st = nb * blockDim.x;
    const MgLevel& F = a.lv[0];
    const int n1 = a.l1list && a.L > 1 ? *a.l1n : -1;  // level 1's listed FLUID cells
    float* b0 = F.b;  // FP32 copy of r: the V-cycle's right-hand side
    float* z = F.x;   // FP32 preconditioned residual
    double* r = a.r;
    int red = 0;      // reduction counter (partial buffers double-buffered by parity)
    auto partial = [&](double v0, double v1, double v2) {
        double3 bs = block_sum3(v0, v1, v2);
        double* pp = a.part + (red & 1) * 3 * nb;
        if (threadIdx.x == 0) { pp[blockIdx.x] = bs.x; pp[nb + blockIdx.x] = bs.y; pp[2 * nb + blockIdx.x] = bs.z; }
    };
    auto total = [&]() { double3 t = grid_sum3(a.part + (red & 1) * 3 * nb, nb); ++red; return t; };
    const int sy = F.sy, sz = F.sz;
    __shared__ BlkLevel s_lv[MG_MAX_LEVELS];  // the shared-memory block levels
    const int nl = a.smem ? block_levels_init(a, s_lv) : a.L;  // every block: its own copy

    // level codes: level 0 on its FLUID cells (zero elsewhere, restored at the
    // end), the dense grid-wide levels (and, without shared-memory copies, the
    // block levels) over all their cells
    for (int l = 1; l <= (a.smem ? a.G : a.L - 1); ++l) op_codes(a.lv[l], t0, st);
    cache_cells(a.fidx, a.diag, nf, t0, st, 1 + sy + sz);
    // r = rhs, the V-cycle's right-hand side and first sweep, the level-0
    // codes and the guess.  A dense guess (the previous pressure, zero off the
    // current fluid and outside the grid) also gets its stencil A g and the
    // dot products here: it was complete before the launch, so its
    // neighbours need no grid barrier.  A compact guess needs one.
    const bool dense_guess = a.pprev != nullptr;
    double rrl = 0.0, xb = 0.0, xq = 0.0;
    constexpr int UI = 2;
    for (int base = t0, q0 = 0; base < nf; base += UI * st, q0 += UI) {
        Cells<UI> k;
        load_cells(k, a.fidx, a.diag, nf, base, q0, st, 1 + sy + sz);
        float bvf[UI], g[UI];
        double qv[UI];
#pragma unroll
        for (int u = 0; u < UI; ++u) {
            const int n = base + u * st;
            bvf[u] = k.ok[u] ? a.rhs[n] : 0.0f;
            g[u] = 0.0f;
            qv[u] = 0.0;
            if (!k.ok[u]) continue;
            if (a.x0) {
                g[u] = a.x0[n];
            } else if (dense_guess) {
                const int c = k.c[u];
                const int i = c % sy - 1, j = (c / sy) % (F.H + 2) - 1, kk = c / sz - 1;
                const int64_t e = (int64_t(kk) * F.H + j) * F.W + i, sY = F.W, sZ = int64_t(F.W) * F.H;
                auto gv = [&](bool in, int64_t off) {
                    const float v = in ? a.pprev[e + off] : 0.0f;
                    return isfinite(v) ? double(v) : 0.0;
                };
                const double gc = gv(true, 0);
                g[u] = float(gc);
                qv[u] = double(k.db[u] & 0x7F) * gc - ((gv(i + 1 < F.W, 1) + gv(i > 0, -1)) +
                                                        (gv(j + 1 < F.H, sY) + gv(j > 0, -sY)) +
                                                        (gv(kk + 1 < F.D, sZ) + gv(kk > 0, -sZ)));
            }
        }
#pragma unroll
        for (int u = 0; u < UI; ++u) {
            if (!k.ok[u]) continue;
            const int c = k.c[u];
            const double rv = double(bvf[u]);
            F.code[c] = uint8_t(1 + (k.db[u] & 0x7F));
            r[c] = rv;
            b0[c] = float(rv);
            z[c] = first_red0(float(rv), k.db[u]);  // the V-cycle's first sweep
            a.xs[c] = double(g[u]);
            if (dense_guess) {
                a.q[c] = qv[u];
                xb += double(g[u]) * rv;
                xq += double(g[u]) * qv[u];
            }
            rrl += rv * rv;
        }
    }
    const bool guess = a.x0 || a.pprev;
    double bb_warm = 0.0;  // ||b||^2 when started from a guess
    // With a guess g the solve's first flexible-CG step uses g as its
    // preconditioned residual: z0 = g, p0 = z0, alpha0 = (r0, z0) / (p0, A p0)
    // -- the energy-optimal scaling -- and x1 = alpha0 g.  For the network's
    // guess N(b) (the learned preconditioner), p0, A p0, gamma0 = (r0, z0) and
    // (p0, A p0) stay in the recurrence, so the next direction (from the
    // V-cycle) is made A-conjugate to p0 by the Polak-Ribiere beta.  The
    // previous step's pressure restarts the recurrence instead: kept in it, it
    // cost iterations (11.2 against 10.8 per warm-started solve at 128^3).
    bool dir0 = false;
    double gam0 = 0.0, alpha0 = 0.0, den0 = 0.0;
    if (guess) {
        // Scale the guess by its energy-optimal factor alpha = (x0, b) / (x0, A x0):
        // the A-norm error of alpha x0 is never above that of x = 0.  Then r = b - A x.
        if (a.x0) {
            if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
            for (int n = t0; n < nf; n += st) {
                const int c = a.fidx[n];
                const double* xp = a.xs + c;
                const double qc = double(a.diag[n] & 0x7F) * xp[0] -
                                  ((xp[1] + xp[-1]) + (xp[sy] + xp[-sy]) + (xp[sz] + xp[-sz]));
                a.q[c] = qc;
                xb += xp[0] * r[c];
                xq += xp[0] * qc;
            }
        }
        partial(xb, xq, rrl);
        if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
        const double3 t = total();
        const double alpha = (t.y > 0.0 && isfinite(t.x / t.y)) ? t.x / t.y : 0.0;
        dir0 = alpha != 0.0 && a.x0 != nullptr;  // the learned guess only (see above)
        gam0 = t.x; alpha0 = alpha; den0 = t.y;
        bb_warm = t.z;  // all reads of x ended before the barrier above
        rrl = 0.0;
        for (int base = t0, q0 = 0; base < nf; base += UI * st, q0 += UI) {
            Cells<UI> k;
            load_cells(k, a.fidx, a.diag, nf, base, q0, st, 1 + sy + sz);
            double xv[UI], rv0[UI], qc[UI];
#pragma unroll
            for (int u = 0; u < UI; ++u) {
                xv[u] = a.xs[k.c[u]];
                rv0[u] = r[k.c[u]];
                qc[u] = a.q[k.c[u]];
            }
#pragma unroll
            for (int u = 0; u < UI; ++u) {
                if (!k.ok[u]) continue;
                const int c = k.c[u];
                a.xs[c] = xv[u] * alpha;
                if (a.x0) a.p[c] = xv[u];  // the learned guess: p0 = g; q holds A p0
                const double rv = rv0[u] - alpha * qc[u];
                r[c] = rv;
                b0[c] = float(rv);
                z[c] = first_red0(float(rv), k.db[u]);
                rrl += rv * rv;
            }
        }
    }
    partial(rrl, 0.0, 0.0);
    if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
    double rr = total().x;
    const double bb = guess ? bb_warm : rr;
    const double rr0 = rr;
    const double thr = a.tol * a.tol * bb;
    // Flexible preconditioned CG in the Chronopoulos-Gear form: after the
    // V-cycle one pass forms w = A z, gamma = (r, z), delta = (z, w) and
    // zeta = (z, s_old); one more updates p = z + beta p, s = w + beta s
    // (= A p), x += alpha p, r -= alpha s and starts the next cycle.  beta is
    // the Polak-Ribiere choice (z, r - r_old) / gamma_old = -alpha_old zeta /
    // gamma_old, and (p, A p) = delta + 2 beta zeta + beta^2 (p, A p)_old holds
    // for any beta, so alpha = gamma / (p, A p) needs no symmetry of the
    // V-cycle (over-relaxed smoothing makes it slightly non-symmetric).  Two
    // grid-wide passes per iteration besides the cycle.  w is kept in the
    // compact X buffer (the solution is written there only at the end); s
    // lives in q.
    double* w = a.X;
    double gam = 0.0, gam_old = gam0, alpha_old = dir0 ? alpha0 : 1.0, den_old = dir0 ? den0 : 1.0;
    int it = 0, stt = DEV_OK;
    while (rr > thr && bb > 0.0) {
        if (it >= a.maxit) { stt = DEV_MAXIT; break; }
        if (!vcycle(a, s_lv, nl, n1)) return;  // z = M^-1 r
        double gl = 0.0, dl = 0.0, sl = 0.0;
        constexpr int U3 = 3;  // three cells in flight fit the register budget with FP64 sums
        for (int base = t0, q0 = 0; base < nf; base += U3 * st, q0 += U3) {
            Cells<U3> k;
            load_cells(k, a.fidx, a.diag, nf, base, q0, st, 1 + sy + sz);
            float zc[U3];
            double zn[U3], rc[U3], sc[U3];  // A z exactly: FP32 values summed in FP64
#pragma unroll
            for (int u = 0; u < U3; ++u) {
                const float* zp = z + k.c[u];
                zc[u] = zp[0];
                zn[u] = (double(zp[1]) + double(zp[-1])) + (double(zp[sy]) + double(zp[-sy])) +
                        (double(zp[sz]) + double(zp[-sz]));
                rc[u] = r[k.c[u]];
                sc[u] = a.q[k.c[u]];
            }
#pragma unroll
            for (int u = 0; u < U3; ++u) {
                if (!k.ok[u]) continue;
                const double zv = double(zc[u]);
                const double wv = double(k.db[u] & 0x7F) * zv - zn[u];
                w[base + u * st] = wv;
                gl += rc[u] * zv;
                dl += zv * wv;
                sl += zv * sc[u];
            }
        }
        partial(gl, dl, sl);
        if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
        const double3 t = total();
        gam = t.x;
        if (isnan(t.x) || isnan(t.y) || isnan(t.z)) { stt = DEV_NAN; break; }
        const bool coupled = it > 0 || dir0;  // a previous direction to conjugate against
        const double beta = coupled ? -alpha_old * t.z / gam_old : 0.0;
        const double den = coupled ? t.y + beta * (2.0 * t.z + beta * den_old) : t.y;
        if (!(den > 0.0)) { stt = DEV_BREAKDOWN; break; }
        const double alpha = gam / den;
        rrl = 0.0;
        constexpr int U2 = 2;  // FP64: two cells in flight fit the register budget
        for (int base = t0, q0 = 0; base < nf; base += U2 * st, q0 += U2) {
            Cells<U2> k;
            load_cells(k, a.fidx, a.diag, nf, base, q0, st, 1 + sy + sz);
            double pv[U2], sv[U2], xv[U2], rv[U2], wv[U2];
            float zc[U2];
#pragma unroll
            for (int u = 0; u < U2; ++u) {
                const int c = k.c[u];
                zc[u] = z[c];
                pv[u] = a.p[c];
                sv[u] = a.q[c];
                xv[u] = a.xs[c];
                rv[u] = r[c];
                wv[u] = k.ok[u] ? w[base + u * st] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U2; ++u) {
                if (!k.ok[u]) continue;
                const int c = k.c[u];
                const double pn = coupled ? double(zc[u]) + beta * pv[u] : double(zc[u]);
                const double sn = coupled ? wv[u] + beta * sv[u] : wv[u];
                a.p[c] = pn;
                a.q[c] = sn;
                a.xs[c] = xv[u] + alpha * pn;
                const double rn = rv[u] - alpha * sn;
                r[c] = rn;
                b0[c] = float(rn);
                z[c] = first_red0(float(rn), k.db[u]);
                rrl += rn * rn;
            }
        }
        partial(rrl, 0.0, 0.0);
        if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
        rr = total().x;
        ++it;
        if (isnan(rr)) { stt = DEV_NAN; break; }
        gam_old = gam;
        alpha_old = alpha;
        den_old = den;
    }
    // The true residual of the FP64 solution, ||rhs - A x||^2 and ||rhs||^2,
    // then the compact and dense solution; zero the level-0 work grids at the
    // FLUID cells so the next solve starts from zero whatever cells are fluid.
    if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
    {
        double e2 = 0.0, b2 = 0.0;
        for (int n = t0; n < nf; n += st) {
            const int c = a.fidx[n];
            const double* xp = a.xs + c;
            const double ax = double(a.diag[n] & 0x7F) * xp[0] -
                              ((xp[1] + xp[-1]) + (xp[sy] + xp[-sy]) + (xp[sz] + xp[-sz]));
            const double bv = double(a.rhs[n]), e = bv - ax;
            e2 += e * e;
            b2 += bv * bv;
        }
        partial(e2, b2, 0.0);
    }
    if (!grid_barrier(a.bar, unsigned(nb), a.status)) return;
    {
        const double3 t = total();
        if (blockIdx.x == 0 && threadIdx.x == 0) { a.red[0] = t.x; a.red[1] = t.y; }
    }
    for (int n = t0; n < nf; n += st) {
        const int c = a.fidx[n];
        const double xv = a.xs[c];
        a.X[n] = xv;
        if (a.pout) {
            const int i = c % sy - 1, j = (c / sy) % (F.H + 2) - 1, k = c / sz - 1;
            a.pout[(int64_t(k) * F.H + j) * F.W + i] = float(xv);
        }
        a.xs[c] = fmin(fabs(xv), 0.0);  // +0 computed from the load (a constant store would wait on it)
        a.p[c] = 0.0; a.q[c] = 0.0; r[c] = 0.0; b0[c] = 0.0f; z[c] = 0.0f; F.code[c] = 0;
    }
    for (int t = t0; t < n1; t += st) {  // level 1's FLUID cells: x and b back to zero
        const int c = a.l1list[t];
        a.lv[1].x[c] = 0.0f;
        a.lv[1].b[c] = 0.0f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out->iters = it;
        atomicCAS(a.status, DEV_OK, stt);
        a.out->rr = rr;
        a.out->bb = bb;
        a.out->rz = gam;
        a.out->rr0 = rr0;
    }
}

// Coarse labels with Dirichlet priority: AIR if any child AIR, else FLUID if
// any child FLUID, else SOLID.
__global__ void k_coarsen(MgLevel F, MgLevel Cl) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < Cl.W * Cl.H * Cl.D) coarsen_cell(F, Cl, t);
}

// Level 1 straight from the cell labels, by the same rule (BODY, like SOLID,
// is neither AIR nor FLUID); level 0 itself needs no padded label copy, as
// its operations read the FLUID list's diagonal bytes and codes.
// It also appends level 1's FLUID cells (padded indices) to list, one atomic
// per block, in no fixed order: every use of the list treats its cells
// independently.  *nlist must be zero before the launch; at most cap entries
// are written.
constexpr int COARSEN_THREADS = 256;
__global__ void __launch_bounds__(COARSEN_THREADS) k_coarsen_cells(const uint8_t* __restrict__ lab, Dims g, MgLevel Cl,
                                                                   int* __restrict__ list, int* __restrict__ nlist,
                                                                   int cap) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    bool listed = false;
    int cc = 0;
    if (t < Cl.W * Cl.H * Cl.D) {
        int I, J, K;
        cc = lv_cell(Cl, t, I, J, K);
        bool air = false, fluid = false;
        for (int c3 = 0; c3 < 2; ++c3)
            for (int b3 = 0; b3 < 2; ++b3)
                for (int a3 = 0; a3 < 2; ++a3) {
                    const int i = 2 * I + a3, j = 2 * J + b3, k = 2 * K + c3;
                    if (i >= g.W || j >= g.H || k >= g.D) continue;
                    const uint8_t l = lab[int64_t(i) + int64_t(j) * g.W + int64_t(k) * g.W * g.H];
                    air |= l == AIR;
                    fluid |= l == FLUID;
                }
        Cl.lab[cc] = air ? AIR : (fluid ? FLUID : SOLID);
        listed = fluid && !air;
    }
    if (!list) return;  // uniform across the block
    __shared__ int s_off[COARSEN_THREADS / 32];
    __shared__ int s_base;
    const unsigned m = __ballot_sync(0xffffffffu, listed);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_off[wid] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < COARSEN_THREADS / 32; ++w) { const int c = s_off[w]; s_off[w] = tot; tot += c; }
        s_base = tot > 0 ? atomicAdd(nlist, tot) : 0;
    }
    __syncthreads();
    const int slot = s_base + s_off[wid] + __popc(m & ((1u << lane) - 1u));
    if (listed && slot < cap) list[slot] = cc;
}

}  // namespace

int mg_levels_for(int W, int H, int D, MgLevel* lv) {
    int L = 0;
    int w = W, h = H, d = D;
    while (L < MG_MAX_LEVELS) {
        lv[L].W = w; lv[L].H = h; lv[L].D = d;
        lv[L].sy = w + 2; lv[L].sz = (w + 2) * (h + 2);
        ++L;
        if (w <= 2 && h <= 2 && d <= 2) break;
        w = (w + 1) / 2; h = (h + 1) / 2; d = (d + 1) / 2;
    }
    return L;
}

int mg_max_blocks() {
    static DeviceMemo memo;
    return memo.get([](int dev) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_pcg_mg, cudaFuncAttributeMaxDynamicSharedMemorySize, MG_SMEM_BUDGET);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_mg, MG_THREADS, MG_SMEM_BUDGET);
        return sms * std::max(1, per);
    });
}

int mg_split(const MgLevel* lv, int L, int* smem_bytes) {
    *smem_bytes = 0;
    if (L <= 1) return 0;
    int G = 1;  // level 0 is always swept grid-wide on its FLUID list
    for (int l = 0; l < L; ++l)
        if (int64_t(lv[l].W) * lv[l].H * lv[l].D > MG_BLOCK_CELLS) G = std::max(G, l + 1);
    for (G = std::min(G, L - 1); G < L; ++G) {
        const int b = mg_smem_bytes(lv, G, L);
        // the FLUID lists hold padded indices in 16 bits
        if (b <= MG_SMEM_BUDGET && mg_npad(lv[G]) <= 65535) { *smem_bytes = b; return G; }
    }
    return L - 1;  // not even the coarsest level fits: the block levels stay in global memory
}

int launch_mg_setup(const uint8_t* labels, Dims g, MgLevel* lv, int L, int* l1list, int* l1n, cudaStream_t st) {
    int smem = 0;
    const int G = mg_split(lv, L, &smem);
    const int last = smem ? G : L - 1;  // deeper shared-memory levels: coarsened by the solver kernel
    for (int l = 1; l <= last; ++l) {
        const int n = lv[l].W * lv[l].H * lv[l].D;
        if (l == 1) {
            if (l1list) cudaMemsetAsync(l1n, 0, sizeof(int), st);
            k_coarsen_cells<<<(n + COARSEN_THREADS - 1) / COARSEN_THREADS, COARSEN_THREADS, 0, st>>>(labels, g, lv[1],
                                                                                                   l1list, l1n, n);
        }
        else k_coarsen<<<(n + 255) / 256, 256, 0, st>>>(lv[l - 1], lv[l]);
    }
    return last;
}

int launch_pcg_mg(Dims g, PressureBufs& pb, MgLevel* lv, int L, const int* l1list, const int* l1n, double* p,
                  double* q, double* xs, double* r, const float* rhs, double tol, int maxit, cudaStream_t st,
                  const float* x0, int nu0, const float* pprev, float* pout, unsigned wait_polls) {
    // One block per 4096 cells (each thread's UNR cells per trip), at most one
    // per SM: a small grid waits at cheaper barriers (one block: __syncthreads).
    const int64_t want = (g.nc() + int64_t(MG_THREADS) * UNR - 1) / (int64_t(MG_THREADS) * UNR);
    const int nb = int(std::max<int64_t>(1, std::min<int64_t>(mg_max_blocks(), want)));
    int* status = &pb.out->status;
    launch_reset_barrier(pb.bar, status, wait_polls, st);
    MgArgs a;
    a.L = L;
    a.G = mg_split(lv, L, &a.smem);
    for (int l = 0; l < L; ++l) a.lv[l] = lv[l];
    a.rscale = g.D > 1 ? 0.25f : 0.5f;
    // The piecewise-constant prolongation underestimates the coarse correction;
    // scaling it by 1.7 roughly halves the PCG iterations (29 -> 15 at 128^3,
    // 31 -> 14 at 256^2 in a float64 model of this V-cycle).  Any omega > 0
    // keeps the preconditioner symmetric; in that model PCG converged for
    // every omega up to 2 on dam-break, pool and random-box scenes.  With the
    // over-relaxed smoother, 1.8 was as fast as 1.9 on the dam break and
    // faster on random boxes (14 against 15 iterations); with two sweep pairs
    // on the block levels and SOR 1.2, 1.7 is best (1.9: 10.55, 2.0: 10.75
    // iterations per warm-started solve at 128^3).
    a.omega = MG_OMEGA;
    a.nu_coarse = MG_NU_COARSE;
    a.nu0 = std::max(1, nu0);
    a.nu_grid = MG_NU_GRID;
    a.nu_block = MG_NU_BLOCK;
    a.p = p; a.q = q; a.xs = xs; a.r = r; a.rhs = rhs; a.x0 = x0; a.pprev = x0 ? nullptr : pprev;
    a.fidx = pb.fidx; a.diag = pb.diag; a.nf = pb.nf;
    a.l1list = l1list; a.l1n = l1n;
    a.X = static_cast<double*>(pb.X);
    a.pout = pout;
    a.red = pb.red;
    a.part = pb.part; a.bar = pb.bar; a.status = status; a.out = pb.out;
    a.tol = tol; a.maxit = maxit;
    void* args[] = {&a};
    cudaError_t e =
        cudaLaunchCooperativeKernel((const void*)k_pcg_mg, dim3(nb), dim3(MG_THREADS), args, size_t(a.smem), st);
    return e == cudaSuccess ? 0 : int(e);
}

}  // namespace fp
