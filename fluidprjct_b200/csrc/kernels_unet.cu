// kernels_unet.cu -- kernels of the learned pressure preconditioner (a 3D
// U-Net; the layer table is in unet.hpp).
//
// The forward and backward-data convolutions run on tcgen05
// (kernels_unet_tma.cu).  This file holds the rest, with the weight gradient
// on the BF16 mma.sync path (m16n8k16, FP32 accumulation):
//   k_corr3  weight gradients dw[t][co][ci] = sum_v g[v][co] x[v+off(t)][ci]
//            (M = COUT, N = CIN, K = voxels), over bricks of 8x8x4 voxels
//            whose zero-padded input halo (10x10x6, every input channel) is
//            staged with cp.async.  The input may be the concatenation
//            [up2(xa) | xb] of a 2x-upsampled coarse tensor and a same-level
//            one: the upsampling is an index shift in the halo load.  Each
//            CTA accumulates its tap group over its bricks in registers and
//            writes one partial.  The partials are summed in a fixed order,
//            so gradients are deterministic.
// Smem rows are padded by 16 bytes, so each 8-row ldmatrix phase hits eight
// distinct 16-byte bank groups.
#include <algorithm>
#include <cstdio>

#include "device_memo.hpp"
#include "unet.hpp"

namespace fp {
namespace unet {
namespace {

constexpr int BX = 8, BY = 8, BZ = 4;
constexpr int HX = BX + 2, HY = BY + 2, HZ = BZ + 2, HALO = HX * HY * HZ;  // 600
constexpr int THREADS = 256;
constexpr int BRICK = BX * BY * BZ;  // 256 voxels = 16 M-tiles of 16

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool pred) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(pred ? 16 : 0));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void ldsm_x4_t(unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3, unsigned addr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2_t(unsigned& r0, unsigned& r1, unsigned addr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(addr));
}
__device__ __forceinline__ void mma16816(float* c, unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                         unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Stage the zero-padded input halo of the brick at (x0, y0, z0) (its -1
// corner) into sx, rows of RS bf16.  Channels [0, CA) come from the coarse
// tensor at (x>>1, y>>1, z>>1), channels [CA, CA+CB) from the same level.
template <int CA, int CB, int RS>
__device__ __forceinline__ void load_halo(bf16* sx, const bf16* __restrict__ xa, const bf16* __restrict__ xb,
                                          const Lvl& lv, const Lvl& lc, int x0, int y0, int z0) {
    constexpr int CH = (CA + CB) / 8;
    for (int i = threadIdx.x; i < HALO * CH; i += THREADS) {
        const int ch = i % CH, hv = i / CH;
        const int gx = x0 + hv % HX, gy = y0 + (hv / HX) % HY, gz = z0 + hv / (HX * HY);
        const bool in = gx >= 0 && gx < lv.W && gy >= 0 && gy < lv.H && gz >= 0 && gz < lv.D;
        const bf16* src;
        if (CA > 0 && ch * 8 < CA)
            src = in ? xa + blk8(lc.n(), (int64_t(gz >> 1) * lc.H + (gy >> 1)) * lc.W + (gx >> 1), ch) : xa;
        else
            src = in ? xb + blk8(lv.n(), (int64_t(gz) * lv.H + gy) * lv.W + gx, ch - CA / 8) : xb;
        cp_async16(sx + hv * RS + ch * 8, src, in);
    }
}

template <int CA, int CB, int COUT, int TPC>
__global__ void __launch_bounds__(THREADS) k_corr3(CorrArgs a) {
    constexpr int CIN = CA + CB;
    constexpr int RS = CIN + 8;
    constexpr int GS = COUT + 8;
    constexpr int TILES = TPC * (COUT / 16) * (CIN / 8);
    constexpr int NTW = (TILES + 7) / 8;
    static_assert(27 % TPC == 0 && COUT % 16 == 0 && CIN % 16 == 0, "tiling");
    extern __shared__ __align__(16) unsigned char smem[];
    bf16* sx = reinterpret_cast<bf16*>(smem);
    bf16* sg = sx + HALO * RS;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tap0 = blockIdx.y * TPC;
    const int nbx = (a.lv.W + BX - 1) / BX, nby = (a.lv.H + BY - 1) / BY, nbz = (a.lv.D + BZ - 1) / BZ;
    const int nbricks = nbx * nby * nbz;
    // A (= g^T, 16 channels x 16 voxels) via ldmatrix.trans: voxel row, channel offset
    const int akr = (lane & 7) + 8 * (lane >> 4), amoff = 8 * ((lane >> 3) & 1);
    // B (= shifted x, 16 voxels x 8 channels) via ldmatrix.x2.trans
    const int bkr = (lane & 7) + 8 * ((lane >> 3) & 1);
    const unsigned sx_s = smem_addr(sx), sg_s = smem_addr(sg);

    float acc[NTW][4];
#pragma unroll
    for (int i = 0; i < NTW; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0f;

    for (int brick = blockIdx.x; brick < nbricks; brick += gridDim.x) {
        const int bx = brick % nbx, by = (brick / nbx) % nby, bz = brick / (nbx * nby);
        load_halo<CA, CB, RS>(sx, a.xa, a.xb, a.lv, a.lc, bx * BX - 1, by * BY - 1, bz * BZ - 1);
        for (int i = tid; i < BRICK * (COUT / 8); i += THREADS) {
            const int ch = i % (COUT / 8), v = i / (COUT / 8);
            const int gx = bx * BX + (v & 7), gy = by * BY + ((v >> 3) & 7), gz = bz * BZ + (v >> 6);
            const bool in = gx < a.lv.W && gy < a.lv.H && gz < a.lv.D;
            const bf16* src = in ? a.g + blk8(a.lv.n(), (int64_t(gz) * a.lv.H + gy) * a.lv.W + gx, ch) : a.g;
            cp_async16(sg + v * GS + ch * 8, src, in);
        }
        cp_async_wait_all();
        __syncthreads();
#pragma unroll 1
        for (int ks = 0; ks < 16; ++ks) {
            const int z = ks >> 2, yy = (ks & 3) * 2;
            const int av = (z * BY + yy + (akr >> 3)) * BX + (akr & 7);
            const int bh = ((z + 1) * HY + (yy + (bkr >> 3) + 1)) * HX + ((bkr & 7) + 1);
#pragma unroll
            for (int i = 0; i < NTW; ++i) {
                const int tile = warp + 8 * i;
                if (TILES % 8 != 0 && tile >= TILES) continue;
                const int tl = tile / ((COUT / 16) * (CIN / 8));
                const int rem = tile % ((COUT / 16) * (CIN / 8));
                const int cot = rem / (CIN / 8), cit = rem % (CIN / 8);
                const int tap = tap0 + tl;
                const int toff = ((tap / 9 - 1) * HY + ((tap / 3) % 3 - 1)) * HX + (tap % 3 - 1);
                unsigned a0, a1, a2, a3, b0, b1;
                ldsm_x4_t(a0, a1, a2, a3, sg_s + (av * GS + cot * 16 + amoff) * 2);
                ldsm_x2_t(b0, b1, sx_s + ((bh + toff) * RS + cit * 8) * 2);
                mma16816(acc[i], a0, a1, a2, a3, b0, b1);
            }
        }
        __syncthreads();
    }
    const int g = lane >> 2, tq = lane & 3;
    float* part = a.part + int64_t(blockIdx.x) * 27 * COUT * CIN;
#pragma unroll
    for (int i = 0; i < NTW; ++i) {
        const int tile = warp + 8 * i;
        if (tile >= TILES) continue;
        const int tl = tile / ((COUT / 16) * (CIN / 8));
        const int rem = tile % ((COUT / 16) * (CIN / 8));
        const int cot = rem / (CIN / 8), cit = rem % (CIN / 8);
        const int tap = tap0 + tl;
        const int co = cot * 16 + g, ci = cit * 8 + 2 * tq;
        float* p0 = part + (int64_t(tap) * COUT + co) * CIN + ci;
        p0[0] = acc[i][0];
        p0[1] = acc[i][1];
        p0[8 * CIN] = acc[i][2];
        p0[8 * CIN + 1] = acc[i][3];
    }
}

__global__ void k_reduce_partials(const float* __restrict__ part, int nblk, int64_t n, float* __restrict__ out) {
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        float s = 0.0f;
        for (int b = 0; b < nblk; ++b) s += part[int64_t(b) * n + j];
        out[j] = s;
    }
}

// ---------------------------------------------------------------- small kernels
constexpr int RED_BLOCKS = 256;

template <int N>
__device__ __forceinline__ void block_sum_d(double (&v)[N], double* sh) {
    // fixed-order tree over a 256-thread block; result in thread 0's v
#pragma unroll
    for (int k = 0; k < N; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) sh[warp * N + k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double s = 0.0;
            for (int w = 0; w < THREADS / 32; ++w) s += sh[w * N + k];
            v[k] = s;
        }
    __syncthreads();
}

__device__ __forceinline__ uint8_t label_net(const uint8_t* __restrict__ lab, const Lvl& real, int i, int j, int k) {
    if (i >= real.W || j >= real.H || k >= real.D) return 0;  // padding counts as SOLID
    return lab[(int64_t(k) * real.H + j) * real.W + i];
}

__global__ void __launch_bounds__(THREADS) k_rhs_scale_part(const uint8_t* __restrict__ lab,
                                                             const float* __restrict__ rhs, Lvl real,
                                                             double* __restrict__ red) {
    __shared__ double sh[2 * THREADS / 32];
    double v[2] = {0.0, 0.0};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < real.n(); t += int64_t(gridDim.x) * blockDim.x)
        if (lab[t] == 1) {
            const double r = rhs[t];
            v[0] += r * r;
            v[1] += 1.0;
        }
    block_sum_d<2>(v, sh);
    if (threadIdx.x == 0) {
        red[blockIdx.x] = v[0];
        red[RED_BLOCKS + blockIdx.x] = v[1];
    }
}
__global__ void k_rhs_scale_final(const double* __restrict__ red, float* __restrict__ scal) {
    if (threadIdx.x != 0) return;
    double ss = 0.0, n = 0.0;
    for (int b = 0; b < RED_BLOCKS; ++b) {
        ss += red[b];
        n += red[RED_BLOCKS + b];
    }
    const double s = (n > 0.0 && ss > 0.0) ? sqrt(ss / n) : 1.0;
    scal[0] = float(s);
    scal[1] = float(1.0 / s);
}

__global__ void k_input(const uint8_t* __restrict__ lab, const float* __restrict__ rhs, Lvl real, Lvl net,
                        const float* __restrict__ scal, bf16* __restrict__ x0) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= net.n()) return;
    const int i = int(t % net.W), j = int((t / net.W) % net.H), k = int(t / (int64_t(net.W) * net.H));
    const uint8_t l = label_net(lab, real, i, j, k);
    const float c0 = l == 1 ? __fmul_rn(rhs[(int64_t(k) * real.H + j) * real.W + i], scal[1]) : 0.0f;
    __align__(16) bf16 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16_rn(0.0f);
    v[0] = __float2bfloat16_rn(c0);
    v[1] = __float2bfloat16_rn(l == 1 ? 1.0f : 0.0f);
    v[2] = __float2bfloat16_rn(l == 2 ? 1.0f : 0.0f);
    v[3] = __float2bfloat16_rn((l == 0 || l == 3) ? 1.0f : 0.0f);
    *reinterpret_cast<uint4*>(x0 + blk8(net.n(), t, 0)) = reinterpret_cast<const uint4*>(v)[0];
    *reinterpret_cast<uint4*>(x0 + blk8(net.n(), t, 1)) = reinterpret_cast<const uint4*>(v)[1];
}

__device__ __forceinline__ void load8(const bf16* p, float* f) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float2 x = __bfloat1622float2(h[q]);
        f[2 * q] = x.x;
        f[2 * q + 1] = x.y;
    }
}
__device__ __forceinline__ void store8(bf16* p, const float* f) {
    uint4 u;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
    for (int q = 0; q < 4; ++q) h[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
    *reinterpret_cast<uint4*>(p) = u;
}

// One thread per (coarse voxel, 8 channels), voxels fastest.  Fine dims are even.
__global__ void k_pool(const bf16* __restrict__ e, Lvl fine, int C, bf16* __restrict__ q) {
    const int CH = C / 8;
    const Lvl cl{fine.W / 2, fine.H / 2, fine.D / 2};
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= cl.n() * CH) return;
    const int64_t V = t % cl.n();
    const int ch = int(t / cl.n());
    const int I = int(V % cl.W), J = int((V / cl.W) % cl.H), K = int(V / (int64_t(cl.W) * cl.H));
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                float f[8];
                load8(e + blk8(fine.n(), (int64_t(2 * K + dz) * fine.H + 2 * J + dy) * fine.W + 2 * I + dx, ch), f);
#pragma unroll
                for (int c = 0; c < 8; ++c) s[c] += f[c];
            }
#pragma unroll
    for (int c = 0; c < 8; ++c) s[c] *= 0.125f;
    store8(q + blk8(cl.n(), V, ch), s);
}

// g[V][c] = (sum over the 8 children of raw[child][c]) * (act[V][c] > 0), c < C.
__global__ void k_sum_children_mask(const bf16* __restrict__ raw, Lvl fine, int ctot, int C,
                                    const bf16* __restrict__ act, bf16* __restrict__ gout) {
    const int CH = C / 8;
    const Lvl cl{fine.W / 2, fine.H / 2, fine.D / 2};
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= cl.n() * CH) return;
    const int64_t V = t % cl.n();
    const int ch = int(t / cl.n());
    const int I = int(V % cl.W), J = int((V / cl.W) % cl.H), K = int(V / (int64_t(cl.W) * cl.H));
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                float f[8];
                load8(raw + blk8(fine.n(), (int64_t(2 * K + dz) * fine.H + 2 * J + dy) * fine.W + 2 * I + dx, ch), f);
#pragma unroll
                for (int c = 0; c < 8; ++c) s[c] += f[c];
            }
    float m[8];
    load8(act + blk8(cl.n(), V, ch), m);
#pragma unroll
    for (int c = 0; c < 8; ++c) s[c] = m[c] > 0.0f ? s[c] : 0.0f;
    store8(gout + blk8(cl.n(), V, ch), s);
}

// g[v][c] = (raw[v][ca + c] + gq[v>>1][c] / 8) * (act[v][c] > 0), c < C.
__global__ void k_skip_combine(const bf16* __restrict__ raw, Lvl fine, int ctot, int ca, int C,
                               const bf16* __restrict__ gq, const bf16* __restrict__ act, bf16* __restrict__ gout) {
    const int CH = C / 8;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= fine.n() * CH) return;
    const int64_t v = t % fine.n();
    const int ch = int(t / fine.n());
    const int i = int(v % fine.W), j = int((v / fine.W) % fine.H), k = int(v / (int64_t(fine.W) * fine.H));
    const Lvl cl{fine.W / 2, fine.H / 2, fine.D / 2};
    float r[8], q[8], m[8];
    load8(raw + blk8(fine.n(), v, ca / 8 + ch), r);
    load8(gq + blk8(cl.n(), (int64_t(k >> 1) * cl.H + (j >> 1)) * cl.W + (i >> 1), ch), q);
    load8(act + blk8(fine.n(), v, ch), m);
#pragma unroll
    for (int c = 0; c < 8; ++c) r[c] = m[c] > 0.0f ? r[c] + 0.125f * q[c] : 0.0f;
    store8(gout + blk8(fine.n(), v, ch), r);
}

__global__ void __launch_bounds__(THREADS) k_loss_part(const uint8_t* __restrict__ lab, const float* __restrict__ p,
                                                        Lvl real, Lvl net, const float* __restrict__ out,
                                                        const float* __restrict__ scal, double* __restrict__ red) {
    __shared__ double sh[2 * THREADS / 32];
    double v[2] = {0.0, 0.0};
    const float inv_s = scal[1];
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < real.n();
         t += int64_t(gridDim.x) * blockDim.x) {
        if (lab[t] != 1) continue;
        const int i = int(t % real.W), j = int((t / real.W) % real.H), k = int(t / (int64_t(real.W) * real.H));
        const float tv = __fmul_rn(p[t], inv_s);
        const double e = double(out[(int64_t(k) * net.H + j) * net.W + i]) - double(tv);
        v[0] += e * e;
        v[1] += double(tv) * double(tv);
    }
    block_sum_d<2>(v, sh);
    if (threadIdx.x == 0) {
        red[blockIdx.x] = v[0];
        red[RED_BLOCKS + blockIdx.x] = v[1];
    }
}
__global__ void k_loss_final(double* __restrict__ red, float* __restrict__ scal) {
    if (threadIdx.x != 0) return;
    double ee = 0.0, tt = 0.0;
    for (int b = 0; b < RED_BLOCKS; ++b) {
        ee += red[b];
        tt += red[RED_BLOCKS + b];
    }
    if (!(tt > 0.0)) tt = 1.0;
    red[2 * RED_BLOCKS] = ee / tt;  // loss
    scal[2] = float(2.0 / tt);
}

__global__ void __launch_bounds__(THREADS) k_head_bwd(const uint8_t* __restrict__ lab, const float* __restrict__ p,
                                                       Lvl real, Lvl net, const float* __restrict__ out,
                                                       const bf16* __restrict__ d0, const float* __restrict__ hw,
                                                       const float* __restrict__ scal, bf16* __restrict__ g9,
                                                       float* __restrict__ hpart) {
    __shared__ double sh[16 * THREADS / 32];
    double hp[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) hp[c] = 0.0;
    const float inv_s = scal[1], k2 = scal[2];
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < net.n(); t += int64_t(gridDim.x) * blockDim.x) {
        const int i = int(t % net.W), j = int((t / net.W) % net.H), k = int(t / (int64_t(net.W) * net.H));
        const uint8_t l = label_net(lab, real, i, j, k);
        float go = 0.0f;
        if (l == 1) {
            const float tv = __fmul_rn(p[(int64_t(k) * real.H + j) * real.W + i], inv_s);
            go = (out[t] - tv) * k2;
        }
        float f[16], o[16];
        load8(d0 + blk8(net.n(), t, 0), f);
        load8(d0 + blk8(net.n(), t, 1), f + 8);
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            o[c] = f[c] > 0.0f ? go * hw[c] : 0.0f;
            hp[c] += double(go) * double(f[c]);
        }
        store8(g9 + blk8(net.n(), t, 0), o);
        store8(g9 + blk8(net.n(), t, 1), o + 8);
    }
    block_sum_d<16>(hp, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int c = 0; c < 16; ++c) hpart[blockIdx.x * 16 + c] = float(hp[c]);
}

__global__ void k_output_dense(const uint8_t* __restrict__ lab, Lvl real, Lvl net, const float* __restrict__ out,
                               const float* __restrict__ scal, float* __restrict__ x) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= real.n()) return;
    const int i = int(t % real.W), j = int((t / real.W) % real.H), k = int(t / (int64_t(real.W) * real.H));
    x[t] = lab[t] == 1 ? out[(int64_t(k) * net.H + j) * net.W + i] * scal[0] : 0.0f;
}

__global__ void k_output_compact(const int* __restrict__ nf_p, const int* __restrict__ fidx, Lvl real, Lvl net,
                                 const float* __restrict__ out, const float* __restrict__ scal,
                                 float* __restrict__ x0) {
    const int nf = *nf_p;
    const float s = scal[0];
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) {
        const int c = fidx[n];
        const int i = c % (real.W + 2) - 1, j = (c / (real.W + 2)) % (real.H + 2) - 1,
                  k = c / ((real.W + 2) * (real.H + 2)) - 1;
        x0[n] = out[(int64_t(k) * net.H + j) * net.W + i] * s;
    }
}

__global__ void k_rhs_dense(const int* __restrict__ nf_p, const int* __restrict__ fidx, Lvl real,
                            const float* __restrict__ b, float* __restrict__ dense) {
    const int nf = *nf_p;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += gridDim.x * blockDim.x) {
        const int c = fidx[n];
        const int i = c % (real.W + 2) - 1, j = (c / (real.W + 2)) % (real.H + 2) - 1,
                  k = c / ((real.W + 2) * (real.H + 2)) - 1;
        dense[(int64_t(k) * real.H + j) * real.W + i] = b[n];
    }
}

// Global gradient norm (fixed-order, FP64) and the clipping factor
// min(1, clip / norm) in scal[3]; the norm itself goes to red[2 * RED_BLOCKS + 1].
__global__ void __launch_bounds__(THREADS) k_gnorm_part(const float* __restrict__ g, int64_t n,
                                                         double* __restrict__ red) {
    __shared__ double sh[THREADS / 32];
    double v[1] = {0.0};
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        v[0] += double(g[i]) * double(g[i]);
    block_sum_d<1>(v, sh);
    if (threadIdx.x == 0) red[blockIdx.x] = v[0];
}
__global__ void k_gnorm_final(double* __restrict__ red, float clip, float* __restrict__ scal) {
    if (threadIdx.x != 0) return;
    double ss = 0.0;
    for (int b = 0; b < RED_BLOCKS; ++b) ss += red[b];
    const double nrm = sqrt(ss);
    red[2 * RED_BLOCKS + 1] = nrm;
    scal[3] = (nrm > double(clip) && isfinite(nrm)) ? float(double(clip) / nrm) : (isfinite(nrm) ? 1.0f : 0.0f);
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, const float* __restrict__ scal, int64_t n, float lr, float b1,
                       float b2, float eps, float bc1, float bc2) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] * scal[3];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// BF16 copies of the 3x3x3 weights: wf in the forward layout [t][co][ci] and
// wt, the backward-data layout [26 - t][ci][co].
struct LayerTable {
    int64_t off[kLayers + 1];
    int cin[kLayers], cout[kLayers];
};
__global__ void k_weights_bf16(const float* __restrict__ w, bf16* __restrict__ wf, bf16* __restrict__ wt,
                               LayerTable lt) {
    const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= lt.off[kLayers]) return;
    int l = 0;
    while (l + 1 < kLayers && idx >= lt.off[l + 1]) ++l;
    const int64_t r = idx - lt.off[l];
    const int cin = lt.cin[l], cout = lt.cout[l];
    const int ci = int(r % cin), co = int((r / cin) % cout), t = int(r / (int64_t(cin) * cout));
    const bf16 b = __float2bfloat16_rn(w[idx]);
    wf[idx] = b;
    wt[lt.off[l] + (int64_t(26 - t) * cin + ci) * cout + co] = b;
}

// ---------------------------------------------------------------- dispatch
int sm_count() {
    static DeviceMemo memo;
    const int n = memo.get([](int dev) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        return std::max(sms, 0);
    });
    return n > 0 ? n : 148;
}

int nbricks_of(const Lvl& lv) {
    return ((lv.W + BX - 1) / BX) * ((lv.H + BY - 1) / BY) * ((lv.D + BZ - 1) / BZ);
}

template <int CA, int CB, int COUT, int TPC>
int run_corr(const CorrArgs& a, int nblk, cudaStream_t st) {
    constexpr int CIN = CA + CB;
    constexpr size_t smem = size_t(HALO * (CIN + 8) + BRICK * (COUT + 8)) * sizeof(bf16);
    static DeviceMemo memo;
    auto kern = k_corr3<CA, CB, COUT, TPC>;
    memo.get([&](int) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        return 1;
    });
    kern<<<dim3(nblk, 27 / TPC), THREADS, smem, st>>>(a);
    return int(cudaPeekAtLastError());
}

constexpr int kTpc[kLayers] = {27, 27, 9, 9, 3, 3, 3, 9, 9, 27};

}  // namespace

int corr_blocks(int layer, const Lvl& lv) {
    const int groups = 27 / kTpc[layer];
    return std::max(1, std::min(nbricks_of(lv), 2 * sm_count() / groups));
}

int corr_layer(int layer, const CorrArgs& a, int nblk, cudaStream_t st) {
    switch (layer) {
        case 0: case 1: case 9: return run_corr<0, 16, 16, 27>(a, nblk, st);
        case 2: return run_corr<0, 16, 32, 9>(a, nblk, st);
        case 3: case 7: return run_corr<0, 32, 32, 9>(a, nblk, st);
        case 4: return run_corr<0, 32, 64, 3>(a, nblk, st);
        case 5: return run_corr<0, 64, 64, 3>(a, nblk, st);
        case 6: return run_corr<64, 32, 32, 3>(a, nblk, st);
        case 8: return run_corr<32, 16, 16, 9>(a, nblk, st);
    }
    return int(cudaErrorInvalidValue);
}

void reduce_partials(const float* part, int nblk, int64_t n, float* out, cudaStream_t st) {
    const int blocks = int(std::min<int64_t>((n + 255) / 256, 4 * sm_count()));
    k_reduce_partials<<<blocks, 256, 0, st>>>(part, nblk, n, out);
}

void launch_rhs_scale(const uint8_t* labels, const float* rhs, Lvl real, double* red, float* scal, cudaStream_t st) {
    k_rhs_scale_part<<<RED_BLOCKS, THREADS, 0, st>>>(labels, rhs, real, red);
    k_rhs_scale_final<<<1, 32, 0, st>>>(red, scal);
}

void launch_input(const uint8_t* labels, const float* rhs, Lvl real, Lvl net, const float* scal, bf16* x0,
                  cudaStream_t st) {
    k_input<<<unsigned((net.n() + 255) / 256), 256, 0, st>>>(labels, rhs, real, net, scal, x0);
}

void launch_pool(const bf16* e, Lvl fine, int C, bf16* q, cudaStream_t st) {
    const int64_t n = fine.n() / 8 * (C / 8);
    k_pool<<<unsigned((n + 255) / 256), 256, 0, st>>>(e, fine, C, q);
}

void launch_sum_children_mask(const bf16* raw, Lvl fine, int ctot, int C, const bf16* act, bf16* g, cudaStream_t st) {
    const int64_t n = fine.n() / 8 * (C / 8);
    k_sum_children_mask<<<unsigned((n + 255) / 256), 256, 0, st>>>(raw, fine, ctot, C, act, g);
}

void launch_skip_combine(const bf16* raw, Lvl fine, int ctot, int ca, int C, const bf16* gq, const bf16* act,
                         bf16* g, cudaStream_t st) {
    const int64_t n = fine.n() * (C / 8);
    k_skip_combine<<<unsigned((n + 255) / 256), 256, 0, st>>>(raw, fine, ctot, ca, C, gq, act, g);
}

void launch_loss(const uint8_t* labels, const float* p, Lvl real, Lvl net, const float* out, double* red, float* scal,
                 cudaStream_t st) {
    k_loss_part<<<RED_BLOCKS, THREADS, 0, st>>>(labels, p, real, net, out, scal, red);
    k_loss_final<<<1, 32, 0, st>>>(red, scal);
}

int head_blocks(Lvl net) { return int(std::min<int64_t>((net.n() + THREADS - 1) / THREADS, 2 * sm_count())); }

void launch_head_backward(const uint8_t* labels, const float* p, Lvl real, Lvl net, const float* out, const bf16* d0,
                          const float* head_w, const float* scal, bf16* g9, float* head_part, int nblk,
                          cudaStream_t st) {
    k_head_bwd<<<nblk, THREADS, 0, st>>>(labels, p, real, net, out, d0, head_w, scal, g9, head_part);
}

void launch_output_dense(const uint8_t* labels, Lvl real, Lvl net, const float* out, const float* scal, float* x,
                         cudaStream_t st) {
    k_output_dense<<<unsigned((real.n() + 255) / 256), 256, 0, st>>>(labels, real, net, out, scal, x);
}

void launch_output_compact(const int* nf, const int* fidx, Lvl real, Lvl net, const float* out, const float* scal,
                           float* x0, cudaStream_t st) {
    k_output_compact<<<4 * sm_count(), 256, 0, st>>>(nf, fidx, real, net, out, scal, x0);
}

void launch_rhs_dense(const int* nf, const int* fidx, Lvl real, const float* b, float* dense, cudaStream_t st) {
    cudaMemsetAsync(dense, 0, sizeof(float) * size_t(real.n()), st);
    k_rhs_dense<<<4 * sm_count(), 256, 0, st>>>(nf, fidx, real, b, dense);
}

void launch_adam(float* w, float* m, float* v, const float* g, int64_t n, float lr, float b1, float b2, float eps,
                 float bc1, float bc2, float clip, double* red, float* scal, cudaStream_t st) {
    k_gnorm_part<<<RED_BLOCKS, THREADS, 0, st>>>(g, n, red);
    k_gnorm_final<<<1, 32, 0, st>>>(red, clip, scal);
    k_adam<<<unsigned((n + 255) / 256), 256, 0, st>>>(w, m, v, g, scal, n, lr, b1, b2, eps, bc1, bc2);
}

void launch_weights_bf16(const float* w32, bf16* wf, bf16* wt, cudaStream_t st) {
    LayerTable lt;
    for (int l = 0; l <= kLayers; ++l) lt.off[l] = layer_offset(l);
    for (int l = 0; l < kLayers; ++l) {
        lt.cin[l] = kSpec[l].ca + kSpec[l].cb;
        lt.cout[l] = kSpec[l].cout;
    }
    const int64_t n = lt.off[kLayers];
    k_weights_bf16<<<unsigned((n + 255) / 256), 256, 0, st>>>(w32, wf, wt, lt);
}

}  // namespace unet
}  // namespace fp
