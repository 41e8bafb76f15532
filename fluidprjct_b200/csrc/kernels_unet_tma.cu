// kernels_unet_tma.cu -- the U-Net's 3x3x3 convolutions on the fifth-generation
// tensor cores, fed by the Tensor Memory Accelerator.
//
// One persistent CTA walks output bricks of 8x16x4 voxels (four M = 128
// tiles: row m of a tile is voxel (x = m % 8, y = m / 8) of one z slice) in
// 16-channel input groups.  With N = 16 one MMA is too small to hide its
// latency, so the four tiles' accumulation chains are interleaved.  Five warps, each with one job:
//   warp 4, one thread: the producer and MMA issuer.  For each step (brick,
//     group) it waits until a shared-memory stage is free, then loads the
//     group's zero-padded halo with two TMA tensor loads.  Each load is one
//     8-channel plane of a 10x18x6 box; TMA fills the out-of-grid part with
//     zeros.  NST - 1 steps behind the loads, it issues the step's 27 tap MMAs
//     per tile (tcgen05.mma kind::f16, M = 128, N = NCO, K = 16) into the
//     brick's TMEM accumulator set, and commits them to the stage's "empty"
//     barrier (and, after the brick's last group, to the set's "full" barrier).
//   warps 0-3: the epilogue.  Each reads its 32 TMEM lanes (tcgen05.ld
//     32x32b): every thread holds one voxel's NCO outputs, applies ReLU, the
//     backward mask or the fused 16->1 head, and stores 16-byte vectors.  Then
//     it frees the accumulator set.  There are two sets, so a brick's epilogue
//     overlaps the next brick's MMAs.
// A TMA box plane is exactly the K-major no-swizzle UMMA layout ([halo voxel]
// rows of 8 channels = 16 bytes): the operand of tap (dz, dy, dx) is the plane
// shifted by the tap's halo offset, with core matrices of successive y rows
// 160 bytes apart (SBO) and the two 8-channel halves of a K step one plane
// apart (LBO).  The CTA's output-channel group of the weights ([tap][chunk]
// [co][8], the K-major layout of B) is staged once and stays resident.
// Every wait is bounded; a wait that gives up sets *status, the CTA stops
// issuing, waits (bounded) for its own MMAs, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "device_memo.hpp"
#include "unet.hpp"

namespace fp {
namespace unet {
namespace {

constexpr int TX = 8, TY = 16, TZ = 4;           // brick: four 128-voxel tiles, four MMA chains
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2;
constexpr int HVOX = HX * HY * HZ;             // 1080 halo voxels
constexpr int PLANE_BYTES = HVOX * 16;         // one 8-channel plane: 17,280 bytes
constexpr int STAGE_BYTES = 2 * PLANE_BYTES;   // one 16-channel group
constexpr int EPI_THREADS = 128, THREADS = 160;
constexpr long long kSpinLimit = 1ll << 26;
constexpr int DEV_TIMEOUT_CODE = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity) {
    for (long long i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;\n" ::"r"(bytes), "r"(mbar) : "memory");
}
// One 4D tensor tile (channels, x, y, z) into shared memory, completing on mbar.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t mbar, int c, int x, int y,
                                            int z) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(mbar), "r"(c), "r"(x), "r"(y), "r"(z)
        : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Layers with 16 output channels stack the three z taps in N ("dz in N"):
// halo plane p (0 <= p < HZ), shifted by (dy, dx), is multiplied once by
// [W(dz=-1); W(0); W(+1)] (N = 48) into its own 48 accumulator columns; the
// dz block of plane p feeds output tile zo = p - 1 - dz.  Output tile zo adds
// plane zo's dz=-1 block, plane zo+1's dz=0 block and plane zo+2's dz=+1
// block: the same TMEM lanes, so the sum stays in one thread.  Each A tile is
// read 9 times per group instead of 27, which is what the 16-wide MMAs are
// bound by (their shared-memory operand reads).  Every MMA has the same shape
// (changing N between consecutive MMAs stalls the tensor pipe).  The edge
// planes' unused dz blocks overlap in pairs: plane 0 uses only dz = -1 and
// plane 5 only dz = +1, plane 1 drops dz = +1 and plane 4 dz = -1, so one
// set needs 240 columns instead of 288:
//   plane   0    5    1    4    2    3
//   column  0   16   64   96  144  192     (blocks of 16 per dz = -1, 0, +1)
static_assert(TZ == 4, "the dz-in-N column table is laid out for four tiles");
__host__ __device__ constexpr int dzn_col(int p) {
    return p == 0 ? 0 : p == 5 ? 16 : p == 1 ? 64 : p == 4 ? 96 : p == 2 ? 144 : 192;
}
constexpr int DZN_SET_COLS = 240;
// first column of output tile zo's dz partial
__host__ __device__ constexpr int dzn_block_col(int zo, int dz) { return dzn_col(zo + 1 + dz) + (dz + 1) * 16; }

// NSET accumulator sets of TZ tiles x NCO columns, or of the dz-in-N
// blocks, allocated as a power of two >= 32.  Two sets let a brick's
// epilogue overlap the next brick's MMAs inside the CTA; one set leaves
// room for two CTAs per SM, whose MMA streams then interleave.
template <int NCO>
constexpr int set_cols() { return NCO == 16 ? DZN_SET_COLS : TZ * NCO; }
template <int NCO, int NSET>
constexpr int tmem_cols() {
    constexpr int c = NSET * set_cols<NCO>();
    return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512;
}
template <int CIN, int NCO, int NST>
constexpr size_t smem_bytes() {
    // stages + weights + barriers (2 NST + 5) and the TMEM slot + 128-byte alignment slack
    return size_t(NST) * STAGE_BYTES + size_t(27) * CIN * NCO * 2 + 8 * (2 * NST + 5) + 16 + 128;
}

template <int CIN, int COUT, int NCO, int EPI, int NST, int NSET>
__global__ void __launch_bounds__(THREADS) k_conv3_tma(const __grid_constant__ CUtensorMap tin, TmaConvArgs a) {
    constexpr int G = CIN / 16;
    // loads issued ahead of the MMAs; with four or more stages two MMA batches
    // stay in flight (the stage wait then covers the batch before the last)
    constexpr int LA = NST >= 4 ? NST - 2 : NST - 1;
    constexpr int NCOLS = tmem_cols<NCO, NSET>();
    static_assert(NSET == 1 || NSET == 2, "accumulator sets");
    constexpr bool DZN = NCO == 16;
    constexpr uint32_t SET = uint32_t(set_cols<NCO>());
    constexpr uint32_t IDESC = umma_idesc_bf16(NCO);
    static_assert(CIN % 16 == 0 && NCO % 16 == 0 && NCO <= 48 && COUT % NCO == 0 && NST >= 2, "tiling");
    static_assert(EPI != EPI_HEAD || (NCO == 16 && COUT == 16), "the head needs all 16 channels");
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 127u) & ~127u;
    unsigned char* sbase = smem_raw + (base - raw);
    const uint32_t sStage = base;
    const uint32_t sB = base + uint32_t(NST * STAGE_BYTES);
    const uint32_t bars = sB + uint32_t(27 * CIN * NCO * 2);
    // barriers, 8 bytes each: full[NST], empty[NST], acc_full[2], acc_empty[2], spare
    const uint32_t full0 = bars, empty0 = bars + 8u * NST, accf0 = bars + 16u * NST, acce0 = accf0 + 16u;
    const uint32_t spare = acce0 + 16u;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sbase + (NST * STAGE_BYTES + 27 * CIN * NCO * 2 + 8 * (2 * NST + 5)));
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cog = blockIdx.y;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(NCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        s_abort = 0;
        for (int q = 0; q < NST; ++q) {
            mbar_init(full0 + 8u * q, 1);
            mbar_init(empty0 + 8u * q, 1);
        }
        for (int q = 0; q < 2; ++q) {
            mbar_init(accf0 + 8u * q, 1);
            mbar_init(acce0 + 8u * q, EPI_THREADS / 32);
        }
        mbar_init(spare, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // weights, K-major: [tap][chunk][co][8], or [dy,dx][chunk][dz][co][8] for dz in N
    for (int i = tid; i < 27 * NCO * (CIN / 8); i += THREADS) {
        int co, c, tap;
        if constexpr (DZN) {
            co = i % 16;
            const int dz = (i / 16) % 3;
            c = (i / 48) % (CIN / 8);
            tap = dz * 9 + i / (48 * (CIN / 8));
        } else {
            co = i % NCO;
            c = (i / NCO) % (CIN / 8);
            tap = i / (NCO * (CIN / 8));
        }
        cp_async16(sB + uint32_t(i * 16), a.w + (int64_t(tap) * COUT + cog * NCO + co) * CIN + c * 8);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;

    const int nbx = (a.lv.W + TX - 1) / TX, nby = (a.lv.H + TY - 1) / TY, nbz = (a.lv.D + TZ - 1) / TZ;
    const int nbricks = nbx * nby * nbz;
    const int mine = int(blockIdx.x) < nbricks ? (nbricks - 1 - int(blockIdx.x)) / int(gridDim.x) + 1 : 0;
    const int steps = mine * G;

    if (warp == 4) {
        if (lane == 0) {
            bool ok = true;
            auto fail = [&]() {
                ok = false;
                if (a.status) atomicExch(a.status, DEV_TIMEOUT_CODE);
                atomicExch(&s_abort, 1);
            };
            auto mma_step = [&](int t) {
                const int sl = t % NST, use = t / NST, i = t / G, g = t % G;
                if (!mbar_wait_bounded(full0 + 8u * sl, uint32_t(use & 1))) return fail();
                if (g == 0 && i >= NSET &&
                    !mbar_wait_bounded(acce0 + 8u * (i % NSET), uint32_t((i / NSET - 1) & 1)))
                    return fail();
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t stage = sStage + uint32_t(sl * STAGE_BYTES);
                const uint32_t set = uint32_t(i % NSET) * SET;
                if constexpr (DZN) {
                    // shifts outer, planes inner: six accumulation chains interleave
#pragma unroll 1
                    for (int sh = 0; sh < 9; ++sh) {
                        const int dy = sh / 3 - 1, dx = sh % 3 - 1;
                        const uint64_t bd =
                            umma_desc(sB + uint32_t((sh * (CIN / 8) + 2 * g) * 3 * 16 * 16), 3 * 16 * 16, 128);
#pragma unroll
                        for (int p = 0; p < HZ; ++p) {
                            const int hv0 = (p * HY + (1 + dy)) * HX + (1 + dx);
                            const uint64_t ad = umma_desc(stage + uint32_t(hv0 * 16), PLANE_BYTES, HX * 16);
                            umma_bf16(tmem + set + uint32_t(dzn_col(p)), ad, bd, umma_idesc_bf16(48),
                                      (g | sh) != 0 ? 1u : 0u);
                        }
                    }
                } else {
                    // taps outer, tiles inner: the tiles' accumulation chains interleave
#pragma unroll 1
                    for (int tap = 0; tap < 27; ++tap) {
                        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                        const uint64_t bd = umma_desc(sB + uint32_t((tap * (CIN / 8) + 2 * g) * NCO * 16), NCO * 16, 128);
#pragma unroll
                        for (int zo = 0; zo < TZ; ++zo) {
                            const int hv0 = ((zo + 1 + dz) * HY + (1 + dy)) * HX + (1 + dx);
                            const uint64_t ad = umma_desc(stage + uint32_t(hv0 * 16), PLANE_BYTES, HX * 16);
                            umma_bf16(tmem + set + uint32_t(zo * NCO), ad, bd, IDESC, (g | tap) != 0 ? 1u : 0u);
                        }
                    }
                }
                umma_commit(empty0 + 8u * sl);
                if (g == G - 1) umma_commit(accf0 + 8u * (i % NSET));
            };
            for (int s = 0; s < steps && ok; ++s) {
                const int sl = s % NST, use = s / NST, i = s / G, g = s % G;
                if (use >= 1 && !mbar_wait_bounded(empty0 + 8u * sl, uint32_t((use - 1) & 1))) {
                    fail();
                    break;
                }
                const int brick = int(blockIdx.x) + i * int(gridDim.x);
                const int bx = brick % nbx, by = (brick / nbx) % nby, bz = brick / (nbx * nby);
                const uint32_t stage = sStage + uint32_t(sl * STAGE_BYTES);
                mbar_expect_tx(full0 + 8u * sl, STAGE_BYTES);
                // (8 channels x 10 voxels) rows of 160 bytes; x = 8 (bx TX - 1) is a multiple of 8 elements
                tma_load_4d(stage, &tin, full0 + 8u * sl, 8 * (bx * TX - 1), by * TY - 1, bz * TZ - 1, 2 * g);
                tma_load_4d(stage + PLANE_BYTES, &tin, full0 + 8u * sl, 8 * (bx * TX - 1), by * TY - 1, bz * TZ - 1,
                            2 * g + 1);
                if (s >= LA) mma_step(s - LA);
            }
            for (int t = max(0, steps - LA); t < steps && ok; ++t) mma_step(t);
            if (!ok) {
                // one more bounded wait: the spare barrier completes once every
                // MMA issued so far has completed
                umma_commit(spare);
                mbar_wait_bounded(spare, 0u);
            }
        }
    } else {
        // epilogue warps: TMEM lanes 32 * warp .. 32 * warp + 31
        for (int i = 0; i < mine; ++i) {
            bool got = true;
            if (lane == 0) got = mbar_wait_bounded(accf0 + 8u * (i % NSET), uint32_t((i / NSET) & 1));
            got = __shfl_sync(0xffffffffu, got ? 1 : 0, 0) != 0;
            if (!got || *(volatile int*)&s_abort) {
                if (lane == 0 && !got && a.status) atomicExch(a.status, DEV_TIMEOUT_CODE);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const int brick = int(blockIdx.x) + i * int(gridDim.x);
            const int bx = brick % nbx, by = (brick / nbx) % nby, bz = brick / (nbx * nby);
            const uint32_t set = uint32_t(i % NSET) * SET;
            const uint32_t lanes = tmem + (uint32_t(warp * 32) << 16) + set;
#pragma unroll
            for (int zo = 0; zo < TZ; ++zo) {
                float v[NCO];
                if constexpr (DZN) {
                    float v1[16], v2[16];
                    tmem_ld16(lanes + uint32_t(dzn_block_col(zo, -1)), v);
                    tmem_ld16(lanes + uint32_t(dzn_block_col(zo, 0)), v1);
                    tmem_ld16(lanes + uint32_t(dzn_block_col(zo, 1)), v2);
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                    for (int q = 0; q < 16; ++q) v[q] = (v[q] + v1[q]) + v2[q];
                } else {
#pragma unroll
                    for (int j = 0; j < NCO / 16; ++j) tmem_ld16(lanes + uint32_t(zo * NCO + 16 * j), v + 16 * j);
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                }
                const int m = warp * 32 + lane;
                const int gx = bx * TX + (m & 7), gy = by * TY + (m >> 3), gz = bz * TZ + zo;
                if (gx >= a.lv.W || gy >= a.lv.H || gz >= a.lv.D) continue;
                const int64_t vox = (int64_t(gz) * a.lv.H + gy) * a.lv.W + gx;
                const int64_t nv = a.lv.n();
                if (EPI == EPI_RELU || EPI == EPI_HEAD) {
#pragma unroll
                    for (int q = 0; q < NCO; ++q) v[q] = fmaxf(v[q], 0.0f);
                }
                if (EPI == EPI_MASK) {
#pragma unroll
                    for (int q = 0; q < NCO / 8; ++q) {
                        const uint4 mk = *reinterpret_cast<const uint4*>(a.mask + blk8(nv, vox, cog * (NCO / 8) + q));
                        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&mk);
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float2 f = __bfloat1622float2(h[e]);
                            if (!(f.x > 0.0f)) v[8 * q + 2 * e] = 0.0f;
                            if (!(f.y > 0.0f)) v[8 * q + 2 * e + 1] = 0.0f;
                        }
                    }
                }
                float hsum = 0.0f;
#pragma unroll
                for (int q = 0; q < NCO / 8; ++q) {
                    uint4 u;
                    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        h[e] = __floats2bfloat162_rn(v[8 * q + 2 * e], v[8 * q + 2 * e + 1]);
                        if (EPI == EPI_HEAD) {
                            const float2 f = __bfloat1622float2(h[e]);
                            hsum += f.x * a.head_w[8 * q + 2 * e] + f.y * a.head_w[8 * q + 2 * e + 1];
                        }
                    }
                    *reinterpret_cast<uint4*>(a.y + blk8(nv, vox, cog * (NCO / 8) + q)) = u;
                }
                if (EPI == EPI_HEAD) a.head_out[vox] = hsum;
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(acce0 + 8u * (i % NSET));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(NCOLS));
}

// up2(coarse) into the first ca / 8 channel blocks of a decoder layer's input
// [up2(coarse) | skip]; the skip tensor already lives in the blocks after
// them.  One thread per (fine voxel, 8 channels), voxels fastest.
__global__ void k_upcat(const bf16* __restrict__ coarse, int ca, Lvl fine, bf16* __restrict__ out) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= fine.n() * (ca / 8)) return;
    const int64_t v = t % fine.n();
    const int c = int(t / fine.n());
    const int i = int(v % fine.W), j = int((v / fine.W) % fine.H), k = int(v / (int64_t(fine.W) * fine.H));
    const Lvl cl{fine.W / 2, fine.H / 2, fine.D / 2};
    *reinterpret_cast<uint4*>(out + blk8(fine.n(), v, c)) = *reinterpret_cast<const uint4*>(
        coarse + blk8(cl.n(), (int64_t(k >> 1) * cl.H + (j >> 1)) * cl.W + (i >> 1), c));
}

// ---- host side
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    return g_encode;
}

// Tensor map of a channel-blocked [C/8][D][H][W][8] bf16 tensor seen as
// (8 W, H, D, C / 8): one box is an 8-channel halo plane of HX x HY x HZ
// voxels, HY * HZ rows of 160 contiguous bytes.
bool make_map(CUtensorMap* map, const bf16* ptr, int C, const Lvl& lv) {
    auto enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[4] = {cuuint64_t(lv.W) * 8, cuuint64_t(lv.H), cuuint64_t(lv.D), cuuint64_t(C / 8)};
    const cuuint64_t strides[3] = {cuuint64_t(lv.W) * 16, cuuint64_t(lv.H) * lv.W * 16,
                                   cuuint64_t(lv.D) * lv.H * lv.W * 16};
    const cuuint32_t box[4] = {8 * HX, HY, HZ, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(ptr), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Pipelines: wide layers (NCO >= 32) run two CTAs per SM with two stages and
// two accumulator sets; 16-wide layers with CIN <= 48 run two CTAs per SM
// with one set; wider inputs run one CTA per SM with two sets and 4-5 stages.
template <int CIN, int NCO>
constexpr int pick_nst() { return NCO != 16 || CIN <= 48 ? 2 : CIN <= 64 ? 5 : 4; }
template <int CIN, int NCO>
constexpr int pick_nset() { return NCO == 16 && CIN <= 48 ? 1 : 2; }

template <int CIN, int COUT, int NCO, int EPI, int NST = pick_nst<CIN, NCO>(), int NSET = pick_nset<CIN, NCO>()>
int run_tma(const bf16* in, const TmaConvArgs& a, cudaStream_t st) {
    constexpr size_t smem = smem_bytes<CIN, NCO, NST>();
    static_assert(smem <= 232448, "shared memory of one CTA");
    static DeviceMemo memo;
    auto kern = k_conv3_tma<CIN, COUT, NCO, EPI, NST, NSET>;
    // resident CTAs on the device: shared memory (1 KB reserved per CTA),
    // threads and the 512 TMEM columns per SM (the CTAs never wait on each
    // other, so a grid above the true residency only queues)
    const int resident = memo.get([&](int dev) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        int sms = 0, smem_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        if (smem_sm <= 0) smem_sm = 233472;
        return sms * std::max(1, std::min({smem_sm / int(smem + 1024), 2048 / THREADS,
                                           512 / tmem_cols<NCO, NSET>()}));
    });
    CUtensorMap map;
    std::memset(&map, 0, sizeof map);
    if (!make_map(&map, in, CIN, a.lv)) return int(cudaErrorNotSupported);
    const int groups = COUT / NCO;
    const int nb = ((a.lv.W + TX - 1) / TX) * ((a.lv.H + TY - 1) / TY) * ((a.lv.D + TZ - 1) / TZ);
    const int gx = std::max(1, std::min(nb, resident / groups));
    kern<<<dim3(gx, groups), THREADS, smem, st>>>(map, a);
    return int(cudaPeekAtLastError());
}

}  // namespace

// Every layer runs in 16-channel output groups (blockIdx.y): the dz-in-N
// MMAs, and for CIN <= 48 two CTAs per SM.
int conv_forward_layer_tma(int layer, const bf16* in, const TmaConvArgs& a, cudaStream_t st) {
    switch (layer) {
        case 0: case 1: return run_tma<16, 16, 16, EPI_RELU>(in, a, st);
        case 2: return run_tma<16, 32, 16, EPI_RELU>(in, a, st);
        case 3: case 7: return run_tma<32, 32, 16, EPI_RELU>(in, a, st);
        case 4: return run_tma<32, 64, 16, EPI_RELU>(in, a, st);
        case 5: return run_tma<64, 64, 16, EPI_RELU>(in, a, st);
        case 6: return run_tma<96, 32, 16, EPI_RELU>(in, a, st);
        case 8: return run_tma<48, 16, 16, EPI_RELU>(in, a, st);
        case 9: return run_tma<16, 16, 16, EPI_HEAD>(in, a, st);
    }
    return int(cudaErrorInvalidValue);
}

int conv_backward_layer_tma(int layer, const bf16* in, const TmaConvArgs& a, cudaStream_t st) {
    switch (layer) {
        case 9: case 1: return run_tma<16, 16, 16, EPI_MASK>(in, a, st);
        case 8: return run_tma<16, 48, 16, EPI_RAW>(in, a, st);
        case 7: case 3: return run_tma<32, 32, 16, EPI_MASK>(in, a, st);
        case 6: return run_tma<32, 96, 16, EPI_RAW>(in, a, st);
        case 5: return run_tma<64, 64, 16, EPI_MASK>(in, a, st);
        case 4: return run_tma<64, 32, 16, EPI_RAW>(in, a, st);
        case 2: return run_tma<32, 16, 16, EPI_RAW>(in, a, st);
    }
    return int(cudaErrorInvalidValue);
}

void launch_upcat(const bf16* coarse, int ca, Lvl fine, bf16* out, cudaStream_t st) {
    const int64_t n = fine.n() * (ca / 8);
    k_upcat<<<unsigned((n + 255) / 256), 256, 0, st>>>(coarse, ca, fine, out);
}

}  // namespace unet
}  // namespace fp
