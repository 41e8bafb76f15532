// kernels_unet_tc.cu -- the U-Net's 3x3x3 convolutions on the fifth-generation
// tensor cores (tcgen05.mma, BF16 operands from shared memory, FP32
// accumulators in tensor memory).
//
// One persistent CTA of 128 threads walks output bricks of 8x16x2 voxels.
// A brick is two M = 128 tiles, one per z slice: row m of a tile is the voxel
// (x = m % 8, y = m / 8).  Per brick and 16-channel input group:
//   1. all threads stage that group of the zero-padded input halo (10x18x4
//      voxels) in one of two shared-memory stages with cp.async.  The layout is
//      chunk-major ([8-channel chunk][halo voxel][8 channels]), the K-major
//      no-swizzle UMMA layout: any 8 consecutive voxels of a halo row form one
//      8x16-byte core matrix.  The operand of tap (dz, dy, dx) is then the
//      same layout shifted by that tap's halo offset: core matrices of
//      successive y rows lie 160 bytes apart (SBO), the two K halves of a
//      16-channel step one chunk plane apart (LBO).
//   2. one thread issues the group's 27 tap MMAs per tile (M = 128, N = NCO,
//      K = 16) into the brick's TMEM accumulator set, then commits them to
//      the stage's mbarrier; loading the next group overlaps these MMAs.
//   3. once the brick's last commit has arrived, each warp reads its 32 TMEM lanes
//      (tcgen05.ld 32x32b): every thread then holds one voxel's NCO outputs
//      and writes them as contiguous 16-byte vectors.  Two accumulator sets
//      let this epilogue overlap the next brick's MMAs.
// The CTA's output-channel group of the weights ([tap][chunk][co][8], the
// K-major layout of B) is loaded once and stays resident.  The waits are
// bounded: a wait that gives up sets *status, waits again (bounded) for the
// CTA's own MMAs, frees the TMEM and returns.
#include <algorithm>

#include "unet.hpp"

namespace fp {
namespace unet {
namespace {

constexpr int TX = 8, TY = 16, TZ = 2;                 // brick (two 128-voxel tiles)
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2;   // 10 x 18 x 4 halo
constexpr int HVOX = HX * HY * HZ;                     // 720
constexpr int TC_THREADS = 128;
constexpr long long kSpinLimit = 1ll << 26;            // mbarrier polls before giving up
constexpr int DEV_TIMEOUT_CODE = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool pred) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(pred ? 16 : 0));
}

// UMMA shared-memory descriptor, K-major, no swizzle (sm_100 layout: start
// address, leading and stride byte offsets in 16-byte units, version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor: D FP32, A and B BF16, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}

// D (+)= A * B^T with every output lane enabled (zero disable-lane mask).
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
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

// Thread 0 alone polls the barrier (bounded); the other warps wait at the
// block barrier, which costs them no issue slots.  Every thread returns the
// same verdict.
__device__ __forceinline__ bool block_wait(uint32_t mbar, uint32_t parity) {
    int got = 1;
    if (threadIdx.x == 0) got = mbar_wait_bounded(mbar, parity) ? 1 : 0;
    return __syncthreads_and(got) != 0;
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

// Two accumulator sets (one per brick in flight), each two tiles of NCO columns.
template <int NCO>
constexpr int tmem_cols() {
    return (4 * NCO <= 32) ? 32 : (4 * NCO <= 64) ? 64 : (4 * NCO <= 128) ? 128 : 256;
}

constexpr int STAGE_BYTES = HVOX * 2 * 16;  // one 16-channel K group of the halo: 23,040 bytes

template <int CA, int CB, int COUT, int NCO, int NST>
constexpr size_t tc_smem_bytes() {
    // NST halo stages + resident weights + five mbarriers and the TMEM slot + alignment slack
    return size_t(NST) * STAGE_BYTES + size_t(27) * (CA + CB) * NCO * 2 + 48 + 128;
}

// Pipeline of one CTA: the steps are (brick i, 16-channel group g) in order.
// Step s loads its group's halo into stage s % NST; with two stages that load
// overlaps the MMAs of step s - 1.  A stage is reused once the MMAs that read
// it have completed (commit to that stage's mbarrier).  One stage keeps the
// footprint small, so that more CTAs share an SM and overlap each other.  Brick i accumulates into TMEM set i & 1; its
// epilogue runs after the first MMAs of brick i + 1 are issued, once the
// commit after its last group has arrived on that set's mbarrier.
template <int CA, int CB, int COUT, int NCO, int EPI, int NST>
__global__ void __launch_bounds__(TC_THREADS) k_conv3_tc(ConvArgs a) {
    constexpr int CIN = CA + CB;
    constexpr int G = CIN / 16;  // K groups per brick
    constexpr int NCOLS = tmem_cols<NCO>();
    constexpr uint32_t IDESC = umma_idesc_bf16(NCO);
    static_assert(CIN % 16 == 0 && NCO % 16 == 0 && NCO <= 48 && COUT % NCO == 0, "channel tiling");
    static_assert(EPI != EPI_HEAD || (NCO == 16 && COUT == 16), "the head needs all 16 channels");
    static_assert(NST == 1 || NST == 2, "one or two halo stages");
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 127u) & ~127u;
    unsigned char* sbase = smem_raw + (base - raw);
    const uint32_t sStage = base;                            // NST x [2 chunks][HVOX][8 channels]
    const uint32_t sB = base + uint32_t(NST * STAGE_BYTES);  // [tap][chunk][co][8]
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(sbase + NST * STAGE_BYTES + 27 * CIN * NCO * 2);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 5);
    // barriers (8 bytes apart): stage 0, stage 1, accumulator set 0, set 1, spare
    const uint32_t bar_stage0 = smem_u32(bars), bar_acc0 = smem_u32(bars + 2), bar_spare = smem_u32(bars + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cog = blockIdx.y;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(NCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int b = 0; b < 5; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_stage0 + 8u * b));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    for (int i = tid; i < 27 * NCO * (CIN / 8); i += TC_THREADS) {
        const int co = i % NCO, c = (i / NCO) % (CIN / 8), tap = i / (NCO * (CIN / 8));
        cp_async16(sB + uint32_t(((tap * (CIN / 8) + c) * NCO + co) * 16),
                   a.w + (int64_t(tap) * COUT + cog * NCO + co) * CIN + c * 8, true);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;

    const int nbx = (a.lv.W + TX - 1) / TX, nby = (a.lv.H + TY - 1) / TY, nbz = (a.lv.D + TZ - 1) / TZ;
    const int nbricks = nbx * nby * nbz;
    const int mine = int(blockIdx.x) < nbricks ? (nbricks - 1 - int(blockIdx.x)) / int(gridDim.x) + 1 : 0;

    // epilogue of this CTA's brick i (TMEM set i & 1)
    auto epilogue = [&](int i) {
        const int brick = int(blockIdx.x) + i * int(gridDim.x);
        const int bx = brick % nbx, by = (brick / nbx) % nby, bz = brick / (nbx * nby);
        const uint32_t set = uint32_t(i & 1) * uint32_t(2 * NCO);
#pragma unroll 1
        for (int zo = 0; zo < TZ; ++zo) {
            float v[NCO];
#pragma unroll
            for (int j = 0; j < NCO / 16; ++j)
                tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + set + uint32_t(zo * NCO + 16 * j), v + 16 * j);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            const int m = warp * 32 + lane;
            const int gx = bx * TX + (m & 7), gy = by * TY + (m >> 3), gz = bz * TZ + zo;
            if (gx >= a.lv.W || gy >= a.lv.H || gz >= a.lv.D) continue;
            const int64_t vox = (int64_t(gz) * a.lv.H + gy) * a.lv.W + gx;
            if (EPI == EPI_RELU || EPI == EPI_HEAD) {
#pragma unroll
                for (int q = 0; q < NCO; ++q) v[q] = fmaxf(v[q], 0.0f);
            }
            if (EPI == EPI_MASK) {
#pragma unroll
                for (int q = 0; q < NCO / 8; ++q) {
                    const uint4 mk = *reinterpret_cast<const uint4*>(a.mask + vox * COUT + cog * NCO + 8 * q);
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
                *reinterpret_cast<uint4*>(a.y + vox * COUT + cog * NCO + 8 * q) = u;
            }
            if (EPI == EPI_HEAD) a.head_out[vox] = hsum;
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    };

    bool ok = true;
    const int steps = mine * G;
    for (int s = 0; s < steps && ok; ++s) {
        const int i = s / G, g = s % G;
        const int brick = int(blockIdx.x) + i * int(gridDim.x);
        const int bx = brick % nbx, by = (brick / nbx) % nby, bz = brick / (nbx * nby);
        const int sl = s % NST, use = s / NST;  // stage slot, and how often it has been filled before
        const uint32_t stage = sStage + uint32_t(sl * STAGE_BYTES);
        // the stage's previous MMAs (step s - NST) must be done before it is overwritten
        if (use >= 1 && !block_wait(bar_stage0 + 8u * uint32_t(sl), uint32_t((use - 1) & 1))) {
            ok = false;
            break;
        }
        // channels [16 g, 16 g + 16) of the halo, voxel-fastest
        const int x0 = bx * TX - 1, y0 = by * TY - 1, z0 = bz * TZ - 1;
        for (int t = tid; t < HVOX * 2; t += TC_THREADS) {
            const int hv = t % HVOX, cl = t / HVOX;
            const int c = 2 * g + cl;  // 8-channel chunk of the full input
            const int gx = x0 + hv % HX, gy = y0 + (hv / HX) % HY, gz = z0 + hv / (HX * HY);
            const bool in = gx >= 0 && gx < a.lv.W && gy >= 0 && gy < a.lv.H && gz >= 0 && gz < a.lv.D;
            const bf16* src;
            if (CA > 0 && c * 8 < CA)
                src = in ? a.xa + ((int64_t(gz >> 1) * a.lc.H + (gy >> 1)) * a.lc.W + (gx >> 1)) * CA + c * 8 : a.xa;
            else
                src = in ? a.xb + ((int64_t(gz) * a.lv.H + gy) * a.lv.W + gx) * CB + (c * 8 - CA) : a.xb;
            cp_async16(stage + uint32_t((cl * HVOX + hv) * 16), src, in);
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // generic-proxy writes -> tensor core
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (tid == 0) {
            const uint32_t set = uint32_t(i & 1) * uint32_t(2 * NCO);
#pragma unroll 1
            for (int zo = 0; zo < TZ; ++zo) {
#pragma unroll 1
                for (int tap = 0; tap < 27; ++tap) {
                    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    const int hv0 = ((zo + 1 + dz) * HY + (1 + dy)) * HX + (1 + dx);
                    const uint64_t ad = umma_desc(stage + uint32_t(hv0 * 16), HVOX * 16, HX * 16);
                    const uint64_t bd = umma_desc(sB + uint32_t((tap * (CIN / 8) + 2 * g) * NCO * 16), NCO * 16, 128);
                    umma_bf16(tmem + set + uint32_t(zo * NCO), ad, bd, IDESC, (g | tap) != 0 ? 1u : 0u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             bar_stage0 + 8u * uint32_t(sl))
                         : "memory");
            if (g == G - 1)
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 bar_acc0 + 8u * uint32_t(i & 1))
                             : "memory");
        }
        // the previous brick's epilogue overlaps this brick's first MMAs
        if (g == 0 && i >= 1) {
            if (!block_wait(bar_acc0 + 8u * uint32_t((i - 1) & 1), uint32_t(((i - 1) >> 1) & 1))) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            epilogue(i - 1);
        }
    }
    if (ok && mine > 0) {
        const int i = mine - 1;
        if (block_wait(bar_acc0 + 8u * uint32_t(i & 1), uint32_t((i >> 1) & 1))) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            epilogue(i);
        } else {
            ok = false;
        }
    }
    if (!ok && tid == 0) {
        if (a.status) atomicExch(a.status, DEV_TIMEOUT_CODE);
        // one more bounded wait for this CTA's own MMAs: a final commit arrives
        // on the spare barrier once every MMA issued so far has completed
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar_spare)
                     : "memory");
        mbar_wait_bounded(bar_spare, 0u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(NCOLS));
}

int g_tc_sms = 0;

template <int CA, int CB, int COUT, int NCO, int EPI, int NST = 1>
int run_conv_tc(const ConvArgs& a, cudaStream_t st) {
    constexpr size_t smem = tc_smem_bytes<CA, CB, COUT, NCO, NST>();
    static_assert(smem <= 232448, "shared memory of one CTA");
    static int per_sm = -1;
    auto kern = k_conv3_tc<CA, CB, COUT, NCO, EPI, NST>;
    if (per_sm < 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        // all of the SM's unified memory as shared memory, so that several
        // CTAs are resident (the default carveout fits only one)
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        int dev = 0, smem_sm = 0;
        cudaGetDevice(&dev);
        if (!g_tc_sms) {
            cudaDeviceGetAttribute(&g_tc_sms, cudaDevAttrMultiProcessorCount, dev);
            if (g_tc_sms <= 0) g_tc_sms = 148;
        }
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        if (smem_sm <= 0) smem_sm = 233472;
        // resident CTAs per SM: shared memory (1 KB reserved per CTA), threads,
        // and the 512 TMEM columns they must share
        // (the CTAs never wait on each other, so a grid above the true residency
        // only queues; a TMEM allocation waits for CTAs that finish regardless)
        per_sm = std::max(1, std::min({smem_sm / int(smem + 1024), 2048 / TC_THREADS, 512 / tmem_cols<NCO>()}));
    }
    const int groups = COUT / NCO;
    const int nb = ((a.lv.W + TX - 1) / TX) * ((a.lv.H + TY - 1) / TY) * ((a.lv.D + TZ - 1) / TZ);
    const int gx = std::max(1, std::min(nb, per_sm * g_tc_sms / groups));
    kern<<<dim3(gx, groups), TC_THREADS, smem, st>>>(a);
    return int(cudaPeekAtLastError());
}

}  // namespace

int conv_forward_layer_tc(int layer, const ConvArgs& a, cudaStream_t st) {
    switch (layer) {
        case 0: case 1: return run_conv_tc<0, 16, 16, 16, EPI_RELU>(a, st);
        case 2: return run_conv_tc<0, 16, 32, 32, EPI_RELU>(a, st);
        case 3: case 7: return run_conv_tc<0, 32, 32, 32, EPI_RELU>(a, st);
        case 4: return run_conv_tc<0, 32, 64, 32, EPI_RELU>(a, st);
        case 5: return run_conv_tc<0, 64, 64, 16, EPI_RELU>(a, st);
        case 6: return run_conv_tc<64, 32, 32, 16, EPI_RELU>(a, st);
        case 8: return run_conv_tc<32, 16, 16, 16, EPI_RELU>(a, st);
        case 9: return run_conv_tc<0, 16, 16, 16, EPI_HEAD>(a, st);
    }
    return int(cudaErrorInvalidValue);
}

int conv_backward_layer_tc(int layer, const ConvArgs& a, cudaStream_t st) {
    switch (layer) {
        case 9: case 1: return run_conv_tc<0, 16, 16, 16, EPI_MASK>(a, st);
        case 8: return run_conv_tc<0, 16, 48, 48, EPI_RAW>(a, st);
        case 7: case 3: return run_conv_tc<0, 32, 32, 32, EPI_MASK>(a, st);
        case 6: return run_conv_tc<0, 32, 96, 32, EPI_RAW>(a, st);
        case 5: return run_conv_tc<0, 64, 64, 16, EPI_MASK>(a, st);
        case 4: return run_conv_tc<0, 64, 32, 16, EPI_RAW>(a, st);
        case 2: return run_conv_tc<0, 32, 16, 16, EPI_RAW>(a, st);
    }
    return int(cudaErrorInvalidValue);
}

}  // namespace unet
}  // namespace fp
