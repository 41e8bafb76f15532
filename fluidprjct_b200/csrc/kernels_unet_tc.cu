// kernels_unet_tc.cu -- the U-Net's 3x3x3 convolutions on the fifth-generation
// tensor cores (tcgen05.mma, BF16 operands from shared memory, FP32
// accumulators in tensor memory).
//
// One persistent CTA of 128 threads walks output bricks of 8x16x2 voxels.
// A brick is two M = 128 tiles, one per z slice: row m of a tile is the voxel
// (x = m % 8, y = m / 8).  Per brick:
//   1. all threads stage the zero-padded input halo (10x18x4 voxels, every
//      input channel) in shared memory with cp.async.  The layout is
//      chunk-major ([8-channel chunk][halo voxel][8 channels]), the K-major
//      no-swizzle UMMA layout: any 8 consecutive voxels of a halo row form one
//      8x16-byte core matrix.  The operand of tap (dz, dy, dx) is then the
//      same layout shifted by that tap's halo offset: core matrices of
//      successive y rows lie 160 bytes apart (SBO), the two K halves of a
//      16-channel step one chunk plane apart (LBO).
//   2. one thread issues 27 taps x CIN/16 MMAs per tile (M = 128, N = NCO,
//      K = 16) into the tile's TMEM columns, then commits them to an
//      mbarrier.
//   3. after the mbarrier completes, each warp reads its 32 TMEM lanes
//      (tcgen05.ld 32x32b): every thread then holds one voxel's NCO outputs
//      and writes them as contiguous 16-byte vectors.
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

template <int NCO>
constexpr int tmem_cols() {
    return (2 * NCO <= 32) ? 32 : (2 * NCO <= 64) ? 64 : (2 * NCO <= 128) ? 128 : 256;
}

template <int CA, int CB, int COUT, int NCO>
constexpr size_t tc_smem_bytes() {
    // halo + weights + mbarrier/TMEM slot + alignment slack
    return size_t(HVOX) * (CA + CB) * 2 + size_t(27) * (CA + CB) * NCO * 2 + 16 + 128;
}

template <int CA, int CB, int COUT, int NCO, int EPI>
__global__ void __launch_bounds__(TC_THREADS) k_conv3_tc(ConvArgs a) {
    constexpr int CIN = CA + CB;
    constexpr int CH = CIN / 8;
    constexpr int NCOLS = tmem_cols<NCO>();
    constexpr uint32_t IDESC = umma_idesc_bf16(NCO);
    static_assert(CIN % 16 == 0 && NCO % 16 == 0 && NCO <= 48 && COUT % NCO == 0, "channel tiling");
    static_assert(EPI != EPI_HEAD || (NCO == 16 && COUT == 16), "the head needs all 16 channels");
    extern __shared__ unsigned char smem_raw[];
    // 128-byte aligned operand area: halo, then weights, then the barrier word
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 127u) & ~127u;
    unsigned char* sbase = smem_raw + (base - raw);
    const uint32_t sA = base;
    const uint32_t sB = sA + uint32_t(HVOX * CH * 16);
    unsigned long long* mbar_p = reinterpret_cast<unsigned long long*>(sbase + HVOX * CH * 16 + 27 * CH * NCO * 16);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar_p + 1);
    const uint32_t mbar = smem_u32(mbar_p);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cog = blockIdx.y;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(NCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // weights of this output-channel group: [tap][chunk][co][8]
    for (int i = tid; i < 27 * NCO * CH; i += TC_THREADS) {
        const int co = i % NCO, c = (i / NCO) % CH, tap = i / (NCO * CH);
        cp_async16(sB + uint32_t(((tap * CH + c) * NCO + co) * 16),
                   a.w + (int64_t(tap) * COUT + cog * NCO + co) * CIN + c * 8, true);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;

    const int nbx = (a.lv.W + TX - 1) / TX, nby = (a.lv.H + TY - 1) / TY, nbz = (a.lv.D + TZ - 1) / TZ;
    const int nbricks = nbx * nby * nbz;
    uint32_t phase = 0;
    bool ok = true;
    for (int brick = blockIdx.x; brick < nbricks && ok; brick += gridDim.x) {
        const int bx = brick % nbx, by = (brick / nbx) % nby, bz = brick / (nbx * nby);
        const int x0 = bx * TX - 1, y0 = by * TY - 1, z0 = bz * TZ - 1;
        // 1. halo, voxel-fastest so the shared-memory writes are contiguous
        for (int i = tid; i < HVOX * CH; i += TC_THREADS) {
            const int hv = i % HVOX, c = i / HVOX;
            const int gx = x0 + hv % HX, gy = y0 + (hv / HX) % HY, gz = z0 + hv / (HX * HY);
            const bool in = gx >= 0 && gx < a.lv.W && gy >= 0 && gy < a.lv.H && gz >= 0 && gz < a.lv.D;
            const bf16* src;
            if (CA > 0 && c * 8 < CA)
                src = in ? a.xa + ((int64_t(gz >> 1) * a.lc.H + (gy >> 1)) * a.lc.W + (gx >> 1)) * CA + c * 8 : a.xa;
            else
                src = in ? a.xb + ((int64_t(gz) * a.lv.H + gy) * a.lv.W + gx) * CB + (c * 8 - CA) : a.xb;
            cp_async16(sA + uint32_t((c * HVOX + hv) * 16), src, in);
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // generic-proxy writes -> tensor core
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        // 2. one thread issues the MMAs of both tiles
        if (tid == 0) {
#pragma unroll 1
            for (int zo = 0; zo < TZ; ++zo) {
#pragma unroll 1
                for (int tap = 0; tap < 27; ++tap) {
                    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    const int hv0 = ((zo + 1 + dz) * HY + (1 + dy)) * HX + (1 + dx);
#pragma unroll
                    for (int kc = 0; kc < CIN / 16; ++kc) {
                        const uint64_t ad = umma_desc(sA + uint32_t((2 * kc * HVOX + hv0) * 16), HVOX * 16, HX * 16);
                        const uint64_t bd = umma_desc(sB + uint32_t((tap * CH + 2 * kc) * NCO * 16), NCO * 16, 128);
                        umma_bf16(tmem + uint32_t(zo * NCO), ad, bd, IDESC, (tap | kc) != 0 ? 1u : 0u);
                    }
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
                         : "memory");
        }
        // 3. wait for the MMAs (every thread observes the barrier; the block
        // agrees on the outcome), then the epilogue from TMEM
        const bool got = mbar_wait_bounded(mbar, phase);
        if (!__syncthreads_and(got ? 1 : 0)) {
            if (tid == 0) {
                if (a.status) atomicExch(a.status, DEV_TIMEOUT_CODE);
                mbar_wait_bounded(mbar, phase);  // one more bounded wait for this CTA's own MMAs
            }
            ok = false;
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll 1
        for (int zo = 0; zo < TZ; ++zo) {
            float v[NCO];
#pragma unroll
            for (int j = 0; j < NCO / 16; ++j)
                tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(zo * NCO + 16 * j), v + 16 * j);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            const int m = warp * 32 + lane;
            const int gx = bx * TX + (m & 7), gy = by * TY + (m >> 3), gz = bz * TZ + zo;
            if (gx >= a.lv.W || gy >= a.lv.H || gz >= a.lv.D) continue;
            const int64_t vox = (int64_t(gz) * a.lv.H + gy) * a.lv.W + gx;
            if (EPI == EPI_RELU || EPI == EPI_HEAD) {
#pragma unroll
                for (int i = 0; i < NCO; ++i) v[i] = fmaxf(v[i], 0.0f);
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
        // every thread's TMEM reads and shared-memory use end before the next brick
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(NCOLS));
}

int g_tc_sms = 0;

template <int CA, int CB, int COUT, int NCO, int EPI>
int run_conv_tc(const ConvArgs& a, cudaStream_t st) {
    constexpr size_t smem = tc_smem_bytes<CA, CB, COUT, NCO>();
    static_assert(smem <= 232448, "shared memory of one CTA");
    static int per_sm = -1;
    auto kern = k_conv3_tc<CA, CB, COUT, NCO, EPI>;
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
