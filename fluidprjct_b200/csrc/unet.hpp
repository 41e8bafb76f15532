// unet.hpp -- the learned pressure preconditioner: a 3-level 3D U-Net
// (16/32/64 channels, 3x3x3 convolutions, BF16 weights and activations, FP32
// accumulation) that maps (labels, divergence) to an initial pressure guess.
//
// Layer table (CA = channels of the 2x-upsampled coarse input, CB = channels
// of the same-level input, COUT = output channels):
//   L0 16->16, L1 16->16 = e0 -> avgpool2 -> q0                 level 0
//   L2 16->32, L3 32->32 = e1 -> avgpool2 -> q1                 level 1
//   L4 32->64, L5 64->64 = e2                                   level 2
//   L6 [up2(e2) | e1] 96->32, L7 32->32 = d1                    level 1
//   L8 [up2(d1) | e0] 48->16, L9 16->16 = d0, head 16->1        level 0
// Every 3x3x3 convolution is followed by ReLU; there are no biases.  Tensors
// are channels-last bf16 ([z][y][x][c]) on grids padded to multiples of 4.
// Weights are [27][COUT][CIN] with tap = (dz+1)*9 + (dy+1)*3 + (dx+1), and
// the flat parameter vector is L0..L9 followed by the 16 head weights.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

struct fp_unet;

namespace fp {
namespace unet {

using bf16 = __nv_bfloat16;

constexpr int kLayers = 10;
constexpr int kHead = 16;
constexpr int kInCh = 16;

struct LayerSpec {
    int level, ca, cb, cout;
};
constexpr LayerSpec kSpec[kLayers] = {
    {0, 0, 16, 16}, {0, 0, 16, 16}, {1, 0, 16, 32}, {1, 0, 32, 32}, {2, 0, 32, 64},
    {2, 0, 64, 64}, {1, 64, 32, 32}, {1, 0, 32, 32}, {0, 32, 16, 16}, {0, 0, 16, 16},
};
constexpr int64_t layer_size(int l) { return int64_t(27) * kSpec[l].cout * (kSpec[l].ca + kSpec[l].cb); }
constexpr int64_t layer_offset(int l) { return l == 0 ? 0 : layer_offset(l - 1) + layer_size(l - 1); }
constexpr int64_t kParams = layer_offset(kLayers) + kHead;  // 359,440

struct Lvl {
    int W, H, D;
    __host__ __device__ int64_t n() const { return int64_t(W) * H * D; }
};

// Activations and their gradients are channel-blocked: channel c of voxel v
// on a level of n voxels is element blk8(n, v, c / 8) + c % 8.  Eight channels
// of a row of voxels are then contiguous, which is what the convolutions'
// tensor maps read, and a channel concatenation [A | B] is A's blocks
// followed by B's.
__host__ __device__ inline int64_t blk8(int64_t n, int64_t v, int cb) { return (int64_t(cb) * n + v) * 8; }

// Arguments of the weight-gradient kernel: dw[t][co][ci] = sum_v g[v][co] x[v + off(t)][ci].
struct CorrArgs {
    const bf16* xa;
    const bf16* xb;
    const bf16* g;         // [V][COUT]
    float* part;           // [gridDim.x][27][COUT][CIN] partial sums
    Lvl lv, lc;
};

enum { EPI_RELU = 0, EPI_MASK = 1, EPI_RAW = 2, EPI_HEAD = 3 };

// Arguments of the TMA-fed convolution (kernels_unet_tma.cu); its input is
// one [V][CIN] tensor read through a tensor map.
struct TmaConvArgs {
    bf16* y;               // output [V][COUT]
    const bf16* mask;      // EPI_MASK: output is zeroed where mask[V][c] <= 0
    const float* head_w;   // EPI_HEAD: 16 head weights
    float* head_out;       // EPI_HEAD: one FP32 value per voxel
    const bf16* w;         // [27][COUT][CIN]
    Lvl lv;                // the level of input and output
    int* status;           // set to nonzero if a bounded device wait gave up
};
int conv_forward_layer_tma(int layer, const bf16* in, const TmaConvArgs& a, cudaStream_t st);
int conv_backward_layer_tma(int layer, const bf16* in, const TmaConvArgs& a, cudaStream_t st);
// The first ca / 8 channel blocks of out = up2(coarse) on the fine level.
void launch_upcat(const bf16* coarse, int ca, Lvl fine, bf16* out, cudaStream_t st);

// Launchers (kernels_unet.cu).  Each returns 0 or a cudaError_t value.
int corr_layer(int layer, const CorrArgs& a, int nblk, cudaStream_t st);
int corr_blocks(int layer, const Lvl& lv);                               // gridDim.x for corr_layer
void reduce_partials(const float* part, int nblk, int64_t n, float* out, cudaStream_t st);

void launch_rhs_scale(const uint8_t* labels, const float* rhs, Lvl real, double* red, float* scal, cudaStream_t st);
void launch_input(const uint8_t* labels, const float* rhs, Lvl real, Lvl net, const float* scal, bf16* x0,
                  cudaStream_t st);
void launch_pool(const bf16* e, Lvl fine, int C, bf16* q, cudaStream_t st);
void launch_sum_children_mask(const bf16* raw, Lvl fine, int ctot, int C, const bf16* act, bf16* g, cudaStream_t st);
void launch_skip_combine(const bf16* raw, Lvl fine, int ctot, int ca, int C, const bf16* gq, const bf16* act,
                         bf16* g, cudaStream_t st);
void launch_loss(const uint8_t* labels, const float* p, Lvl real, Lvl net, const float* out, double* red, float* scal,
                 cudaStream_t st);
void launch_head_backward(const uint8_t* labels, const float* p, Lvl real, Lvl net, const float* out, const bf16* d0,
                          const float* head_w, const float* scal, bf16* g9, float* head_part, int nblk,
                          cudaStream_t st);
int head_blocks(Lvl net);
void launch_output_dense(const uint8_t* labels, Lvl real, Lvl net, const float* out, const float* scal, float* x,
                         cudaStream_t st);
// Compact initial guess for the pressure solver: x0[n] = s * out at the n-th
// FLUID cell, whose index in the (W+2)(H+2)(D+2) padded grid is fidx[n].
void launch_output_compact(const int* nf, const int* fidx, Lvl real, Lvl net, const float* out, const float* scal,
                           float* x0, cudaStream_t st);
// Dense right-hand side from the solver's compact one (zero off FLUID cells).
void launch_rhs_dense(const int* nf, const int* fidx, Lvl real, const float* b, float* dense, cudaStream_t st);
// Adam on the gradient scaled by min(1, clip / ||g||) (global norm, computed
// on the device; scal[3] receives the factor, red the norm).
void launch_adam(float* w, float* m, float* v, const float* g, int64_t n, float lr, float b1, float b2, float eps,
                 float bc1, float bc2, float clip, double* red, float* scal, cudaStream_t st);
void launch_weights_bf16(const float* w32, bf16* wf, bf16* wt, cudaStream_t st);

// Forward pass of a network made by fp_unet_create on the stream st; leaves
// the head output on the padded level-0 grid and (s, 1/s) on the device.
int forward_on(fp_unet* u, const uint8_t* labels, const float* rhs, cudaStream_t st);
Lvl net_level0(const fp_unet* u);
const float* net_out(const fp_unet* u);
const float* net_scal(const fp_unet* u);
const int* net_status(const fp_unet* u);  // device word, nonzero after a timed-out wait

}  // namespace unet
}  // namespace fp
