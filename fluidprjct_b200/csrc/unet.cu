// unet.cu -- host side of the learned pressure preconditioner: buffers, the
// forward and backward schedules, Adam, weight files and the fp_unet_* C ABI.
//
// The network has no counterpart in the reference (its pressure solve is the
// cuDSS factorisation of FluidSolver3D.cu:1930-2008).  Training pairs
// (labels, divergence) -> pressure come from the plain PCG solver.  Inside
// the solver the network gives the initial guess of the MG-preconditioned
// PCG, and the plain PCG is the fallback.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/fluidprjct.h"
#include "unet.hpp"

using namespace fp::unet;

namespace {
constexpr int kRedLoss = 2 * 256;  // index of the loss in the reduction buffer (the gradient norm follows)
constexpr float kClip = 1.0f;      // global gradient-norm clip of the training step
constexpr char kMagic[8] = {'F', 'P', 'U', 'N', 'E', 'T', '0', '1'};
}  // namespace

struct fp_unet {
    Lvl real{}, L[3]{};
    bool train = false;
    cudaStream_t st = nullptr;
    std::vector<void*> allocs;
    bool alloc_failed = false;
    float *w32 = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *part = nullptr, *hpart = nullptr;
    bf16 *wf = nullptr, *wt = nullptr;
    double* red = nullptr;
    float* scal = nullptr;  // s, 1/s, 2/sum(t^2)
    int* d_status = nullptr;  // nonzero once a bounded wait in a convolution gave up
    int* h_status = nullptr;
    double* h_loss = nullptr;
    // forward
    bf16 *X0, *a0, *e0, *q0, *a1, *e1, *q1, *a2, *e2, *d1a, *d1, *d0a, *d0;
    bf16 *cat6, *cat8;  // [up2(e2) | e1] and [up2(d1) | e0], the decoder layers' inputs
    float* out = nullptr;
    // backward
    bf16 *g9, *g8, *raw8, *g7, *g6, *raw6, *g5, *g4, *gq1, *g3, *g2, *gq0, *g1, *g0;
    int hblk = 0;
    int64_t step = 0;
    std::string err;

    template <class T>
    T* alloc(int64_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * size_t(std::max<int64_t>(n, 1))) != cudaSuccess) {
            alloc_failed = true;
            return nullptr;
        }
        allocs.push_back(p);
        return static_cast<T*>(p);
    }
    int fail(int code, const std::string& msg) {
        err = msg;
        return code;
    }
    int cuda_check(const char* what) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(FP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        return FP_OK;
    }
};

namespace fp {
namespace unet {

Lvl net_level0(const fp_unet* u) { return u->L[0]; }
const float* net_out(const fp_unet* u) { return u->out; }
const float* net_scal(const fp_unet* u) { return u->scal; }
const int* net_status(const fp_unet* u) { return u->d_status; }

// A 3x3x3 convolution layer.  A decoder layer reads [up2(xa) | xb] through
// one TMA tensor map from u->cat6 / u->cat8: the skip tensor xb (e1, e0) is
// written there by its own layer (the channel blocks after up2(xa)), and
// up2(xa) is filled in here.
static int conv_fwd(fp_unet* u, int l, const bf16* xa, const bf16* xb, bf16* y, cudaStream_t st) {
    TmaConvArgs a{};
    a.w = u->wf + layer_offset(l);
    a.y = y;
    a.lv = u->L[kSpec[l].level];
    a.head_w = u->w32 + layer_offset(kLayers);
    a.head_out = u->out;
    a.status = u->d_status;
    const bf16* in = xb;
    if (kSpec[l].ca > 0) {
        bf16* cat = l == 6 ? u->cat6 : u->cat8;
        launch_upcat(xa, kSpec[l].ca, a.lv, cat, st);
        in = cat;
    }
    return conv_forward_layer_tma(l, in, a, st);
}

// Forward pass: u->out (net level 0) and u->scal (s, 1/s).
int forward_on(fp_unet* u, const uint8_t* labels, const float* rhs, cudaStream_t st) {
    launch_rhs_scale(labels, rhs, u->real, u->red, u->scal, st);
    launch_input(labels, rhs, u->real, u->L[0], u->scal, u->X0, st);
    int e = 0;
    e |= conv_fwd(u, 0, nullptr, u->X0, u->a0, st);
    e |= conv_fwd(u, 1, nullptr, u->a0, u->e0, st);
    launch_pool(u->e0, u->L[0], 16, u->q0, st);
    e |= conv_fwd(u, 2, nullptr, u->q0, u->a1, st);
    e |= conv_fwd(u, 3, nullptr, u->a1, u->e1, st);
    launch_pool(u->e1, u->L[1], 32, u->q1, st);
    e |= conv_fwd(u, 4, nullptr, u->q1, u->a2, st);
    e |= conv_fwd(u, 5, nullptr, u->a2, u->e2, st);
    e |= conv_fwd(u, 6, u->e2, u->e1, u->d1a, st);
    e |= conv_fwd(u, 7, nullptr, u->d1a, u->d1, st);
    e |= conv_fwd(u, 8, u->d1, u->e0, u->d0a, st);
    e |= conv_fwd(u, 9, nullptr, u->d0a, u->d0, st);
    return e;
}

int forward_kernel_count() { return 2 + 10 + 2 + 2; }

}  // namespace unet
}  // namespace fp

namespace {

// Reads the device status after the stream is synchronised.
int device_status(fp_unet* u, const char* what) {
    if (cudaMemcpy(u->h_status, u->d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return u->cuda_check(what);
    if (*u->h_status) return u->fail(FP_ERR_TIMEOUT, std::string(what) + ": a bounded tensor-core wait gave up");
    return FP_OK;
}

int conv_bwd(fp_unet* u, int l, const bf16* g, const bf16* mask, bf16* y, cudaStream_t st) {
    TmaConvArgs a{};
    a.w = u->wt + layer_offset(l);
    a.y = y;
    a.mask = mask;
    a.lv = u->L[kSpec[l].level];
    a.status = u->d_status;
    return conv_backward_layer_tma(l, g, a, st);
}

int wgrad(fp_unet* u, int l, const bf16* xa, const bf16* xb, const bf16* g, cudaStream_t st) {
    CorrArgs a{};
    a.xa = xa;
    a.xb = xb;
    a.g = g;
    a.part = u->part;
    a.lv = u->L[kSpec[l].level];
    a.lc = kSpec[l].level < 2 ? u->L[kSpec[l].level + 1] : a.lv;
    const int nblk = corr_blocks(l, a.lv);
    int e = corr_layer(l, a, nblk, st);
    reduce_partials(u->part, nblk, layer_size(l), u->grad + layer_offset(l), st);
    return e;
}

// Loss and gradient of the last forward pass against the pressure p.
int backward(fp_unet* u, const uint8_t* labels, const float* p, cudaStream_t st) {
    const Lvl* L = u->L;
    launch_loss(labels, p, u->real, L[0], u->out, u->red, u->scal, st);
    launch_head_backward(labels, p, u->real, L[0], u->out, u->d0, u->w32 + layer_offset(kLayers), u->scal, u->g9,
                         u->hpart, u->hblk, st);
    reduce_partials(u->hpart, u->hblk, kHead, u->grad + layer_offset(kLayers), st);
    int e = 0;
    e |= wgrad(u, 9, nullptr, u->d0a, u->g9, st);
    e |= conv_bwd(u, 9, u->g9, u->d0a, u->g8, st);
    e |= wgrad(u, 8, u->d1, u->e0, u->g8, st);
    e |= conv_bwd(u, 8, u->g8, nullptr, u->raw8, st);
    launch_sum_children_mask(u->raw8, L[0], 48, 32, u->d1, u->g7, st);
    e |= wgrad(u, 7, nullptr, u->d1a, u->g7, st);
    e |= conv_bwd(u, 7, u->g7, u->d1a, u->g6, st);
    e |= wgrad(u, 6, u->e2, u->e1, u->g6, st);
    e |= conv_bwd(u, 6, u->g6, nullptr, u->raw6, st);
    launch_sum_children_mask(u->raw6, L[1], 96, 64, u->e2, u->g5, st);
    e |= wgrad(u, 5, nullptr, u->a2, u->g5, st);
    e |= conv_bwd(u, 5, u->g5, u->a2, u->g4, st);
    e |= wgrad(u, 4, nullptr, u->q1, u->g4, st);
    e |= conv_bwd(u, 4, u->g4, nullptr, u->gq1, st);
    launch_skip_combine(u->raw6, L[1], 96, 64, 32, u->gq1, u->e1, u->g3, st);
    e |= wgrad(u, 3, nullptr, u->a1, u->g3, st);
    e |= conv_bwd(u, 3, u->g3, u->a1, u->g2, st);
    e |= wgrad(u, 2, nullptr, u->q0, u->g2, st);
    e |= conv_bwd(u, 2, u->g2, nullptr, u->gq0, st);
    launch_skip_combine(u->raw8, L[0], 48, 32, 16, u->gq0, u->e0, u->g1, st);
    e |= wgrad(u, 1, nullptr, u->a0, u->g1, st);
    e |= conv_bwd(u, 1, u->g1, u->a0, u->g0, st);
    e |= wgrad(u, 0, nullptr, u->X0, u->g0, st);
    return e;
}

void init_weights(std::vector<float>& w, uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    w.assign(size_t(kParams), 0.0f);
    for (int l = 0; l < kLayers; ++l) {
        const double sd = std::sqrt(2.0 / (27.0 * (kSpec[l].ca + kSpec[l].cb)));
        for (int64_t i = 0; i < layer_size(l); ++i) w[size_t(layer_offset(l) + i)] = float(nd(rng) * sd);
    }
    for (int c = 0; c < kHead; ++c) w[size_t(layer_offset(kLayers) + c)] = float(nd(rng) * 0.25);
}

int upload_weights(fp_unet* u, const float* host) {
    if (cudaMemcpyAsync(u->w32, host, sizeof(float) * size_t(kParams), cudaMemcpyHostToDevice, u->st) != cudaSuccess)
        return u->cuda_check("weight upload");
    launch_weights_bf16(u->w32, u->wf, u->wt, u->st);
    if (u->train) {
        cudaMemsetAsync(u->m, 0, sizeof(float) * size_t(kParams), u->st);
        cudaMemsetAsync(u->v, 0, sizeof(float) * size_t(kParams), u->st);
        u->step = 0;
    }
    if (cudaStreamSynchronize(u->st) != cudaSuccess) return u->cuda_check("weight upload");
    return FP_OK;
}

}  // namespace

extern "C" {

int64_t fp_unet_num_params(void) { return kParams; }

int fp_unet_create(int W, int H, int D, int train, uint64_t seed, fp_unet** out) {
    if (!out || W < 4 || H < 4 || D < 4) return FP_ERR_ARG;
    *out = nullptr;
    fp_unet* u = new fp_unet();
    u->train = train != 0;
    u->real = Lvl{W, H, D};
    u->L[0] = Lvl{(W + 3) / 4 * 4, (H + 3) / 4 * 4, (D + 3) / 4 * 4};
    u->L[1] = Lvl{u->L[0].W / 2, u->L[0].H / 2, u->L[0].D / 2};
    u->L[2] = Lvl{u->L[0].W / 4, u->L[0].H / 4, u->L[0].D / 4};
    if (cudaStreamCreateWithFlags(&u->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete u;
        return FP_ERR_CUDA;
    }
    const int64_t n0 = u->L[0].n(), n1 = u->L[1].n(), n2 = u->L[2].n();
    u->w32 = u->alloc<float>(kParams);
    u->wf = u->alloc<bf16>(kParams);
    u->wt = u->alloc<bf16>(kParams);
    u->red = u->alloc<double>(1024);
    u->scal = u->alloc<float>(4);
    u->d_status = u->alloc<int>(1);
    u->X0 = u->alloc<bf16>(n0 * 16);
    u->a0 = u->alloc<bf16>(n0 * 16);
    u->cat8 = u->alloc<bf16>(n0 * 48);
    u->e0 = u->cat8 ? u->cat8 + n0 * 32 : nullptr;  // channel blocks 4-5 of [up2(d1) | e0]
    u->q0 = u->alloc<bf16>(n1 * 16);
    u->a1 = u->alloc<bf16>(n1 * 32);
    u->cat6 = u->alloc<bf16>(n1 * 96);
    u->e1 = u->cat6 ? u->cat6 + n1 * 64 : nullptr;  // channel blocks 8-11 of [up2(e2) | e1]
    u->q1 = u->alloc<bf16>(n2 * 32);
    u->a2 = u->alloc<bf16>(n2 * 64);
    u->e2 = u->alloc<bf16>(n2 * 64);
    u->d1a = u->alloc<bf16>(n1 * 32);
    u->d1 = u->alloc<bf16>(n1 * 32);
    u->d0a = u->alloc<bf16>(n0 * 16);
    u->d0 = u->alloc<bf16>(n0 * 16);
    u->out = u->alloc<float>(n0);
    if (u->train) {
        u->m = u->alloc<float>(kParams);
        u->v = u->alloc<float>(kParams);
        u->grad = u->alloc<float>(kParams);
        u->g9 = u->alloc<bf16>(n0 * 16);
        u->g8 = u->alloc<bf16>(n0 * 16);
        u->raw8 = u->alloc<bf16>(n0 * 48);
        u->g7 = u->alloc<bf16>(n1 * 32);
        u->g6 = u->alloc<bf16>(n1 * 32);
        u->raw6 = u->alloc<bf16>(n1 * 96);
        u->g5 = u->alloc<bf16>(n2 * 64);
        u->g4 = u->alloc<bf16>(n2 * 64);
        u->gq1 = u->alloc<bf16>(n2 * 32);
        u->g3 = u->alloc<bf16>(n1 * 32);
        u->g2 = u->alloc<bf16>(n1 * 32);
        u->gq0 = u->alloc<bf16>(n1 * 16);
        u->g1 = u->alloc<bf16>(n0 * 16);
        u->g0 = u->alloc<bf16>(n0 * 16);
        int64_t pf = 0;
        for (int l = 0; l < kLayers; ++l)
            pf = std::max(pf, int64_t(corr_blocks(l, u->L[kSpec[l].level])) * layer_size(l));
        u->part = u->alloc<float>(pf);
        u->hblk = head_blocks(u->L[0]);
        u->hpart = u->alloc<float>(int64_t(u->hblk) * kHead);
    }
    if (cudaMallocHost(&u->h_loss, sizeof(double)) != cudaSuccess) u->alloc_failed = true;
    if (cudaMallocHost(&u->h_status, sizeof(int)) != cudaSuccess) u->alloc_failed = true;
    if (!u->alloc_failed && cudaMemsetAsync(u->d_status, 0, sizeof(int), u->st) != cudaSuccess) u->alloc_failed = true;
    if (u->alloc_failed) {
        fp_unet_destroy(u);
        return FP_ERR_CUDA;
    }
    std::vector<float> w;
    init_weights(w, seed);
    if (upload_weights(u, w.data()) != FP_OK) {
        fp_unet_destroy(u);
        return FP_ERR_CUDA;
    }
    *out = u;
    return FP_OK;
}

void fp_unet_destroy(fp_unet* u) {
    if (!u) return;
    if (u->st) cudaStreamSynchronize(u->st);
    for (void* p : u->allocs) cudaFree(p);
    if (u->h_loss) cudaFreeHost(u->h_loss);
    if (u->h_status) cudaFreeHost(u->h_status);
    if (u->st) cudaStreamDestroy(u->st);
    delete u;
}

const char* fp_unet_last_error(const fp_unet* u) { return u ? u->err.c_str() : "null network"; }

void* fp_unet_cuda_stream(const fp_unet* u) { return u ? static_cast<void*>(u->st) : nullptr; }

int fp_unet_get_params(fp_unet* u, float* out, int64_t n) {
    if (!u || !out || n != kParams) return FP_ERR_ARG;
    if (cudaMemcpyAsync(out, u->w32, sizeof(float) * size_t(kParams), cudaMemcpyDeviceToHost, u->st) != cudaSuccess ||
        cudaStreamSynchronize(u->st) != cudaSuccess)
        return u->cuda_check("fp_unet_get_params");
    return FP_OK;
}

int fp_unet_set_params(fp_unet* u, const float* in, int64_t n) {
    if (!u || !in || n != kParams) return FP_ERR_ARG;
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(in[i])) return u->fail(FP_ERR_ARG, "non-finite weight at index " + std::to_string(i));
    return upload_weights(u, in);
}

int fp_unet_save(fp_unet* u, const char* path) {
    if (!u || !path) return FP_ERR_ARG;
    std::vector<float> w(static_cast<size_t>(kParams));
    int rc = fp_unet_get_params(u, w.data(), kParams);
    if (rc) return rc;
    FILE* f = std::fopen(path, "wb");
    if (!f) return u->fail(FP_ERR_IO, std::string("cannot write ") + path);
    const int64_t n = kParams;
    bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&n, sizeof n, 1, f) == 1 &&
              std::fwrite(w.data(), sizeof(float), w.size(), f) == w.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? FP_OK : u->fail(FP_ERR_IO, std::string("short write to ") + path);
}

int fp_unet_load(fp_unet* u, const char* path) {
    if (!u || !path) return FP_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return u->fail(FP_ERR_IO, std::string("cannot open ") + path);
    char magic[8];
    int64_t n = 0;
    std::vector<float> w(static_cast<size_t>(kParams));
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
              std::fread(&n, sizeof n, 1, f) == 1 && n == kParams &&
              std::fread(w.data(), sizeof(float), w.size(), f) == w.size();
    std::fclose(f);
    if (!ok) return u->fail(FP_ERR_IO, std::string("not a U-Net weight file of this layout: ") + path);
    return fp_unet_set_params(u, w.data(), kParams);
}

int fp_unet_forward(fp_unet* u, const uint8_t* d_labels, const float* d_rhs, float* d_x) {
    if (!u || !d_labels || !d_rhs || !d_x) return FP_ERR_ARG;
    if (forward_on(u, d_labels, d_rhs, u->st)) return u->cuda_check("U-Net forward");
    launch_output_dense(d_labels, u->real, u->L[0], u->out, u->scal, d_x, u->st);
    if (cudaStreamSynchronize(u->st) != cudaSuccess) return u->cuda_check("U-Net forward");
    if (int rc = u->cuda_check("U-Net forward")) return rc;
    return device_status(u, "U-Net forward");
}

int fp_unet_loss_grad(fp_unet* u, const uint8_t* d_labels, const float* d_rhs, const float* d_p, double* loss,
                      float* grad) {
    if (!u || !d_labels || !d_rhs || !d_p) return FP_ERR_ARG;
    if (!u->train) return u->fail(FP_ERR_STATE, "network was created without training buffers");
    int e = forward_on(u, d_labels, d_rhs, u->st);
    e |= backward(u, d_labels, d_p, u->st);
    if (e) return u->cuda_check("U-Net backward");
    cudaMemcpyAsync(u->h_loss, u->red + kRedLoss, sizeof(double), cudaMemcpyDeviceToHost, u->st);
    if (grad) cudaMemcpyAsync(grad, u->grad, sizeof(float) * size_t(kParams), cudaMemcpyDeviceToHost, u->st);
    if (cudaStreamSynchronize(u->st) != cudaSuccess) return u->cuda_check("U-Net backward");
    if (loss) *loss = *u->h_loss;
    if (int rc = u->cuda_check("U-Net backward")) return rc;
    return device_status(u, "U-Net backward");
}

int fp_unet_train_step(fp_unet* u, const uint8_t* d_labels, const float* d_rhs, const float* d_p, float lr,
                       double* loss) {
    if (!u || !d_labels || !d_rhs || !d_p || !(lr > 0.0f)) return FP_ERR_ARG;
    if (!u->train) return u->fail(FP_ERR_STATE, "network was created without training buffers");
    int e = forward_on(u, d_labels, d_rhs, u->st);
    e |= backward(u, d_labels, d_p, u->st);
    if (e) return u->cuda_check("U-Net training step");
    ++u->step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = float(1.0 - std::pow(double(b1), double(u->step)));
    const float bc2 = float(1.0 - std::pow(double(b2), double(u->step)));
    launch_adam(u->w32, u->m, u->v, u->grad, kParams, lr, b1, b2, 1e-8f, bc1, bc2, kClip, u->red, u->scal, u->st);
    launch_weights_bf16(u->w32, u->wf, u->wt, u->st);
    if (loss) {
        cudaMemcpyAsync(u->h_loss, u->red + kRedLoss, sizeof(double), cudaMemcpyDeviceToHost, u->st);
        if (cudaStreamSynchronize(u->st) != cudaSuccess) return u->cuda_check("U-Net training step");
        *loss = *u->h_loss;
        if (int rc = device_status(u, "U-Net training step")) return rc;
    }
    return u->cuda_check("U-Net training step");
}

}  // extern "C"
