// kernels_extrap.cu -- velocity extrapolation by wavefronts
// (extrapolateGridFluidData, FluidSolver2D.cu:1207-1295; its calls in the 2D
// step, :1309-1310 and :1325-1326, are commented out, so it is opt-in here).
//
// On one face grid of nx x ny x nz values: marker 0 for known values,
// "unknown" otherwise.  Wave 1 is every unknown value with a known neighbour;
// wave k+1 every unknown value next to wave k.  A wave-k value becomes the
// mean of its neighbours with a smaller marker, summed in the fixed neighbour
// order (x offset -1, 0, 1; y offset +1, 0, -1; z offset -1, 0, 1), which in
// 2D is the reference's list {-1,1},{-1,0},{-1,-1},{0,1},{0,-1},{1,1},{1,0},
// {1,-1}.  A wave reads only strictly older markers and values, so each wave
// is two race-free launches: mark the front, then average it.
//
// The reference's initial-front test reads neighbour markers at stride
// gridWidth whatever the grid (checkNeighbors, :1049-1066), which is the
// wrong stride for the (W+1)-wide u grid; front_stride restates that.
#include <climits>

#include "kernels.hpp"

namespace fp {
namespace {

constexpr float kVelUnknown = -2147483648.0f;
constexpr int kUnknown = INT_MAX;

__global__ void k_ext_known_value(const float* __restrict__ v, int64_t n, int* __restrict__ mark) {
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c < n) mark[c] = v[c] != kVelUnknown ? 0 : kUnknown;
}

// 3D scheme: a face is known when a FLUID cell lies on either side.
__global__ void k_ext_known_fluid(const uint8_t* __restrict__ lab, Dims g, int axis, int* __restrict__ mark) {
    const int nx = g.W + (axis == 0), ny = g.H + (axis == 1), nz = g.D + (axis == 2);
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= int64_t(nx) * ny * nz) return;
    const int i = int(c % nx), j = int((c / nx) % ny), k = int(c / (int64_t(nx) * ny));
    const uint8_t a = label_at(lab, g, i, j, k);
    const uint8_t b = label_at(lab, g, i - (axis == 0), j - (axis == 1), k - (axis == 2));
    mark[c] = (a == FLUID || b == FLUID) ? 0 : kUnknown;
}

__global__ void k_ext_front(int* __restrict__ mark, int nx, int ny, int nz, int wave, int front_stride) {
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= int64_t(nx) * ny * nz || mark[c] != kUnknown) return;
    const int i = int(c % nx), j = int((c / nx) % ny), k = int(c / (int64_t(nx) * ny));
    const int sy = wave == 1 ? front_stride : nx;
    for (int ox = -1; ox <= 1; ++ox)
        for (int oy = 1; oy >= -1; --oy)
            for (int oz = -1; oz <= 1; ++oz) {
                if (ox == 0 && oy == 0 && oz == 0) continue;
                const int a = i + ox, b = j + oy, e = k + oz;
                if (a < 0 || a >= nx || b < 0 || b >= ny || e < 0 || e >= nz) continue;
                if (mark[a + int64_t(b) * sy + int64_t(e) * nx * ny] == wave - 1) {
                    mark[c] = wave;  // wave != wave - 1: other threads' tests are unaffected
                    return;
                }
            }
}

__global__ void k_ext_average(float* __restrict__ v, const int* __restrict__ mark, int nx, int ny, int nz, int wave) {
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= int64_t(nx) * ny * nz || mark[c] != wave) return;
    const int i = int(c % nx), j = int((c / nx) % ny), k = int(c / (int64_t(nx) * ny));
    float avg = 0.0f;
    int used = 0;
    for (int ox = -1; ox <= 1; ++ox)
        for (int oy = 1; oy >= -1; --oy)
            for (int oz = -1; oz <= 1; ++oz) {
                if (ox == 0 && oy == 0 && oz == 0) continue;
                const int a = i + ox, b = j + oy, e = k + oz;
                if (a < 0 || a >= nx || b < 0 || b >= ny || e < 0 || e >= nz) continue;
                const int64_t q = a + int64_t(b) * nx + int64_t(e) * nx * ny;
                if (mark[q] < wave) {
                    avg = __fadd_rn(avg, v[q]);
                    ++used;
                }
            }
    // used is 0 only for a first-front value that the stride-W test admitted
    // without a truly known neighbour: 0/0 = NaN, as in the reference
    v[c] = __fdiv_rn(avg, float(used));
}

unsigned blocks(int64_t n) { return unsigned((n + 255) / 256); }

void run_waves(float* v, int* mark, int nx, int ny, int nz, int depth, int front_stride, cudaStream_t st) {
    const int64_t n = int64_t(nx) * ny * nz;
    for (int w = 1; w <= depth; ++w) {
        k_ext_front<<<blocks(n), 256, 0, st>>>(mark, nx, ny, nz, w, front_stride);
        k_ext_average<<<blocks(n), 256, 0, st>>>(v, mark, nx, ny, nz, w);
    }
}

}  // namespace

int launch_extrapolate_unknown(float* v, int nx, int ny, int depth, int front_stride, int* mark, cudaStream_t st) {
    const int64_t n = int64_t(nx) * ny;
    k_ext_known_value<<<blocks(n), 256, 0, st>>>(v, n, mark);
    run_waves(v, mark, nx, ny, 1, depth, front_stride, st);
    return 1 + 2 * depth;
}

int launch_extrapolate_from_fluid(float* v, int axis, const uint8_t* labels, Dims g, int depth, int* mark,
                                  cudaStream_t st) {
    const int nx = g.W + (axis == 0), ny = g.H + (axis == 1), nz = g.D + (axis == 2);
    k_ext_known_fluid<<<blocks(int64_t(nx) * ny * nz), 256, 0, st>>>(labels, g, axis, mark);
    run_waves(v, mark, nx, ny, nz, depth, nx, st);
    return 1 + 2 * depth;
}

}  // namespace fp
