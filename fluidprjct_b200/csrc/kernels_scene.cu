// kernels_scene.cu -- scene generation on the device: labels from level sets
// and the seabed scene.
//
// Level sets (DistrGen/fluidLevelSets.py + fluidLabels.py): a solid and a
// fluid signed-distance grid combine into labels, SOLID where phi_solid < 0,
// else FLUID where phi_fluid < 0, else AIR (generate_combined_labels_simple).
//
// Seabed: SOLID walls, a bed of height base + amp * noise(x, z) and water to
// y < level for x >= water_xmin (the wave-tank scene; no reference
// counterpart).  The noise is multi-octave value noise whose lattice values
// come from a splitmix64 hash of (seed, octave, i, j), evaluated in double with
// explicit round-to-nearest operations, so that the Python generator
// (fluidprjct_b200/scenes.py) produces the same labels bit for bit.
#include "kernels.hpp"

namespace fp {
namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// lattice value in [0, 1) at integer point (a, b) of octave o
__device__ __forceinline__ double lattice(uint64_t seed, int o, int a, int b) {
    const uint64_t key = (uint64_t(o) << 42) ^ (uint64_t(uint32_t(a)) << 21) ^ uint64_t(uint32_t(b));
    return double(splitmix64(seed ^ splitmix64(key)) >> 11) * 0x1.0p-53;
}
__device__ __forceinline__ double smooth(double f) { return __dmul_rn(__dmul_rn(f, f), __dsub_rn(3.0, __dmul_rn(2.0, f))); }
__device__ __forceinline__ double lerp(double a, double b, double f) {
    return __dadd_rn(__dmul_rn(a, __dsub_rn(1.0, f)), __dmul_rn(b, f));
}

// value noise in [0, 1] at column (i, k) of an nx x nz grid (octaves 4, 8, 16, ... lattice cells)
__device__ double value_noise(int i, int k, int nx, int nz, int octaves, uint64_t seed) {
    double out = 0.0, amp = 1.0, tot = 0.0;
    for (int o = 0; o < octaves; ++o) {
        const int cells = 4 << o;
        const double zs = __dmul_rn(double(k), __ddiv_rn(double(cells), double(nz)));
        const double xs = __dmul_rn(double(i), __ddiv_rn(double(cells), double(nx)));
        const int z0 = int(zs), x0 = int(xs);
        const double fz = smooth(__dsub_rn(zs, double(z0))), fx = smooth(__dsub_rn(xs, double(x0)));
        const double top = lerp(lattice(seed, o, z0, x0), lattice(seed, o, z0, x0 + 1), fx);
        const double bot = lerp(lattice(seed, o, z0 + 1, x0), lattice(seed, o, z0 + 1, x0 + 1), fx);
        out = __dadd_rn(out, __dmul_rn(amp, lerp(top, bot, fz)));
        tot = __dadd_rn(tot, amp);
        amp = __dmul_rn(amp, 0.5);
    }
    return __ddiv_rn(out, tot);
}

// One thread per (x, z) column.
__global__ void k_seabed_labels(uint8_t* __restrict__ lab, int W, int H, int D, double dx, double level,
                                double bed_base, double bed_amp, uint64_t seed, double water_xmin) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(W) * D) return;
    const int i = int(t % W), k = int(t / W);
    const double bed = __dadd_rn(bed_base, __dmul_rn(bed_amp, value_noise(i, k, W, D, 4, seed)));
    const double x = __dmul_rn(__dadd_rn(double(i), 0.5), dx);
    for (int j = 0; j < H; ++j) {
        const double y = __dmul_rn(__dadd_rn(double(j), 0.5), dx);
        uint8_t l;
        if (i == 0 || i == W - 1 || j == 0 || j == H - 1 || k == 0 || k == D - 1 || y < bed) l = SOLID;
        else if (y < level && x >= water_xmin) l = FLUID;
        else l = AIR;
        lab[i + int64_t(j) * W + int64_t(k) * W * H] = l;
    }
}

__global__ void k_levelset_labels(const float* __restrict__ solid, const float* __restrict__ fluid, int64_t n,
                                  uint8_t* __restrict__ lab) {
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= n) return;
    lab[c] = solid[c] < 0.0f ? SOLID : fluid[c] < 0.0f ? FLUID : AIR;
}

}  // namespace

void launch_seabed_labels(uint8_t* labels, int W, int H, int D, double dx, double level, double bed_base,
                          double bed_amp, uint64_t seed, double water_xmin, cudaStream_t st) {
    const int64_t n = int64_t(W) * D;
    k_seabed_labels<<<unsigned((n + 127) / 128), 128, 0, st>>>(labels, W, H, D, dx, level, bed_base, bed_amp, seed,
                                                                water_xmin);
}

void launch_levelset_labels(const float* solid, const float* fluid, int64_t n, uint8_t* labels, cudaStream_t st) {
    k_levelset_labels<<<unsigned((n + 255) / 256), 256, 0, st>>>(solid, fluid, n, labels);
}

}  // namespace fp
