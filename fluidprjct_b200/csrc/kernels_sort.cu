// kernels_sort.cu -- labelling and the counting sort of particles by cell.
//
// Replaces labelGrid (FluidSolver3D.cu:340-397: ClearNonSolidFunctor,
// MarkBodyCellsFunctor, MarkFluidCellsFunctor).  The cell key is the
// reference's floorf(p/dx) with its clamp, so labels are bit-identical; the
// FLUID mark falls out of the per-cell particle counts that the sort needs
// anyway.  The sort is a counting sort: one atomic per particle for its rank
// in its cell, a three-pass exclusive scan of the counts into cell offsets,
// and a scatter of the particle records into cell order.
#include "kernels.hpp"
#include "scan.cuh"

namespace fp {

namespace {
constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

// Particles arrive nearly in cell order (sorted last step, moved less than a
// cell), so a warp's lanes share a few cells: one atomic per distinct cell of
// the warp (lanes grouped by __match_any_sync), each lane's rank the group's
// base plus its place among the group's lanes.  The order of a cell's
// particles is arbitrary either way.  Every lane of every warp reaches the
// match (the block size is a multiple of 32; lanes past np carry key -1).
template <bool P2>
__global__ void k_bin(const float4* __restrict__ pos, int64_t np, Dims g, int* __restrict__ counts,
                      int* __restrict__ key, int* __restrict__ rank) {
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool ok = q < np;
    int c = -1;
    if (ok) {
        const float4 p = pos[q];
        c = cell_key<P2>(p.x, p.y, p.z, g);
    }
    const unsigned grp = __match_any_sync(0xffffffffu, c);
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    int base = 0;
    if (ok && lane == leader) base = atomicAdd(&counts[c], __popc(grp));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (ok) {
        key[q] = c;
        rank[q] = base + __popc(grp & ((1u << lane) - 1u));
    }
}

__device__ __forceinline__ uint8_t label_of(uint8_t base, uint8_t body, int count) {
    if (base == SOLID) return SOLID;        // ClearNonSolidFunctor keeps SOLID
    if (body) return BODY;                  // MarkBodyCellsFunctor
    return count > 0 ? FLUID : AIR;         // MarkFluidCellsFunctor
}

// Pass 1: labels and the per-tile sums of the counts.
__global__ void __launch_bounds__(SCAN_BLOCK) k_label_tiles(const uint8_t* __restrict__ base,
                                                            const uint8_t* __restrict__ body,
                                                            const int* __restrict__ counts,
                                                            uint8_t* __restrict__ labels, int64_t nc,
                                                            int* __restrict__ tile_sums) {
    int64_t e0 = int64_t(blockIdx.x) * SCAN_TILE + int64_t(threadIdx.x) * SCAN_ITEMS;
    int s = 0;
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; ++t) {
        int64_t e = e0 + t;
        if (e < nc) {
            int c = counts[e];
            s += c;
            labels[e] = label_of(base[e], body ? body[e] : 0, c);
        }
    }
    int total;
    block_exclusive_scan<SCAN_BLOCK>(s, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Pass 3: exclusive scan inside each tile plus the tile offset.
__global__ void __launch_bounds__(SCAN_BLOCK) k_start_tiles(const int* __restrict__ counts, int64_t nc,
                                                            const int* __restrict__ tile_offsets,
                                                            int* __restrict__ start) {
    int64_t e0 = int64_t(blockIdx.x) * SCAN_TILE + int64_t(threadIdx.x) * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; ++t) {
        int64_t e = e0 + t;
        v[t] = e < nc ? counts[e] : 0;
        s += v[t];
    }
    int total;
    int pre = block_exclusive_scan<SCAN_BLOCK>(s, total) + tile_offsets[blockIdx.x];
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; ++t) {
        int64_t e = e0 + t;
        if (e < nc) start[e] = pre;
        pre += v[t];
    }
}

__global__ void k_scatter(const float4* __restrict__ pos, const float4* __restrict__ vel,
                          const int* __restrict__ key, const int* __restrict__ rank,
                          const int* __restrict__ start, int64_t np, float4* __restrict__ pos2,
                          float4* __restrict__ vel2) {
    int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= np) return;
    int slot = start[key[q]] + rank[q];
    pos2[slot] = pos[q];
    vel2[slot] = vel[q];
}
}  // namespace

__global__ void k_scan_single_block(int* data, int n, int* total) {
    int carry = 0;
    for (int base = 0; base < n; base += 1024) {
        int i = base + threadIdx.x;
        int v = i < n ? data[i] : 0;
        int tot;
        int pre = block_exclusive_scan<1024>(v, tot);
        if (i < n) data[i] = carry + pre;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

void launch_bin(const float4* pos, int64_t np, Dims g, int* counts, int* key, int* rank, cudaStream_t st) {
    if (np == 0) return;
    const unsigned nb = unsigned((np + 255) / 256);
    if (g.idx != 0.0f) k_bin<true><<<nb, 256, 0, st>>>(pos, np, g, counts, key, rank);
    else k_bin<false><<<nb, 256, 0, st>>>(pos, np, g, counts, key, rank);
}

void launch_label_scan(const uint8_t* base, const uint8_t* body_mark, const int* counts, uint8_t* labels, int* start,
                       int* tile_sums, Dims g, cudaStream_t st) {
    int64_t nc = g.nc();
    int ntiles = int((nc + SCAN_TILE - 1) / SCAN_TILE);
    k_label_tiles<<<ntiles, SCAN_BLOCK, 0, st>>>(base, body_mark, counts, labels, nc, tile_sums);
    k_scan_single_block<<<1, 1024, 0, st>>>(tile_sums, ntiles, start + nc);  // start[nc] = np
    k_start_tiles<<<ntiles, SCAN_BLOCK, 0, st>>>(counts, nc, tile_sums, start);
}

void launch_scatter(const float4* pos, const float4* vel, const int* key, const int* rank, const int* start, int64_t np,
                    float4* pos2, float4* vel2, cudaStream_t st) {
    if (np == 0) return;
    k_scatter<<<unsigned((np + 255) / 256), 256, 0, st>>>(pos, vel, key, rank, start, np, pos2, vel2);
}

}  // namespace fp
