// ref3d_harness.cu -- runs phases of the reference's own 3D solver
// (src/FluidSim/FluidSolver3D.cu, compiled unmodified beside this file) on
// given particles, to produce golden fixtures for the oracle.
//
// TEST INFRASTRUCTURE ONLY (the checker's pins).  Built into oracle/_ref/ by
// the Makefile beside this file, from the reference sources of a checkout
// named by FLUIDPRJCT_REFERENCE; tests/golden/make_refrun_golden.py calls it
// once on a GPU and commits what it returns.  The step phases are private
// members of FluidSolver3D, so this file alone makes them accessible by
// defining `private` as `public` around the class header; the class layout is
// the same in both translation units.
//
// ref3d_run: FluidSolver3D(5, 5, 5, dx, dt) with activeBody off, then the
// reference's init(label_file) (grid sizing, label reading, its own seeding,
// replaced at once by the given particles), then labelGrid,
// particlesToGrid, saveVelocities, applyForces (FluidSolver3D.cu:340-761),
// copying the labels and the face grids out after P2G and after the forces;
// then, with the given face grids u, v, w, u*, v*, w* in place,
// gridToParticles(alpha) and advectParticles(C) (:803-1357), copying the
// particles out.  pressureSolve and applyPressure are never called (they need
// cuDSS, and their border reads assume more than a solid wall).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <cusparse.h>
#include <thrust/copy.h>
#include <thrust/count.h>
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/for_each.h>
#include <thrust/functional.h>
#include <thrust/generate.h>
#include <thrust/host_vector.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/permutation_iterator.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/random.h>
#include <thrust/sort.h>
#include <thrust/transform.h>

#include "cudss.h"

#define private public
#define protected public
#include "FluidSolver3D.cuh"
#undef protected
#undef private

namespace {

void grid_out(Utility::Grid3D<float>& g, float* out) {
    thrust::host_vector<float> h = g.device_data;
    for (size_t i = 0; i < h.size(); ++i) out[i] = h[i];
}
void grid_in(Utility::Grid3D<float>& g, const float* in) {
    thrust::host_vector<float> h(g.device_data.size());
    for (size_t i = 0; i < h.size(); ++i) h[i] = in[i];
    g.device_data = h;
}

}  // namespace

extern "C" int ref3d_run(const char* label_file, float dx, float dt, float alpha, float C, int64_t np,
                         const float* pos, const float* vel, const float* g2p_grids, int* labels_out,
                         float* p2g_out, float* forces_out, float* pos_out, float* vel_out) {
    try {
        FluidSolver3D s(5, 5, 5, dx, dt);
        s.activeBody = false;
        s.init(label_file);
        const int W = s.gridWidth, H = s.gridHeight, D = s.gridDepth;
        const size_t nu = size_t(W + 1) * H * D, nv = size_t(W) * (H + 1) * D, nw = size_t(W) * H * (D + 1);
        s.h_particles.clear();
        for (int64_t q = 0; q < np; ++q)
            s.h_particles.push_back(Utility::Particle3D(make_float3(pos[3 * q], pos[3 * q + 1], pos[3 * q + 2]),
                                                        make_float3(vel[3 * q], vel[3 * q + 1], vel[3 * q + 2])));
        s.d_particles = s.h_particles;
        if (s.labelGrid() != 0) return -2;
        {
            thrust::host_vector<int> h = s.labels.device_data;
            for (size_t i = 0; i < h.size(); ++i) labels_out[i] = h[i];
        }
        s.particlesToGrid();
        grid_out(s.u, p2g_out);
        grid_out(s.v, p2g_out + nu);
        grid_out(s.w, p2g_out + nu + nv);
        s.saveVelocities();
        s.applyForces();
        grid_out(s.u, forces_out);
        grid_out(s.v, forces_out + nu);
        grid_out(s.w, forces_out + nu + nv);
        if (g2p_grids) {
            const float* g = g2p_grids;
            grid_in(s.u, g); g += nu;
            grid_in(s.v, g); g += nv;
            grid_in(s.w, g); g += nw;
            grid_in(s.uSaved, g); g += nu;
            grid_in(s.vSaved, g); g += nv;
            grid_in(s.wSaved, g);
        }
        s.gridToParticles(alpha);
        s.advectParticles(C);
        thrust::host_vector<Utility::Particle3D> out = s.d_particles;
        for (int64_t q = 0; q < np; ++q) {
            pos_out[3 * q] = out[q].pos.x; pos_out[3 * q + 1] = out[q].pos.y; pos_out[3 * q + 2] = out[q].pos.z;
            vel_out[3 * q] = out[q].vel.x; vel_out[3 * q + 1] = out[q].vel.y; vel_out[3 * q + 2] = out[q].vel.z;
        }
        return cudaDeviceSynchronize() == cudaSuccess ? 0 : -3;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref3d_run: %s\n", e.what());
        return -1;
    }
}
