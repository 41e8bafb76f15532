// io.hpp -- host-side scene and particle I/O in the reference's formats.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fluidprjct.h"

namespace fp::io {

// 3D label file (FluidSolver3D::init, FluidSolver3D.cu:81-153): "W H D" then
// W*H*D characters S/F/A read in fully reversed order (k, j, i descending).
// Unknown characters and truncation are errors (the reference leaves such
// cells at their zero-initialised value, SOLID, or reads past the end).
bool read_labels3d(const std::string& path, int& W, int& H, int& D, std::vector<uint8_t>& out, std::string& err);
// 2D label file (FluidSolver2D::init, FluidSolver2D.cu:52-104): "W H" then rows
// from the top (j = H-1) to the bottom, columns ascending.
bool read_labels2d(const std::string& path, int& W, int& H, std::vector<uint8_t>& out, std::string& err);
// 2D level-set file of DistrGen/fluidLevelSets.py: "<S|F> w h", then h rows of
// w floats from the top row (j = h-1) down; out[i + j*w].
bool read_levelset2d(const std::string& path, char& kind, int& W, int& H, std::vector<float>& out, std::string& err);

// PLY vertices (ascii or binary_little_endian; float or double x y z and
// optional vx vy vz).  The reference writes ascii positions only
// (utility.cu:91-109) and has no reader.
bool read_ply(const std::string& path, std::vector<float>& pos, std::vector<float>& vel, bool& has_vel, std::string& err);
// format: FP_OUT_PLY (ascii, positions; utility.cu:91-109), FP_OUT_OFF
// (utility.cu:111-127), FP_OUT_PLY_BINARY (little-endian float x y z vx vy vz).
// A frame from records x y z vx vy vz (6 floats per particle): binary PLY
// writes them as they are; ASCII PLY / OFF format the positions.
bool write_frame_records(const std::string& path, const float* rec, int64_t n, int format, std::string& err);
bool write_particles(const std::string& path, const float* pos, const float* vel, int64_t n, int format,
                     std::string& err);

// seedParticles (FluidSolver3D.cu:213-297) with std::mt19937(seed): for every
// FLUID cell in i-fastest order, ppc particles at a random octant centre
// jittered by U(-0.24, 0.24)*dx and clamped to the cell.  2D
// (FluidSolver2D.cu:114-158): quadrants instead of octants.
int64_t seed_particles(const uint8_t* labels, int W, int H, int D, float dx, int ppc, uint32_t seed,
                       std::vector<float>& pos);

// Reference config.json (main.cpp:17-52) plus the added keys.
bool load_config_json(const std::string& path, fp_config& cfg, std::string* label_path, int* frames, std::string& err);

// Body SDF text file (RigidBody::loadSDF, utility.cuh:231-338): "w h d",
// origin, cell size, then w*h*d floats in i-fastest order.
bool read_sdf(const std::string& path, int& w, int& h, int& d, float origin[3], float& cell, std::vector<float>& data,
              std::string& err);

}  // namespace fp::io
