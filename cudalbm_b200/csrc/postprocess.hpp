// postprocess.hpp -- cut planes and the VTS (VTK structured grid) writer of
// the fieldConvert post-processor (reference applications/fieldConvert and
// src/postProcess/VTS.cuh), host side.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace lbm {

using FieldSet = std::vector<std::vector<float>>;  // [variable][node], node = x + nx*(y + ny*z)

// [field][block-tiled node] (the .LBMBin order) -> global order.
// Reference: fileIO::deinterleaveAoS (src/fileIO/fileInput.cuh:776-822).
FieldSet tiled_to_global(const std::vector<float> &tiled, uint64_t nx, uint64_t ny, uint64_t nz);

// Plane normal to `axis` (0 x, 1 y, 2 z) at `coordinate` in units of the
// domain length (0 = first node, 1 = last node when L = 1), linearly
// interpolated between the two bracketing node planes.  Output layout per
// variable: x-cut [z][y], y-cut [z][x], z-cut [y][x].
//   reference_weight = true: the reference's arithmetic
//   (applications/fieldConvert/fieldConvert.cuh:236-326): float index
//   (n-1)*(coordinate*L), floor/ceil, and weight = coordinate - floor(index),
//   which equals the true weight only when the index is an integer (a plane
//   through nodes) and extrapolates otherwise; kept for drop-in output.
//   reference_weight = false: weight = index - floor(index).
// Throws CaseError if the index falls outside [0, n-1].
FieldSet cut_plane(const FieldSet &fields, uint64_t nx, uint64_t ny, uint64_t nz, const float L[3], int axis,
                   float coordinate, bool reference_weight);

// Interleaved point coordinates (x, y, z per node) of a mesh, as the
// reference computes them (src/postProcess/postProcess.cuh:73-100): in double,
// L * i / (n - 1), and 0 along a dimension with a single node.
std::vector<float> mesh_coordinates(uint64_t nx, uint64_t ny, uint64_t nz, const float L[3]);

// Bytes of the .vts file write_vts produces.
uint64_t vts_file_bytes(uint64_t nx, uint64_t ny, uint64_t nz, const std::vector<std::string> &names);

// VTK XML structured grid, appended raw binary data with UInt64 block
// headers (the reference's VTS writer, src/postProcess/VTS.cuh:68-136 and postProcess.cuh:218-226).
void write_vts(const std::string &path, const FieldSet &fields, const std::vector<std::string> &names, uint64_t nx,
               uint64_t ny, uint64_t nz, const float L[3]);

}  // namespace lbm
