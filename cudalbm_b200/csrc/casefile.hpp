// casefile.hpp -- reader of the cudaLBM case files.
//
// Same grammar and lookup rules as the reference (src/strings.cuh,
// src/programControl/programControl.cuh, src/latticeMesh/latticeMesh.cuh,
// src/boundaryConditions/boundaryValue.cuh, src/functionObjects/
// functionObjects.cuh), so every case directory the reference runs is read
// to the same values:
//   * "key value;" lines are found by substring match on the key; the value
//     is the second space-separated token without its last character;
//   * "name { ... };" blocks are located by a line that starts with the name
//     and delimited by brace counting, "//" starting a comment;
//   * function objects are enabled by an exact "S;" / "kMean;" ... line
//     inside functionObjectList (commented lines do not match).
// Errors throw lbm::CaseError with the reference's message where it has one.
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace lbm {

struct CaseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

using Lines = std::vector<std::string>;

Lines read_lines(const std::string &path);
std::string trim(const std::string &s, bool strip_semicolon = false);
std::string parameter_string(const Lines &lines, const std::string &name);
Lines extract_block(const Lines &lines, const std::string &name);
bool is_number(const std::string &s);

struct ProgramControl {
    std::string caseName;
    float Re = 0.0f;
    float u_inf = 0.0f;
    uint64_t nTimeSteps = 0, saveInterval = 1, infoInterval = 1;
};

struct LatticeMesh {
    uint64_t nx = 0, ny = 0, nz = 0;
    float Lx = 0, Ly = 0, Lz = 0;
};

ProgramControl read_program_control(const std::string &dir);
LatticeMesh read_lattice_mesh(const std::string &dir);

// region values [field][region], fields in moment order, regions
// internalField, North, South, East, West, Front, Back, scaled as stored
// (rho as is, u*3, m_aa*4.5, m_ab*9; equilibrium = 4.5*u_a*u_b/rho0).
std::array<float, 70> read_initial_conditions(const std::string &dir);

// LBM_FO_* mask from the functionObjects file (0 if the file is absent).
uint32_t read_function_objects(const std::string &dir);

// Time indices of <prefix>_<n>.LBMBin files in dir, sorted (fileIO.cuh:98-233).
std::vector<uint64_t> time_indices(const std::string &dir, const std::string &prefix);

// The programControl and latticeMesh blocks every reference executable prints
// on start-up (programControl.cuh:86-120 without its banner, latticeMesh.cuh:95-104);
// latestTime = the last saved time of the case (0 if none).
void print_program_control(const ProgramControl &pc, const std::string &program, const std::vector<int> &devices,
                           uint64_t latest);
void print_lattice_mesh(const LatticeMesh &mesh);

// -GPU <ids> of the command line ("0,1"); `required` as for the solvers,
// else device 0 when absent (the post-processors, inputControl.cuh:204-226).
std::vector<int> parse_gpu_list(int argc, char **argv, bool required);

}  // namespace lbm
