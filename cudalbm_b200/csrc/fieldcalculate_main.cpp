// fieldcalculate_main.cpp -- the fieldCalculate post-processor's checks.
//
// Drop-in for the reference's applications/fieldCalculate
// (fieldCalculate.cu:52-105, fieldCalculate.cuh:74-170) for its two
// reductions.  Run inside a case directory:
//
//   fieldCalculate -calculationType containsNaN|spatialMean [-latestTime] [-GPU id]
//
// For every <caseName>_<t>.LBMBin (only the last with -latestTime) it reads
// the ten moment fields and prints, per time, the reference's block:
// containsNaN names every field holding a NaN (or says there is none),
// spatialMean prints mean(<field>) for each field -- the reference's
// left-to-right float sum in global node order over float(nodes), computed
// on the GPU by lbm_field_statistics, so the digits are the reference's.
// The start-up blocks (programControl, latticeMesh) are printed as the
// solvers print them.  -GPU is optional (device 0), as in the reference.
// The reference's other calculation types (vorticity, div[U]) are not
// provided: they fail with a message; an absent or unknown -calculationType
// does nothing, as in the reference.
#include <filesystem>
#include <iostream>
#include <string>
#include <vector>

#include "casefile.hpp"
#include "lbm_b200.h"
#include "lbmbin.hpp"

namespace fs = std::filesystem;

namespace {

const std::vector<std::string> kMoments = {"rho", "u", "v", "w", "m_xx", "m_xy", "m_xz", "m_yy", "m_yz", "m_zz"};

bool present(int argc, char **argv, const std::string &name)
{
    for (int i = 1; i < argc; i++)
        if (name == argv[i])
            return true;
    return false;
}

std::string value(int argc, char **argv, const std::string &name)
{
    for (int i = 1; i + 1 < argc; i++)
        if (name == argv[i])
            return argv[i + 1];
    throw lbm::CaseError("Input argument " + name + " has not been supplied with a value");
}

void check(lbm_status s)
{
    if (s != LBM_OK)
        throw lbm::CaseError(std::string(lbm_status_string(s)) + ": " + lbm_last_error());
}

int run(int argc, char **argv)
{
    const std::vector<int> gpus = lbm::parse_gpu_list(argc, argv, false);
    const lbm::ProgramControl pc = lbm::read_program_control(".");
    const std::vector<uint64_t> times = lbm::time_indices(".", pc.caseName);
    lbm::print_program_control(pc, argv[0], gpus, times.empty() ? 0 : times.back());
    const lbm::LatticeMesh mesh = lbm::read_lattice_mesh(".");
    lbm::print_lattice_mesh(mesh);

    const std::string type = present(argc, argv, "-calculationType") ? value(argc, argv, "-calculationType") : "";
    if (type == "vorticity" || type == "div[U]")
        throw lbm::CaseError("-calculationType " + type + " is not provided (containsNaN and spatialMean are)");
    if (type != "containsNaN" && type != "spatialMean")
        return 0;
    const bool nan_check = type == "containsNaN";
    const uint64_t n = mesh.nx * mesh.ny * mesh.nz;
    const size_t first = present(argc, argv, "-latestTime") && !times.empty() ? times.size() - 1 : 0;
    for (size_t k = first; k < times.size(); k++) {
        const std::string src = pc.caseName + "_" + std::to_string(times[k]) + ".LBMBin";
        const lbm::FieldFileHeader h = lbm::read_field_header(src);
        if (h.nx != mesh.nx || h.ny != mesh.ny || h.nz != mesh.nz)
            throw lbm::CaseError(src + " does not match the mesh in latticeMesh");
        std::vector<float> tiled;
        tiled.reserve(kMoments.size() * n);
        for (const std::string &name : kMoments) {
            const std::vector<float> f = lbm::read_field_by_name(src, name);
            tiled.insert(tiled.end(), f.begin(), f.end());
        }
        const int nf = int(kMoments.size());
        std::vector<int32_t> nan(nf);
        std::vector<float> mean_ref(nf);
        std::vector<double> mean(nf);
        check(lbm_field_statistics(gpus[0], tiled.data(), int64_t(mesh.nx), int64_t(mesh.ny), int64_t(mesh.nz), nf,
                                   LBM_ORDER_TILED, nan.data(), mean_ref.data(), mean.data()));
        std::cout << "Time: " << times[k] << std::endl << "{" << std::endl;
        if (nan_check) {
            int fields_with_nan = 0;
            for (int f = 0; f < nf; f++)
                if (nan[f] > 0) {
                    std::cout << "    NaN detected in field " << kMoments[f] << std::endl;
                    fields_with_nan++;
                }
            if (fields_with_nan == 0)
                std::cout << "    No NaN values detected in any field." << std::endl;
            else
                std::cout << "    Total number of fields with NaN values: " << fields_with_nan << std::endl;
        } else {
            for (int f = 0; f < nf; f++)
                std::cout << "    mean(" << kMoments[f] << "): " << mean_ref[f] << ";" << std::endl;
        }
        std::cout << "};" << std::endl << std::endl;
    }
    std::cout << "End" << std::endl << std::endl;
    return 0;
}

}  // namespace

int main(int argc, char **argv)
{
    try {
        return run(argc, argv);
    } catch (const std::exception &e) {
        std::cerr << fs::path(argv[0]).filename().string() << ": " << e.what() << std::endl;
        return 1;
    }
}
