// fieldconvert_main.cpp -- the fieldConvert post-processor: .LBMBin -> VTS.
//
// Drop-in for the reference's applications/fieldConvert (fieldConvert.cu:52-113,
// fieldConvert.cuh) for its VTS writer and cut planes.  Run inside a case
// directory:
//
//   fieldConvert -fileType vts [-fieldName S|SMean|k|kMean|momentsMean]
//                [-cutPlane x=0.5|y=...|z=...] [-latestTime] [-GPU ids]
//
// For every <prefix>_<t>.LBMBin (prefix = the case name, or -fieldName) it
// writes postProcess/<prefix>_<t>.vts, or with -cutPlane
// postProcess/<prefix>CutPlane_<d>=<c>_<t>.vts holding the plane (a mesh one
// node thick).  The files match the reference's byte for byte, including its
// cut-plane interpolation weight (see postprocess.hpp).  Other -fileType
// values of the reference (vtu, tecplot) are not provided.  The start-up
// blocks (programControl, latticeMesh) are printed as the solvers print them.
// -GPU is optional (device 0) and only printed: nothing here runs on a GPU.
#include <cstdio>
#include <filesystem>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "casefile.hpp"
#include "lbmbin.hpp"
#include "postprocess.hpp"

namespace fs = std::filesystem;

namespace {

const std::vector<std::string> kMoments = {"rho", "u", "v", "w", "m_xx", "m_xy", "m_xz", "m_yy", "m_yz", "m_zz"};

// functionObjects::fieldComponentsMap of the reference (functionObjects.cuh:65-70)
const std::map<std::string, std::vector<std::string>> kFieldComponents = {
    {"momentsMean", {"rhoMean", "uMean", "vMean", "wMean", "m_xxMean", "m_xyMean", "m_xzMean", "m_yyMean", "m_yzMean",
                     "m_zzMean"}},
    {"S", {"S_xx", "S_xy", "S_xz", "S_yy", "S_yz", "S_zz"}},
    {"SMean", {"S_xxMean", "S_xyMean", "S_xzMean", "S_yyMean", "S_yzMean", "S_zzMean"}},
    {"k", {"k"}},
    {"kMean", {"kMean"}}};

struct Args {
    std::string program;
    std::vector<int> gpus;
    std::vector<std::string> v;
    bool present(const std::string &name) const
    {
        for (const auto &a : v)
            if (a == name)
                return true;
        return false;
    }
    std::string value(const std::string &name) const
    {
        for (size_t i = 0; i + 1 < v.size(); i++)
            if (v[i] == name)
                return v[i + 1];
        throw lbm::CaseError("Input argument " + name + " has not been supplied with a value");
    }
};

// -cutPlane d=c: direction character before an '=' at position 1
// (fieldConvert.cuh:165-191), coordinate parsed as long double then float.
bool parse_cut_plane(const std::string &s, int &axis, float &coord)
{
    if (s.size() < 3 || s[1] != '=' || s.find('=') != 1)
        return false;
    if (s[0] == 'x')
        axis = 0;
    else if (s[0] == 'y')
        axis = 1;
    else if (s[0] == 'z')
        axis = 2;
    else
        return false;
    coord = static_cast<float>(std::stold(s.substr(2)));
    return true;
}

void report_write(const std::string &file, uint64_t bytes, bool dir_existed)
{
    std::cout << "vtsWriter:" << std::endl << "{" << std::endl;
    std::cout << "    fileName: " << file << ";" << std::endl;
    if (dir_existed)
        std::cout << "    directoryStatus: OK;" << std::endl;
    std::cout << "    fileSize: " << double(bytes) / (1024.0 * 1024.0) << " MiB;" << std::endl;
    std::cout << "    ofstreamStatus: OK;" << std::endl;
    std::cout << "    writeStatus: success;" << std::endl << "};" << std::endl << std::endl;
}

int run(const Args &args)
{
    const lbm::ProgramControl pc = lbm::read_program_control(".");
    const std::vector<uint64_t> saved = lbm::time_indices(".", pc.caseName);
    lbm::print_program_control(pc, args.program, args.gpus, saved.empty() ? 0 : saved.back());
    const lbm::LatticeMesh mesh = lbm::read_lattice_mesh(".");
    lbm::print_lattice_mesh(mesh);
    const bool custom = args.present("-fieldName");
    const std::string prefix = custom ? args.value("-fieldName") : pc.caseName;
    std::vector<std::string> names = kMoments;
    if (custom) {
        auto it = kFieldComponents.find(prefix);
        if (it == kFieldComponents.end())
            throw lbm::CaseError("Invalid argument passed to -fieldName");
        names = it->second;
    }
    const std::string type = args.value("-fileType");
    if (type != "vts")
        throw lbm::CaseError("Unsupported conversion format: " + type + "\nSupported formats are: vts");
    const bool cut = args.present("-cutPlane");
    int axis = 0;
    float coord = 0.0f;
    std::string cut_arg;
    if (cut) {
        cut_arg = args.value("-cutPlane");
        if (!parse_cut_plane(cut_arg, axis, coord))
            throw lbm::CaseError("Invalid cardinal direction");
    }
    const std::vector<uint64_t> times = lbm::time_indices(".", prefix);
    if (times.empty())
        throw lbm::CaseError("No " + prefix + "_<t>.LBMBin files in the case directory");
    const float L[3] = {mesh.Lx, mesh.Ly, mesh.Lz};
    const uint64_t n = mesh.nx * mesh.ny * mesh.nz;
    const size_t first = args.present("-latestTime") ? times.size() - 1 : 0;
    for (size_t k = first; k < times.size(); k++) {
        const std::string src = prefix + "_" + std::to_string(times[k]) + ".LBMBin";
        const lbm::FieldFileHeader h = lbm::read_field_header(src);
        if (h.nx != mesh.nx || h.ny != mesh.ny || h.nz != mesh.nz)
            throw lbm::CaseError(src + " does not match the mesh in latticeMesh");
        std::vector<float> tiled;
        tiled.reserve(names.size() * n);
        for (const std::string &name : names) {
            const std::vector<float> f = lbm::read_field_by_name(src, name);
            tiled.insert(tiled.end(), f.begin(), f.end());
        }
        lbm::FieldSet fields = lbm::tiled_to_global(tiled, mesh.nx, mesh.ny, mesh.nz);
        uint64_t ox = mesh.nx, oy = mesh.ny, oz = mesh.nz;
        std::string out_name = prefix + "_" + std::to_string(times[k]);
        if (cut) {
            fields = lbm::cut_plane(fields, mesh.nx, mesh.ny, mesh.nz, L, axis, coord, true);
            (axis == 0 ? ox : axis == 1 ? oy : oz) = 1;
            out_name = prefix + "CutPlane_" + cut_arg + "_" + std::to_string(times[k]);
        }
        const bool existed = fs::is_directory("postProcess");
        if (!existed && !fs::create_directory("postProcess"))
            throw lbm::CaseError("unable to create directory postProcess");
        const std::string path = "postProcess/" + out_name + ".vts";
        lbm::write_vts(path, fields, names, ox, oy, oz, L);
        report_write(path, lbm::vts_file_bytes(ox, oy, oz, names), existed);
    }
    return 0;
}

}  // namespace

int main(int argc, char **argv)
{
    Args args;
    args.program = argv[0];
    for (int i = 1; i < argc; i++)
        args.v.emplace_back(argv[i]);
    try {
        args.gpus = lbm::parse_gpu_list(argc, argv, false);
        return run(args);
    } catch (const std::exception &e) {
        std::cerr << fs::path(argv[0]).filename().string() << ": " << e.what() << std::endl;
        return 1;
    }
}
