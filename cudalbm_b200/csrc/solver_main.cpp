// solver_main.cpp -- the momentBasedD3Q19 / momentBasedD3Q27 executables.
//
// Drop-in replacements for the reference's applications/momentBasedD3Q19 and
// momentBasedD3Q27 (momentBasedD3Q19.cu:56-140): run inside a case directory
// with `momentBasedD3Q19 -GPU <id>`, read programControl, latticeMesh,
// initialConditions and functionObjects, restart from the latest
// <caseName>_<t>.LBMBin if there is one, and write the same .LBMBin files at
// the same steps.  The lattice is fixed at compile time (LBM_LATTICE).
//
// The time loop keeps the reference's order -- at step t: print if
// t % infoInterval == 0, save if t % saveInterval == 0, then advance -- but
// queues the steps between two such events without synchronising the device.
//
// Optional file b200Options (ignored by the reference) may set
//   meanPrecision 64;   double-precision running means;
//   restoreMeans 1;     on restart, read the function-object fields saved at
//                       the restart time (momentsMean, S, SMean, k, kMean --
//                       those the functionObjects list enables) back into the
//                       device accumulators, so that a restarted run continues
//                       its running means exactly as an uninterrupted run.
// Without restoreMeans the running means restart from zero while their count
// 1/(t+1) keeps the absolute step, as in the reference
// (src/functionObjects/strainRateTensor.cuh:331; src/array/hostArray.cuh:264-276
// restores the moments only).
#include <algorithm>
#include <array>
#include <chrono>
#include <limits>
#include <sstream>
#include <cstdio>
#include <ctime>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "casefile.hpp"
#include "lbm_b200.h"
#include "lbmbin.hpp"

#ifndef LBM_LATTICE
#define LBM_LATTICE 19
#endif

namespace {

struct Failure {
    int code;
    std::string msg;
};

void check(lbm_status s)
{
    if (s != LBM_OK)
        throw Failure{int(s), std::string(lbm_status_string(s)) + ": " + lbm_last_error()};
}

void print_velocity_set()
{
    static const int cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    static const int cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
    static const int cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    const int Q = LBM_LATTICE;
    std::cout << "D3Q" << Q << " {w, cx, cy, cz}:\n{\n";
    for (int q = 0; q < Q; q++) {
        const int n = (cx[q] != 0) + (cy[q] != 0) + (cz[q] != 0);
        const double w = Q == 19 ? (n == 0 ? 1.0 / 3 : n == 1 ? 1.0 / 18 : 1.0 / 36)
                                 : (n == 0 ? 8.0 / 27 : n == 1 ? 2.0 / 27 : n == 2 ? 1.0 / 54 : 1.0 / 216);
        std::cout << "    [" << q << "] = {" << w << ", " << cx[q] << ", " << cy[q] << ", " << cz[q] << "};\n";
    }
    std::cout << "};\n" << std::endl;
}

const std::vector<std::string> kMoments = {"rho", "u", "v", "w", "m_xx", "m_xy", "m_xz", "m_yy", "m_yz", "m_zz"};

std::vector<std::string> with_suffix(std::vector<std::string> v, const std::string &s)
{
    for (auto &x : v)
        x += s;
    return v;
}

struct Saver {
    lbm_handle *h;
    const lbm::LatticeMesh &mesh;
    uint64_t N;
    uint32_t fo;
    int mean_bits;

    void field(lbm_field_set set, const std::string &prefix, const std::vector<std::string> &names, uint64_t t,
               bool mean) const
    {
        const size_t count = names.size() * N;
        const std::string path = prefix + "_" + std::to_string(t) + ".LBMBin";
        if (mean && mean_bits == 64) {
            std::vector<double> buf(count);
            check(lbm_read_fields(h, set, buf.data(), count, LBM_F64, LBM_ORDER_TILED));
            lbm::write_field_file(path, mesh.nx, mesh.ny, mesh.nz, names, buf.data(), t, true);
        } else {
            std::vector<float> buf(count);
            check(lbm_read_fields(h, set, buf.data(), count, LBM_F32, LBM_ORDER_TILED));
            lbm::write_field_file(path, mesh.nx, mesh.ny, mesh.nz, names, buf.data(), t, mean);
        }
    }

    // the case file and then the function objects, in the reference's order
    // (objectRegistry.cuh:150-198: momentsMean, S, SMean, k, kMean)
    void all(const std::string &caseName, uint64_t t) const
    {
        field(LBM_FIELDS_MOMENTS, caseName, kMoments, t, false);
        const std::vector<std::string> S = {"S_xx", "S_xy", "S_xz", "S_yy", "S_yz", "S_zz"};
        if (fo & LBM_FO_MOMENTSMEAN)
            field(LBM_FIELDS_MOMENTSMEAN, "momentsMean", with_suffix(kMoments, "Mean"), t, true);
        if (fo & LBM_FO_S)
            field(LBM_FIELDS_S, "S", S, t, false);
        if (fo & LBM_FO_SMEAN)
            field(LBM_FIELDS_SMEAN, "SMean", with_suffix(S, "Mean"), t, true);
        if (fo & LBM_FO_K)
            field(LBM_FIELDS_K, "k", {"k"}, t, false);
        if (fo & LBM_FO_KMEAN)
            field(LBM_FIELDS_KMEAN, "kMean", {"kMean"}, t, true);
    }
};

// The function-object fields saved at step t, read back into the handle's
// accumulators (the files' names and field names as Saver::all writes them;
// 32- or 64-bit files, any mean precision of the handle).
void restore_function_objects(lbm_handle *h, uint32_t fo, uint64_t t, uint64_t N)
{
    const std::vector<std::string> S = {"S_xx", "S_xy", "S_xz", "S_yy", "S_yz", "S_zz"};
    struct Item {
        uint32_t bit;
        lbm_field_set set;
        std::string prefix;
        std::vector<std::string> names;
    };
    const Item items[] = {{LBM_FO_MOMENTSMEAN, LBM_FIELDS_MOMENTSMEAN, "momentsMean", with_suffix(kMoments, "Mean")},
                          {LBM_FO_S, LBM_FIELDS_S, "S", S},
                          {LBM_FO_SMEAN, LBM_FIELDS_SMEAN, "SMean", with_suffix(S, "Mean")},
                          {LBM_FO_K, LBM_FIELDS_K, "k", {"k"}},
                          {LBM_FO_KMEAN, LBM_FIELDS_KMEAN, "kMean", {"kMean"}}};
    for (const Item &it : items) {
        if (!(fo & it.bit))
            continue;
        const std::string file = it.prefix + "_" + std::to_string(t) + ".LBMBin";
        if (!std::filesystem::exists(file))
            throw lbm::CaseError("restoreMeans: " + file + " not found (saved function objects are needed at the restart time)");
        std::vector<double> all(it.names.size() * N);
        for (size_t f = 0; f < it.names.size(); f++) {
            const std::vector<double> v = lbm::read_field_by_name_f64(file, it.names[f]);
            if (v.size() != N)
                throw lbm::CaseError("Field size mismatch in " + file);
            std::copy(v.begin(), v.end(), all.begin() + f * N);
        }
        check(lbm_write_fields(h, it.set, all.data(), all.size(), LBM_F64, LBM_ORDER_TILED));
    }
}

std::string hms(long long s)
{
    std::ostringstream o;
    o << s / 3600 << ":" << std::setfill('0') << std::setw(2) << (s % 3600) / 60 << ":" << std::setfill('0')
      << std::setw(2) << s % 60;
    return o.str();
}

int run(int argc, char **argv)
{
    const std::vector<int> gpus = lbm::parse_gpu_list(argc, argv, true);
    const lbm::ProgramControl pc = lbm::read_program_control(".");
    const std::vector<uint64_t> times = lbm::time_indices(".", pc.caseName);
    const uint64_t latest = times.empty() ? 0 : times.back();

    lbm::print_program_control(pc, argv[0], gpus, latest);
    const lbm::LatticeMesh mesh = lbm::read_lattice_mesh(".");
    lbm::print_lattice_mesh(mesh);
    if (mesh.nx % 8 || mesh.ny % 8 || mesh.nz % 8 || !mesh.nx || !mesh.ny || !mesh.nz)
        throw lbm::CaseError("block::nx() * mesh.nxBlocks() not equal to mesh.nx()\nMesh dimensions should be multiples of 8");
    print_velocity_set();

    lbm_config cfg;
    lbm_config_default(&cfg);
    cfg.lattice = LBM_LATTICE;
    cfg.device = gpus[0];
    cfg.nx = int64_t(mesh.nx);
    cfg.ny = int64_t(mesh.ny);
    cfg.nz = int64_t(mesh.nz);
    cfg.Re = pc.Re;
    cfg.u_inf = pc.u_inf;
    cfg.function_objects = lbm::read_function_objects(".");
    cfg.start_step = int64_t(latest);
    bool restore_means = false;
    // kernel shape: the autotuner times the compiled variants on this run's
    // own state and restores it (every variant computes the same bits); by
    // default only for runs long enough to repay the trial steps
    const uint64_t steps_to_run = pc.nTimeSteps > latest ? pc.nTimeSteps - latest : 0;
    bool autotune = steps_to_run >= 1000;
    if (std::filesystem::exists("b200Options")) {
        const lbm::Lines L = lbm::read_lines("b200Options");
        try {
            cfg.mean_bits = std::stoi(lbm::parameter_string(L, "meanPrecision"));
        } catch (const lbm::CaseError &) {
        }
        try {
            restore_means = std::stoi(lbm::parameter_string(L, "restoreMeans")) != 0;
        } catch (const lbm::CaseError &) {
        }
        try {
            autotune = std::stoi(lbm::parameter_string(L, "autotune")) != 0;
        } catch (const lbm::CaseError &) {
        }
    }
    lbm_handle *h = nullptr;
    check(lbm_create(&cfg, &h));
    const uint64_t N = mesh.nx * mesh.ny * mesh.nz;

    if (!times.empty()) {
        // restart: every moment from the latest file, by name (hostArray.cuh:264-276)
        const std::string file = pc.caseName + "_" + std::to_string(latest) + ".LBMBin";
        std::vector<float> all(10 * N);
        for (int f = 0; f < 10; f++) {
            const std::vector<float> v = lbm::read_field_by_name(file, kMoments[f]);
            if (v.size() != N)
                throw lbm::CaseError("Field size mismatch in " + file);
            std::copy(v.begin(), v.end(), all.begin() + f * N);
        }
        check(lbm_write_fields(h, LBM_FIELDS_MOMENTS, all.data(), all.size(), LBM_F32, LBM_ORDER_TILED));
        // running means: from the saved files with restoreMeans, else from
        // zero as in the reference (their count keeps the absolute step)
        if (restore_means)
            restore_function_objects(h, cfg.function_objects, latest, N);
    } else {
        const std::array<float, 70> region = lbm::read_initial_conditions(".");
        check(lbm_init_regions(h, region.data()));
    }

    if (autotune) {
        // a failure here (e.g. no room for the state copy the trials need)
        // leaves the default shape in place
        lbm_tuning tuning;
        if (lbm_autotune(h, 10, &tuning) != LBM_OK)
            std::cerr << "autotune skipped: " << lbm_last_error() << std::endl;
    }

    const Saver save{h, mesh, N, cfg.function_objects, cfg.mean_bits};
    std::cout << "Time loop start\n" << std::endl;
    const auto start = std::chrono::high_resolution_clock::now();
    uint64_t t = latest;
    while (t < pc.nTimeSteps) {
        if (t % pc.infoInterval == 0) {
            check(lbm_synchronize(h));
            std::cout << "Time: " << t << std::endl;
        }
        if (t % pc.saveInterval == 0)
            save.all(pc.caseName, t);
        // advance to the next step that prints or saves
        uint64_t next = std::min(pc.nTimeSteps, std::min((t / pc.infoInterval + 1) * pc.infoInterval,
                                                         (t / pc.saveInterval + 1) * pc.saveInterval));
        check(lbm_step(h, next - t));
        t = next;
    }
    check(lbm_synchronize(h));
    const auto end = std::chrono::high_resolution_clock::now();
    const long long secs = std::chrono::duration_cast<std::chrono::seconds>(end - start).count();
    const double wall = std::chrono::duration<double>(end - start).count();
    const uint64_t nsteps = pc.nTimeSteps > latest ? pc.nTimeSteps - latest : 0;
    std::cout << "\nElapsed time: " << hms(secs) << "\n" << std::endl;
    // the reference's figure: integer seconds, nt - latestTime - 1 steps (runTimeIO.cuh:144-165)
    const double ref_mlups = secs > 0 ? double(N) * double(nsteps > 0 ? nsteps - 1 : 0) / (1e6 * double(secs))
                                      : std::numeric_limits<double>::infinity();
    std::cout << "MLUPS: " << ref_mlups << "\n" << std::endl;
    std::cout << "MLUPS (wall clock, " << nsteps << " steps incl. IO): " << (wall > 0 ? double(N) * nsteps / wall / 1e6 : 0)
              << "\n" << std::endl;
    std::cout << "End\n" << std::endl;
    lbm_destroy(h);
    return 0;
}

}  // namespace

int main(int argc, char **argv)
{
    try {
        return run(argc, argv);
    } catch (const Failure &f) {
        std::cerr << f.msg << std::endl;
        return f.code;
    } catch (const std::exception &e) {
        std::cerr << "terminate called after throwing an instance of 'std::runtime_error'\n  what():  " << e.what()
                  << std::endl;
        return 134;
    }
}
