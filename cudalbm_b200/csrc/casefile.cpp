// casefile.cpp -- see casefile.hpp.
#include "casefile.hpp"

#include <algorithm>
#include <cctype>
#include <charconv>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>

#include "lbm_b200.h"

namespace lbm {

namespace fs = std::filesystem;

Lines read_lines(const std::string &path)
{
    if (!fs::exists(path))
        throw CaseError(path + " file not opened");
    std::ifstream in(path);
    if (!in)
        throw CaseError(path + " file not opened");
    Lines out;
    std::string s;
    while (std::getline(in, s))
        out.push_back(s);
    return out;
}

std::string trim(const std::string &s, bool strip_semicolon)
{
    const char *ws = " \t\n\r\f\v";
    const size_t b = s.find_first_not_of(ws);
    if (b == std::string::npos)
        return "";
    const size_t e = s.find_last_not_of(strip_semicolon ? " \t\n\r\f\v;" : ws);
    if (e == std::string::npos || e < b)
        return "";
    return s.substr(b, e - b + 1);
}

static std::string strip_comment(const std::string &s)
{
    const size_t p = s.find("//");
    return p == std::string::npos ? s : s.substr(0, p);
}

bool is_number(const std::string &s)
{
    // [+-]digits[.digits] (reference strings.cuh isNumber)
    if (s.empty())
        return false;
    size_t i = 0;
    if (s[0] == '+' || s[0] == '-') {
        if (s.size() == 1)
            return false;
        i = 1;
    }
    bool digits = false, dot = false;
    for (; i < s.size(); i++) {
        if (std::isdigit(static_cast<unsigned char>(s[i])))
            digits = true;
        else if (s[i] == '.' && !dot)
            dot = true;
        else
            return false;
    }
    return digits;
}

std::string parameter_string(const Lines &lines, const std::string &name)
{
    for (const auto &line : lines) {
        if (line.find(name) == std::string::npos)
            continue;
        std::vector<std::string> tok;
        std::string cur;
        for (char c : line) {
            if (c == ' ') {
                if (!cur.empty())
                    tok.push_back(cur);
                cur.clear();
            } else {
                cur.push_back(c);
            }
        }
        if (!cur.empty())
            tok.push_back(cur);
        if (tok.size() < 2 || tok[1].empty())
            throw CaseError("Parameter " + name + " has no value");
        return tok[1].substr(0, tok[1].size() - 1);
    }
    throw CaseError("Parameter " + name + " not found");
}

static size_t find_block_line(const Lines &lines, const std::string &name)
{
    for (size_t i = 0; i < lines.size(); i++) {
        const std::string t = trim(strip_comment(lines[i]));
        if (t.compare(0, name.size(), name) != 0)
            continue;
        const std::string rest = trim(t.substr(name.size()));
        if (rest.empty() || rest[0] == '{' || rest[0] == ';')
            return i;
        std::istringstream iss(rest);
        std::string next;
        iss >> next;
        if (next.empty() || next == "{" || next == ";")
            return i;
    }
    throw CaseError("Field block \"" + name + "\" not defined");
}

Lines extract_block(const Lines &lines, const std::string &name)
{
    const size_t at = find_block_line(lines, name);
    Lines out;
    size_t open = 0;
    bool found = false;
    if (strip_comment(lines[at]).find('{') != std::string::npos) {
        open = at;
        found = true;
    } else {
        for (size_t i = at + 1; i < lines.size(); i++) {
            const std::string p = strip_comment(lines[i]);
            if (p.find('}') != std::string::npos)
                throw CaseError("Found closing brace before opening brace for block '" + name + "'");
            const std::string t = trim(p);
            if (!t.empty() && t.find('{') == std::string::npos)
                throw CaseError("Non-whitespace content found between block declaration and opening brace for block '" +
                                name + "'");
            if (p.find('{') != std::string::npos) {
                open = i;
                found = true;
                break;
            }
        }
    }
    if (!found)
        throw CaseError("Opening brace not found for block '" + name + "'");
    out.push_back(lines[open]);
    int depth = 1;
    for (size_t i = open + 1; i < lines.size(); i++) {
        for (char c : strip_comment(lines[i])) {
            if (c == '{')
                depth++;
            else if (c == '}')
                depth--;
        }
        out.push_back(lines[i]);
        if (depth == 0)
            return out;
    }
    throw CaseError("Unbalanced braces for block '" + name + "'");
}

template <typename T>
static T to_unsigned(const std::string &s)
{
    // extractParameter<integral>: non-numbers read as 0 in the reference
    if (!is_number(s))
        return 0;
    return static_cast<T>(std::stoull(s));
}

static float to_float(const std::string &s)
{
    try {
        return static_cast<float>(std::stold(s));
    } catch (const std::exception &) {
        throw CaseError("Invalid floating point value " + s);
    }
}

static std::string join(const std::string &dir, const char *f)
{
    return (fs::path(dir) / f).string();
}

ProgramControl read_program_control(const std::string &dir)
{
    const Lines L = read_lines(join(dir, "programControl"));
    ProgramControl p;
    p.caseName = parameter_string(L, "caseName");
    p.Re = to_float(parameter_string(L, "Re"));
    p.u_inf = to_float(parameter_string(L, "u_inf"));
    p.nTimeSteps = to_unsigned<uint64_t>(parameter_string(L, "nTimeSteps"));
    p.saveInterval = to_unsigned<uint64_t>(parameter_string(L, "saveInterval"));
    p.infoInterval = to_unsigned<uint64_t>(parameter_string(L, "infoInterval"));
    if (p.saveInterval == 0 || p.infoInterval == 0)
        throw CaseError("saveInterval and infoInterval must be positive");
    return p;
}

LatticeMesh read_lattice_mesh(const std::string &dir)
{
    const Lines L = read_lines(join(dir, "latticeMesh"));
    LatticeMesh m;
    m.nx = to_unsigned<uint64_t>(parameter_string(L, "nx"));
    m.ny = to_unsigned<uint64_t>(parameter_string(L, "ny"));
    m.nz = to_unsigned<uint64_t>(parameter_string(L, "nz"));
    m.Lx = to_float(parameter_string(L, "Lx"));
    m.Ly = to_float(parameter_string(L, "Ly"));
    m.Lz = to_float(parameter_string(L, "Lz"));
    return m;
}

static const char *kFields[10] = {"rho", "u", "v", "w", "m_xx", "m_xy", "m_xz", "m_yy", "m_yz", "m_zz"};
static const char *kRegions[7] = {"internalField", "North", "South", "East", "West", "Front", "Back"};

static std::string region_value(const Lines &L, const std::string &field, const std::string &region)
{
    const Lines fb = extract_block(L, "field " + field);
    const Lines rb = extract_block(fb, region);
    return parameter_string(rb, "value");
}

std::array<float, 70> read_initial_conditions(const std::string &dir)
{
    const Lines L = read_lines(join(dir, "initialConditions"));
    std::array<float, 70> out{};
    for (int f = 0; f < 10; f++) {
        const std::string name = kFields[f];
        for (int r = 0; r < 7; r++) {
            const std::string v = region_value(L, name, kRegions[r]);
            float value;
            if (is_number(v)) {
                const float raw = to_float(v);
                if (f == 0)
                    value = raw;
                else if (f <= 3)
                    value = raw * 3.0f;
                else if (f == 4 || f == 7 || f == 9)
                    value = raw * 4.5f;
                else
                    value = raw * 9.0f;
            } else if (v == "equilibrium" && f >= 4) {
                // second-order equilibrium from the same region's raw velocities;
                // the reference scales every component by 4.5 here
                static const int pa[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
                static const int pb[10] = {0, 0, 0, 0, 1, 2, 3, 2, 3, 3};
                auto vel = [&](int k) {
                    const std::string s = region_value(L, kFields[k], kRegions[r]);
                    if (!is_number(s))
                        throw CaseError("Invalid boundary value " + s + ". Value must be a number.");
                    return to_float(s);
                };
                const float ua = vel(pa[f]), ub = vel(pb[f]);
                value = 4.5f * (ua * ub) / 1.0f;
            } else {
                throw CaseError("Entry for " + name + " in region " + kRegions[r] +
                                " not a valid numerical value and not an equilibrium moment");
            }
            out[size_t(f) * 7 + r] = value;
        }
    }
    return out;
}

uint32_t read_function_objects(const std::string &dir)
{
    const std::string path = join(dir, "functionObjects");
    if (!fs::exists(path))
        return 0;
    Lines block = extract_block(read_lines(path), "functionObjectList");
    if (block.size() < 3 || block.front() != "{" || block.back() != "};")
        throw CaseError("functionObjectList must be '{', entries, '};' on separate lines");
    uint32_t mask = 0;
    const std::pair<const char *, uint32_t> names[] = {{"S", LBM_FO_S},
                                                       {"SMean", LBM_FO_SMEAN},
                                                       {"k", LBM_FO_K},
                                                       {"kMean", LBM_FO_KMEAN},
                                                       {"momentsMean", LBM_FO_MOMENTSMEAN}};
    for (size_t i = 1; i + 1 < block.size(); i++) {
        const std::string t = trim(block[i], true);
        for (const auto &n : names)
            if (t == n.first)
                mask |= n.second;
    }
    return mask;
}

std::vector<uint64_t> time_indices(const std::string &dir, const std::string &prefix)
{
    std::vector<uint64_t> out;
    const std::string pre = prefix + "_";
    for (const auto &e : fs::directory_iterator(dir.empty() ? "." : dir)) {
        if (!e.is_regular_file() || e.path().extension() != ".LBMBin")
            continue;
        const std::string stem = e.path().stem().string();
        if (stem.size() <= pre.size() || stem.compare(0, pre.size(), pre) != 0)
            continue;
        const std::string num = stem.substr(pre.size());
        if (num.empty() || !std::all_of(num.begin(), num.end(), [](unsigned char c) { return std::isdigit(c); }))
            continue;
        uint64_t v = 0;
        std::from_chars(num.data(), num.data() + num.size(), v);
        out.push_back(v);
    }
    std::sort(out.begin(), out.end());
    return out;
}

void print_program_control(const ProgramControl &pc, const std::string &program, const std::vector<int> &devices,
                           uint64_t latest)
{
    const std::time_t now = std::time(nullptr);
    std::cout << "programControl:\n{\n"
              << "    programName: " << program << ";\n"
              << "    launchTime: " << std::put_time(std::localtime(&now), "%Y-%m-%d %H:%M:%S") << ";\n"
              << "    launchDirectory: " << fs::current_path().string() << ";\n"
              << "    deviceList: [";
    for (size_t i = 0; i < devices.size(); i++)
        std::cout << devices[i] << (i + 1 < devices.size() ? ", " : "");
    std::cout << "];\n    caseName: " << pc.caseName << ";\n    Re = " << pc.Re << ";\n    nTimeSteps = " << pc.nTimeSteps
              << ";\n    saveInterval = " << pc.saveInterval << ";\n    infoInterval = " << pc.infoInterval
              << ";\n    latestTime = " << latest << ";\n    scalarType: 32 bit;\n    labelType: uint64_t;\n};\n"
              << std::endl;
}

void print_lattice_mesh(const LatticeMesh &mesh)
{
    std::cout << "latticeMesh:\n{\n    nx = " << mesh.nx << ";\n    ny = " << mesh.ny << ";\n    nz = " << mesh.nz
              << ";\n    Lx = " << mesh.Lx << ";\n    Ly = " << mesh.Ly << ";\n    Lz = " << mesh.Lz << ";\n};\n"
              << std::endl;
}

std::vector<int> parse_gpu_list(int argc, char **argv, bool required)
{
    const std::string exe = fs::path(argv[0]).filename().string();
    for (int i = 1; i < argc; i++) {
        if (std::string(argv[i]) != "-GPU")
            continue;
        if (i + 1 >= argc)
            throw CaseError("Input argument -GPU has not been supplied with a value; the correct syntax is -GPU 0,1 for example");
        std::vector<int> ids;
        std::string s = argv[i + 1], cur;
        for (char c : s + ",") {
            if (c == ',') {
                if (!cur.empty()) {
                    if (!is_number(cur) || cur.find('.') != std::string::npos)
                        throw CaseError("-GPU is not numeric");
                    ids.push_back(std::stoi(cur));
                }
                cur.clear();
            } else {
                cur.push_back(c);
            }
        }
        if (ids.empty())
            throw CaseError("-GPU is not numeric");
        return ids;
    }
    if (!required)
        return {0};
    throw CaseError("Error: The -GPU argument is mandatory for the " + exe + " executable.");
}

}  // namespace lbm
