// lbmbin.cpp -- see lbmbin.hpp.
#include "lbmbin.hpp"

#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>

#include "casefile.hpp"

namespace lbm {

template <typename T>
static void write_impl(const std::string &path, uint64_t nx, uint64_t ny, uint64_t nz,
                       const std::vector<std::string> &names, const T *values, uint64_t time_step, bool time_average)
{
    const uint64_t nvars = names.size();
    const uint64_t total = nvars * nx * ny * nz;
    {
        // the reference refuses to write without room for the data (fileOutput.cuh:103-110)
        std::error_code ec;
        const auto parent = std::filesystem::absolute(path).parent_path();
        const auto sp = std::filesystem::space(parent, ec);
        if (!ec && sp.available < total * sizeof(T))
            throw CaseError("Insufficient disk space to write file " + path);
    }
    std::ofstream out(path, std::ios::binary);
    if (!out)
        throw CaseError("Cannot open file: " + path);
    out << "systemInformation\n{\n\tbinaryType\tlittleEndian;\n\n\tscalarType\t" << (sizeof(T) == 4 ? "32" : "64")
        << " bit;\n};\n\n";
    out << "fieldInformation\n{\n\ttimeStep\t" << time_step << ";\n\n\ttimeType\t"
        << (time_average ? "timeAverage" : "instantaneous") << ";\n\n\tfieldNames[" << nvars << "]\n\t{\n";
    for (const auto &n : names)
        out << "\t\t" << n << ";\n";
    out << "\t};\n};\n\n";
    out << "fieldData\n{\n\tfieldType\tnonUniform;\n\n\tfield[" << total << "][" << nvars << "][" << nz << "][" << ny
        << "][" << nx << "]\n\t{\n";
    out.write(reinterpret_cast<const char *>(values), std::streamsize(total * sizeof(T)));
    out << "\n\t};\n};\n";
    if (!out)
        throw CaseError("Error writing file: " + path);
}

void write_field_file(const std::string &path, uint64_t nx, uint64_t ny, uint64_t nz,
                      const std::vector<std::string> &names, const float *values, uint64_t time_step, bool time_average)
{
    write_impl(path, nx, ny, nz, names, values, time_step, time_average);
}
void write_field_file(const std::string &path, uint64_t nx, uint64_t ny, uint64_t nz,
                      const std::vector<std::string> &names, const double *values, uint64_t time_step,
                      bool time_average)
{
    write_impl(path, nx, ny, nz, names, values, time_step, time_average);
}

FieldFileHeader read_field_header(const std::string &path)
{
    std::ifstream in(path, std::ios::binary);
    if (!in)
        throw CaseError("Cannot open file: " + path);
    in.seekg(0, std::ios::end);
    const uint64_t size = uint64_t(in.tellg());
    in.seekg(0, std::ios::beg);
    FieldFileHeader h;
    std::string line;
    bool in_names = false, have_scalar = false, have_dims = false;
    uint64_t total = 0, nvars = 0;
    while (std::getline(in, line)) {
        const std::string t = trim(line);
        if (t.empty())
            continue;
        if (t.rfind("binaryType", 0) == 0) {
            h.little_endian = t.find("littleEndian") != std::string::npos;
        } else if (t.rfind("scalarType", 0) == 0) {
            if (t.find("32 bit") != std::string::npos)
                h.scalar_bytes = 4;
            else if (t.find("64 bit") != std::string::npos)
                h.scalar_bytes = 8;
            else
                throw CaseError("Invalid scalarType in " + path);
            have_scalar = true;
        } else if (t.rfind("timeStep", 0) == 0) {
            std::istringstream iss(t.substr(8));
            iss >> h.time_step;
        } else if (t.rfind("timeType", 0) == 0) {
            h.time_type = trim(t.substr(8), true);
        } else if (t.rfind("fieldNames[", 0) == 0) {
            in_names = true;
        } else if (in_names) {
            if (t == "{")
                continue;
            if (t == "};") {
                in_names = false;
                continue;
            }
            h.names.push_back(trim(t, true));
        } else if (t.rfind("field[", 0) == 0) {
            std::vector<uint64_t> d;
            size_t p = 0;
            while ((p = t.find('[', p)) != std::string::npos) {
                const size_t e = t.find(']', p);
                if (e == std::string::npos)
                    throw CaseError("Unclosed bracket in " + path);
                d.push_back(std::stoull(t.substr(p + 1, e - p - 1)));
                p = e + 1;
            }
            if (d.size() < 5)
                throw CaseError("Invalid field dimensions in " + path);
            total = d[0];
            nvars = d[1];
            h.nz = d[2];
            h.ny = d[3];
            h.nx = d[4];
            if (!std::getline(in, line) || trim(line) != "{")
                throw CaseError("Malformed fieldData block in " + path);
            h.data_offset = uint64_t(in.tellg());
            have_dims = true;
            break;
        }
    }
    if (!have_scalar || !have_dims)
        throw CaseError("Incomplete header in " + path);
    if (total != nvars * h.nx * h.ny * h.nz || nvars != h.names.size())
        throw CaseError("Dimension mismatch in " + path);
    if (!h.little_endian)
        throw CaseError("Big-endian field files are not supported: " + path);
    if (h.data_offset + total * uint64_t(h.scalar_bytes) > size)
        throw CaseError("Truncated field file: " + path);
    return h;
}

namespace {
// Position of field `name` among the file's fields.
size_t field_index(const FieldFileHeader &h, const std::string &path, const std::string &name)
{
    size_t k = 0;
    while (k < h.names.size() && h.names[k] != name)
        k++;
    if (k == h.names.size())
        throw CaseError("Field " + name + " not found in " + path);
    return k;
}

template <typename T>
std::vector<T> read_field_as(const std::string &path, const std::string &name)
{
    const FieldFileHeader h = read_field_header(path);
    const size_t k = field_index(h, path, name);
    const uint64_t n = h.nx * h.ny * h.nz;
    std::ifstream in(path, std::ios::binary);
    in.seekg(std::streamoff(h.data_offset + k * n * uint64_t(h.scalar_bytes)));
    std::vector<T> out(n);
    if (h.scalar_bytes == int(sizeof(T))) {
        in.read(reinterpret_cast<char *>(out.data()), std::streamsize(n * sizeof(T)));
    } else if (h.scalar_bytes == 4) {
        std::vector<float> tmp(n);
        in.read(reinterpret_cast<char *>(tmp.data()), std::streamsize(n * 4));
        for (uint64_t i = 0; i < n; i++)
            out[i] = T(tmp[i]);
    } else {
        std::vector<double> tmp(n);
        in.read(reinterpret_cast<char *>(tmp.data()), std::streamsize(n * 8));
        for (uint64_t i = 0; i < n; i++)
            out[i] = T(tmp[i]);
    }
    if (!in)
        throw CaseError("Truncated field file: " + path);
    return out;
}
}  // namespace

std::vector<float> read_field_by_name(const std::string &path, const std::string &name)
{
    return read_field_as<float>(path, name);
}

std::vector<double> read_field_by_name_f64(const std::string &path, const std::string &name)
{
    return read_field_as<double>(path, name);
}

}  // namespace lbm
