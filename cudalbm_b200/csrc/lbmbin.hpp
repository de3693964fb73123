// lbmbin.hpp -- the .LBMBin field-file format.
//
// Writer: byte for byte the layout of the reference's fileIO::writeFile
// (src/fileIO/fileOutput.cuh:82-183): ASCII systemInformation,
// fieldInformation and fieldData headers, then the raw little-endian values
// ordered [field][block-tiled node], then "\n\t};\n};\n".
// Reader: parses the same header (src/fileIO/fileInput.cuh:99-489) and returns
// fields by name (readFieldByName, :608-761), keeping the tiled node order.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace lbm {

struct FieldFileHeader {
    uint64_t time_step = 0;
    std::string time_type;
    std::vector<std::string> names;
    uint64_t nx = 0, ny = 0, nz = 0;
    int scalar_bytes = 4;
    bool little_endian = true;
    uint64_t data_offset = 0;
};

// values: nvars * nx*ny*nz floats in [field][tiled node] order.
void write_field_file(const std::string &path, uint64_t nx, uint64_t ny, uint64_t nz,
                      const std::vector<std::string> &names, const float *values, uint64_t time_step,
                      bool time_average);
void write_field_file(const std::string &path, uint64_t nx, uint64_t ny, uint64_t nz,
                      const std::vector<std::string> &names, const double *values, uint64_t time_step,
                      bool time_average);

FieldFileHeader read_field_header(const std::string &path);

// One field (tiled order) converted to float.
std::vector<float> read_field_by_name(const std::string &path, const std::string &name);
// One field (tiled order) as double: exact for 32- and 64-bit files alike.
std::vector<double> read_field_by_name_f64(const std::string &path, const std::string &name);

}  // namespace lbm
