// postprocess.cpp -- cut planes and the VTS writer (see postprocess.hpp).
#include "postprocess.hpp"

#include <cmath>
#include <fstream>
#include <sstream>

#include "casefile.hpp"

namespace lbm {

FieldSet tiled_to_global(const std::vector<float> &tiled, uint64_t nx, uint64_t ny, uint64_t nz)
{
    const uint64_t n = nx * ny * nz;
    if (n == 0 || tiled.size() % n)
        throw CaseError("field data size is not a multiple of the node count");
    const uint64_t nvars = tiled.size() / n, nbx = nx / 8, nby = ny / 8;
    FieldSet out(nvars, std::vector<float>(n));
    for (uint64_t v = 0; v < nvars; v++) {
        const float *src = tiled.data() + v * n;
        for (uint64_t z = 0; z < nz; z++)
            for (uint64_t y = 0; y < ny; y++)
                for (uint64_t x = 0; x < nx; x++) {
                    const uint64_t t =
                        (x & 7) + 8 * ((y & 7) + 8 * ((z & 7) + 8 * ((x >> 3) + nbx * ((y >> 3) + nby * (z >> 3)))));
                    out[v][x + nx * (y + ny * z)] = src[t];
                }
    }
    return out;
}

FieldSet cut_plane(const FieldSet &fields, uint64_t nx, uint64_t ny, uint64_t nz, const float L[3], int axis,
                   float coordinate, bool reference_weight)
{
    if (axis < 0 || axis > 2)
        throw CaseError("cut plane direction must be x, y or z");
    const uint64_t dims[3] = {nx, ny, nz};
    const uint64_t n = dims[axis];
    // index coordinate in float, as the reference evaluates it
    const float index = static_cast<float>(n - 1) * (coordinate * L[axis]);
    if (!(index >= 0.0f) || index > static_cast<float>(n - 1))
        throw CaseError("cut plane coordinate lies outside the mesh");
    const uint64_t i0 = static_cast<uint64_t>(std::floor(index));
    const uint64_t i1 = static_cast<uint64_t>(std::ceil(index));
    const float w = reference_weight ? coordinate - static_cast<float>(i0) : index - static_cast<float>(i0);
    const float one_w = 1.0f - w;
    // plane extents (a, b): x-cut (y, z), y-cut (x, z), z-cut (x, y)
    const uint64_t na = axis == 0 ? ny : nx, nb = axis == 2 ? ny : nz;
    auto node = [&](uint64_t i, uint64_t a, uint64_t b) {
        const uint64_t x = axis == 0 ? i : a;
        const uint64_t y = axis == 0 ? a : (axis == 1 ? i : b);
        const uint64_t z = axis == 2 ? i : b;
        return x + nx * (y + ny * z);
    };
    FieldSet out(fields.size(), std::vector<float>(na * nb));
    for (size_t v = 0; v < fields.size(); v++)
        for (uint64_t b = 0; b < nb; b++)
            for (uint64_t a = 0; a < na; a++) {
                const float f0 = fields[v][node(i0, a, b)];
                const float f1 = fields[v][node(i1, a, b)];
                out[v][a + na * b] = (one_w * f0) + (w * f1);
            }
    return out;
}

std::vector<float> mesh_coordinates(uint64_t nx, uint64_t ny, uint64_t nz, const float L[3])
{
    std::vector<float> c(3 * nx * ny * nz);
    auto coord = [](float l, uint64_t i, uint64_t n) {
        const uint64_t many = n > 1 ? 1 : 0;
        return static_cast<float>((static_cast<double>(l) * static_cast<double>(i * many)) /
                                  static_cast<double>(n - many));
    };
    for (uint64_t k = 0; k < nz; k++)
        for (uint64_t j = 0; j < ny; j++)
            for (uint64_t i = 0; i < nx; i++) {
                const uint64_t idx = (k * ny + j) * nx + i;
                c[3 * idx + 0] = coord(L[0], i, nx);
                c[3 * idx + 1] = coord(L[1], j, ny);
                c[3 * idx + 2] = coord(L[2], k, nz);
            }
    return c;
}

namespace {

std::string vts_header(uint64_t nx, uint64_t ny, uint64_t nz, const std::vector<std::string> &names)
{
    const uint64_t n = nx * ny * nz;
    std::ostringstream x;
    const std::string extent =
        "0 " + std::to_string(nx - 1) + " 0 " + std::to_string(ny - 1) + " 0 " + std::to_string(nz - 1);
    x << "<?xml version=\"1.0\"?>\n";
    x << "<VTKFile type=\"StructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    x << "  <StructuredGrid WholeExtent=\"" << extent << "\">\n";
    x << "    <Piece Extent=\"" << extent << "\">\n";
    x << "      <PointData Scalars=\"" << (names.empty() ? "" : names[0]) << "\">\n";
    uint64_t offset = 0;
    for (const std::string &name : names) {
        x << "        <DataArray type=\"Float32\" Name=\"" << name << "\" format=\"appended\" offset=\"" << offset
          << "\"/>\n";
        offset += 8 + n * 4;
    }
    x << "      </PointData>\n";
    x << "      <Points>\n";
    x << "        <DataArray type=\"Float32\" Name=\"Coordinates\" NumberOfComponents=\"3\" format=\"appended\" offset=\""
      << offset << "\"/>\n";
    x << "      </Points>\n";
    x << "    </Piece>\n";
    x << "  </StructuredGrid>\n";
    x << "  <AppendedData encoding=\"raw\">_";
    return x.str();
}

const char kVtsTrailer[] = "</AppendedData>\n</VTKFile>\n";

void write_block(std::ofstream &out, const float *data, uint64_t count)
{
    const uint64_t bytes = count * sizeof(float);
    out.write(reinterpret_cast<const char *>(&bytes), sizeof(bytes));
    out.write(reinterpret_cast<const char *>(data), std::streamsize(bytes));
}

}  // namespace

uint64_t vts_file_bytes(uint64_t nx, uint64_t ny, uint64_t nz, const std::vector<std::string> &names)
{
    const uint64_t n = nx * ny * nz;
    return vts_header(nx, ny, nz, names).size() + names.size() * (8 + 4 * n) + (8 + 12 * n) +
           (sizeof(kVtsTrailer) - 1);
}

void write_vts(const std::string &path, const FieldSet &fields, const std::vector<std::string> &names, uint64_t nx,
               uint64_t ny, uint64_t nz, const float L[3])
{
    const uint64_t n = nx * ny * nz;
    if (fields.size() != names.size())
        throw CaseError("the number of fields (" + std::to_string(fields.size()) +
                        ") does not match the number of names (" + std::to_string(names.size()) + ")");
    for (size_t v = 0; v < fields.size(); v++)
        if (fields[v].size() != n)
            throw CaseError("field " + names[v] + " has " + std::to_string(fields[v].size()) + " values, expected " +
                            std::to_string(n));
    std::ofstream out(path, std::ios::binary);
    if (!out)
        throw CaseError("cannot open " + path + " for writing");
    out << vts_header(nx, ny, nz, names);
    for (const auto &f : fields)
        write_block(out, f.data(), n);
    const std::vector<float> points = mesh_coordinates(nx, ny, nz, L);
    write_block(out, points.data(), points.size());
    out << kVtsTrailer;
    if (!out)
        throw CaseError("write failed: " + path);
}

}  // namespace lbm
