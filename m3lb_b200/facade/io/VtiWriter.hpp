// VTK ImageData output for the drop-in headers (the reference's
// src/io/VtiWriter.hpp interface: write_vti, VtiArray, write_vti_bin,
// write_pvd).  The files are byte-for-byte those the reference writes for
// the same values, so ParaView state files and downstream scripts keep
// working: the same XML header text, x-fastest point order, ASCII numbers
// at 9 significant digits, and for the binary writer raw appended Float32
// blocks each led by a UInt32 byte count, offsets counted from the byte
// after the '_' that opens AppendedData.
#pragma once
#include <cstdint>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "core/Types.hpp"
#include "grid/Domain.hpp"

namespace lbm {

namespace vti_detail {
inline void extent(std::ostream& f, Index nx, Index ny, Index nz) {
  f << "0 " << nx - 1 << " 0 " << ny - 1 << " 0 " << nz - 1;
}
}  // namespace vti_detail

// ASCII file of one solver's rho, u and cell flags (refreshed through
// compute_macroscopic()).
template <class Solver>
void write_vti(const std::string& path, Solver& s) {
  s.compute_macroscopic();
  const Domain& d = s.domain();
  const auto rho = s.rho();
  const auto ux = s.ux();
  const auto uy = s.uy();
  const auto uz = s.uz();
  const auto fl = s.flags();
  std::ofstream out(path);
  out.precision(9);
  out << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
      << "  <ImageData WholeExtent=\"";
  vti_detail::extent(out, d.nx, d.ny, d.nz);
  out << "\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n    <Piece Extent=\"";
  vti_detail::extent(out, d.nx, d.ny, d.nz);
  out << "\">\n      <PointData Scalars=\"rho\" Vectors=\"u\">\n";
  auto each = [&](auto&& emit) {
    for (Index z = 0; z < d.nz; ++z)
      for (Index y = 0; y < d.ny; ++y)
        for (Index x = 0; x < d.nx; ++x) emit(d.id(x, y, z));
  };
  out << "        <DataArray type=\"Float64\" Name=\"rho\" format=\"ascii\">\n";
  each([&](Index n) { out << rho(n) << ' '; });
  out << "\n        </DataArray>\n"
      << "        <DataArray type=\"Float64\" Name=\"u\" NumberOfComponents=\"3\" format=\"ascii\">\n";
  each([&](Index n) { out << ux(n) << ' ' << uy(n) << ' ' << uz(n) << ' '; });
  out << "\n        </DataArray>\n"
      << "        <DataArray type=\"UInt8\" Name=\"flag\" format=\"ascii\">\n";
  each([&](Index n) { out << int(fl(n)) << ' '; });
  out << "\n        </DataArray>\n"
      << "      </PointData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n";
}

// One named point array: npoints * ncomp floats, x fastest, then y, then z.
struct VtiArray {
  std::string name;
  int ncomp = 1;
  std::vector<float> data;
};

// Binary (raw appended) file of any named arrays on an nx * ny * nz grid;
// `spacing` is the cell size on every axis.
inline void write_vti_bin(const std::string& path, Index nx, Index ny, Index nz,
                          const std::vector<VtiArray>& arrays, double spacing = 1.0) {
  const std::size_t np = std::size_t(nx) * std::size_t(ny) * std::size_t(nz);
  for (const VtiArray& a : arrays) {
    const std::size_t want = np * std::size_t(a.ncomp);
    if (a.data.size() != want)
      throw std::runtime_error("write_vti_bin: array '" + a.name + "' has " +
                               std::to_string(a.data.size()) + " values, expected " +
                               std::to_string(want));
  }
  // the first one- and three-component arrays are the ones ParaView shows
  const VtiArray* scalar = nullptr;
  const VtiArray* vector = nullptr;
  for (const VtiArray& a : arrays) {
    if (a.ncomp == 1 && !scalar) scalar = &a;
    if (a.ncomp == 3 && !vector) vector = &a;
  }
  std::ofstream out(path, std::ios::binary);
  out << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\""
         " header_type=\"UInt32\">\n"
      << "  <ImageData WholeExtent=\"";
  vti_detail::extent(out, nx, ny, nz);
  out << "\" Origin=\"0 0 0\" Spacing=\"" << spacing << ' ' << spacing << ' ' << spacing
      << "\">\n    <Piece Extent=\"";
  vti_detail::extent(out, nx, ny, nz);
  out << "\">\n      <PointData";
  if (scalar) out << " Scalars=\"" << scalar->name << '"';
  if (vector) out << " Vectors=\"" << vector->name << '"';
  out << ">\n";
  std::size_t offset = 0;
  for (const VtiArray& a : arrays) {
    out << "        <DataArray type=\"Float32\" Name=\"" << a.name << "\" NumberOfComponents=\""
        << a.ncomp << "\" format=\"appended\" offset=\"" << offset << "\"/>\n";
    offset += sizeof(std::uint32_t) + a.data.size() * sizeof(float);
  }
  out << "      </PointData>\n    </Piece>\n  </ImageData>\n"
      << "  <AppendedData encoding=\"raw\">\n_";
  for (const VtiArray& a : arrays) {
    const std::uint32_t bytes = std::uint32_t(a.data.size() * sizeof(float));
    out.write(reinterpret_cast<const char*>(&bytes), sizeof bytes);
    out.write(reinterpret_cast<const char*>(a.data.data()), std::streamsize(bytes));
  }
  out << "\n  </AppendedData>\n</VTKFile>\n";
}

// ParaView time series: (time, file) per frame, paths written as given.
inline void write_pvd(const std::string& path,
                      const std::vector<std::pair<double, std::string>>& frames) {
  std::ofstream out(path);
  out.precision(9);
  out << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
      << "  <Collection>\n";
  for (const auto& fr : frames)
    out << "    <DataSet timestep=\"" << fr.first << "\" group=\"\" part=\"0\" file=\""
        << fr.second << "\"/>\n";
  out << "  </Collection>\n</VTKFile>\n";
}

}  // namespace lbm
