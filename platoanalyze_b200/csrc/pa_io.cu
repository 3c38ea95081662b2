// pa_io.cu -- visualisation output: the mesh, the displacement and the control
// as a VTK XML unstructured grid (.vtu), the role Plato::write /
// Plato::output play for the reference through Omega_h's VTK writer
// (src/AnalyzeOutput.hpp:469-482: vertex tags "Control" and "Displacements").
//
// Format: VTKFile type="UnstructuredGrid" version 1.0, little-endian,
// header_type UInt64, every DataArray format="binary": base64 of a UInt64
// byte count followed by the raw values.  Cells are VTK_TETRA (10); points
// Float64 x 3; connectivity and offsets Int64.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pa_problem.cuh"

namespace pa {

namespace {

// RFC 4648 base64 of a byte range (no line breaks).
std::string base64(const unsigned char* p, size_t n) {
  static const char* k = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
  std::string out;
  out.reserve((n + 2) / 3 * 4);
  size_t i = 0;
  for (; i + 3 <= n; i += 3) {
    const uint32_t v = (uint32_t(p[i]) << 16) | (uint32_t(p[i + 1]) << 8) | uint32_t(p[i + 2]);
    out += k[(v >> 18) & 63];
    out += k[(v >> 12) & 63];
    out += k[(v >> 6) & 63];
    out += k[v & 63];
  }
  if (i < n) {
    uint32_t v = uint32_t(p[i]) << 16;
    if (i + 1 < n) v |= uint32_t(p[i + 1]) << 8;
    out += k[(v >> 18) & 63];
    out += k[(v >> 12) & 63];
    out += (i + 1 < n) ? k[(v >> 6) & 63] : '=';
    out += '=';
  }
  return out;
}

// One binary DataArray: UInt64 byte count + values, base64 together.
template <typename T>
void data_array(FILE* f, const char* type, const char* name, int comps, const T* v, size_t count) {
  std::vector<unsigned char> buf(sizeof(uint64_t) + count * sizeof(T));
  const uint64_t bytes = uint64_t(count * sizeof(T));
  std::memcpy(buf.data(), &bytes, sizeof(bytes));
  if (count) std::memcpy(buf.data() + sizeof(bytes), v, count * sizeof(T));
  std::fprintf(f, "        <DataArray type=\"%s\"", type);
  if (name) std::fprintf(f, " Name=\"%s\"", name);
  if (comps > 1) std::fprintf(f, " NumberOfComponents=\"%d\"", comps);
  std::fprintf(f, " format=\"binary\">\n          %s\n        </DataArray>\n", base64(buf.data(), buf.size()).c_str());
}

// Host copy of a caller array (host or device).
std::vector<double> host_copy(const double* p, size_t n) {
  std::vector<double> h(n);
  if (n == 0) return h;
  cudaPointerAttributes a{};
  const bool dev = cudaPointerGetAttributes(&a, p) == cudaSuccess &&
                   (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged);
  if (!dev) cudaGetLastError();
  if (dev)
    PA_CUDA(cudaMemcpy(h.data(), p, n * sizeof(double), cudaMemcpyDeviceToHost));
  else
    std::memcpy(h.data(), p, n * sizeof(double));
  return h;
}

}  // namespace

void write_vtu(const Mesh& m, const std::string& path, const double* u, const double* control, int control_layout) {
  const std::vector<double> uh = u ? host_copy(u, size_t(3 * m.N)) : std::vector<double>();
  const size_t nctl = control_layout == PA_CONTROL_CELL ? size_t(m.C) : size_t(m.N);
  const std::vector<double> zh = control ? host_copy(control, nctl) : std::vector<double>();
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw Error(PA_ERR_INVALID_ARG, "cannot open '" + path + "' for writing");
  std::fprintf(f, "<?xml version=\"1.0\"?>\n");
  std::fprintf(f,
               "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" "
               "header_type=\"UInt64\">\n  <UnstructuredGrid>\n");
  std::fprintf(f, "    <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\">\n", (long long)m.N, (long long)m.C);
  std::fprintf(f, "      <PointData%s>\n", u ? " Vectors=\"Displacements\"" : "");
  if (u) data_array(f, "Float64", "Displacements", 3, uh.data(), uh.size());
  if (control && control_layout != PA_CONTROL_CELL) data_array(f, "Float64", "Control", 1, zh.data(), zh.size());
  std::fprintf(f, "      </PointData>\n      <CellData>\n");
  if (control && control_layout == PA_CONTROL_CELL) data_array(f, "Float64", "Control", 1, zh.data(), zh.size());
  std::fprintf(f, "      </CellData>\n      <Points>\n");
  data_array(f, "Float64", nullptr, 3, m.coords.data(), m.coords.size());
  std::fprintf(f, "      </Points>\n      <Cells>\n");
  std::vector<int64_t> conn(m.cells.begin(), m.cells.end()), offs(size_t(m.C));
  for (int64_t c = 0; c < m.C; ++c) offs[size_t(c)] = 4 * (c + 1);
  std::vector<uint8_t> types(size_t(m.C), uint8_t(10));  // VTK_TETRA
  data_array(f, "Int64", "connectivity", 1, conn.data(), conn.size());
  data_array(f, "Int64", "offsets", 1, offs.data(), offs.size());
  data_array(f, "UInt8", "types", 1, types.data(), types.size());
  std::fprintf(f, "      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n");
  const bool ok = std::ferror(f) == 0;
  if (std::fclose(f) != 0 || !ok) throw Error(PA_ERR_INVALID_ARG, "write to '" + path + "' failed");
}

}  // namespace pa
