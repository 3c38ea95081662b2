// pa_exodus.cu -- Exodus II mesh input: the role Omega_h::exodus::read plays
// for the reference (src/PlatoDriver.hpp:76, the mesh and its node sets).
//
// Exodus II files are netCDF files; this reads the netCDF classic container
// (CDF-1, CDF-2 "64-bit offset" and CDF-5 "64-bit data"; big-endian header
// and data, non-record variables stored contiguously at their offsets) on the
// host, without the netCDF or SEACAS libraries, which are not in this image.
// netCDF-4 files (HDF5 containers) are refused.  From the Exodus conventions
// it takes: num_dim (must be 3); the coordinates (coordx / coordy / coordz or
// coord[num_dim][num_nodes]); the element blocks connect1..connectB with
// their elem_type attribute (4-node tetrahedra only: the hot path is linear
// tets), concatenated in block order; the node sets node_ns1..node_nsS with
// their names (ns_names) or, unnamed, "ns_<id>" from ns_prop1.  Connectivity
// and node-set entries are 1-based in the file and 0-based here.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "pa_internal.cuh"

struct pa_exodus {
  std::vector<double> coords;   // N x 3
  std::vector<int32_t> cells;   // C x 4, 0-based
  std::vector<std::string> set_names;
  std::vector<std::vector<int32_t>> sets;  // 0-based node ids
};

namespace pa {
namespace {

enum NcType { kByte = 1, kChar = 2, kShort = 3, kInt = 4, kFloat = 5, kDouble = 6, kUByte = 7, kUShort = 8,
              kUInt = 9, kInt64 = 10, kUInt64 = 11 };

size_t type_size(int t) {
  switch (t) {
    case kByte: case kChar: case kUByte: return 1;
    case kShort: case kUShort: return 2;
    case kInt: case kFloat: case kUInt: return 4;
    case kDouble: case kInt64: case kUInt64: return 8;
    default: throw Error(PA_ERR_INVALID_ARG, "netCDF: unknown data type " + std::to_string(t));
  }
}

struct NcVar {
  std::string name;
  std::vector<int64_t> dims;
  int type = 0;
  uint64_t begin = 0;
  std::string elem_type;  // the "elem_type" text attribute, if any
};

struct NcFile {
  std::vector<unsigned char> buf;
  size_t pos = 0;
  int version = 1;
  std::vector<std::pair<std::string, int64_t>> dims;  // length 0: the record dimension
  std::vector<NcVar> vars;

  void need(size_t n) const {
    if (pos + n > buf.size()) throw Error(PA_ERR_INVALID_ARG, "netCDF: truncated header");
  }
  uint64_t be(size_t n) {
    need(n);
    uint64_t v = 0;
    for (size_t i = 0; i < n; ++i) v = (v << 8) | buf[pos + i];
    pos += n;
    return v;
  }
  uint64_t count() { return be(version == 5 ? 8 : 4); }
  std::string name() {
    const uint64_t n = count();
    need(n);
    std::string s(reinterpret_cast<const char*>(&buf[pos]), size_t(n));
    pos += (n + 3) / 4 * 4;
    return s;
  }
  // attribute list; returns the text of attribute `want` if present
  std::string attributes(const char* want) {
    const uint64_t tag = be(4);
    const uint64_t n = count();
    if (tag == 0) {
      if (n != 0) throw Error(PA_ERR_INVALID_ARG, "netCDF: bad attribute list");
      return {};
    }
    if (tag != 0x0C) throw Error(PA_ERR_INVALID_ARG, "netCDF: bad attribute list tag");
    std::string found;
    for (uint64_t a = 0; a < n; ++a) {
      const std::string an = name();
      const int t = int(be(4));
      const uint64_t m = count();
      const size_t bytes = size_t(m) * type_size(t);
      need(bytes);
      if (want && an == want && t == kChar) found.assign(reinterpret_cast<const char*>(&buf[pos]), bytes);
      pos += (bytes + 3) / 4 * 4;
    }
    return found;
  }
  void parse() {
    if (buf.size() >= 4 && buf[0] == 0x89 && buf[1] == 'H' && buf[2] == 'D' && buf[3] == 'F')
      throw Error(PA_ERR_INVALID_ARG, "netCDF-4 (HDF5) files are not supported; write the Exodus file as netCDF classic");
    if (buf.size() < 8 || buf[0] != 'C' || buf[1] != 'D' || buf[2] != 'F')
      throw Error(PA_ERR_INVALID_ARG, "not a netCDF classic file");
    version = buf[3];
    if (version != 1 && version != 2 && version != 5)
      throw Error(PA_ERR_INVALID_ARG, "netCDF: unknown format version " + std::to_string(version));
    pos = 4;
    count();  // numrecs
    // dimensions
    uint64_t tag = be(4), n = count();
    if (tag == 0x0A) {
      for (uint64_t d = 0; d < n; ++d) {
        std::string dn = name();
        const int64_t len = int64_t(count());
        dims.emplace_back(std::move(dn), len);
      }
    } else if (tag != 0 || n != 0) {
      throw Error(PA_ERR_INVALID_ARG, "netCDF: bad dimension list");
    }
    attributes(nullptr);  // global attributes
    tag = be(4);
    n = count();
    if (tag == 0x0B) {
      for (uint64_t v = 0; v < n; ++v) {
        NcVar var;
        var.name = name();
        const uint64_t nd = count();
        for (uint64_t k = 0; k < nd; ++k) {
          const uint64_t id = count();
          if (id >= dims.size()) throw Error(PA_ERR_INVALID_ARG, "netCDF: bad dimension id");
          var.dims.push_back(int64_t(id));
        }
        var.elem_type = attributes("elem_type");
        var.type = int(be(4));
        count();  // vsize
        var.begin = be(version == 1 ? 4 : 8);
        vars.push_back(std::move(var));
      }
    } else if (tag != 0 || n != 0) {
      throw Error(PA_ERR_INVALID_ARG, "netCDF: bad variable list");
    }
  }
  int64_t dim(const std::string& dn, bool required = true) const {
    for (const auto& d : dims)
      if (d.first == dn) return d.second;
    if (required) throw Error(PA_ERR_INVALID_ARG, "Exodus: missing dimension " + dn);
    return -1;
  }
  const NcVar* var(const std::string& vn) const {
    for (const auto& v : vars)
      if (v.name == vn) return &v;
    return nullptr;
  }
  // all values of a non-record variable as doubles (integers exactly up to 2^53)
  std::vector<double> values(const NcVar& v) const {
    size_t count = 1;
    for (int64_t id : v.dims) {
      const int64_t len = dims[size_t(id)].second;
      if (len == 0) throw Error(PA_ERR_INVALID_ARG, "Exodus: variable " + v.name + " is a record variable");
      count *= size_t(len);
    }
    const size_t ts = type_size(v.type);
    if (v.begin + count * ts > buf.size()) throw Error(PA_ERR_INVALID_ARG, "Exodus: variable " + v.name + " truncated");
    std::vector<double> out(count);
    const unsigned char* p = buf.data() + v.begin;
    for (size_t i = 0; i < count; ++i, p += ts) {
      uint64_t u = 0;
      for (size_t b = 0; b < ts; ++b) u = (u << 8) | p[b];
      double x = 0.0;
      switch (v.type) {
        case kByte: x = double(int8_t(u)); break;
        case kUByte: x = double(uint8_t(u)); break;
        case kShort: x = double(int16_t(u)); break;
        case kUShort: x = double(uint16_t(u)); break;
        case kInt: x = double(int32_t(u)); break;
        case kUInt: x = double(uint32_t(u)); break;
        case kInt64: x = double(int64_t(u)); break;
        case kUInt64: x = double(u); break;
        case kFloat: { const uint32_t w = uint32_t(u); float f; std::memcpy(&f, &w, 4); x = f; break; }
        case kDouble: std::memcpy(&x, &u, 8); break;
        default: throw Error(PA_ERR_INVALID_ARG, "Exodus: variable " + v.name + " is not numeric");
      }
      out[i] = x;
    }
    return out;
  }
  std::vector<double> values(const std::string& vn) const {
    const NcVar* v = var(vn);
    if (!v) throw Error(PA_ERR_INVALID_ARG, "Exodus: missing variable " + vn);
    return values(*v);
  }
};

bool is_tet4(std::string t) {
  while (!t.empty() && (t.back() == '\0' || t.back() == ' ')) t.pop_back();
  for (char& c : t) c = char(std::toupper(static_cast<unsigned char>(c)));
  return t == "TETRA" || t == "TETRA4" || t == "TET4" || t == "TET";
}

std::unique_ptr<pa_exodus> read_exodus(const char* path) {
  PA_CHECK(path, "null path");
  NcFile f;
  {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) throw Error(PA_ERR_INVALID_ARG, std::string("cannot open ") + path);
    std::fseek(fp, 0, SEEK_END);
    const long sz = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    f.buf.resize(size_t(sz > 0 ? sz : 0));
    const size_t got = sz > 0 ? std::fread(f.buf.data(), 1, f.buf.size(), fp) : 0;
    std::fclose(fp);
    if (got != f.buf.size()) throw Error(PA_ERR_INVALID_ARG, std::string("cannot read ") + path);
  }
  f.parse();
  PA_CHECK(f.dim("num_dim") == 3, "Exodus: only 3-D meshes are supported");
  const int64_t N = f.dim("num_nodes");
  auto ex = std::make_unique<pa_exodus>();
  ex->coords.resize(size_t(3 * N));
  if (f.var("coordx")) {
    const char* names[3] = {"coordx", "coordy", "coordz"};
    for (int d = 0; d < 3; ++d) {
      const std::vector<double> c = f.values(names[d]);
      PA_CHECK(int64_t(c.size()) == N, "Exodus: coordinate length");
      for (int64_t i = 0; i < N; ++i) ex->coords[size_t(3 * i + d)] = c[size_t(i)];
    }
  } else {
    const std::vector<double> c = f.values("coord");
    PA_CHECK(int64_t(c.size()) == 3 * N, "Exodus: coordinate length");
    for (int d = 0; d < 3; ++d)
      for (int64_t i = 0; i < N; ++i) ex->coords[size_t(3 * i + d)] = c[size_t(d * N + i)];
  }
  const int64_t B = f.dim("num_el_blk");
  for (int64_t b = 1; b <= B; ++b) {
    const int64_t ne = f.dim("num_el_in_blk" + std::to_string(b), false);
    if (ne <= 0) continue;
    const NcVar* cv = f.var("connect" + std::to_string(b));
    PA_CHECK(cv, "Exodus: missing connect" + std::to_string(b));
    const int64_t npe = f.dim("num_nod_per_el" + std::to_string(b));
    if (npe != 4 || !is_tet4(cv->elem_type))
      throw Error(PA_ERR_INVALID_ARG, "Exodus: element block " + std::to_string(b) + " is '" + cv->elem_type +
                                          "' with " + std::to_string(npe) + " nodes; only 4-node tetrahedra");
    const std::vector<double> conn = f.values(*cv);
    PA_CHECK(int64_t(conn.size()) == 4 * ne, "Exodus: connectivity length");
    for (double v : conn) {
      if (!(v >= 1.0 && v <= double(N))) throw Error(PA_ERR_INVALID_ARG, "Exodus: connectivity entry out of range");
      ex->cells.push_back(int32_t(v) - 1);
    }
  }
  PA_CHECK(!ex->cells.empty(), "Exodus: no elements");
  const int64_t S = f.dim("num_node_sets", false);
  std::vector<double> ids;
  if (S > 0 && f.var("ns_prop1")) ids = f.values("ns_prop1");
  std::vector<std::string> names;
  if (S > 0 && f.var("ns_names")) {
    const NcVar& nv = *f.var("ns_names");
    PA_CHECK(nv.type == kChar && nv.dims.size() == 2, "Exodus: ns_names");
    const int64_t len = f.dims[size_t(nv.dims[1])].second;
    PA_CHECK(nv.begin + uint64_t(S * len) <= f.buf.size(), "Exodus: ns_names truncated");
    for (int64_t s = 0; s < S; ++s) {
      std::string nm(reinterpret_cast<const char*>(f.buf.data() + nv.begin + uint64_t(s * len)), size_t(len));
      nm = nm.substr(0, nm.find('\0'));
      names.push_back(nm);
    }
  }
  for (int64_t s = 1; s <= S; ++s) {
    std::string nm = size_t(s - 1) < names.size() ? names[size_t(s - 1)] : std::string();
    if (nm.empty())
      nm = "ns_" + std::to_string(size_t(s - 1) < ids.size() ? int64_t(ids[size_t(s - 1)]) : s);
    std::vector<int32_t> nodes;
    if (f.dim("num_nod_ns" + std::to_string(s), false) > 0) {
      for (double v : f.values("node_ns" + std::to_string(s))) {
        if (!(v >= 1.0 && v <= double(N))) throw Error(PA_ERR_INVALID_ARG, "Exodus: node set entry out of range");
        nodes.push_back(int32_t(v) - 1);
      }
    }
    ex->set_names.push_back(nm);
    ex->sets.push_back(std::move(nodes));
  }
  return ex;
}

template <typename F>
pa_status host_guard(F&& f) {
  try {
    f();
    return PA_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return PA_ERR_INVALID_ARG;
  }
}

}  // namespace
}  // namespace pa

extern "C" {

pa_status pa_exodus_open(const char* path, pa_exodus** out) {
  return pa::host_guard([&] {
    PA_CHECK(out, "null output");
    *out = pa::read_exodus(path).release();
  });
}

pa_status pa_exodus_sizes(const pa_exodus* ex, int64_t* num_nodes, int64_t* num_cells, int32_t* num_node_sets) {
  return pa::host_guard([&] {
    PA_CHECK(ex, "null Exodus handle");
    if (num_nodes) *num_nodes = int64_t(ex->coords.size() / 3);
    if (num_cells) *num_cells = int64_t(ex->cells.size() / 4);
    if (num_node_sets) *num_node_sets = int32_t(ex->sets.size());
  });
}

pa_status pa_exodus_mesh(const pa_exodus* ex, double* coords, int32_t* cells2nodes) {
  return pa::host_guard([&] {
    PA_CHECK(ex && coords && cells2nodes, "null argument");
    std::memcpy(coords, ex->coords.data(), sizeof(double) * ex->coords.size());
    std::memcpy(cells2nodes, ex->cells.data(), sizeof(int32_t) * ex->cells.size());
  });
}

pa_status pa_exodus_node_set(const pa_exodus* ex, int32_t index, char* name, int32_t name_capacity, int64_t* count,
                             int32_t* nodes) {
  return pa::host_guard([&] {
    PA_CHECK(ex, "null Exodus handle");
    PA_CHECK(index >= 0 && size_t(index) < ex->sets.size(), "node set index out of range");
    const std::string& nm = ex->set_names[size_t(index)];
    if (name && name_capacity > 0) {
      const size_t k = std::min(nm.size(), size_t(name_capacity - 1));
      std::memcpy(name, nm.data(), k);
      name[k] = '\0';
    }
    if (count) *count = int64_t(ex->sets[size_t(index)].size());
    if (nodes) std::memcpy(nodes, ex->sets[size_t(index)].data(), sizeof(int32_t) * ex->sets[size_t(index)].size());
  });
}

void pa_exodus_close(pa_exodus* ex) { delete ex; }

}  // extern "C"
