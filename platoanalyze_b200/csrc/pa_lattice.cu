// pa_lattice.cu -- recognise a structured box in a mesh given as arrays.
//
// The reference builds its boxes with Omega_h build_box and hands this build
// connectivity and coordinates (src/PlatoDriver.hpp:77,
// unit_tests/PlatoTestHelpers.hpp:240-249); the golden 2x2x2 mesh of its
// DerivativeTests splits every hex into the same six tets as mesh_make_box.
// Such a mesh qualifies for the box kernels (pa_box.cuh) under its own node,
// cell and vertex order: this file finds the lattice position of every node
// and the (hex, template tet) slot of every cell, so that the box kernels run
// in lattice order and the solver permutes at its boundary.
//
// Conditions: C = 6 nx ny nz and N = (nx+1)(ny+1)(nz+1); every coordinate on
// an axis-aligned lattice of spacing (hx, hy, hz) to rounding level; the
// nodes fill the lattice once; every cell spans one lattice cube and its four
// corners form one of the six template tets, for one of the eight axis
// reflections of the lattice (a reflection maps the split along one cube
// diagonal onto the split along another); no (hex, tet) slot twice.  Along a
// reflected axis the lattice runs against the caller's axis, so that vector
// component changes sign between the two numberings (the operator is
// invariant under the reflection of the geometry and of the displacements).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "pa_internal.cuh"

namespace pa {

namespace {

// corner sets (bit a + 2b + 4c for corner (a, b, c)) of the six tets of mesh_make_box
int template_of_corners(int mask) {
  static const int tet[6][4][3] = {
      {{0, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 1, 1}}, {{0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}},
      {{0, 0, 0}, {0, 1, 1}, {0, 0, 1}, {1, 1, 1}}, {{0, 0, 0}, {1, 0, 1}, {1, 1, 1}, {0, 0, 1}},
      {{1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {0, 0, 0}}, {{1, 0, 0}, {1, 1, 1}, {1, 1, 0}, {0, 0, 0}}};
  for (int t = 0; t < 6; ++t) {
    int mk = 0;
    for (int n = 0; n < 4; ++n) mk |= 1 << (tet[t][n][0] + 2 * tet[t][n][1] + 4 * tet[t][n][2]);
    if (mk == mask) return t;
  }
  return -1;
}

}  // namespace

void detect_lattice(Mesh& m) {
  m.lat_n[0] = m.lat_n[1] = m.lat_n[2] = 0;
  m.lat_permuted = false;
  m.lat_flip = 0;
  if (m.C % 6 != 0 || m.C < 6) return;
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) lo[a] = hi[a] = m.coords[a];
  for (int64_t v = 0; v < m.N; ++v)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], m.coords[3 * v + a]);
      hi[a] = std::max(hi[a], m.coords[3 * v + a]);
    }
  // spacing from the first cell's extent (a template tet spans its hex)
  double h[3];
  for (int a = 0; a < 3; ++a) {
    double cmin = m.coords[3 * int64_t(m.cells[0]) + a], cmax = cmin;
    for (int n = 1; n < 4; ++n) {
      const double x = m.coords[3 * int64_t(m.cells[n]) + a];
      cmin = std::min(cmin, x);
      cmax = std::max(cmax, x);
    }
    h[a] = cmax - cmin;
    if (!(h[a] > 0.0)) return;
  }
  int n[3];
  for (int a = 0; a < 3; ++a) {
    const double q = (hi[a] - lo[a]) / h[a];
    n[a] = int(std::lround(q));
    if (n[a] < 1 || std::fabs(q - n[a]) > 1e-6 * std::max(1.0, q)) return;
    h[a] = (hi[a] - lo[a]) / n[a];  // the spacing the box kernels use
  }
  const int64_t px = n[0] + 1, py = n[1] + 1, pz = n[2] + 1;
  if (px * py * pz != m.N || 6LL * n[0] * n[1] * n[2] != m.C) return;
  // lattice coordinates of every node, each lattice point once; positions on
  // the lattice to rounding level: within 1e-12 of the spacing plus a few
  // units in the last place of the coordinates (the box kernels use the exact
  // lattice geometry, FP64 results stay within 1e-10)
  constexpr double kEps = 2.220446049250313e-16;
  std::vector<int32_t> ijk(3 * m.N);
  std::vector<uint8_t> hit(size_t(m.N), 0);
  for (int64_t v = 0; v < m.N; ++v) {
    int64_t lin = 0, mul = 1;
    for (int a = 0; a < 3; ++a) {
      const double x = m.coords[3 * v + a];
      const int64_t i = std::llround((x - lo[a]) / h[a]);
      const double tol = 1e-12 * h[a] + 8.0 * kEps * (std::fabs(x) + std::fabs(lo[a]) + std::fabs(hi[a]));
      if (i < 0 || i > n[a] || std::fabs(x - (lo[a] + double(i) * h[a])) > tol) return;
      ijk[3 * v + a] = int32_t(i);
      lin += i * mul;
      mul *= a == 0 ? px : py;
    }
    if (hit[size_t(lin)]) return;
    hit[size_t(lin)] = 1;
  }
  // the reflection under which every cell is a template tet of its cube
  std::vector<int32_t> slot_cell(size_t(m.C));
  for (int refl = 0; refl < 8; ++refl) {
    std::fill(slot_cell.begin(), slot_cell.end(), -1);
    bool ok = true;
    for (int64_t c = 0; c < m.C && ok; ++c) {
      int p[4][3], mn[3] = {1 << 30, 1 << 30, 1 << 30}, mx[3] = {-1, -1, -1};
      for (int k = 0; k < 4; ++k)
        for (int a = 0; a < 3; ++a) {
          const int i = ijk[3 * int64_t(m.cells[4 * c + k]) + a];
          p[k][a] = ((refl >> a) & 1) ? n[a] - i : i;
          mn[a] = std::min(mn[a], p[k][a]);
          mx[a] = std::max(mx[a], p[k][a]);
        }
      for (int a = 0; a < 3; ++a) ok = ok && mx[a] - mn[a] == 1;
      if (!ok) break;
      int mask = 0;
      for (int k = 0; k < 4; ++k) mask |= 1 << ((p[k][0] - mn[0]) + 2 * (p[k][1] - mn[1]) + 4 * (p[k][2] - mn[2]));
      const int t = template_of_corners(mask);
      if (t < 0) {
        ok = false;
        break;
      }
      const int64_t hx = mn[0] + int64_t(n[0]) * (mn[1] + int64_t(n[1]) * mn[2]);
      int32_t& sc = slot_cell[size_t(6 * hx + t)];
      if (sc >= 0) {
        ok = false;
        break;
      }
      sc = int32_t(c);
    }
    if (!ok) continue;
    // lattice numbering under this reflection
    std::vector<int32_t> lat_of(size_t(m.N)), node_of(size_t(m.N));
    bool identity = refl == 0;
    for (int64_t v = 0; v < m.N; ++v) {
      int q[3];
      for (int a = 0; a < 3; ++a) q[a] = ((refl >> a) & 1) ? n[a] - ijk[3 * v + a] : ijk[3 * v + a];
      const int64_t b = q[0] + px * (q[1] + py * int64_t(q[2]));
      lat_of[size_t(v)] = int32_t(b);
      node_of[size_t(b)] = int32_t(v);
      identity = identity && b == v;
    }
    for (int64_t k = 0; k < m.C && identity; ++k) identity = slot_cell[size_t(k)] == k;
    for (int a = 0; a < 3; ++a) {
      m.lat_n[a] = n[a];
      m.lat_l[a] = h[a] * n[a];
    }
    m.lat_permuted = !identity;
    m.lat_flip = refl;
    if (m.lat_permuted) {
      m.d_lat_node.upload(node_of.data(), node_of.size());
      m.d_lat_of_node.upload(lat_of.data(), lat_of.size());
      m.d_lat_cell.upload(slot_cell.data(), slot_cell.size());
      m.h_lat_of_node.swap(lat_of);
    }
    return;
  }
}

}  // namespace pa
