// pa_mesh.cu -- mesh set-up on the host: block-CRS graph, cell -> CRS block
// map, and the shared-memory cell tiles of the matrix-free kernel.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <numeric>

#include "pa_problem.cuh"

namespace pa {

namespace {

inline uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
  v &= 0x1fffffULL;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}

struct Cluster {
  int32_t cell0;        // first user cell (hex: the 6 cells in template order below)
  int32_t hex_cells[6]; // hex only: user cells of template tets T0..T5
  int32_t nodes[8];     // hex: slot s = a + 2b + 4c; single: its 4 nodes
  bool hex;
  int32_t part;
  uint64_t key;
};

// Six consecutive cells form a hex cluster when their union has 8 nodes, two
// of which (the diagonal) belong to all six tets and the other six form a
// ring in which consecutive tets share one node.  Labeling: diagonal ->
// slots 0 and 7, ring r0..r5 -> slots 3, 2, 6, 4, 5, 1, so that tet
// {d0, d1, r_k, r_k+1} is template tet T_k of hex_slot().
bool match_hex(const Mesh& m, int64_t c0, Cluster& out) {
  int32_t nodes[24];
  for (int j = 0; j < 6; ++j)
    for (int n = 0; n < 4; ++n) nodes[4 * j + n] = m.cells[4 * (c0 + j) + n];
  int32_t uniq[24];
  int nu = 0;
  for (int i = 0; i < 24; ++i) {
    bool seen = false;
    for (int k = 0; k < nu && !seen; ++k) seen = uniq[k] == nodes[i];
    if (!seen) uniq[nu++] = nodes[i];
  }
  if (nu != 8) return false;
  auto has = [&](int j, int32_t v) {
    for (int n = 0; n < 4; ++n)
      if (nodes[4 * j + n] == v) return true;
    return false;
  };
  int32_t diag[2];
  int nd = 0;
  for (int k = 0; k < 8; ++k) {
    bool all = true;
    for (int j = 0; j < 6 && all; ++j) all = has(j, uniq[k]);
    if (all) {
      if (nd == 2) return false;
      diag[nd++] = uniq[k];
    }
  }
  if (nd != 2) return false;
  // ring nodes of each tet
  int32_t ring[6][2];
  for (int j = 0; j < 6; ++j) {
    int r = 0;
    for (int n = 0; n < 4; ++n) {
      const int32_t v = nodes[4 * j + n];
      if (v == diag[0] || v == diag[1]) continue;
      if (r == 2) return false;
      ring[j][r++] = v;
    }
    if (r != 2 || ring[j][0] == ring[j][1]) return false;
  }
  // walk the cycle: tet order t_0..t_5 with ring nodes (r_k, r_k+1)
  int order[6];
  int32_t rn[7];
  bool used[6] = {false, false, false, false, false, false};
  order[0] = 0;
  used[0] = true;
  rn[0] = ring[0][0];
  rn[1] = ring[0][1];
  for (int k = 1; k < 6; ++k) {
    int next = -1;
    for (int j = 0; j < 6; ++j)
      if (!used[j] && (ring[j][0] == rn[k] || ring[j][1] == rn[k])) {
        if (next >= 0) return false;
        next = j;
      }
    if (next < 0) return false;
    used[next] = true;
    order[k] = next;
    rn[k + 1] = ring[next][0] == rn[k] ? ring[next][1] : ring[next][0];
  }
  if (rn[6] != rn[0]) return false;
  for (int a = 0; a < 6; ++a)
    for (int b = a + 1; b < 6; ++b)
      if (rn[a] == rn[b]) return false;
  static const int ring_slot[6] = {3, 2, 6, 4, 5, 1};
  out.hex = true;
  out.cell0 = int32_t(c0);
  out.nodes[0] = diag[0];
  out.nodes[7] = diag[1];
  for (int k = 0; k < 6; ++k) out.nodes[ring_slot[k]] = rn[k];
  for (int k = 0; k < 6; ++k) out.hex_cells[k] = int32_t(c0 + order[k]);
  return true;
}

// Uniform hex geometry: every cluster is a hex and each hex's edge vectors
// E_s = x_slot(s) - x_slot(7) (s = 0..6) equal the first hex's to 1e-9 of its
// largest edge (FP64 rounding of generated coordinates stays far below that).
// Then the per-tet rows of det * J^-1 and 1 / (6 |det|) are the same for all
// hexes; they are computed once here in FP64, in the tile kernel's relative
// form (template tet k = slots 0, ring(k), ring(k+1), 7).
void detect_uniform_hex(Mesh& m, const std::vector<Cluster>& cl) {
  m.uniform_hex = false;
  if (cl.empty()) return;
  for (const Cluster& k : cl)
    if (!k.hex) return;
  auto edges = [&](const Cluster& k, double (&E)[7][3]) {
    const int32_t v7 = k.nodes[7];
    for (int s = 0; s < 7; ++s)
      for (int d = 0; d < 3; ++d) E[s][d] = m.coords[3 * int64_t(k.nodes[s]) + d] - m.coords[3 * int64_t(v7) + d];
  };
  double E0[7][3];
  edges(cl[0], E0);
  double size = 0.0;
  for (int s = 0; s < 7; ++s)
    for (int d = 0; d < 3; ++d) size = std::max(size, std::fabs(E0[s][d]));
  if (!(size > 0.0)) return;
  const double tol = 1e-9 * size;
  double dev = 0.0;
  for (const Cluster& k : cl) {
    double E[7][3];
    edges(k, E);
    for (int s = 0; s < 7; ++s)
      for (int d = 0; d < 3; ++d) {
        const double e = std::fabs(E[s][d] - E0[s][d]);
        if (e > tol) return;
        dev = std::max(dev, e);
      }
  }
  m.hex_geo_dev = dev / size;
  static const int ring[7] = {3, 2, 6, 4, 5, 1, 3};
  auto cross = [](const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
  };
  HexGeo<double> g{};
  for (int k = 0; k < 6; ++k) {
    const double *e0 = E0[0], *ea = E0[ring[k]], *eb = E0[ring[k + 1]];
    cross(ea, eb, &g.h[k][0]);  // h0 = ea x eb
    cross(eb, e0, &g.h[k][3]);  // h1 = eb x e0
    cross(e0, ea, &g.h[k][6]);  // h2 = e0 x ea
    const double det = e0[0] * g.h[k][0] + e0[1] * g.h[k][1] + e0[2] * g.h[k][2];
    if (!(std::fabs(det) > 1e-12 * size * size * size)) return;  // degenerate tet: keep the general path
    g.s[k] = 1.0 / (6.0 * std::fabs(det));
  }
  m.geo64 = g;
  for (int k = 0; k < 6; ++k) {
    for (int i = 0; i < 9; ++i) m.geo32.h[k][i] = float(g.h[k][i]);
    m.geo32.s[k] = float(g.s[k]);
  }
  m.uniform_hex = true;
}

// Clusters (hex groups of six consecutive cells, else single cells), ordered
// along the Morton (Z-order) curve of their centroids, packed greedily into
// tiles of <= tile_clusters clusters and <= 2 tile_clusters nodes.
void build_tiles(Mesh& m) {
  std::vector<Cluster> cl;
  cl.reserve(m.C / 6 + 16);
  for (int64_t c = 0; c < m.C;) {
    Cluster h;
    if (c + 6 <= m.C && match_hex(m, c, h)) {
      cl.push_back(h);
      c += 6;
      continue;
    }
    Cluster s{};
    s.hex = false;
    s.cell0 = int32_t(c);
    for (int n = 0; n < 4; ++n) s.nodes[n] = m.cells[4 * c + n];
    for (int n = 4; n < 8; ++n) s.nodes[n] = -1;
    cl.push_back(s);
    ++c;
  }
  detect_uniform_hex(m, cl);
  if (!m.allow_uniform_geometry) m.uniform_hex = false;
  // part of every cluster (all its nodes must lie in one part)
  std::vector<uint16_t> npart;
  if (m.num_parts > 1) {
    npart.resize(m.N);
    for (int32_t p = 0; p < m.num_parts; ++p)
      for (int64_t v = m.part_node_offsets[p]; v < m.part_node_offsets[p + 1]; ++v) npart[v] = uint16_t(p);
  }
  for (auto& k : cl) {
    k.part = npart.empty() ? 0 : npart[k.nodes[0]];
    const int nn = k.hex ? 8 : 4;
    for (int n = 1; n < nn; ++n)
      if (!npart.empty() && npart[k.nodes[n]] != k.part) throw Error(PA_ERR_INVALID_ARG, "a cell spans two parts");
  }
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t v = 0; v < m.N; ++v)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], m.coords[3 * v + d]);
      hi[d] = std::max(hi[d], m.coords[3 * v + d]);
    }
  double scale[3];
  for (int d = 0; d < 3; ++d) scale[d] = (hi[d] > lo[d]) ? double((1 << 21) - 1) / (hi[d] - lo[d]) : 0.0;
  for (auto& k : cl) {
    const int nn = k.hex ? 8 : 4;
    double ctr[3] = {0, 0, 0};
    for (int n = 0; n < nn; ++n)
      for (int d = 0; d < 3; ++d) ctr[d] += m.coords[3 * int64_t(k.nodes[n]) + d] / nn;
    uint64_t q[3];
    for (int d = 0; d < 3; ++d) q[d] = uint64_t(std::llround((ctr[d] - lo[d]) * scale[d]));
    k.key = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
  }
  std::stable_sort(cl.begin(), cl.end(),
                   [](const Cluster& a, const Cluster& b) { return a.part != b.part ? a.part < b.part : a.key < b.key; });

  const int tile_k = m.tile_clusters, tile_n = 2 * m.tile_clusters;
  std::vector<int32_t> tile_cluster_start{0}, tile_cell_start{0}, tile_hex_count, tile_node_start{0}, perm,
      tile_part;
  int32_t cur_part = 0;
  std::vector<uint32_t> tile_nodes;
  std::vector<uint4> cluster_nodes;
  perm.reserve(m.C);
  std::vector<int32_t> stamp(m.N, -1), local(m.N, 0), node_tiles(m.N, 0), owner(m.N, -1);
  std::vector<int32_t> cur_nodes;
  std::vector<const Cluster*> cur;
  int32_t tile = 0;
  int64_t nhex_total = 0;

  auto close_tile = [&]() {
    std::vector<int32_t> sorted = cur_nodes;
    std::sort(sorted.begin(), sorted.end());
    for (size_t i = 0; i < sorted.size(); ++i) local[sorted[i]] = int32_t(i);
    std::stable_partition(cur.begin(), cur.end(), [](const Cluster* k) { return k->hex; });
    int32_t nh = 0;
    for (const Cluster* k : cur) {
      uint16_t ids[8];
      for (int n = 0; n < 8; ++n) ids[n] = k->nodes[n] >= 0 ? uint16_t(local[k->nodes[n]]) : uint16_t(0xffff);
      uint4 q;
      q.x = uint32_t(ids[0]) | (uint32_t(ids[1]) << 16);
      q.y = uint32_t(ids[2]) | (uint32_t(ids[3]) << 16);
      q.z = uint32_t(ids[4]) | (uint32_t(ids[5]) << 16);
      q.w = uint32_t(ids[6]) | (uint32_t(ids[7]) << 16);
      cluster_nodes.push_back(q);
      if (k->hex) {
        ++nh;
        for (int j = 0; j < 6; ++j) perm.push_back(k->hex_cells[j]);
      } else {
        perm.push_back(k->cell0);
      }
    }
    for (int32_t v : sorted) {
      tile_nodes.push_back(uint32_t(v));
      node_tiles[v] += 1;
      if (owner[v] < 0) owner[v] = tile;
    }
    nhex_total += nh;
    tile_part.push_back(cur_part);
    tile_hex_count.push_back(nh);
    tile_cluster_start.push_back(int32_t(cluster_nodes.size()));
    tile_cell_start.push_back(int32_t(perm.size()));
    tile_node_start.push_back(int32_t(tile_nodes.size()));
    cur_nodes.clear();
    cur.clear();
    ++tile;
  };

  for (const Cluster& k : cl) {
    const int nn = k.hex ? 8 : 4;
    int fresh = 0;
    for (int n = 0; n < nn; ++n) fresh += stamp[k.nodes[n]] == tile ? 0 : 1;
    if (int(cur.size()) >= tile_k || int(cur_nodes.size()) + fresh > tile_n || (!cur.empty() && k.part != cur_part))
      close_tile();
    cur_part = k.part;
    for (int n = 0; n < nn; ++n) {
      const int32_t v = k.nodes[n];
      if (stamp[v] != tile) {
        stamp[v] = tile;
        cur_nodes.push_back(v);
      }
    }
    cur.push_back(&k);
  }
  if (!cur.empty()) close_tile();
  if (int64_t(perm.size()) != m.C) throw Error(PA_ERR_INVALID_ARG, "cluster build lost cells");
  // Structural checks the kernel relies on (every shared-memory index in range,
  // every cell exactly once).
  {
    std::vector<uint8_t> seen(m.C, 0);
    for (int32_t c : perm) {
      if (c < 0 || c >= m.C || seen[c]) throw Error(PA_ERR_INVALID_ARG, "cell permutation is not a bijection");
      seen[c] = 1;
    }
    for (int32_t t = 0; t < tile; ++t) {
      const int32_t nn = tile_node_start[t + 1] - tile_node_start[t];
      const int32_t nk = tile_cluster_start[t + 1] - tile_cluster_start[t];
      const int32_t nc = tile_cell_start[t + 1] - tile_cell_start[t];
      if (nn > tile_n || nk > tile_k || tile_hex_count[t] > nk || nc > 6 * tile_k ||
          nc != 6 * tile_hex_count[t] + (nk - tile_hex_count[t]))
        throw Error(PA_ERR_INVALID_ARG, "tile exceeds its shared-memory capacity");
      for (int32_t k = tile_cluster_start[t]; k < tile_cluster_start[t + 1]; ++k) {
        const uint4 q = cluster_nodes[k];
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
        const int used = (k - tile_cluster_start[t]) < tile_hex_count[t] ? 8 : 4;
        for (int n = 0; n < used; ++n) {
          const uint32_t id = (w[n / 2] >> (16 * (n % 2))) & 0xffffu;
          if (int32_t(id) >= nn) throw Error(PA_ERR_INVALID_ARG, "cluster node id outside its tile");
        }
      }
    }
  }

  // The table kernel accumulates node sums slot by slot without atomics: it
  // needs, in every tile, the nodes of any one slot to be distinct across the
  // tile's hexes (true for translates, unless hexes are duplicated).
  if (m.uniform_hex) {
    std::vector<int32_t> mark(tile_n, -1);
    for (int32_t t = 0; t < tile && m.uniform_hex; ++t)
      for (int s = 0; s < 8 && m.uniform_hex; ++s) {
        const int32_t stamp = 8 * t + s;
        for (int32_t k = tile_cluster_start[t]; k < tile_cluster_start[t + 1]; ++k) {
          const uint4 q = cluster_nodes[k];
          const uint32_t w[4] = {q.x, q.y, q.z, q.w};
          const uint32_t id = (w[s / 2] >> (16 * (s % 2))) & 0xffffu;
          if (mark[id] == stamp) {
            m.uniform_hex = false;
            break;
          }
          mark[id] = stamp;
        }
      }
  }

  for (int32_t t = 0; t < tile; ++t)
    for (int32_t k = tile_node_start[t]; k < tile_node_start[t + 1]; ++k) {
      const uint32_t v = tile_nodes[k];
      uint32_t f = v;
      if (node_tiles[v] > 1) f |= kShared;
      if (owner[v] == t) f |= kOwner;
      tile_nodes[k] = f;
    }
  m.T = tile;
  m.num_clusters = int64_t(cluster_nodes.size());
  m.num_hex = nhex_total;
  m.h_cell_perm = perm;
  m.d_tile_cluster_start.upload(tile_cluster_start.data(), tile_cluster_start.size());
  m.d_tile_hex_count.upload(tile_hex_count.data(), tile_hex_count.size());
  m.d_tile_node_start.upload(tile_node_start.data(), tile_node_start.size());
  m.d_tile_nodes.upload(tile_nodes.data(), tile_nodes.size());
  m.d_cluster_nodes.upload(cluster_nodes.data(), cluster_nodes.size());
  m.d_tile_cell_start.upload(tile_cell_start.data(), tile_cell_start.size());
  m.h_tile_nodes = tile_nodes;
  m.d_cell_perm.upload(perm.data(), perm.size());
  std::vector<int32_t> iperm(m.C);
  for (int64_t i = 0; i < m.C; ++i) iperm[perm[i]] = int32_t(i);
  m.d_cell_iperm.upload(iperm.data(), iperm.size());
  m.h_tile_part = tile_part;
  if (m.num_parts > 1) {
    m.d_tile_part.upload(tile_part.data(), tile_part.size());
    m.d_node_part.upload(npart.data(), npart.size());
  } else {
    m.d_tile_part.release();
    m.d_node_part.release();
  }
}

// Node-star graph plus diagonal, sorted columns: the pattern CreateBlockMatrix
// builds from Omega_h's star (src/ImplicitFunctors.hpp:735-808).
void build_graph(Mesh& m) {
  std::vector<int32_t> cnt(m.N + 1, 0);
  for (int64_t c = 0; c < m.C; ++c)
    for (int n = 0; n < 4; ++n) cnt[m.cells[4 * c + n] + 1]++;
  for (int64_t v = 0; v < m.N; ++v) cnt[v + 1] += cnt[v];
  std::vector<int32_t> n2c(cnt[m.N]);
  std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
  for (int64_t c = 0; c < m.C; ++c)
    for (int n = 0; n < 4; ++n) n2c[fill[m.cells[4 * c + n]]++] = int32_t(c);
  m.rowmap.assign(m.N + 1, 0);
  m.cols.clear();
  m.cols.reserve(size_t(m.N) * 16);
  std::vector<int32_t> buf;
  for (int64_t v = 0; v < m.N; ++v) {
    buf.clear();
    for (int32_t k = cnt[v]; k < cnt[v + 1]; ++k)
      for (int n = 0; n < 4; ++n) buf.push_back(m.cells[4 * int64_t(n2c[k]) + n]);
    buf.push_back(int32_t(v));
    std::sort(buf.begin(), buf.end());
    buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
    m.cols.insert(m.cols.end(), buf.begin(), buf.end());
    m.rowmap[v + 1] = int32_t(m.cols.size());
  }
  m.B = int64_t(m.cols.size());
}

}  // namespace

// Cell -> CRS block map, 16 entries per cell (row node a, column node b).
void Mesh::build_graph_entries() {
  std::vector<int32_t> ent(size_t(C) * 16);
  for (int64_t c = 0; c < C; ++c)
    for (int a = 0; a < 4; ++a) {
      const int32_t row = cells[4 * c + a];
      for (int b = 0; b < 4; ++b) {
        const int32_t col = cells[4 * c + b];
        int32_t hit = -1;
        for (int32_t k = rowmap[row]; k < rowmap[row + 1]; ++k)
          if (cols[k] == col) { hit = k; break; }
        if (hit < 0) throw Error(PA_ERR_INVALID_ARG, "CRS graph lacks a cell's node pair");
        ent[16 * c + 4 * a + b] = hit;
      }
    }
  d_cell_entry.upload(ent.data(), ent.size());
  d_rowmap.upload(rowmap.data(), rowmap.size());
  d_cols.upload(cols.data(), cols.size());
}

void mesh_rebuild_tiles(Mesh& m) {
  PA_CHECK(m.tile_clusters == 64 || m.tile_clusters == 128 || m.tile_clusters == 256,
           "tile size (clusters per tile) must be 64, 128 or 256");
  build_tiles(m);
  PA_CUDA(cudaDeviceSynchronize());
}

void mesh_make_box(Mesh& m, int nx, int ny, int nz, double lx, double ly, double lz) {
  static const int tet[6][4][3] = {
      {{0, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 1, 1}}, {{0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}},
      {{0, 0, 0}, {0, 1, 1}, {0, 0, 1}, {1, 1, 1}}, {{0, 0, 0}, {1, 0, 1}, {1, 1, 1}, {0, 0, 1}},
      {{1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {0, 0, 0}}, {{1, 0, 0}, {1, 1, 1}, {1, 1, 0}, {0, 0, 0}}};
  const int64_t px = nx + 1, py = ny + 1;
  m.N = px * py * int64_t(nz + 1);
  m.C = 6LL * nx * ny * nz;
  m.coords.resize(3 * m.N);
  m.cells.resize(4 * m.C);
  for (int64_t k = 0; k <= nz; ++k)
    for (int64_t j = 0; j <= ny; ++j)
      for (int64_t i = 0; i <= nx; ++i) {
        const int64_t v = i + px * (j + py * k);
        m.coords[3 * v + 0] = lx * double(i) / nx;
        m.coords[3 * v + 1] = ly * double(j) / ny;
        m.coords[3 * v + 2] = lz * double(k) / nz;
      }
  int64_t c = 0;
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i)
        for (int t = 0; t < 6; ++t, ++c)
          for (int n = 0; n < 4; ++n) {
            const int* o = tet[t][n];
            m.cells[4 * c + n] = int32_t((i + o[0]) + px * ((j + o[1]) + py * (k + o[2])));
          }
  m.box_n[0] = nx;
  m.box_n[1] = ny;
  m.box_n[2] = nz;
  m.box_l[0] = lx;
  m.box_l[1] = ly;
  m.box_l[2] = lz;
  for (int a = 0; a < 3; ++a) {
    m.lat_n[a] = m.box_n[a];
    m.lat_l[a] = m.box_l[a];
  }
  m.lat_permuted = false;
  m.lat_flip = 0;
  mesh_build(m);
}

void mesh_build(Mesh& m) {
  PA_CHECK(m.C > 0 && m.N > 0, "mesh needs at least one cell and one node");
  PA_CHECK(m.N <= int64_t(kNodeIdMask), "too many nodes for 27-bit node ids");
  for (int64_t i = 0; i < 4 * m.C; ++i)
    PA_CHECK(m.cells[i] >= 0 && m.cells[i] < m.N, "cells2nodes entry out of range");
  for (int64_t i = 0; i < 3 * m.N; ++i) PA_CHECK(std::isfinite(m.coords[i]), "non-finite coordinate");
  PA_CUDA(cudaGetDevice(&m.device));
  if (const char* e = std::getenv("PA_TILE_CLUSTERS")) m.tile_clusters = std::atoi(e);
  PA_CHECK(m.tile_clusters == 64 || m.tile_clusters == 128 || m.tile_clusters == 256,
           "tile size (clusters per tile) must be 64, 128 or 256");
  build_graph(m);
  build_tiles(m);
  if (m.box_n[0] == 0) detect_lattice(m);
  m.d_cells.upload(m.cells.data(), m.cells.size());
  m.d_coords.upload(m.coords.data(), m.coords.size());
  std::vector<double> soa(3 * m.N);
  std::vector<float> soa32(3 * m.N);
  for (int64_t v = 0; v < m.N; ++v)
    for (int d = 0; d < 3; ++d) {
      soa[d * m.N + v] = m.coords[3 * v + d];
      soa32[d * m.N + v] = float(m.coords[3 * v + d]);
    }
  m.d_coords_soa.upload(soa.data(), soa.size());
  m.d_coords32_soa.upload(soa32.data(), soa32.size());
  std::vector<float4> aos4(m.N);
  for (int64_t v = 0; v < m.N; ++v)
    aos4[v] = make_float4(float(m.coords[3 * v]), float(m.coords[3 * v + 1]), float(m.coords[3 * v + 2]), 0.0f);
  m.d_coords32_aos4.upload(aos4.data(), aos4.size());
  PA_CUDA(cudaDeviceSynchronize());
}

}  // namespace pa
