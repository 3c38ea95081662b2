// pa_mesh.cu -- mesh set-up on the host: block-CRS graph, cell -> CRS block
// map, and the shared-memory cell tiles of the matrix-free kernel.
#include <algorithm>
#include <cmath>
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

// Cell order for tiling: Morton (Z-order) of the cell centroids, so that
// consecutive cells are spatially compact and a tile of 256 tets touches few
// nodes (about 100 on a structured box).
std::vector<int32_t> morton_order(const Mesh& m) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t v = 0; v < m.N; ++v)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], m.coords[3 * v + d]);
      hi[d] = std::max(hi[d], m.coords[3 * v + d]);
    }
  double scale[3];
  for (int d = 0; d < 3; ++d) scale[d] = (hi[d] > lo[d]) ? double((1 << 21) - 1) / (hi[d] - lo[d]) : 0.0;
  std::vector<std::pair<uint64_t, int32_t>> keys(m.C);
  for (int64_t c = 0; c < m.C; ++c) {
    double ctr[3] = {0, 0, 0};
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) ctr[d] += 0.25 * m.coords[3 * int64_t(m.cells[4 * c + n]) + d];
    uint64_t q[3];
    for (int d = 0; d < 3; ++d) q[d] = uint64_t(std::llround((ctr[d] - lo[d]) * scale[d]));
    keys[c] = {spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2), int32_t(c)};
  }
  std::sort(keys.begin(), keys.end());
  std::vector<int32_t> order(m.C);
  for (int64_t i = 0; i < m.C; ++i) order[i] = keys[i].second;
  return order;
}

void build_tiles(Mesh& m) {
  std::vector<int32_t> order = morton_order(m);
  std::vector<int32_t> tile_cell_start{0}, tile_node_start{0};
  std::vector<uint32_t> tile_nodes, cell_local(m.C);
  std::vector<int32_t> stamp(m.N, -1), local(m.N, 0), node_tiles(m.N, 0), owner(m.N, -1);
  std::vector<int32_t> cur_nodes;
  cur_nodes.reserve(kTileNodes);
  int32_t tile = 0;
  int64_t first_cell = 0;

  auto close_tile = [&](int64_t end_cell) {
    // Sort the tile's nodes by id (coalesced staging loads) and fix local ids.
    std::vector<int32_t> sorted = cur_nodes;
    std::sort(sorted.begin(), sorted.end());
    for (size_t i = 0; i < sorted.size(); ++i) local[sorted[i]] = int32_t(i);
    for (int64_t i = first_cell; i < end_cell; ++i) {
      const int32_t c = order[i];
      uint32_t packed = 0;
      for (int n = 0; n < 4; ++n) packed |= uint32_t(local[m.cells[4 * int64_t(c) + n]]) << (8 * n);
      cell_local[i] = packed;
    }
    for (int32_t v : sorted) {
      tile_nodes.push_back(uint32_t(v));
      node_tiles[v] += 1;
      if (owner[v] < 0) owner[v] = tile;
    }
    tile_cell_start.push_back(int32_t(end_cell));
    tile_node_start.push_back(int32_t(tile_nodes.size()));
    cur_nodes.clear();
    ++tile;
    first_cell = end_cell;
  };

  for (int64_t i = 0; i < m.C; ++i) {
    const int32_t c = order[i];
    int fresh = 0;
    for (int n = 0; n < 4; ++n) {
      const int32_t v = m.cells[4 * int64_t(c) + n];
      bool seen = stamp[v] == tile;
      for (int k = 0; k < n && !seen; ++k) seen = (m.cells[4 * int64_t(c) + k] == v);
      fresh += seen ? 0 : 1;
    }
    if (i - first_cell >= kTileCells || int(cur_nodes.size()) + fresh > kTileNodes) close_tile(i);
    for (int n = 0; n < 4; ++n) {
      const int32_t v = m.cells[4 * int64_t(c) + n];
      if (stamp[v] != tile) {
        stamp[v] = tile;
        cur_nodes.push_back(v);
      }
    }
  }
  if (m.C > first_cell) close_tile(m.C);

  // Flags: shared (written by atomics) and owner (exactly one tile per node).
  for (int32_t t = 0; t < tile; ++t)
    for (int32_t k = tile_node_start[t]; k < tile_node_start[t + 1]; ++k) {
      const uint32_t v = tile_nodes[k];
      uint32_t f = v;
      if (node_tiles[v] > 1) f |= kShared;
      if (owner[v] == t) f |= kOwner;
      tile_nodes[k] = f;
    }
  m.T = tile;
  m.h_cell_perm = order;
  m.d_tile_cell_start.upload(tile_cell_start.data(), tile_cell_start.size());
  m.d_tile_node_start.upload(tile_node_start.data(), tile_node_start.size());
  m.d_tile_nodes.upload(tile_nodes.data(), tile_nodes.size());
  m.d_cell_local.upload(cell_local.data(), cell_local.size());
  m.d_cell_perm.upload(order.data(), order.size());
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

void mesh_build(Mesh& m) {
  PA_CHECK(m.C > 0 && m.N > 0, "mesh needs at least one cell and one node");
  PA_CHECK(m.N < int64_t(kNodeMask), "too many nodes for 30-bit node ids");
  for (int64_t i = 0; i < 4 * m.C; ++i)
    PA_CHECK(m.cells[i] >= 0 && m.cells[i] < m.N, "cells2nodes entry out of range");
  for (int64_t i = 0; i < 3 * m.N; ++i) PA_CHECK(std::isfinite(m.coords[i]), "non-finite coordinate");
  PA_CUDA(cudaGetDevice(&m.device));
  build_graph(m);
  build_tiles(m);
  m.d_cells.upload(m.cells.data(), m.cells.size());
  m.d_coords.upload(m.coords.data(), m.coords.size());
  std::vector<float> c32(m.coords.begin(), m.coords.end());
  m.d_coords32.upload(c32.data(), c32.size());
  PA_CUDA(cudaDeviceSynchronize());
}

}  // namespace pa
