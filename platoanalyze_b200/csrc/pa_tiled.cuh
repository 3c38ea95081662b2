// pa_tiled.cuh -- tile-staged, hex-clustered matrix-free K.x: the hot kernel
// of the solve.
//
// Mesh layout (built once on the host, pa_mesh.cu):
//  * cells are grouped into clusters: a "hex" cluster is six tets that form
//    the six-tet split of one hexahedron around a diagonal (the split every
//    hex-derived tet mesh, e.g. a structured box, has); any other cell is a
//    "single" cluster.  A hex cluster touches 8 nodes for 6 cells, a single
//    one 4 nodes for 1 cell.
//  * clusters are ordered along a Morton curve and packed into tiles of at
//    most kTileClusters clusters touching at most kTileNodes nodes.
//
// Kernel (a persistent grid, a multiple of the SM count, walks the tiles):
//  1. stage the tile's nodes in shared memory (coordinates, input vector,
//     Dirichlet mask) in one coalesced pass over the tile's sorted node list;
//  2. one thread per cluster: read the cluster's nodes from shared memory
//     into registers once, evaluate its tets (geometry, strain, stress, SIMP
//     weight, divergence) and accumulate the node sums in registers -- a hex
//     cluster reads 8 nodes and issues 24 shared-memory atomics for 6 tets,
//     instead of 24 node reads and 72 atomics cell by cell;
//  3. write each node sum once: a plain store for nodes only this tile
//     touches, a global atomic add for nodes shared with other tiles.
// The PCG variant (MODE 1) forms p = D^-1 r + beta p_old while staging (the
// owner tile writes p once) and reduces p.Kp = sum_cells p_e^T K_e p_e from
// the per-tet energies, so the search-direction update and the first dot
// product need no extra pass over the vectors.
#pragma once
#include "pa_cell.cuh"

namespace pa {

constexpr int kApplyThreads = kTileClusters;

template <typename T>
struct ApplyArgs {
  TileView tv;
  const T* coords;          // N*3
  const T* w;               // C, SIMP weight per cell, internal order
  const uint8_t* node_mask; // N (bit d: dof d constrained) or null
  Iso<T> iso;
  const T* x;               // plain: input vector; pcg: p_old
  T* y;                     // output, zero on entry
  // PCG fusion (mode 1)
  const T* r;
  const T* dinv;
  T* p_new;
  PcgScalars* sc;
  double* partials;
  unsigned int* counter;
};

__device__ __forceinline__ double block_sum(double v, double* smem /*>= 32*/) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? smem[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;  // valid in thread 0
}

// Returns true in every thread of the block that arrives last.
__device__ __forceinline__ bool last_block_arrive(unsigned int* counter) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  return s_last;
}

// Six tets of a hex cluster in slot numbering s = a + 2b + 4c of corner (a,b,c);
// a constant expression, so that after unrolling every register index is static.
__host__ __device__ constexpr int hex_slot(int j, int n) {
  constexpr int t[6][4] = {{0, 3, 2, 7}, {0, 2, 6, 7}, {0, 6, 4, 7}, {0, 5, 7, 4}, {1, 5, 7, 0}, {1, 7, 3, 0}};
  return t[j][n];
}

// One tet: contributions r[4][3] for its nodes from xs (coords) and us (input);
// returns the tet's energy sig:eps (for p.Kp).
template <typename T>
__device__ __forceinline__ T tet_apply(const Iso<T>& iso, T w, const T (&xc)[4][3], const T (&u)[12], T (&r)[12]) {
  T g[4][3], vol, e[6], sig[6];
  tet_geometry(xc, g, vol);
  tet_strain(g, u, e);
  tet_stress(iso, vol * w, e, sig);
  tet_divergence(g, sig, r);
  return voigt_dot(sig, e);
}

template <typename T, int MODE>
__global__ void __launch_bounds__(kApplyThreads, 1) k_apply_tiled(ApplyArgs<T> a) {
  __shared__ T s_c[kTileNodes * 3];
  __shared__ T s_x[kTileNodes * 3];
  __shared__ T s_y[kTileNodes * 3];
  __shared__ uint32_t s_node[kTileNodes];
  __shared__ uint8_t s_mask[kTileNodes];
  __shared__ double s_red[32];

  T beta = T(0);
  if (MODE == 1) {
    if (a.sc->done) return;
    beta = T(a.sc->beta);
  }
  double pap = 0.0;

  for (int tile = blockIdx.x; tile < a.tv.num_tiles; tile += gridDim.x) {
    const int n0 = a.tv.tile_node_start[tile], nn = a.tv.tile_node_start[tile + 1] - n0;
    const int k0 = a.tv.tile_cluster_start[tile], nk = a.tv.tile_cluster_start[tile + 1] - k0;
    const int nhex = a.tv.tile_hex_count[tile];
    // 1. stage nodes
    for (int i = threadIdx.x; i < nn; i += blockDim.x) {
      const uint32_t f = a.tv.tile_nodes[n0 + i];
      const int64_t gid = f & kNodeMask;
      const uint8_t mk = a.node_mask ? a.node_mask[gid] : uint8_t(0);
      s_node[i] = f;
      s_mask[i] = mk;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int64_t dof = 3 * gid + d;
        s_c[3 * i + d] = a.coords[dof];
        s_y[3 * i + d] = T(0);
        T v;
        if (MODE == 0) {
          v = (mk >> d) & 1 ? T(0) : a.x[dof];
        } else {
          v = (mk >> d) & 1 ? T(0) : a.dinv[dof] * a.r[dof] + beta * a.x[dof];
          if (f & kOwner) a.p_new[dof] = v;
        }
        s_x[3 * i + d] = v;
      }
    }
    __syncthreads();
    // 2. one cluster per thread
    const int t = threadIdx.x;
    if (t < nk) {
      const int k = k0 + t;
      const uint4 q = a.tv.cluster_nodes[k];
      const int c0 = a.tv.cluster_cell_start[k];
      int ln[8] = {int(q.x & 0xffff), int(q.x >> 16), int(q.y & 0xffff), int(q.y >> 16),
                   int(q.z & 0xffff), int(q.z >> 16), int(q.w & 0xffff), int(q.w >> 16)};
      if (t < nhex) {
        T X[8][3], U[8][3], Y[8][3];
#pragma unroll
        for (int s = 0; s < 8; ++s)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            X[s][d] = s_c[3 * ln[s] + d];
            U[s][d] = s_x[3 * ln[s] + d];
            Y[s][d] = T(0);
          }
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          T xc[4][3], u[12], r[12];
#pragma unroll
          for (int n = 0; n < 4; ++n)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              xc[n][d] = X[hex_slot(j, n)][d];
              u[3 * n + d] = U[hex_slot(j, n)][d];
            }
          const T en = tet_apply(a.iso, a.w[c0 + j], xc, u, r);
          if (MODE == 1) pap += double(en);
#pragma unroll
          for (int n = 0; n < 4; ++n)
#pragma unroll
            for (int d = 0; d < 3; ++d) Y[hex_slot(j, n)][d] += r[3 * n + d];
        }
#pragma unroll
        for (int s = 0; s < 8; ++s)
#pragma unroll
          for (int d = 0; d < 3; ++d) atomicAdd(&s_y[3 * ln[s] + d], Y[s][d]);
      } else {
        T xc[4][3], u[12], r[12];
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            xc[n][d] = s_c[3 * ln[n] + d];
            u[3 * n + d] = s_x[3 * ln[n] + d];
          }
        const T en = tet_apply(a.iso, a.w[c0], xc, u, r);
        if (MODE == 1) pap += double(en);
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
          for (int d = 0; d < 3; ++d) atomicAdd(&s_y[3 * ln[n] + d], r[3 * n + d]);
      }
    }
    __syncthreads();
    // 3. write node sums
    for (int i = threadIdx.x; i < nn; i += blockDim.x) {
      const uint32_t f = s_node[i];
      const int64_t gid = f & kNodeMask;
      const uint8_t mk = s_mask[i];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if ((mk >> d) & 1) continue;
        const T v = s_y[3 * i + d];
        if (f & kShared)
          atomicAdd(&a.y[3 * gid + d], v);
        else
          a.y[3 * gid + d] = v;
      }
    }
    __syncthreads();
  }

  if (MODE == 1) {
    const double bsum = block_sum(pap, s_red);
    if (threadIdx.x == 0) a.partials[blockIdx.x] = bsum;
    if (last_block_arrive(a.counter)) {
      double v = 0.0;
      for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) v += __ldcg(&a.partials[i]);
      v = block_sum(v, s_red);
      if (threadIdx.x == 0) {
        PcgScalars* sc = a.sc;
        sc->pap = v;
        if (!(v > 0.0) || !isfinite(v)) {
          sc->breakdown = 1;
          sc->done = 1;
          sc->alpha = 0.0;
        } else {
          sc->alpha = sc->rz / v;
        }
        *a.counter = 0u;
      }
    }
  }
}

}  // namespace pa
