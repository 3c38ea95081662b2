// pa_tiled.cuh -- tile-staged matrix-free K.x, the hot kernel of the solve.
//
// Design (B200): a persistent grid of CTAs (a multiple of the SM count) walks
// the cell tiles.  For each tile the CTA
//   1. stages the tile's nodes (<= 256) in shared memory: coordinates, input
//      vector, Dirichlet mask -- one coalesced pass over the tile's sorted
//      node list, so each node's data is read from HBM/L2 once per tile
//      instead of once per incident cell (about 24 tets share a node);
//   2. evaluates one tet per thread entirely in registers (geometry, strain,
//      stress, SIMP weight, divergence), reading its 4 nodes through 1-byte
//      local ids (4 bytes of connectivity per cell instead of 16);
//   3. accumulates the 12 cell results into shared-memory node sums
//      (shared-memory atomics, no global contention);
//   4. writes each node sum once: a plain store for nodes only this tile
//      touches, one global atomic add per dof for nodes shared with other
//      tiles (~1 atomic per cell instead of the reference's 12,
//      src/Assembly.hpp:1189-1209).
// The PCG variant additionally forms p = D^-1 r + beta p_old while staging
// (the owner tile writes p once) and reduces p.Kp = sum_cells p_e^T K_e p_e
// from the per-cell energies, so the search-direction update and the first
// dot product need no extra pass over the vectors.
#pragma once
#include "pa_cell.cuh"

namespace pa {

constexpr int kApplyThreads = kTileCells;

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

template <typename T, int MODE>
__global__ void __launch_bounds__(kApplyThreads, 2) k_apply_tiled(ApplyArgs<T> a) {
  __shared__ T s_x[kTileNodes * 3];
  __shared__ T s_c[kTileNodes * 3];
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
    const int c0 = a.tv.tile_cell_start[tile], nc = a.tv.tile_cell_start[tile + 1] - c0;
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
    if (threadIdx.x < nc) {
      const int c = c0 + threadIdx.x;
      const uint32_t loc = a.tv.cell_local[c];
      int ln[4];
      T xc[4][3], u[12];
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        ln[n] = (loc >> (8 * n)) & 0xff;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          xc[n][d] = s_c[3 * ln[n] + d];
          u[3 * n + d] = s_x[3 * ln[n] + d];
        }
      }
      T g[4][3], vol, e[6], sig[6], r[12];
      tet_geometry(xc, g, vol);
      tet_strain(g, u, e);
      tet_stress(a.iso, vol * a.w[c], e, sig);
      if (MODE == 1) pap += double(voigt_dot(sig, e));
      tet_divergence(g, sig, r);
#pragma unroll
      for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int d = 0; d < 3; ++d) atomicAdd(&s_y[3 * ln[n] + d], r[3 * n + d]);
    }
    __syncthreads();
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
