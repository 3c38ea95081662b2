// pa_tiled.cuh -- tile-staged, hex-clustered, software-pipelined matrix-free
// K.x: the hot kernel of the solve.
//
// Mesh layout (built once on the host, pa_mesh.cu):
//  * cells are grouped into clusters: a "hex" cluster is six tets that form
//    the six-tet split of one hexahedron around a diagonal (the split every
//    hex-derived tet mesh, e.g. a structured box, has); any other cell is a
//    "single" cluster.  A hex cluster touches 8 nodes for 6 cells, a single
//    one 4 nodes for 1 cell.
//  * clusters are ordered along a Morton curve and packed into tiles of at
//    at most TILE clusters (64, 128 or 256) touching at most 2 TILE nodes; a tile's
//    cells are contiguous in the internal cell order.
//
// Kernel: a persistent grid (a multiple of the SM count) walks the tiles.  For
// each tile the CTA
//  1. has the tile's data already in shared memory: input vectors (gathered
//     through the tile's sorted node list), node coordinates (unless the mesh
//     has the uniform hex geometry table, below), cluster records and penalty
//     weights -- brought in by cp.async while the previous tile was computing
//     (two data buffers; tile headers and node-id lists run further ahead), so
//     the gathers' latency is hidden behind arithmetic;
//  2. forms the input vector (PCG mode: p = D^-1 r + beta p_old, masked; the
//     owner tile writes p once);
//  3. one thread per cluster: reads the cluster's nodes from shared memory into
//     registers once, evaluates its tets (geometry, strain, stress, SIMP
//     weight, divergence) and accumulates 8 node sums in registers.  With the
//     geometry table (GEO: every hex a translate of the first) the per-tet
//     geometry comes from the kernel's parameter block, and the node sums go
//     to shared memory slot by slot without atomics (a slot's nodes are
//     distinct across a tile's hexes); otherwise 24 shared atomics per hex;
//  4. writes each node sum once: a plain store for nodes only this tile
//     touches, a `red.global.add` for nodes shared with other tiles.
// PCG mode also reduces p.Kp = sum_cells p_e^T K_e p_e from the per-tet
// energies; the last CTA to finish turns it into alpha.
#pragma once
#include <algorithm>

#include "pa_cell.cuh"

namespace pa {

// Vectors are stored component-major (SoA): v[d * N + node].
template <typename T>
struct ApplyArgs {
  TileView tv;
  const uint32_t* tile_nodes;  // flagged node ids (mask bits set for the problem's BCs, or none)
  int64_t N;                   // nodes (SoA stride)
  const T* coords;             // 3N, SoA
  const float4* coords4;       // FP32 PCG modes: N x (x, y, z, 0), one 16-byte gather per node (or null)
  const float4* dinv4;         // FP32 PCG modes: D^-1 as N x (x, y, z, 0) (required there)
  const T* w;                  // C, SIMP weight per cell, internal order
  const T* plas;               // null (elastic) or 8 per cell, internal order: J2 tangent record
  Iso<T> iso;
  HexGeo<T> geo;               // uniform hex geometry (filled by the launcher when the mesh has it)
  const T* x;                  // plain: input vector; pcg: p_old
  T* y;                        // output, zero on entry
  // PCG fusion (mode 1)
  const T* r;
  const T* dinv;
  T* p_new;
  PcgScalars* sc;
  double* partials;
  unsigned int* counter;
  // batched PCG (mode 2): one CG per mesh part
  const int32_t* tile_part;  // T
  PartScalars* psc;          // P
  double* pacc;              // P, zero between launches
  int32_t num_parts;
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

// One tet: node contributions r from coordinates xc and input u; returns the
// tet's energy sig:eps (for p.Kp).
template <typename T>
__device__ __forceinline__ T tet_apply(const Iso<T>& iso, T w, const T (&xc)[4][3], const T (&u)[12], T (&r)[12]) {
  T g[4][3], vol, e[6], sig[6];
  tet_geometry(xc, g, vol);
  tet_strain(g, u, e);
  tet_stress(iso, vol * w, e, sig);
  tet_divergence(g, sig, r);
  return voigt_dot(sig, e);
}

// One tet in "relative" form, vertices (v0, va, vb, v3) with edge vectors
// e0 = x_v0 - x_v3, ea, eb and input differences du = u - u_v3.  With
// h0 = ea x eb, h1 = eb x e0, h2 = e0 x ea (the rows of det * J^-1, since J has
// columns e0, ea, eb) and det = e0 . h0, the reference's per-cell chain
// (ComputeGradientWorkset, Strain, LinearStress, ApplyWeighting,
// StressDivergence) becomes
//   eps_u = sum_n h_n (x) du_n        (= det * strain; Voigt, engineering shears)
//   sig'  = s C eps_u,  s = w / (6 |det|)
//   r_n   = h_n . sig'  for n = 0..2,  r_v3 = -(r_0 + r_1 + r_2)
// i.e. vol * w * B^T C B u with vol = |det| / 6, one reciprocal per tet and no
// per-entry scaling of the gradients.  Returns eps_u : sig' = p_e^T K_e p_e.
// h1 and h2 are passed in because a hex cluster shares them between tets.
// With `pl` non-null the stress is the J2 consistent tangent instead of the
// elastic one: pl = {n (6, tensor Voigt), theta1, theta2} of the cell's last
// return mapping and
//   sigma = w [kappa tr(eps) 1 + 2 mu (1 - theta1) dev(eps) - 2 mu (theta2 - theta1) (n : eps) n],
// theta1 = sqrt(6) mu_p dgamma / |eta_trial|, theta2 = 3 mu_p / (3 mu_p + H_iso,p + H_kin,p)
// (zero for an elastic cell).
//
// tet_core is the part after the geometry: rows h0, h1, h2 and the scale
// sc = w / (6 |det|) given.
template <typename T>
__device__ __forceinline__ T tet_core(const Iso<T>& iso, T sc, const T (&h0)[3], const T (&h1)[3], const T (&h2)[3],
                                      const T (&d0)[3], const T (&da)[3], const T (&db)[3], T (&r0)[3], T (&ra)[3],
                                      T (&rb)[3], const T* __restrict__ pl) {
  // eps_u = sum_n h_n (x) du_n
  const T exx = h0[0] * d0[0] + h1[0] * da[0] + h2[0] * db[0];
  const T eyy = h0[1] * d0[1] + h1[1] * da[1] + h2[1] * db[1];
  const T ezz = h0[2] * d0[2] + h1[2] * da[2] + h2[2] * db[2];
  const T gyz = h0[1] * d0[2] + h0[2] * d0[1] + h1[1] * da[2] + h1[2] * da[1] + h2[1] * db[2] + h2[2] * db[1];
  const T gxz = h0[0] * d0[2] + h0[2] * d0[0] + h1[0] * da[2] + h1[2] * da[0] + h2[0] * db[2] + h2[2] * db[0];
  const T gxy = h0[0] * d0[1] + h0[1] * d0[0] + h1[0] * da[1] + h1[1] * da[0] + h2[0] * db[1] + h2[1] * db[0];
  T sxx, syy, szz, syz, sxz, sxy;
  if (pl == nullptr) {
    const T lam = iso.lam * sc, mu = iso.mu * sc, two_mu = mu + mu;
    const T ltr = lam * (exx + eyy + ezz);
    sxx = ltr + two_mu * exx;
    syy = ltr + two_mu * eyy;
    szz = ltr + two_mu * ezz;
    syz = mu * gyz;
    sxz = mu * gxz;
    sxy = mu * gxy;
  } else {
    const T n0 = pl[0], n1 = pl[1], n2 = pl[2], n3 = pl[3], n4 = pl[4], n5 = pl[5], t1 = pl[6], t2 = pl[7];
    const T tr = exx + eyy + ezz, m = tr * (T(1) / T(3));
    const T k = (iso.lam + iso.mu * (T(2) / T(3))) * sc;
    const T ma = iso.mu * (T(1) - t1) * sc, two_ma = ma + ma;
    const T bne = T(2) * iso.mu * (t2 - t1) * sc * (n0 * exx + n1 * eyy + n2 * ezz + n3 * gyz + n4 * gxz + n5 * gxy);
    const T ktr = k * tr;
    sxx = ktr + two_ma * (exx - m) - bne * n0;
    syy = ktr + two_ma * (eyy - m) - bne * n1;
    szz = ktr + two_ma * (ezz - m) - bne * n2;
    syz = ma * gyz - bne * n3;
    sxz = ma * gxz - bne * n4;
    sxy = ma * gxy - bne * n5;
  }
  r0[0] = h0[0] * sxx + h0[1] * sxy + h0[2] * sxz;
  r0[1] = h0[0] * sxy + h0[1] * syy + h0[2] * syz;
  r0[2] = h0[0] * sxz + h0[1] * syz + h0[2] * szz;
  ra[0] = h1[0] * sxx + h1[1] * sxy + h1[2] * sxz;
  ra[1] = h1[0] * sxy + h1[1] * syy + h1[2] * syz;
  ra[2] = h1[0] * sxz + h1[1] * syz + h1[2] * szz;
  rb[0] = h2[0] * sxx + h2[1] * sxy + h2[2] * sxz;
  rb[1] = h2[0] * sxy + h2[1] * syy + h2[2] * syz;
  rb[2] = h2[0] * sxz + h2[1] * syz + h2[2] * szz;
  return sxx * exx + syy * eyy + szz * ezz + syz * gyz + sxz * gxz + sxy * gxy;
}

template <typename T>
__device__ __forceinline__ T tet_rel(const Iso<T>& iso, T w, const T (&e0)[3], const T (&ea)[3], const T (&eb)[3],
                                     const T (&h1)[3], const T (&h2)[3], const T (&d0)[3], const T (&da)[3],
                                     const T (&db)[3], T (&r0)[3], T (&ra)[3], T (&rb)[3],
                                     const T* __restrict__ pl = nullptr) {
  T h0[3];
  h0[0] = ea[1] * eb[2] - ea[2] * eb[1];
  h0[1] = ea[2] * eb[0] - ea[0] * eb[2];
  h0[2] = ea[0] * eb[1] - ea[1] * eb[0];
  const T det = e0[0] * h0[0] + e0[1] * h0[1] + e0[2] * h0[2];
  const T sc = w / (T(6) * fabs(det));
  return tet_core(iso, sc, h0, h1, h2, d0, da, db, r0, ra, rb, pl);
}

template <typename T>
__device__ __forceinline__ void cross3(const T (&a)[3], const T (&b)[3], T (&c)[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Ring of a hex cluster: tet k has vertices (slot 0, ring(k), ring(k+1), slot 7),
// the same vertex sets as hex_slot(k, .).
__host__ __device__ constexpr int hex_ring(int k) {
  constexpr int r[7] = {3, 2, 6, 4, 5, 1, 3};
  return r[k];
}

// Fire-and-forget global reduction (no returned value, so nothing waits on
// it); the address is converted to the global window explicitly.
__device__ __forceinline__ void red_add_global(float* p, float v) {
  asm volatile("red.global.add.f32 [%0], %1;\n" ::"l"(__cvta_generic_to_global(p)), "f"(v) : "memory");
}
__device__ __forceinline__ void red_add_global(double* p, double v) {
  asm volatile("red.global.add.f64 [%0], %1;\n" ::"l"(__cvta_generic_to_global(p)), "d"(v) : "memory");
}

// ---------------------------------------------------------------- cp.async --
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Packed node records in shared memory: coordinates + first input
// component in one 16-byte (FP32) / two 16-byte (FP64) loads, the other two
// input components in one 8- / 16-byte load.
template <typename T>
struct alignas(16) Node4 {
  T x, y, z, u0;
};
template <typename T>
struct alignas(2 * sizeof(T)) Node2 {
  T u1, u2;
};

// Shared-memory layout of one CTA (dynamic shared memory); TILE clusters
// (threads) and up to 2 * TILE nodes per tile.  GEO (uniform hex geometry):
// xc holds the input vector (u0, u1, u2, 0) and uu is not used.
template <typename T, int MODE, int TILE, bool GEO = false>
struct TileSmem {
  static constexpr int kTileNodes = 2 * TILE;
  static constexpr int kRawBufs = MODE >= 1 ? 2 : 1;
  // node records: gathered by cp.async (two buffers), except in the GEO PCG
  // modes, where the formation step writes them (one buffer)
  static constexpr int kXcBufs = (GEO && MODE >= 1) ? 1 : 2;
  Node4<T> xc[kXcBufs][kTileNodes];       // coordinates + input (component 0)
  Node2<T> uu[2][GEO ? 1 : kTileNodes];   // input components 1, 2
  // PCG modes: r, D^-1, p_old gathered for the tile.  FP32 keeps D^-1 as one
  // 16-byte record per node (dv) and only r and p_old in raw.
  static constexpr bool kPackedD = sizeof(T) == 4 && MODE >= 1;
  static constexpr int kRawRows = kPackedD ? 6 : 9;
  static constexpr int kRowD = 3, kRowP = kPackedD ? 3 : 6;
  T raw[kRawBufs][kRawRows][kTileNodes];
  float4 dv[kPackedD ? 2 : 1][kPackedD ? kTileNodes : 1];
  // node sums of the current tile: the PCG modes keep them in the r rows of
  // the tile's gather buffer (raw[b][0..2], dead once the input is formed)
  T y[MODE >= 1 ? 1 : 3][MODE >= 1 ? 1 : kTileNodes];
  T w[2][6 * TILE];                       // penalty weights of the tile's cells
  // tile headers and node ids: three buffers, fetched two tiles ahead (the
  // data gathers of tile k+1 read the ids of tile k+1 while tile k still uses
  // its own); cluster records travel with the data (two buffers)
  uint4 rec[2][TILE];                     // cluster node ids
  uint32_t ids[3][kTileNodes];            // flagged node ids
  int32_t meta[3][8];                     // n0, nn, k0, nk, nhex, cell0, ncell
  double red[32];
};

// Row d of the current tile's node sums (data buffer b).
template <typename T, int MODE, int TILE, bool GEO>
__device__ __forceinline__ T* node_sums(TileSmem<T, MODE, TILE, GEO>& S, int b, int d) {
  if constexpr (MODE >= 1)
    return S.raw[b][d];
  else
    return S.y[d];
}

template <typename T, int MODE, int TILE, bool GEO>
constexpr size_t tile_smem_bytes() {
  return sizeof(TileSmem<T, MODE, TILE, GEO>);
}

// Header of one tile (node, cluster and cell ranges), loaded into registers
// one tile before its ids are fetched so that the loads' latency is hidden.
struct TileHead {
  int n0, nn, k0, nk, nhex, c0, nc;
};

__device__ __forceinline__ TileHead load_head(const TileView& tv, int tile) {
  TileHead h;
  h.n0 = __ldg(&tv.tile_node_start[tile]);
  h.nn = __ldg(&tv.tile_node_start[tile + 1]) - h.n0;
  h.k0 = __ldg(&tv.tile_cluster_start[tile]);
  h.nk = __ldg(&tv.tile_cluster_start[tile + 1]) - h.k0;
  h.nhex = __ldg(&tv.tile_hex_count[tile]);
  h.c0 = __ldg(&tv.tile_cell_start[tile]);
  h.nc = __ldg(&tv.tile_cell_start[tile + 1]) - h.c0;
  return h;
}

// Issue the loads of one tile's node ids and cluster records into id buffer ib.
template <typename T, int MODE, int TILE, bool GEO>
__device__ __forceinline__ void prefetch_ids(const ApplyArgs<T>& a, TileSmem<T, MODE, TILE, GEO>& S,
                                             const TileHead& h, int ib) {
  if (threadIdx.x == 0) {
    S.meta[ib][0] = h.n0;
    S.meta[ib][1] = h.nn;
    S.meta[ib][2] = h.k0;
    S.meta[ib][3] = h.nk;
    S.meta[ib][4] = h.nhex;
    S.meta[ib][5] = h.c0;
    S.meta[ib][6] = h.nc;
  }
  for (int i = threadIdx.x; i < h.nn; i += blockDim.x) cp_async<4>(&S.ids[ib][i], &a.tile_nodes[h.n0 + i]);
  cp_async_commit();
}

// Issue the gathers of the node data and weights of the tile whose ids sit in buffer b.
// GEO (uniform hex geometry): no coordinates; the node record holds the
// input vector (u0, u1, u2, 0).
template <typename T, int MODE, int TILE, bool GEO>
__device__ __forceinline__ void prefetch_data(const ApplyArgs<T>& a, TileSmem<T, MODE, TILE, GEO>& S, int ib,
                                              int b) {
  const int nn = S.meta[ib][1];
  const int64_t N = a.N;
  for (int i = threadIdx.x; i < nn; i += blockDim.x) {
    const int64_t g = int64_t(S.ids[ib][i] & kNodeIdMask);
    if constexpr (!GEO) {
      bool packed = false;
      if constexpr (sizeof(T) == 4 && MODE >= 1) {
        // (x, y, z, 0) in one copy; the fourth slot is the input component 0,
        // which the PCG modes write after this copy has landed
        if (a.coords4) {
          cp_async<16>(&S.xc[b][i], &a.coords4[g]);
          packed = true;
        }
      }
      if (!packed) {
        cp_async<sizeof(T)>(&S.xc[b][i].x, &a.coords[g]);
        cp_async<sizeof(T)>(&S.xc[b][i].y, &a.coords[N + g]);
        cp_async<sizeof(T)>(&S.xc[b][i].z, &a.coords[2 * N + g]);
      }
    }
    if constexpr (MODE == 0 && GEO) {
      cp_async<sizeof(T)>(&S.xc[b][i].x, &a.x[g]);
      cp_async<sizeof(T)>(&S.xc[b][i].y, &a.x[N + g]);
      cp_async<sizeof(T)>(&S.xc[b][i].z, &a.x[2 * N + g]);
    } else if constexpr (MODE == 0) {
      cp_async<sizeof(T)>(&S.xc[b][i].u0, &a.x[g]);
      cp_async<sizeof(T)>(&S.uu[b][i].u1, &a.x[N + g]);
      cp_async<sizeof(T)>(&S.uu[b][i].u2, &a.x[2 * N + g]);
    } else {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        cp_async<sizeof(T)>(&S.raw[b][d][i], &a.r[d * N + g]);
        if constexpr (!TileSmem<T, MODE, TILE>::kPackedD)
          cp_async<sizeof(T)>(&S.raw[b][TileSmem<T, MODE, TILE>::kRowD + d][i], &a.dinv[d * N + g]);
        cp_async<sizeof(T)>(&S.raw[b][TileSmem<T, MODE, TILE>::kRowP + d][i], &a.x[d * N + g]);
      }
      if constexpr (TileSmem<T, MODE, TILE>::kPackedD) cp_async<16>(&S.dv[b][i], &a.dinv4[g]);
    }
  }
  const int c0 = S.meta[ib][5], nc = S.meta[ib][6];
  for (int i = threadIdx.x; i < nc; i += blockDim.x) cp_async<sizeof(T)>(&S.w[b][i], &a.w[c0 + i]);
  const int k0 = S.meta[ib][2], nk = S.meta[ib][3];
  for (int i = threadIdx.x; i < nk; i += blockDim.x) cp_async<16>(&S.rec[b][i], &a.tv.cluster_nodes[k0 + i]);
  cp_async_commit();
}

// FP32 instances ask for 640 resident threads per SM (<= 96 registers, 20
// warps), the GEO PCG instances of 256-cluster tiles for three CTAs (768
// threads, <= 85 registers; their shared memory fits three); FP64 instances
// are register-bound at one or two CTAs.
template <typename T, int MODE, int TILE, bool GEO>
constexpr int apply_min_blocks() {
  return sizeof(T) != 4 ? 1 : (GEO && MODE >= 1 && TILE == 256) ? 3 : 640 / TILE;
}

template <typename T, int MODE, int TILE, bool GEO>
__global__ void __launch_bounds__(TILE, (apply_min_blocks<T, MODE, TILE, GEO>())) k_apply_tiled(ApplyArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileSmem<T, MODE, TILE, GEO>& S = *reinterpret_cast<TileSmem<T, MODE, TILE, GEO>*>(smem_raw);

  T beta = T(0);
  if (MODE >= 1) {
    if (a.sc->done) return;
    beta = T(a.sc->beta);
  }
  double pap = 0.0;
  const int stride = gridDim.x;
  int tile = blockIdx.x;

  // Pipeline (tile k of this CTA at the top of iteration k): data of tile k
  // and ids of tile k+1 have landed; the iteration issues the data gathers of
  // tile k+1 and the id loads of tile k+2, and loads the header of tile k+3
  // into registers, then computes tile k.  Id buffers rotate over three
  // slots, data buffers over two.
  const int T_ = a.tv.num_tiles;
  TileHead head_next{};  // header of tile k+2 at the top of iteration k
  if (tile < T_) {
    prefetch_ids(a, S, load_head(a.tv, tile), 0);
    cp_async_wait_all();
    __syncthreads();
    prefetch_data<T, MODE, TILE, GEO>(a, S, 0, 0);
    if (tile + stride < T_) prefetch_ids(a, S, load_head(a.tv, tile + stride), 1);
    if (tile + 2 * stride < T_) head_next = load_head(a.tv, tile + 2 * stride);
  }

  int ib = 0;  // id buffer of tile k (k mod 3)
  for (int k = 0; tile < T_; ++k, tile += stride, ib = ib == 2 ? 0 : ib + 1) {
    const int b = k & 1;
    const int xb = TileSmem<T, MODE, TILE, GEO>::kXcBufs == 1 ? 0 : b;  // node-record buffer
    const int ib1 = ib == 2 ? 0 : ib + 1, ib2 = ib1 == 2 ? 0 : ib1 + 1;
    cp_async_wait_all();  // data of this tile, ids of the next
    __syncthreads();
    if (tile + stride < T_) prefetch_data<T, MODE, TILE, GEO>(a, S, ib1, b ^ 1);
    if (tile + 2 * stride < T_) {
      // slot ib2 held the ids of tile k-1, finished before the barrier above
      prefetch_ids(a, S, head_next, ib2);
      if (tile + 3 * stride < T_) head_next = load_head(a.tv, tile + 3 * stride);
    }
    // batched mode: this tile's part, its beta, and whether it has converged
    int part = 0;
    bool skip = false;
    if constexpr (MODE == 2) {
      part = a.tile_part[tile];
      skip = a.psc[part].done != 0;
      beta = T(a.psc[part].beta);
      pap = 0.0;
      if (skip) {
        // a stopped part keeps its direction: p_new = p_old on its owned nodes,
        // so both p buffers stay current if the part resumes
        const int nn = S.meta[ib][1];
        for (int i = threadIdx.x; i < nn; i += blockDim.x) {
          const uint32_t f = S.ids[ib][i];
          const int64_t g = int64_t(f & kNodeIdMask);
          if ((f & kOwner) && g < a.N) {
#pragma unroll
            for (int d = 0; d < 3; ++d) a.p_new[d * a.N + g] = S.raw[b][TileSmem<T, MODE, TILE>::kRowP + d][i];
          }
        }
      }
    }
    if (!skip) {

    // 2. input vector of this tile; zero its sums
    const int nn = S.meta[ib][1];
    for (int i = threadIdx.x; i < nn; i += blockDim.x) {
      const uint32_t f = S.ids[ib][i];
      const uint32_t mk = (f >> kMaskShift) & 7u;
      if constexpr (MODE == 0 && GEO) {
        if (mk) {
          if (mk & 1u) S.xc[xb][i].x = T(0);
          if (mk & 2u) S.xc[xb][i].y = T(0);
          if (mk & 4u) S.xc[xb][i].z = T(0);
        }
      } else if constexpr (MODE == 0) {
        if (mk) {
          if (mk & 1u) S.xc[xb][i].u0 = T(0);
          if (mk & 2u) S.uu[b][i].u1 = T(0);
          if (mk & 4u) S.uu[b][i].u2 = T(0);
        }
      } else {
        T v[3], dinv[3];
        if constexpr (TileSmem<T, MODE, TILE>::kPackedD) {
          const float4 q = S.dv[b][i];
          dinv[0] = q.x;
          dinv[1] = q.y;
          dinv[2] = q.z;
        } else {
#pragma unroll
          for (int d = 0; d < 3; ++d) dinv[d] = S.raw[b][TileSmem<T, MODE, TILE>::kRowD + d][i];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d)
          v[d] = (mk >> d) & 1 ? T(0)
                               : dinv[d] * S.raw[b][d][i] + beta * S.raw[b][TileSmem<T, MODE, TILE>::kRowP + d][i];
        if constexpr (GEO) {
          S.xc[xb][i] = Node4<T>{v[0], v[1], v[2], T(0)};
        } else {
          S.xc[xb][i].u0 = v[0];
          S.uu[b][i].u1 = v[1];
          S.uu[b][i].u2 = v[2];
        }
        if (f & kOwner) {
          const int64_t g = int64_t(f & kNodeIdMask);
#pragma unroll
          for (int d = 0; d < 3; ++d) a.p_new[d * a.N + g] = v[d];
        }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) node_sums(S, b, d)[i] = T(0);  // after this node's r was read
    }
    __syncthreads();

    // 3. one cluster per thread
    const int t = threadIdx.x;
    const int nk = S.meta[ib][3], nhex = S.meta[ib][4];
    T Y[7][3], Y7[3];  // node contributions of this thread's hex (slot order)
    int ln[8];
    const bool act = t < nk;
    if (act) {
      const uint4 q = S.rec[b][t];
      ln[0] = int(q.x & 0xffff);
      ln[1] = int(q.x >> 16);
      ln[2] = int(q.y & 0xffff);
      ln[3] = int(q.y >> 16);
      ln[4] = int(q.z & 0xffff);
      ln[5] = int(q.z >> 16);
      ln[6] = int(q.w & 0xffff);
      ln[7] = int(q.w >> 16);
      if (t < nhex) {
        const T* wv = &S.w[b][6 * t];
        T D[7][3];
        if constexpr (GEO) {
          // input differences relative to slot 7; geometry from the table
          const Node4<T> q7 = S.xc[xb][ln[7]];
#pragma unroll
          for (int s = 0; s < 7; ++s) {
            const Node4<T> q4 = S.xc[xb][ln[s]];
            D[s][0] = q4.x - q7.x;
            D[s][1] = q4.y - q7.y;
            D[s][2] = q4.z - q7.z;
#pragma unroll
            for (int d = 0; d < 3; ++d) Y[s][d] = T(0);
          }
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            const int sa = hex_ring(k), sb = hex_ring(k + 1);
            const T h0[3] = {a.geo.h[k][0], a.geo.h[k][1], a.geo.h[k][2]};
            const T h1[3] = {a.geo.h[k][3], a.geo.h[k][4], a.geo.h[k][5]};
            const T h2[3] = {a.geo.h[k][6], a.geo.h[k][7], a.geo.h[k][8]};
            T r0[3], ra[3], rb[3];
            const T* pl = a.plas ? a.plas + 8 * (int64_t(S.meta[ib][5]) + 6 * t + k) : nullptr;
            const T en = tet_core(a.iso, wv[k] * a.geo.s[k], h0, h1, h2, D[0], D[sa], D[sb], r0, ra, rb, pl);
            if (MODE >= 1) pap += double(en);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              Y[0][d] += r0[d];
              Y[sa][d] += ra[d];
              Y[sb][d] += rb[d];
            }
          }
        } else {
        // edge vectors and input differences relative to slot 7 (the diagonal end)
        T E[7][3];
        {
          const Node4<T> q7 = S.xc[xb][ln[7]];
          const Node2<T> p7 = S.uu[b][ln[7]];
#pragma unroll
          for (int s = 0; s < 7; ++s) {
            const Node4<T> q4 = S.xc[xb][ln[s]];
            const Node2<T> q2 = S.uu[b][ln[s]];
            E[s][0] = q4.x - q7.x;
            E[s][1] = q4.y - q7.y;
            E[s][2] = q4.z - q7.z;
            D[s][0] = q4.u0 - q7.u0;
            D[s][1] = q2.u1 - p7.u1;
            D[s][2] = q2.u2 - p7.u2;
#pragma unroll
            for (int d = 0; d < 3; ++d) Y[s][d] = T(0);
          }
        }
        // C[s] = E[0] x E[s] for the ring slots, shared by the two tets at s
        T Cx[7][3];
#pragma unroll
        for (int k = 0; k < 6; ++k) cross3(E[0], E[hex_ring(k)], Cx[hex_ring(k)]);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          const int sa = hex_ring(k), sb = hex_ring(k + 1);
          T h1[3], r0[3], ra[3], rb[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) h1[d] = -Cx[sb][d];
          const T* pl = a.plas ? a.plas + 8 * (int64_t(S.meta[ib][5]) + 6 * t + k) : nullptr;
          const T en = tet_rel(a.iso, wv[k], E[0], E[sa], E[sb], h1, Cx[sa], D[0], D[sa], D[sb], r0, ra, rb, pl);
          if (MODE >= 1) pap += double(en);
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            Y[0][d] += r0[d];
            Y[sa][d] += ra[d];
            Y[sb][d] += rb[d];
          }
        }
        }  // !GEO
        // slot 7 closes each tet's partition of unity: Y7 = -(Y0 + ... + Y6)
#pragma unroll
        for (int d = 0; d < 3; ++d) Y7[d] = T(0);
#pragma unroll
        for (int s = 0; s < 7; ++s)
#pragma unroll
          for (int d = 0; d < 3; ++d) Y7[d] -= Y[s][d];
        if constexpr (!GEO) {
#pragma unroll
          for (int s = 0; s < 7; ++s)
#pragma unroll
            for (int d = 0; d < 3; ++d) atomicAdd(&node_sums(S, b, d)[ln[s]], Y[s][d]);
#pragma unroll
          for (int d = 0; d < 3; ++d) atomicAdd(&node_sums(S, b, d)[ln[7]], Y7[d]);
        }
      } else if constexpr (!GEO) {
        // single tets follow the hexes: cell index = 6 * nhex + (t - nhex)
        // (a mesh with uniform hex geometry has none)
        T e[3][3], du[3][3], h1[3], h2[3], r[3][3];
        const Node4<T> q3 = S.xc[xb][ln[3]];
        const Node2<T> p3 = S.uu[b][ln[3]];
#pragma unroll
        for (int n = 0; n < 3; ++n) {
          const Node4<T> q4 = S.xc[xb][ln[n]];
          const Node2<T> q2 = S.uu[b][ln[n]];
          e[n][0] = q4.x - q3.x;
          e[n][1] = q4.y - q3.y;
          e[n][2] = q4.z - q3.z;
          du[n][0] = q4.u0 - q3.u0;
          du[n][1] = q2.u1 - p3.u1;
          du[n][2] = q2.u2 - p3.u2;
        }
        cross3(e[2], e[0], h1);
        cross3(e[0], e[1], h2);
        const int cl = 6 * nhex + (t - nhex);
        const T* pl = a.plas ? a.plas + 8 * (int64_t(S.meta[ib][5]) + cl) : nullptr;
        const T en = tet_rel(a.iso, S.w[b][cl], e[0], e[1], e[2], h1, h2, du[0], du[1], du[2], r[0], r[1], r[2], pl);
        if (MODE >= 1) pap += double(en);
#pragma unroll
        for (int n = 0; n < 3; ++n)
#pragma unroll
          for (int d = 0; d < 3; ++d) atomicAdd(&node_sums(S, b, d)[ln[n]], r[n][d]);
#pragma unroll
        for (int d = 0; d < 3; ++d) atomicAdd(&node_sums(S, b, d)[ln[3]], -(r[0][d] + r[1][d] + r[2][d]));
      }
    }
    if constexpr (GEO) {
      // Conflict-free accumulation: two hexes of a tile never share a node in
      // the same slot (the host checks this per tile before it enables the
      // table), so slot by slot the read-add-writes of all threads hit
      // distinct nodes; a barrier separates the slots.  This replaces 24
      // shared float atomics (compare-and-swap loops) per hex.
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        if (act) {
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            T* y = node_sums(S, b, d);
            y[ln[s]] += s < 7 ? Y[s][d] : Y7[d];
          }
        }
        __syncthreads();
      }
    } else {
      __syncthreads();
    }

    // 4. write node sums
    for (int i = threadIdx.x; i < nn; i += blockDim.x) {
      const uint32_t f = S.ids[ib][i];
      const int64_t gid = f & kNodeIdMask;
      const uint32_t mk = (f >> kMaskShift) & 7u;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if ((mk >> d) & 1) continue;
        const T v = node_sums(S, b, d)[i];
        if (f & kShared)
          red_add_global(&a.y[d * a.N + gid], v);
        else
          a.y[d * a.N + gid] = v;
      }
    }
    __syncthreads();
    if constexpr (MODE == 2) {
      // p.Kp of this tile into its part
      const double v = block_sum(pap, S.red);
      if (threadIdx.x == 0) atomicAdd(&a.pacc[part], v);
    }
    }  // !skip
    // a skipped tile read buffers ib and b above; every thread must be done
    // with them before the next iteration refills them (the non-skipped path
    // synchronised after its write-back)
    if (skip) __syncthreads();
  }
  cp_async_wait_all();

  if constexpr (MODE == 2) {
    if (last_block_arrive(a.counter)) {
      for (int p = threadIdx.x; p < a.num_parts; p += blockDim.x) {
        PartScalars& ps = a.psc[p];
        const double v = __ldcg(&a.pacc[p]);
        a.pacc[p] = 0.0;
        if (ps.done) continue;
        ps.pap = v;
        if (!(v > 0.0) || !isfinite(v)) {
          ps.breakdown = 1;
          ps.done = 1;
          ps.alpha = 0.0;
        } else {
          ps.alpha = ps.rz / v;
        }
      }
      if (threadIdx.x == 0) *a.counter = 0u;
    }
  }

  if constexpr (MODE == 1) {
    const double bsum = block_sum(pap, S.red);
    if (threadIdx.x == 0) a.partials[blockIdx.x] = bsum;
    if (last_block_arrive(a.counter)) {
      double v = 0.0;
      for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) v += __ldcg(&a.partials[i]);
      v = block_sum(v, S.red);
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

// Configure dynamic shared memory of one instance; returns the persistent
// grid size (resident CTAs per SM x SMs, capped by the tile count).
template <typename T, int MODE, int TILE, bool GEO>
int apply_grid_for(int num_tiles) {
  const size_t smem = tile_smem_bytes<T, MODE, TILE, GEO>();
  PA_CUDA(cudaFuncSetAttribute(k_apply_tiled<T, MODE, TILE, GEO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(smem)));
  int blocks = 0;
  PA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_apply_tiled<T, MODE, TILE, GEO>, TILE, smem));
  const int grid = std::min(std::max(1, blocks) * num_sms(), num_tiles);
  return std::max(grid, 1);
}

// The FP32 instances take the uniform-geometry form when the mesh has it; the
// FP64 ones only when every hex matches the table to rounding level (their
// parity with the oracle's per-cell FP64 arithmetic is 1e-10).
constexpr double kGeoDevFp64 = 1e-12;
template <typename T>
bool use_uniform_geometry(const Mesh& m) {
  return m.uniform_hex && (sizeof(T) == 4 || m.hex_geo_dev <= kGeoDevFp64);
}

template <typename T, int MODE, bool GEO>
int apply_kernel_setup_geo(const Mesh& m) {
  switch (m.tile_clusters) {
    case 64: return apply_grid_for<T, MODE, 64, GEO>(int(m.T));
    case 128: return apply_grid_for<T, MODE, 128, GEO>(int(m.T));
    default: return apply_grid_for<T, MODE, 256, GEO>(int(m.T));
  }
}

template <typename T, int MODE>
int apply_kernel_setup(const Mesh& m) {
  if (use_uniform_geometry<T>(m)) return apply_kernel_setup_geo<T, MODE, true>(m);
  return apply_kernel_setup_geo<T, MODE, false>(m);
}

template <typename T, int MODE, bool GEO>
void launch_apply_geo(const Mesh& m, int grid, cudaStream_t s, const ApplyArgs<T>& a) {
  switch (m.tile_clusters) {
    case 64: k_apply_tiled<T, MODE, 64, GEO><<<grid, 64, tile_smem_bytes<T, MODE, 64, GEO>(), s>>>(a); break;
    case 128: k_apply_tiled<T, MODE, 128, GEO><<<grid, 128, tile_smem_bytes<T, MODE, 128, GEO>(), s>>>(a); break;
    default: k_apply_tiled<T, MODE, 256, GEO><<<grid, 256, tile_smem_bytes<T, MODE, 256, GEO>(), s>>>(a); break;
  }
}

// Launch (also inside stream capture) the instance matching the mesh's tile
// size and geometry; the grid must come from apply_kernel_setup<T, MODE> of
// the same mesh state.
template <typename T, int MODE>
void launch_apply_kernel(const Mesh& m, int grid, cudaStream_t s, const ApplyArgs<T>& a) {
  if (sizeof(T) == 4 && MODE >= 1 && a.dinv4 == nullptr)
    throw Error(PA_ERR_INVALID_ARG, "FP32 fused apply without the packed D^-1");
  if (use_uniform_geometry<T>(m)) {
    ApplyArgs<T> g = a;
    if constexpr (sizeof(T) == 4)
      g.geo = m.geo32;
    else
      g.geo = m.geo64;
    launch_apply_geo<T, MODE, true>(m, grid, s, g);
    return;
  }
  launch_apply_geo<T, MODE, false>(m, grid, s, a);
}

}  // namespace pa
