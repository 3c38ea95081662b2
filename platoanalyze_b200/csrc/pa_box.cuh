// pa_box.cuh -- matrix-free K x on structured boxes (the hexes of
// mesh_make_box, each split into the six tets of one corner-to-corner
// diagonal), with the node arithmetic of the lattice instead of connectivity.
//
// Operator.  A box of nx x ny x nz equal hexes (edge lengths hx, hy, hz),
// nodes numbered v = i + px (j + py k) (px = nx + 1, ...), vectors component-
// major (x[d N + v]).  Hex h = i + nx (j + ny k) holds tets t = 0..5, each the
// path from corner (0,0,0) to (1,1,1) along the axes in the order
//   t0 (y,x,z)  t1 (y,z,x)  t2 (z,y,x)  t3 (z,x,y)  t4 (x,z,y)  t5 (x,y,z)
// (the split of mesh_make_box; corner c = a + 2b + 4c for offsets (a,b,c)).
// For a path tet with vertices v0 = 0, v1, v2, v3 = 7 the barycentric
// gradients are -e1/h1, e1/h1 - e2/h2, e2/h2 - e3/h3, e3/h3 (e_m the m-th
// axis of the path), so its displacement gradient has column pi_m equal to
// (u[v_m] - u[v_m-1]) / h_m and its nodal forces are the edge fluxes
// S_m = w vol sigma[:, pi_m] / h_m: f[v_m-1] -= S_m, f[v_m] += S_m.  Stress
// sigma = lam tr(G) I + mu (G + G^T) (src/LinearStress.hpp:61-77 with the
// engineering shears of src/Strain.hpp:56-94), vol = hx hy hz / 6 and w the
// tet's SIMP weight (src/Simp.hpp:130-134).  This is the cell chain of
// src/elliptic/ElastostaticResidual.hpp:147-214 for these tets, written in
// edge differences: no geometry arithmetic, no connectivity, no coordinates.
//
// Kernel.  A CTA owns a brick of 31 x 7 nodes in x and y and walks a chunk of
// kz node planes along z.  Warp w, lane L computes hex (i0-1+L, j0-1+w, k) for
// each hex layer k (the hexes around the brick's nodes, one halo layer on the
// low side of every axis); the plane-k forces of a hex are its bottom corners
// plus the top corners of the hex below, carried in registers; the four hexes
// around a node in the plane are combined by a warp shuffle along x and one
// shared-memory exchange between warps along y.  Every node's sum is formed
// by exactly one thread, in a fixed order: no atomics, deterministic, and
// the epilogue sees the final y of its node, so vector updates (Chebyshev
// steps, residuals, CG dot products) fuse into the same kernel.  The input
// vector is formed once per node and plane into shared memory (three plane
// buffers, one barrier per hex layer), its global loads issued a layer
// before they are needed.
#pragma once

#include <cstdint>

#include "pa_internal.cuh"

namespace pa {

constexpr int kBoxX = 31, kBoxY = 7;                 // owned nodes of a CTA along x and y
constexpr int kBoxCols = kBoxX + 2, kBoxRows = kBoxY + 2;
constexpr int kBoxPlane = kBoxCols * kBoxRows;       // formed input nodes per plane (33 x 9)
constexpr int kBoxThreads = 256;                     // 8 warps = 8 hex rows x 32 hex columns

struct BoxDims {
  int nx, ny, nz, px, py, pz;
  int64_t N, H;
};

// lam, mu: Lame parameters times the tet volume (and times 1/h^2 when the
// hexes are cubes, ih unused); ih: 1 / edge length per axis.
template <typename T>
struct BoxGeo {
  T lam, mu;
  T ih[3];
};

// SIMP weights: one per hex (WM = 0) or one per tet, tet-major (WM = 1:
// w[t H + h]).
template <typename T, int WM>
struct BoxW {
  const T* w;
  int64_t H;
};

// Deterministic grid reduction: one partial per CTA, the last CTA to arrive
// sums them in order and calls Out::finish.
struct BoxRed {
  double* partials;
  unsigned int* counter;
};

// Sum over the CTA (valid in thread 0); every thread must call it.
__device__ __forceinline__ double block_sum_box(double v, double* smem /*>= 32*/) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    v = lane < int(blockDim.x >> 5) ? smem[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// One path tet: forces of corner displacements u into f.
template <int P1, int P2, int P3, bool CUBE, typename T>
__device__ __forceinline__ void box_tet(const T (&u)[8][3], T lam, T mu, const T (&ih)[3], T (&f)[8][3]) {
  constexpr int v1 = 1 << P1, v2 = v1 | (1 << P2);
  T G[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    G[c][P1] = u[v1][c] - u[0][c];
    G[c][P2] = u[v2][c] - u[v1][c];
    G[c][P3] = u[7][c] - u[v2][c];
    if constexpr (!CUBE) {
      G[c][P1] *= ih[P1];
      G[c][P2] *= ih[P2];
      G[c][P3] *= ih[P3];
    }
  }
  const T lt = lam * (G[0][0] + G[1][1] + G[2][2]);
  const T m2 = mu + mu;
  T s[3][3];
  s[0][0] = fma(m2, G[0][0], lt);
  s[1][1] = fma(m2, G[1][1], lt);
  s[2][2] = fma(m2, G[2][2], lt);
  s[0][1] = s[1][0] = mu * (G[0][1] + G[1][0]);
  s[0][2] = s[2][0] = mu * (G[0][2] + G[2][0]);
  s[1][2] = s[2][1] = mu * (G[1][2] + G[2][1]);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    T S1 = s[c][P1], S2 = s[c][P2], S3 = s[c][P3];
    if constexpr (!CUBE) {
      S1 *= ih[P1];
      S2 *= ih[P2];
      S3 *= ih[P3];
    }
    f[0][c] -= S1;
    f[v1][c] += S1 - S2;
    f[v2][c] += S2 - S3;
    f[7][c] += S3;
  }
}

// Forces of one hex (six tets) for corner displacements u; w: the hex's
// weight (WM = 0) or its six tet weights.
template <bool CUBE, int WM, typename T>
__device__ __forceinline__ void box_hex(const T (&u)[8][3], const T (&w)[WM ? 6 : 1], const BoxGeo<T>& g,
                                        T (&f)[8][3]) {
#pragma unroll
  for (int c = 0; c < 8; ++c) f[c][0] = f[c][1] = f[c][2] = T(0);
  auto W = [&](int t) { return WM ? w[WM ? t : 0] : w[0]; };
  box_tet<1, 0, 2, CUBE>(u, W(0) * g.lam, W(0) * g.mu, g.ih, f);
  box_tet<1, 2, 0, CUBE>(u, W(1) * g.lam, W(1) * g.mu, g.ih, f);
  box_tet<2, 1, 0, CUBE>(u, W(2) * g.lam, W(2) * g.mu, g.ih, f);
  box_tet<2, 0, 1, CUBE>(u, W(3) * g.lam, W(3) * g.mu, g.ih, f);
  box_tet<0, 2, 1, CUBE>(u, W(4) * g.lam, W(4) * g.mu, g.ih, f);
  box_tet<0, 1, 2, CUBE>(u, W(5) * g.lam, W(5) * g.mu, g.ih, f);
}

// y = K x on the box with a fused input former and epilogue.  Both are split
// into a load part (global loads into registers, issued a hex layer before
// the values are needed) and a compute part:
//   In:  struct Raw;
//        __device__ Raw load(int64_t v, bool owned) const;
//        __device__ void make(const Raw&, int64_t v, int i, int j, int k, bool owned, T (&x)[3]) const;
//        the input vector at node v = (i, j, k), once per CTA, node and plane
//        (`owned`: this CTA owns v, for side outputs);
//   Out: struct Pre;
//        __device__ Pre load(int64_t v) const;
//        __device__ double store(const Pre&, int64_t v, int i, int j, int k, const T (&y)[3]) const;
//        consumes (K x)_v at an owned node and returns its part of the
//        reduction; static constexpr bool kReduce; __device__ void finish(double) const.
// Node plane p is formed three hex layers ahead into buffer (p - k0 + 1) % 3.
// Grid: (ceil(px / 31), ceil(py / 7), ceil(pz / kz)) CTAs of 256 threads.
template <typename T, int WM, bool CUBE, class In, class Out>
__global__ void __launch_bounds__(kBoxThreads) k_box(BoxDims d, BoxGeo<T> g, BoxW<T, WM> bw, int kz, In in,
                                                     Out out, BoxRed red) {
  __shared__ T xs[3][kBoxPlane][3];
  __shared__ T yb[2][8][32][3];
  __shared__ double s_red[32];
  const int L = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int i0 = blockIdx.x * kBoxX, j0 = blockIdx.y * kBoxY, k0 = blockIdx.z * kz;
  const int k1 = min(k0 + kz, d.pz);  // node planes [k0, k1)
  const int i = i0 - 1 + L, j = j0 - 1 + wp;
  const bool hex_ij = i >= 0 && i < d.nx && j >= 0 && j < d.ny;
  const bool own_ij = L >= 1 && wp >= 1 && i < d.px && j < d.py;

  // the (at most two) plane entries this thread forms: e = tid, tid + 256
  constexpr int kSlots = (kBoxPlane + kBoxThreads - 1) / kBoxThreads;
  int fi[kSlots], fj[kSlots];
  bool fin[kSlots], fown[kSlots];
#pragma unroll
  for (int q = 0; q < kSlots; ++q) {
    const int e = threadIdx.x + q * kBoxThreads;
    const int r = e / kBoxCols, c = e - r * kBoxCols;
    fi[q] = i0 - 1 + c;
    fj[q] = j0 - 1 + r;
    fin[q] = e < kBoxPlane && fi[q] >= 0 && fi[q] < d.px && fj[q] >= 0 && fj[q] < d.py;
    fown[q] = e < kBoxPlane && c >= 1 && c <= kBoxX && r >= 1 && r <= kBoxY;
  }
  auto node_of = [&](int ni, int nj, int nk) { return int64_t(ni) + int64_t(d.px) * (nj + int64_t(d.py) * nk); };
  typename In::Raw raw[kSlots];
  // issue the loads of node plane p
  auto form_load = [&](int p) {
#pragma unroll
    for (int q = 0; q < kSlots; ++q)
      if (fin[q] && p >= 0 && p < d.pz) raw[q] = in.load(node_of(fi[q], fj[q], p), fown[q] && p >= k0 && p < k1);
  };
  // finish node plane p into buffer b
  auto form_store = [&](int p, int b) {
#pragma unroll
    for (int q = 0; q < kSlots; ++q) {
      const int e = threadIdx.x + q * kBoxThreads;
      if (e >= kBoxPlane) continue;
      T v[3] = {T(0), T(0), T(0)};
      if (fin[q] && p >= 0 && p < d.pz) {
        const int64_t nv = node_of(fi[q], fj[q], p);
        in.make(raw[q], nv, fi[q], fj[q], p, fown[q] && p >= k0 && p < k1, v);
      }
      xs[b][e][0] = v[0];
      xs[b][e][1] = v[1];
      xs[b][e][2] = v[2];
    }
  };
  // corner (a, b) of this thread's hex from plane buffer pb
  auto corner = [&](int pb, int a, int b, T (&v)[3]) {
    const int e = (wp + b) * kBoxCols + L + a;
    v[0] = xs[pb][e][0];
    v[1] = xs[pb][e][1];
    v[2] = xs[pb][e][2];
  };

  for (int p = 0; p < 3; ++p) {
    form_load(k0 - 1 + p);
    form_store(k0 - 1 + p, p);
  }
  __syncthreads();
  T xb[4][3];  // bottom corners (a + 2b) of the current hex layer
#pragma unroll
  for (int q = 0; q < 4; ++q) corner(0, q & 1, q >> 1, xb[q]);
  __syncthreads();  // the first layer refills buffer 0
  T carry[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q) carry[q][0] = carry[q][1] = carry[q][2] = T(0);
  double acc = 0.0;
  int bt = 1, bf = 0;  // buffer of the top plane (k + 1), buffer to form (k + 3)
  // hex weights, loaded one layer ahead; hex (i, j, k) = h0 + k * layer
  const int64_t layer = int64_t(d.nx) * d.ny, h0 = hex_ij ? int64_t(i) + int64_t(d.nx) * j : 0;
  auto load_w = [&](int k, T (&w)[WM ? 6 : 1]) {
    if (hex_ij && k >= 0 && k < d.nz) {
      const int64_t h = h0 + k * layer;
      if constexpr (WM) {
#pragma unroll
        for (int t = 0; t < 6; ++t) w[t] = bw.w[t * bw.H + h];
      } else {
        w[0] = bw.w[h];
      }
    }
  };
  T wn[WM ? 6 : 1];
  load_w(k0 - 1, wn);
  const int64_t plane = int64_t(d.px) * d.py, v0 = int64_t(i) + int64_t(d.px) * j;
  for (int k = k0 - 1; k < k1; ++k) {
    const bool fwd = k + 3 <= k1;  // plane k + 3 is read by a later layer
    if (fwd) form_load(k + 3);
    const bool own = own_ij && k >= k0;
    const int64_t v = v0 + k * plane;
    typename Out::Pre pre;
    if (own) pre = out.load(v);
    T w[WM ? 6 : 1];
#pragma unroll
    for (int t = 0; t < (WM ? 6 : 1); ++t) w[t] = wn[t];
    load_w(k + 1, wn);
    T u[8][3];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      u[q][0] = xb[q][0];
      u[q][1] = xb[q][1];
      u[q][2] = xb[q][2];
      corner(bt, q & 1, q >> 1, xb[q]);  // top plane, next layer's bottom
      u[q + 4][0] = xb[q][0];
      u[q + 4][1] = xb[q][1];
      u[q + 4][2] = xb[q][2];
    }
    T f[8][3];
    if (hex_ij && k >= 0 && k < d.nz) {
      box_hex<CUBE, WM>(u, w, g, f);
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) f[c][0] = f[c][1] = f[c][2] = T(0);
    }
    // plane-k forces of the four corners: carried top of the layer below + bottom
    T P[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        P[q][c] = carry[q][c] + f[q][c];
        carry[q][c] = f[q + 4][c];
      }
    // along x: node i gets corner a = 0 of hex i and corner a = 1 of hex i - 1
    T G0[3], G1[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      G0[c] = P[0][c] + __shfl_up_sync(0xffffffffu, P[1][c], 1);
      G1[c] = P[2][c] + __shfl_up_sync(0xffffffffu, P[3][c], 1);
    }
    const int yi = (k - k0 + 1) & 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) yb[yi][wp][L][c] = G1[c];
    if (fwd) form_store(k + 3, bf);
    __syncthreads();
    // along y: node j gets corner b = 0 of row j and corner b = 1 of row j - 1
    if (own) {
      T y[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) y[c] = G0[c] + yb[yi][wp - 1][L][c];
      acc += out.store(pre, v, i, j, k, y);
    }
    bt = bt == 2 ? 0 : bt + 1;
    bf = bf == 2 ? 0 : bf + 1;
  }
  if constexpr (Out::kReduce) {
    const double b = block_sum_box(acc, s_red);
    const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
      red.partials[bid] = b;
      __threadfence();
      s_last = atomicAdd(red.counter, 1u) == nb - 1;
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      double t = 0.0;
      for (unsigned p = threadIdx.x; p < nb; p += kBoxThreads) t += __ldcg(&red.partials[p]);
      t = block_sum_box(t, s_red);
      if (threadIdx.x == 0) {
        *red.counter = 0u;
        out.finish(t);
      }
    }
  }
}

}  // namespace pa
