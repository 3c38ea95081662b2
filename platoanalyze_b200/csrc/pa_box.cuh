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
// vector is formed once per node and plane into shared memory (four plane
// buffers, one barrier per hex layer), its global loads issued a layer
// before they are needed.
#pragma once

#include <cstdint>

#include "pa_cell.cuh"
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

// SIMP weights: one per hex (WM = 0), one per tet, tet-major (WM = 1:
// w[t H + h]), or (WM = 2) the per-cell controls themselves in box slot
// order (w[6 h + t]) with the SIMP penalty pmin + (1 - pmin) w^p applied as
// they are loaded.
template <typename T, int WM>
struct BoxW {
  const T* w;
  int64_t H;
  double p = 0.0, pmin = 0.0;
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

// Shared-memory node record: FP32 (x, y, z, unused) in one 16-byte access;
// FP64 (x, y, z) in three 8-byte accesses (24 bytes keep the FP64 kernel's
// plane buffers within 48 KB).
template <typename T>
struct BoxV4;
template <>
struct alignas(16) BoxV4<float> {
  float x, y, z, w;
  __device__ BoxV4() {}
  __device__ BoxV4(float a, float b, float c) : x(a), y(b), z(c), w(0.f) {}
};
template <>
struct BoxV4<double> {
  double x, y, z;
  __device__ BoxV4() {}
  __device__ BoxV4(double a, double b, double c) : x(a), y(b), z(c) {}
};

// Forces of one hex for corner displacements u (corner c = a + 2b + 4c).
// The twelve hex edges carry the displacement differences; tet t (its path
// edges listed below) takes its displacement gradient columns from its three
// edges, and its edge fluxes (stress columns) accumulate per edge; a corner's
// force is the sum of the fluxes of the edges that end there minus those that
// start there:
//   t0 Y00 X10 Z11   t1 Y00 Z01 X11   t2 Z00 Y01 X11
//   t3 Z00 X01 Y11   t4 X00 Z10 Y11   t5 X00 Y10 Z11
// (X_bc: x-edge from corner 2b + 4c; Y_ac: y-edge from a + 4c; Z_ab: z-edge
// from a + 2b).  lw, mw: the six tets' Lame parameters times weight and
// volume (and 1/h^2 for cubes).
template <bool CUBE, typename T>
__device__ __forceinline__ void box_hex(const T (&u)[8][3], const T (&lw)[6], const T (&mw)[6], const T (&ih)[3],
                                        T (&f)[8][3]) {
  T X00[3], X10[3], X01[3], X11[3], Y00[3], Y10[3], Y01[3], Y11[3], Z00[3], Z10[3], Z01[3], Z11[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    X00[c] = u[1][c] - u[0][c];
    X10[c] = u[3][c] - u[2][c];
    X01[c] = u[5][c] - u[4][c];
    X11[c] = u[7][c] - u[6][c];
    Y00[c] = u[2][c] - u[0][c];
    Y10[c] = u[3][c] - u[1][c];
    Y01[c] = u[6][c] - u[4][c];
    Y11[c] = u[7][c] - u[5][c];
    Z00[c] = u[4][c] - u[0][c];
    Z10[c] = u[5][c] - u[1][c];
    Z01[c] = u[6][c] - u[2][c];
    Z11[c] = u[7][c] - u[3][c];
    if constexpr (!CUBE) {
      X00[c] *= ih[0]; X10[c] *= ih[0]; X01[c] *= ih[0]; X11[c] *= ih[0];
      Y00[c] *= ih[1]; Y10[c] *= ih[1]; Y01[c] *= ih[1]; Y11[c] *= ih[1];
      Z00[c] *= ih[2]; Z10[c] *= ih[2]; Z01[c] *= ih[2]; Z11[c] *= ih[2];
    }
  }
  // stress columns (edge fluxes) of a tet with gradient columns gx, gy, gz
  auto tet = [&](const T (&gx)[3], const T (&gy)[3], const T (&gz)[3], T l, T m, T (&sx)[3], T (&sy)[3],
                 T (&sz)[3]) {
    const T lt = l * (gx[0] + gy[1] + gz[2]);
    const T m2 = m + m;
    const T sxy = m * (gy[0] + gx[1]), sxz = m * (gz[0] + gx[2]), syz = m * (gz[1] + gy[2]);
    sx[0] = fma(m2, gx[0], lt);
    sy[1] = fma(m2, gy[1], lt);
    sz[2] = fma(m2, gz[2], lt);
    sx[1] = sy[0] = sxy;
    sx[2] = sz[0] = sxz;
    sy[2] = sz[1] = syz;
    if constexpr (!CUBE) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sx[c] *= ih[0];
        sy[c] *= ih[1];
        sz[c] *= ih[2];
      }
    }
  };
  T qX00[3], qX10[3], qX01[3], qX11[3], qY00[3], qY10[3], qY01[3], qY11[3], qZ00[3], qZ10[3], qZ01[3], qZ11[3];
  T a[3], b[3], c3[3];
  tet(X10, Y00, Z11, lw[0], mw[0], qX10, qY00, qZ11);  // t0
  tet(X11, Y00, Z01, lw[1], mw[1], qX11, a, qZ01);      // t1
#pragma unroll
  for (int c = 0; c < 3; ++c) qY00[c] += a[c];
  tet(X11, Y01, Z00, lw[2], mw[2], a, qY01, qZ00);      // t2
#pragma unroll
  for (int c = 0; c < 3; ++c) qX11[c] += a[c];
  tet(X01, Y11, Z00, lw[3], mw[3], qX01, qY11, a);      // t3
#pragma unroll
  for (int c = 0; c < 3; ++c) qZ00[c] += a[c];
  tet(X00, Y11, Z10, lw[4], mw[4], qX00, a, qZ10);      // t4
#pragma unroll
  for (int c = 0; c < 3; ++c) qY11[c] += a[c];
  tet(X00, Y10, Z11, lw[5], mw[5], b, qY10, c3);        // t5
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    qX00[c] += b[c];
    qZ11[c] += c3[c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    f[0][c] = -(qX00[c] + qY00[c]) - qZ00[c];
    f[1][c] = qX00[c] - qY10[c] - qZ10[c];
    f[2][c] = qY00[c] - qX10[c] - qZ01[c];
    f[3][c] = qX10[c] + qY10[c] - qZ11[c];
    f[4][c] = qZ00[c] - qX01[c] - qY01[c];
    f[5][c] = qX01[c] + qZ10[c] - qY11[c];
    f[6][c] = qY01[c] + qZ01[c] - qX11[c];
    f[7][c] = qX11[c] + qY11[c] + qZ11[c];
  }
}

// The same with the six tet weights and the Lame parameters passed apart, each
// tet forming its own products: fewer live registers, used by the FP64
// per-cell-control instances held to 128 registers (the FP32 instances keep
// the form above, which stays within their 128).
template <bool CUBE, typename T>
__device__ __forceinline__ void box_hex_w(const T (&u)[8][3], const T (&w)[6], T lam, T mu, const T (&ih)[3],
                                          T (&f)[8][3]) {
  T X00[3], X10[3], X01[3], X11[3], Y00[3], Y10[3], Y01[3], Y11[3], Z00[3], Z10[3], Z01[3], Z11[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    X00[c] = u[1][c] - u[0][c];
    X10[c] = u[3][c] - u[2][c];
    X01[c] = u[5][c] - u[4][c];
    X11[c] = u[7][c] - u[6][c];
    Y00[c] = u[2][c] - u[0][c];
    Y10[c] = u[3][c] - u[1][c];
    Y01[c] = u[6][c] - u[4][c];
    Y11[c] = u[7][c] - u[5][c];
    Z00[c] = u[4][c] - u[0][c];
    Z10[c] = u[5][c] - u[1][c];
    Z01[c] = u[6][c] - u[2][c];
    Z11[c] = u[7][c] - u[3][c];
    if constexpr (!CUBE) {
      X00[c] *= ih[0]; X10[c] *= ih[0]; X01[c] *= ih[0]; X11[c] *= ih[0];
      Y00[c] *= ih[1]; Y10[c] *= ih[1]; Y01[c] *= ih[1]; Y11[c] *= ih[1];
      Z00[c] *= ih[2]; Z10[c] *= ih[2]; Z01[c] *= ih[2]; Z11[c] *= ih[2];
    }
  }
  // stress columns (edge fluxes) of a tet with gradient columns gx, gy, gz
  auto tet = [&](const T (&gx)[3], const T (&gy)[3], const T (&gz)[3], T l, T m, T (&sx)[3], T (&sy)[3],
                 T (&sz)[3]) {
    const T lt = l * (gx[0] + gy[1] + gz[2]);
    const T m2 = m + m;
    const T sxy = m * (gy[0] + gx[1]), sxz = m * (gz[0] + gx[2]), syz = m * (gz[1] + gy[2]);
    sx[0] = fma(m2, gx[0], lt);
    sy[1] = fma(m2, gy[1], lt);
    sz[2] = fma(m2, gz[2], lt);
    sx[1] = sy[0] = sxy;
    sx[2] = sz[0] = sxz;
    sy[2] = sz[1] = syz;
    if constexpr (!CUBE) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sx[c] *= ih[0];
        sy[c] *= ih[1];
        sz[c] *= ih[2];
      }
    }
  };
  T qX00[3], qX10[3], qX01[3], qX11[3], qY00[3], qY10[3], qY01[3], qY11[3], qZ00[3], qZ10[3], qZ01[3], qZ11[3];
  T a[3], b[3], c3[3];
  tet(X10, Y00, Z11, w[0] * lam, w[0] * mu, qX10, qY00, qZ11);  // t0
  tet(X11, Y00, Z01, w[1] * lam, w[1] * mu, qX11, a, qZ01);      // t1
#pragma unroll
  for (int c = 0; c < 3; ++c) qY00[c] += a[c];
  tet(X11, Y01, Z00, w[2] * lam, w[2] * mu, a, qY01, qZ00);      // t2
#pragma unroll
  for (int c = 0; c < 3; ++c) qX11[c] += a[c];
  tet(X01, Y11, Z00, w[3] * lam, w[3] * mu, qX01, qY11, a);      // t3
#pragma unroll
  for (int c = 0; c < 3; ++c) qZ00[c] += a[c];
  tet(X00, Y11, Z10, w[4] * lam, w[4] * mu, qX00, a, qZ10);      // t4
#pragma unroll
  for (int c = 0; c < 3; ++c) qY11[c] += a[c];
  tet(X00, Y10, Z11, w[5] * lam, w[5] * mu, b, qY10, c3);        // t5
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    qX00[c] += b[c];
    qZ11[c] += c3[c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    f[0][c] = -(qX00[c] + qY00[c]) - qZ00[c];
    f[1][c] = qX00[c] - qY10[c] - qZ10[c];
    f[2][c] = qY00[c] - qX10[c] - qZ01[c];
    f[3][c] = qX10[c] + qY10[c] - qZ11[c];
    f[4][c] = qZ00[c] - qX01[c] - qY01[c];
    f[5][c] = qX01[c] + qZ10[c] - qY11[c];
    f[6][c] = qY01[c] + qZ01[c] - qX11[c];
    f[7][c] = qX11[c] + qY11[c] + qZ11[c];
  }
}

// y = K x on the box with a fused input former and epilogue.  Both are split
// into a load part (global loads into registers, issued a hex layer before
// the values are needed) and a compute part:
//   In:  struct Raw;
//        __device__ Raw load(int v, bool owned) const;
//        __device__ void make(const Raw&, int v, bool owned, T (&x)[3]) const;
//        the input vector at node v, once per CTA, node and plane (`owned`:
//        this CTA owns v, for side outputs);
//   Out: struct Pre;
//        __device__ Pre load(int v) const;
//        __device__ double store(const Pre&, int v, const T (&y)[3]) const;
//        consumes (K x)_v at an owned node and returns its part of the
//        reduction; static constexpr bool kReduce; __device__ void finish(double) const.
// Node indices are 32-bit (3 N < 2^31).  Node plane p is formed three hex
// layers ahead into buffer (p - k0 + 1) % 4.
// Grid: (ceil(px / 31), ceil(py / 7), ceil(pz / kz)) CTAs of 256 threads.
// Two CTAs of 256 threads per SM (at most 128 registers) for every FP32
// instance and for the FP64 instances with per-cell controls (the per-cell
// entry points): measured on 160x80x80, the FP64 residual 105 -> 87 us with
// the few spills this costs (fewer still with box_hex_w and the late weight
// loads).  The FP64 CG apply (about 210 registers) spills heavily at that
// bound and did not speed up the solve, so those instances keep one CTA per SM.
template <typename T, int WM, bool CUBE, class In, class Out>
__global__ void __launch_bounds__(kBoxThreads, (sizeof(T) == 4 || WM == 2) ? 2 : 1) k_box(BoxDims d, BoxGeo<T> g, BoxW<T, WM> bw, int kz, In in,
                                                     Out out, BoxRed red, const double* skip) {
  // skip (may be null): two flags; the launch is a no-op when either is set
  // (a solve that converged or broke down inside a batch of captured iterations)
  if (skip && (skip[0] != 0.0 || skip[1] != 0.0)) return;
  __shared__ BoxV4<T> xs[4][kBoxPlane];
  __shared__ BoxV4<T> yb[2][8][32];
  __shared__ double s_red[32];
  const int L = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int i0 = blockIdx.x * kBoxX, j0 = blockIdx.y * kBoxY, k0 = blockIdx.z * kz;
  const int k1 = min(k0 + kz, d.pz);  // node planes [k0, k1)
  const int i = i0 - 1 + L, j = j0 - 1 + wp;
  const bool hex_ij = i >= 0 && i < d.nx && j >= 0 && j < d.ny;
  const bool own_ij = L >= 1 && wp >= 1 && i < d.px && j < d.py;
  const int plane = d.px * d.py;

  // the (at most two) plane entries this thread forms: e = tid, tid + 256
  constexpr int kSlots = (kBoxPlane + kBoxThreads - 1) / kBoxThreads;
  int fv[kSlots];
  bool fin[kSlots], fown[kSlots];
#pragma unroll
  for (int q = 0; q < kSlots; ++q) {
    const int e = threadIdx.x + q * kBoxThreads;
    const int r = e / kBoxCols, c = e - r * kBoxCols;
    const int fi = i0 - 1 + c, fj = j0 - 1 + r;
    fin[q] = e < kBoxPlane && fi >= 0 && fi < d.px && fj >= 0 && fj < d.py;
    fown[q] = e < kBoxPlane && c >= 1 && c <= kBoxX && r >= 1 && r <= kBoxY;
    fv[q] = fin[q] ? fi + d.px * fj : 0;  // node of the entry in plane 0
  }
  typename In::Raw raw[kSlots];
  auto form_load = [&](int p) {
#pragma unroll
    for (int q = 0; q < kSlots; ++q)
      if (fin[q] && p >= 0 && p < d.pz) raw[q] = in.load(fv[q] + p * plane, fown[q] && p >= k0 && p < k1);
  };
  auto form_store_from = [&](const typename In::Raw (&rr)[kSlots], int p, int b) {
#pragma unroll
    for (int q = 0; q < kSlots; ++q) {
      const int e = threadIdx.x + q * kBoxThreads;
      if (e >= kBoxPlane) continue;
      T v[3] = {T(0), T(0), T(0)};
      if (fin[q] && p >= 0 && p < d.pz) in.make(rr[q], fv[q] + p * plane, fown[q] && p >= k0 && p < k1, v);
      xs[b][e] = BoxV4<T>(v[0], v[1], v[2]);
    }
  };
  auto form_store = [&](int p, int b) { form_store_from(raw, p, b); };

  // hex weights, loaded one layer ahead; hex (i, j, k) = h0 + k * layer
  const int layer = d.nx * d.ny, h0 = hex_ij ? i + d.nx * j : 0;
  T wn[WM ? 6 : 1];
  auto load_w = [&](int k) {
    if (hex_ij && k >= 0 && k < d.nz) {
      if constexpr (WM == 2) {
        const int64_t hh = h0 + int64_t(k) * layer;
#pragma unroll
        for (int t = 0; t < 6; ++t) wn[t] = T(simp(double(bw.w[6 * hh + t]), bw.p, bw.pmin));
      } else if constexpr (WM == 1) {
#pragma unroll
        for (int t = 0; t < 6; ++t) wn[t] = bw.w[int64_t(t) * bw.H + h0 + k * layer];
      } else {
        wn[0] = bw.w[h0 + k * layer];
      }
    }
  };
  load_w(k0 - 1);  // the first layer's weights, in flight with the planes below

  // the first three planes: every load issued before any is used (a CTA with
  // a one-plane chunk forms nothing else, so these loads are its latency)
  {
    typename In::Raw raw3[3][kSlots];
#pragma unroll
    for (int pl = 0; pl < 3; ++pl) {
      const int p = k0 - 1 + pl;
#pragma unroll
      for (int q = 0; q < kSlots; ++q)
        if (fin[q] && p >= 0 && p < d.pz) raw3[pl][q] = in.load(fv[q] + p * plane, fown[q] && p >= k0 && p < k1);
    }
#pragma unroll
    for (int pl = 0; pl < 3; ++pl) form_store_from(raw3[pl], k0 - 1 + pl, pl);
  }
  __syncthreads();

  const int v0 = i + d.px * j;
  T carry[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q) carry[q][0] = carry[q][1] = carry[q][2] = T(0);
  double acc = 0.0;
  int bb = 0;  // buffer of the bottom plane k; top k + 1 in bb + 1, plane k + 3 formed into bb + 3 (mod 4)
#pragma unroll 2
  for (int k = k0 - 1; k < k1; ++k) {
    const bool fwd = k + 3 <= k1;  // plane k + 3 is read by a later layer
    if (fwd) form_load(k + 3);
    const bool own = own_ij && k >= k0;
    const int v = v0 + k * plane;
    typename Out::Pre pre;
    if (own) pre = out.load(v);
    // FP64 per-cell-control instances (two CTAs per SM at 128 registers): the
    // raw weights go into the hex work and the next layer's load follows it
    constexpr bool kLateW = WM == 2 && sizeof(T) == 8;
    T lw[6], mw[6], w6[6];
    if constexpr (kLateW) {
#pragma unroll
      for (int t = 0; t < 6; ++t) w6[t] = wn[t];
    } else {
      T w[WM ? 6 : 1];
#pragma unroll
      for (int t = 0; t < (WM ? 6 : 1); ++t) w[t] = wn[t];
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        lw[t] = w[WM ? t : 0] * g.lam;
        mw[t] = w[WM ? t : 0] * g.mu;
      }
      load_w(k + 1);
    }
    T f[8][3];
    if (hex_ij && k >= 0 && k < d.nz) {
      T u[8][3];
      const int bt = (bb + 1) & 3;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = (wp + (q >> 1)) * kBoxCols + L + (q & 1);
        const BoxV4<T> lo = xs[bb][e], hi = xs[bt][e];
        u[q][0] = lo.x;
        u[q][1] = lo.y;
        u[q][2] = lo.z;
        u[q + 4][0] = hi.x;
        u[q + 4][1] = hi.y;
        u[q + 4][2] = hi.z;
      }
      if constexpr (kLateW)
        box_hex_w<CUBE>(u, w6, g.lam, g.mu, g.ih, f);
      else
        box_hex<CUBE>(u, lw, mw, g.ih, f);
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) f[c][0] = f[c][1] = f[c][2] = T(0);
    }
    if constexpr (kLateW) load_w(k + 1);
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
    yb[yi][wp][L] = BoxV4<T>(G1[0], G1[1], G1[2]);
    if (fwd) form_store(k + 3, (bb + 3) & 3);
    __syncthreads();
    // along y: node j gets corner b = 0 of row j and corner b = 1 of row j - 1
    if (own) {
      const BoxV4<T> o = yb[yi][wp - 1][L];
      const T y[3] = {G0[0] + o.x, G0[1] + o.y, G0[2] + o.z};
      acc += out.store(pre, v, y);
    }
    bb = (bb + 1) & 3;
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
