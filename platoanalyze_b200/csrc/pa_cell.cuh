// pa_cell.cuh -- per-cell linear-tet mechanics, device side.
//
// One tetrahedron, one quadrature point: the reference evaluates these steps
// as separate Kokkos functors with DRAM temporaries between them
// (ComputeGradientWorkset, Strain, LinearStress, ApplyWeighting,
// StressDivergence, src/elliptic/ElastostaticResidual.hpp:147-214); here they
// are fused in registers.  Derivatives are hand-derived closed forms instead
// of Sacado forward-mode AD.
#pragma once
#include "pa_internal.cuh"

namespace pa {

// Shape-function gradients and weighted volume of a linear tet:
// ComputeGradientWorkset<3> (src/ImplicitFunctors.hpp:165-217).  J has
// columns x_n - x_3, g[n] = row n of J^-1 for n < 3, g[3] = -(g0+g1+g2);
// vol = |det J| / 6 (1-point rule weight, src/LinearTetCubRuleDegreeOne.hpp:72-78).
template <typename T>
__device__ __forceinline__ void tet_geometry(const T x[4][3], T g[4][3], T& vol) {
  const T j11 = x[0][0] - x[3][0], j12 = x[1][0] - x[3][0], j13 = x[2][0] - x[3][0];
  const T j21 = x[0][1] - x[3][1], j22 = x[1][1] - x[3][1], j23 = x[2][1] - x[3][1];
  const T j31 = x[0][2] - x[3][2], j32 = x[1][2] - x[3][2], j33 = x[2][2] - x[3][2];
  const T c11 = j22 * j33 - j23 * j32, c12 = j13 * j32 - j12 * j33, c13 = j12 * j23 - j13 * j22;
  const T det = j11 * c11 + j21 * c12 + j31 * c13;
  const T inv = T(1) / det;
  g[0][0] = c11 * inv;
  g[0][1] = c12 * inv;
  g[0][2] = c13 * inv;
  g[1][0] = (j23 * j31 - j21 * j33) * inv;
  g[1][1] = (j11 * j33 - j13 * j31) * inv;
  g[1][2] = (j13 * j21 - j11 * j23) * inv;
  g[2][0] = (j21 * j32 - j22 * j31) * inv;
  g[2][1] = (j12 * j31 - j11 * j32) * inv;
  g[2][2] = (j11 * j22 - j12 * j21) * inv;
#pragma unroll
  for (int d = 0; d < 3; ++d) g[3][d] = -(g[0][d] + g[1][d] + g[2][d]);
  vol = fabs(det) * (T(1) / T(6));
}

// Voigt strain {xx,yy,zz,yz,xz,xy}, engineering shears (src/Strain.hpp:56-94).
template <typename T>
__device__ __forceinline__ void tet_strain(const T g[4][3], const T u[12], T e[6]) {
  T exx = 0, eyy = 0, ezz = 0, gyz = 0, gxz = 0, gxy = 0;
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const T ux = u[3 * n], uy = u[3 * n + 1], uz = u[3 * n + 2];
    exx += ux * g[n][0];
    eyy += uy * g[n][1];
    ezz += uz * g[n][2];
    gyz += uz * g[n][1] + uy * g[n][2];
    gxz += uz * g[n][0] + ux * g[n][2];
    gxy += uy * g[n][0] + ux * g[n][1];
  }
  e[0] = exx; e[1] = eyy; e[2] = ezz; e[3] = gyz; e[4] = gxz; e[5] = gxy;
}

// Isotropic linear stress (src/LinearStress.hpp:61-77 with the stiffness of
// src/IsotropicLinearElasticMaterial.cpp:86-108), scaled by `s`.
template <typename T>
__device__ __forceinline__ void tet_stress(const Iso<T>& m, T s, const T e[6], T sig[6]) {
  const T tr = m.lam * (e[0] + e[1] + e[2]);
  const T two_mu = m.mu + m.mu;
  sig[0] = s * (tr + two_mu * e[0]);
  sig[1] = s * (tr + two_mu * e[1]);
  sig[2] = s * (tr + two_mu * e[2]);
  sig[3] = s * (m.mu * e[3]);
  sig[4] = s * (m.mu * e[4]);
  sig[5] = s * (m.mu * e[5]);
}

// r[3n+i] = sum_j sig(i,j) g[n][j] (src/StressDivergence.hpp:70-90); the
// caller folds volume and penalty into sig.
template <typename T>
__device__ __forceinline__ void tet_divergence(const T g[4][3], const T sig[6], T r[12]) {
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    r[3 * n + 0] = g[n][0] * sig[0] + g[n][1] * sig[5] + g[n][2] * sig[4];
    r[3 * n + 1] = g[n][0] * sig[5] + g[n][1] * sig[1] + g[n][2] * sig[3];
    r[3 * n + 2] = g[n][0] * sig[4] + g[n][1] * sig[3] + g[n][2] * sig[2];
  }
}

template <typename T>
__device__ __forceinline__ T voigt_dot(const T a[6], const T b[6]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3] + a[4] * b[4] + a[5] * b[5];
}

// x^p; integer exponents 0..4 (the reference's default p is 3) as products,
// which agree with pow to an ulp or two: an FP64 pow costs an exp/log pair,
// and one or two of them per tet made the per-cell kernels FP64-bound.
__device__ __forceinline__ double simp_pow(double x, double p) {
  if (p == 3.0) return x * x * x;
  if (p == 2.0) return x * x;
  if (p == 1.0) return x;
  if (p == 4.0) {
    const double x2 = x * x;
    return x2 * x2;
  }
  if (p == 0.0) return 1.0;
  return pow(x, p);
}

// SIMP penalty and its derivative (src/Simp.hpp:130-134).
__device__ __forceinline__ double simp(double rho, double p, double pmin) {
  return pmin + (1.0 - pmin) * simp_pow(rho, p);
}
__device__ __forceinline__ double simp_deriv(double rho, double p, double pmin) {
  if (rho == 0.0) return p == 1.0 ? (1.0 - pmin) : 0.0;
  return (1.0 - pmin) * p * simp_pow(rho, p - 1.0);
}

// Closed-form 3x3 block (a,b) of the isotropic cell stiffness
// K_ab = s [lam g_a g_b^T + mu g_b g_a^T + mu (g_a . g_b) I], s = vol * penalty.
template <typename T>
__device__ __forceinline__ void tet_kblock(const Iso<T>& m, T s, const T ga[3], const T gb[3], T k[9]) {
  const T d = m.mu * (ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2]);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) k[3 * i + j] = s * (m.lam * ga[i] * gb[j] + m.mu * ga[j] * gb[i] + (i == j ? d : T(0)));
}

}  // namespace pa
