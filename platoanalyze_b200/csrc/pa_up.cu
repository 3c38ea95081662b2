// pa_up.cu -- stabilized u-p J2 plasticity solve (FP64): pseudo-time load
// steps, Newton on the condensed global residual, and the projected pressure
// gradient lagged by one step.
//
// The reference's driver is PlasticityProblem::solveForwardProblem
// (src/PlasticityProblem.hpp:791-846) with NewtonRaphsonSolver::solve
// (src/NewtonRaphsonSolver.hpp:570-640):
//  * each load step starts from the previous converged global and local
//    states (initializeSolver, :335-343) and imposes the Dirichlet increment in
//    the first Newton solve only (applyConstraints, :121-152);
//  * every Newton iterate returns the local states from the previous step's
//    (updateLocalState: the J2 return mapping, closed form for linear
//    hardening, so the local residual H is zero at the returned state);
//  * the tangent is dR/du - dR/dc (dH/dc)^-1 dH/du (:206-290), assembled per
//    cell; here it is formed in closed form per cell: with the return's
//    normal n and theta1 = sqrt(6) mu_l dgamma / |eta_trial|,
//    theta2 = 3 mu_l / (3 mu_l + H_iso + H_kin), d eps_p = theta1 dev(d eps) +
//    (theta2 - theta1) n (n : d eps), so the deviatoric stress
//    s = 2 mu_g dev(eps - eps_p) has ds/d eps = (1 - theta1) D_dev -
//    2 mu_g (theta2 - theta1) n n^T; the pressure rows and columns do not
//    depend on the local states;
//  * after a step converges the projected pressure gradient of the next step
//    is the row-summed (lumped) solve of the projection equation
//    (updateProjectedPressureGradient, :877-897,
//    src/PressureGradientProjectionResidual.hpp): per node, the penalty- and
//    volume-weighted mean of the cells' scaled pressure gradients.
//
// Layout and kernels: one thread per cell forms the return mapping, the 16
// residual entries and the 256 tangent entries, stored component-major
// (entry k of cell c at k C + c, coalesced); assembly is by gather over a
// node -> (cell, vertex) adjacency built once per solve, one thread per node,
// in a fixed order (deterministic, no atomics).  The global tangent is
// symmetric indefinite (a stabilized saddle point), solved by MINRES with the
// inverse absolute diagonal as preconditioner (Paige and Saunders, 1975, in
// the form of Choi, Paige and Saunders's preconditioned recurrence).
#include <algorithm>
#include <cmath>
#include <vector>

#include "pa_cell.cuh"
#include "pa_plastic.cuh"
#include "pa_problem.cuh"

namespace pa {
namespace {

constexpr int kUpT = 128;
constexpr int kRedBlocks = 256;

// Bcol(a, i): the engineering strain (xx, yy, zz, yz, xz, xy) of a unit
// displacement of vertex a along i.
__device__ __forceinline__ void bcol(const double g[3], int i, double b[6]) {
  b[0] = i == 0 ? g[0] : 0.0;
  b[1] = i == 1 ? g[1] : 0.0;
  b[2] = i == 2 ? g[2] : 0.0;
  b[3] = i == 1 ? g[2] : i == 2 ? g[1] : 0.0;
  b[4] = i == 0 ? g[2] : i == 2 ? g[0] : 0.0;
  b[5] = i == 0 ? g[1] : i == 1 ? g[0] : 0.0;
}

// Per cell: the return mapping from `prev` at the state's strain (new local
// states to `cur`), the 16 residual entries at the returned state (rc) and,
// when ke is not null, the 16 x 16 condensed tangent (ke, row-major per cell).
// ppg: the projected pressure gradient per node (3N).
__global__ void __launch_bounds__(kUpT) k_up_cells(const int32_t* __restrict__ cells, const double* __restrict__ coords,
                                                   int64_t C, UpDev q, J2Full j, const double* __restrict__ state,
                                                   const double* __restrict__ prev, const double* __restrict__ ppg,
                                                   const double* __restrict__ z, double* __restrict__ cur,
                                                   double* __restrict__ rc, double* __restrict__ ke) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= C) return;
  const int4 qv = reinterpret_cast<const int4*>(cells)[c];
  const int v[4] = {qv.x, qv.y, qv.z, qv.w};
  double x[4][3], ue[12], p[4], pi[3] = {0.0, 0.0, 0.0}, g[4][3], vol, eps[6];
  double rho = 0.0;
#pragma unroll
  for (int n = 0; n < 4; ++n) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      x[n][d] = coords[3 * int64_t(v[n]) + d];
      ue[3 * n + d] = state[4 * int64_t(v[n]) + d];
      pi[d] += 0.25 * ppg[3 * int64_t(v[n]) + d];
    }
    p[n] = state[4 * int64_t(v[n]) + 3];
    rho += 0.25 * z[v[n]];
  }
  tet_geometry(x, g, vol);
  tet_strain(g, ue, eps);
  double st[kLocal], sig[6], rec[8], pel;
#pragma unroll
  for (int i = 0; i < kLocal; ++i) st[i] = prev[kLocal * c + i];
  j2_cell(j, rho, eps, st, sig, rec, pel);
#pragma unroll
  for (int i = 0; i < kLocal; ++i) cur[kLocal * c + i] = st[i];
  // residual at the returned state (InfinitesimalStrainPlasticityResidual::evaluate)
  double e[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) e[i] = eps[i] - st[2 + i];
  const double pen = simp(rho, q.pe, q.pe_min);
  const double mu_g = pen * q.mu, kappa_p = pen * q.kappa;
  const double tr3 = (e[0] + e[1] + e[2]) * (1.0 / 3.0);
  const double sv[6] = {2.0 * mu_g * (e[0] - tr3), 2.0 * mu_g * (e[1] - tr3), 2.0 * mu_g * (e[2] - tr3),
                        mu_g * e[3], mu_g * e[4], mu_g * e[5]};
  double gp[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int d = 0; d < 3; ++d) gp[d] += p[n] * g[n][d];
  const double ps = q.ps;
  const double pc = ps * 0.25 * (p[0] + p[1] + p[2] + p[3]);
  const double theta = ps * (eps[0] + eps[1] + eps[2] - pc / kappa_p);
  const double cv = cbrt(vol);
  const double tau = cv * cv / (2.0 * q.mu);
  double stab[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) stab[d] = pen * ps * tau * (ps * gp[d] - pi[d]);
  const double S[3][3] = {{sv[0] + pc, sv[5], sv[4]}, {sv[5], sv[1] + pc, sv[3]}, {sv[4], sv[3], sv[2] + pc}};
#pragma unroll
  for (int n = 0; n < 4; ++n) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
      rc[(4 * n + i) * C + c] = vol * (S[i][0] * g[n][0] + S[i][1] * g[n][1] + S[i][2] * g[n][2]);
    rc[(4 * n + 3) * C + c] =
        -vol * (stab[0] * g[n][0] + stab[1] * g[n][1] + stab[2] * g[n][2]) + vol * 0.25 * theta;
  }
  if (!ke) return;
  // condensed tangent: D v = (1 - th1) D_dev v - 2 mu_g (th2 - th1) n (n . v)
  const double th1 = rec[6], th2 = rec[7];
  const double a1 = (1.0 - th1) * mu_g, a2 = 2.0 * mu_g * (th2 - th1);
  const double pp = -vol * ps * ps / (16.0 * kappa_p), ps_stab = vol * pen * ps * ps * tau;
#pragma unroll 1
  for (int a = 0; a < 4; ++a) {
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
      double b[6], t[6];
      bcol(g[a], i, b);
      const double m = (b[0] + b[1] + b[2]) * (1.0 / 3.0);
      const double nb = rec[0] * b[0] + rec[1] * b[1] + rec[2] * b[2] + rec[3] * b[3] + rec[4] * b[4] + rec[5] * b[5];
      t[0] = 2.0 * a1 * (b[0] - m) - a2 * rec[0] * nb;
      t[1] = 2.0 * a1 * (b[1] - m) - a2 * rec[1] * nb;
      t[2] = 2.0 * a1 * (b[2] - m) - a2 * rec[2] * nb;
      t[3] = a1 * b[3] - a2 * rec[3] * nb;
      t[4] = a1 * b[4] - a2 * rec[4] * nb;
      t[5] = a1 * b[5] - a2 * rec[5] * nb;
      const int row = 4 * a + i;
#pragma unroll
      for (int bb = 0; bb < 4; ++bb) {
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
          double bc[6];
          bcol(g[bb], jj, bc);
          const double kv =
              vol * (bc[0] * t[0] + bc[1] * t[1] + bc[2] * t[2] + bc[3] * t[3] + bc[4] * t[4] + bc[5] * t[5]);
          ke[(row * 16 + 4 * bb + jj) * C + c] = kv;
        }
        ke[(row * 16 + 4 * bb + 3) * C + c] = vol * ps * 0.25 * g[a][i];
      }
    }
    const int row = 4 * a + 3;
#pragma unroll
    for (int bb = 0; bb < 4; ++bb) {
#pragma unroll
      for (int jj = 0; jj < 3; ++jj) ke[(row * 16 + 4 * bb + jj) * C + c] = vol * ps * 0.25 * g[bb][jj];
      ke[(row * 16 + 4 * bb + 3) * C + c] =
          pp - ps_stab * (g[a][0] * g[bb][0] + g[a][1] * g[bb][1] + g[a][2] * g[bb][2]);
    }
  }
}

// R[4n + i] (+)= sum over the cells around node n of their entry (vertex, i)
__global__ void k_up_gather(int64_t N, const int32_t* __restrict__ ptr, const int64_t* __restrict__ adj, int64_t C,
                            const double* __restrict__ rc, double* __restrict__ R, int accumulate = 0) {
  const int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (n >= N) return;
  double r[4] = {0.0, 0.0, 0.0, 0.0};
  for (int32_t e = ptr[n]; e < ptr[n + 1]; ++e) {
    const int64_t c = adj[e] >> 2;
    const int a = int(adj[e] & 3);
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] += rc[(4 * a + i) * C + c];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) R[4 * n + i] = (accumulate ? R[4 * n + i] : 0.0) + r[i];
}

__device__ __forceinline__ bool up_masked(const uint8_t* mask, int64_t node, int comp) {
  return mask && ((mask[node] >> comp) & 1);
}

// y = K x with the cell tangents; mask (bit i of node n: dof 4n + i
// constrained; may be null): masked columns zero, masked rows y = x.
__global__ void k_up_apply(int64_t N, const int32_t* __restrict__ ptr, const int64_t* __restrict__ adj,
                           const int32_t* __restrict__ cells, int64_t C, const double* __restrict__ ke,
                           const uint8_t* __restrict__ mask, const double* __restrict__ x, double* __restrict__ y) {
  const int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (n >= N) return;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int32_t e = ptr[n]; e < ptr[n + 1]; ++e) {
    const int64_t c = adj[e] >> 2;
    const int a = int(adj[e] & 3);
    const int4 qv = reinterpret_cast<const int4*>(cells)[c];
    const int v[4] = {qv.x, qv.y, qv.z, qv.w};
    double xv[16];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int j = 0; j < 4; ++j) xv[4 * b + j] = up_masked(mask, v[b], j) ? 0.0 : x[4 * int64_t(v[b]) + j];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double* row = ke + int64_t(4 * a + i) * 16 * C + c;
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 16; ++k) s += row[k * C] * xv[k];
      acc[i] += s;
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) y[4 * n + i] = up_masked(mask, n, i) ? x[4 * n + i] : acc[i];
}

// dinv = 1 / |diag K| (1 on masked dofs and on a zero diagonal)
__global__ void k_up_dinv(int64_t N, const int32_t* __restrict__ ptr, const int64_t* __restrict__ adj, int64_t C,
                          const double* __restrict__ ke, const uint8_t* __restrict__ mask, double* __restrict__ dinv) {
  const int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (n >= N) return;
  double d[4] = {0.0, 0.0, 0.0, 0.0};
  for (int32_t e = ptr[n]; e < ptr[n + 1]; ++e) {
    const int64_t c = adj[e] >> 2;
    const int a = int(adj[e] & 3);
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] += ke[int64_t((4 * a + i) * 16 + 4 * a + i) * C + c];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) dinv[4 * n + i] = (up_masked(mask, n, i) || d[i] == 0.0) ? 1.0 : 1.0 / fabs(d[i]);
}

// Projected pressure gradient of the next step (lumped projection), per node
__global__ void k_up_project(int64_t N, const int32_t* __restrict__ ptr, const int64_t* __restrict__ adj,
                             const int32_t* __restrict__ cells, const double* __restrict__ coords, UpDev q,
                             const double* __restrict__ state, const double* __restrict__ z, double* __restrict__ ppg) {
  const int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (n >= N) return;
  double num[3] = {0.0, 0.0, 0.0}, den = 0.0;
  for (int32_t e = ptr[n]; e < ptr[n + 1]; ++e) {
    const int64_t c = adj[e] >> 2;
    const int4 qv = reinterpret_cast<const int4*>(cells)[c];
    const int v[4] = {qv.x, qv.y, qv.z, qv.w};
    double x[4][3], g[4][3], vol, rho = 0.0, gp[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
      for (int d = 0; d < 3; ++d) x[k][d] = coords[3 * int64_t(v[k]) + d];
      rho += 0.25 * z[v[k]];
    }
    tet_geometry(x, g, vol);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double pk = state[4 * int64_t(v[k]) + 3];
#pragma unroll
      for (int d = 0; d < 3; ++d) gp[d] += pk * g[k][d];
    }
    const double w = simp(rho, q.pe, q.pe_min) * vol;
#pragma unroll
    for (int d = 0; d < 3; ++d) num[d] += w * q.ps * gp[d];
    den += w;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) ppg[3 * n + d] = den > 0.0 ? num[d] / den : 0.0;
}

// partial sums of a . b (masked dofs skipped when mask is given), one per block
__global__ void k_up_dot(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                         const uint8_t* __restrict__ mask, double* __restrict__ partials) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    if (!up_masked(mask, i >> 2, int(i & 3))) s += a[i] * b[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void k_up_sum(int m, const double* __restrict__ partials, double* __restrict__ out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) s += partials[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// out = a x + b y + c w (an input whose coefficient is zero is not read and
// may be null; out may be any of the inputs)
__global__ void k_up_lin3(int64_t n, double* out, double a, const double* x, double b, const double* y, double c,
                          const double* w) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double v = a == 0.0 ? 0.0 : a * x[i];
    if (b != 0.0) v += b * y[i];
    if (c != 0.0) v += c * w[i];
    out[i] = v;
  }
}

// y = d .* x
__global__ void k_up_scale(int64_t n, const double* __restrict__ d, const double* __restrict__ x,
                           double* __restrict__ y) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = d[i] * x[i];
}

// b = masked ? t : -R - y
__global__ void k_up_rhs(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ t,
                         const double* __restrict__ R, const double* __restrict__ y, double* __restrict__ b) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    b[i] = up_masked(mask, i >> 2, int(i & 3)) ? t[i] : -R[i] - y[i];
}

__global__ void k_up_set(int64_t m, const int32_t* __restrict__ dofs, const double* __restrict__ vals, double scale,
                         double* __restrict__ x) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < m) x[dofs[i]] = scale * vals[i];
}

// ---------------------------------------------------------------- adjoint --
// Forward-mode number with one direction, for the pullbacks through the
// return mapping (one pass per input direction).
struct D1 {
  double v, d;
};
__device__ __forceinline__ D1 operator+(D1 a, D1 b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ D1 operator-(D1 a, D1 b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ D1 operator*(D1 a, D1 b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ D1 operator*(double a, D1 b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ D1 operator/(D1 a, D1 b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
__device__ __forceinline__ double val(D1 a) { return a.v; }
__device__ __forceinline__ D1 sqrt_t(D1 a) {
  const double r = sqrt(a.v);
  return {r, r > 0.0 ? a.d / (2.0 * r) : 0.0};
}
__device__ __forceinline__ D1 simp_t(D1 rho, double p, double pmin) {
  return {pmin + (1.0 - pmin) * pow(rho.v, p), (1.0 - pmin) * p * pow(rho.v, p - 1.0) * rho.d};
}
__device__ __forceinline__ double dsimp(double rho, double p, double pmin) {
  return (1.0 - pmin) * p * pow(rho, p - 1.0);
}

// The J2 return mapping c_n = Phi(eps, c_{n-1}, rho) of j2_cell (the local
// state update only) on forward-mode numbers.
template <typename T>
__device__ void j2_phi(const J2Dev& p, T rho, const T e[6], const T prev[kLocal], T cur[kLocal]) {
  const T pe = simp_t(rho, p.pe, p.pe_min);
  const T mu_p = p.mu * pe;
  const T ppen = simp_t(rho, p.pp, p.pp_min);
  const T hi = p.hiso * ppen, hk = p.hkin * ppen;
#pragma unroll
  for (int i = 0; i < kLocal; ++i) cur[i] = prev[i];
  T ee[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) ee[i] = e[i] - prev[2 + i];
  const T tr3 = (1.0 / 3.0) * (ee[0] + ee[1] + ee[2]);
  T n[6];
#pragma unroll
  for (int i = 0; i < 3; ++i) n[i] = 2.0 * mu_p * (ee[i] - tr3) - prev[8 + i];
#pragma unroll
  for (int i = 3; i < 6; ++i) n[i] = mu_p * ee[i] - prev[8 + i];
  const T norm = sqrt_t(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + 2.0 * (n[3] * n[3] + n[4] * n[4] + n[5] * n[5]));
  const double s32 = 1.2247448713915890491, s23 = 0.81649658092772603273;
  const T sy = p.sy0 * ppen + hi * prev[0];
  const T ftr = s32 * norm - sy;
  cur[1] = 0.0 * prev[1];
  if (val(ftr) > 1.0e-10) {
    const T dg = ftr / (3.0 * mu_p + hi + hk);
    cur[1] = dg;
    cur[0] = prev[0] + dg;
    const T m1 = s32 * dg / norm, m2 = s23 * dg * hk / norm;
#pragma unroll
    for (int i = 0; i < 3; ++i) cur[2 + i] = prev[2 + i] + m1 * n[i];
#pragma unroll
    for (int i = 3; i < 6; ++i) cur[2 + i] = prev[2 + i] + 2.0 * m1 * n[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) cur[8 + i] = prev[8 + i] + m2 * n[i];
  }
}

struct UpCell {
  int v[4];
  double g[4][3], vol, rho, eps[6];
};

__device__ __forceinline__ void up_cell_load(const int32_t* cells, const double* coords, const double* x,
                                             const double* z, int64_t c, UpCell& k) {
  const int4 qv = reinterpret_cast<const int4*>(cells)[c];
  k.v[0] = qv.x;
  k.v[1] = qv.y;
  k.v[2] = qv.z;
  k.v[3] = qv.w;
  double xc[4][3], ue[12];
  k.rho = 0.0;
#pragma unroll
  for (int n = 0; n < 4; ++n) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      xc[n][d] = coords[3 * int64_t(k.v[n]) + d];
      ue[3 * n + d] = x[4 * int64_t(k.v[n]) + d];
    }
    k.rho += 0.25 * z[k.v[n]];
  }
  tet_geometry(xc, k.g, k.vol);
  tet_strain(k.g, ue, k.eps);
}

// xc (16 per cell, component-major) = B^T t on the displacement entries, 0 on the pressures
__device__ __forceinline__ void up_store_bt(const UpCell& k, const double t[6], double scale, int64_t C, int64_t c,
                                            double* xc) {
#pragma unroll
  for (int a = 0; a < 4; ++a) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double b[6];
      bcol(k.g[a], i, b);
      xc[(4 * a + i) * C + c] =
          scale * (b[0] * t[0] + b[1] * t[1] + b[2] * t[2] + b[3] * t[3] + b[4] * t[4] + b[5] * t[5]);
    }
    xc[(4 * a + 3) * C + c] = 0.0;
  }
}

// The criterion at the last step: f_c = V sigma . e / 2 (the steps' elastic
// work summed telescopes to the final stored energy), its value per cell,
// and its partials: x (per cell), c_S (cbar) and rho (rbar, written).
__global__ void k_upa_final(const int32_t* __restrict__ cells, const double* __restrict__ coords, int64_t C, UpDev q,
                            double fpe, double fpmin, const double* __restrict__ x, const double* __restrict__ loc,
                            const double* __restrict__ z, double* __restrict__ fcell, double* __restrict__ xc,
                            double* __restrict__ cbar, double* __restrict__ rbar) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= C) return;
  UpCell k;
  up_cell_load(cells, coords, x, z, c, k);
  double e[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) e[i] = k.eps[i] - loc[kLocal * c + 2 + i];
  const double pen = simp(k.rho, fpe, fpmin);
  const double tr = e[0] + e[1] + e[2];
  double sg[6];
#pragma unroll
  for (int i = 0; i < 3; ++i) sg[i] = pen * (q.kappa * tr + 2.0 * q.mu * (e[i] - tr / 3.0));
#pragma unroll
  for (int i = 3; i < 6; ++i) sg[i] = pen * q.mu * e[i];
  double se = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) se += sg[i] * e[i];
  const double f = 0.5 * k.vol * se;
  fcell[c] = f;
  up_store_bt(k, sg, k.vol, C, c, xc);
#pragma unroll
  for (int i = 0; i < kLocal; ++i) cbar[kLocal * c + i] = (i >= 2 && i < 8) ? -k.vol * sg[i - 2] : 0.0;
  rbar[c] = f * dsimp(k.rho, fpe, fpmin) / pen;
}

// Pullback of cbar (the cotangent of c_n) through c_n = Phi(eps(x_n), c_{n-1}, rho)
// onto eps: xc (per cell) = B^T (dPhi/deps)^T cbar.
__global__ void k_upa_phi_eps(const int32_t* __restrict__ cells, const double* __restrict__ coords, int64_t C,
                              J2Dev jd, const double* __restrict__ x, const double* __restrict__ prev,
                              const double* __restrict__ z, const double* __restrict__ cbar, double* __restrict__ xc) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= C) return;
  UpCell k;
  up_cell_load(cells, coords, x, z, c, k);
  double cb[kLocal];
  bool any = false;
#pragma unroll
  for (int i = 0; i < kLocal; ++i) {
    cb[i] = cbar[kLocal * c + i];
    any = any || cb[i] != 0.0;
  }
  double eb[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (any) {
    D1 pv[kLocal], cur[kLocal];
#pragma unroll
    for (int i = 0; i < kLocal; ++i) pv[i] = D1{prev[kLocal * c + i], 0.0};
    const D1 rho{k.rho, 0.0};
#pragma unroll 1
    for (int dir = 0; dir < 6; ++dir) {
      D1 e[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) e[i] = D1{k.eps[i], i == dir ? 1.0 : 0.0};
      j2_phi(jd, rho, e, pv, cur);
      double acc = 0.0;
#pragma unroll
      for (int i = 0; i < kLocal; ++i) acc += cb[i] * cur[i].d;
      eb[dir] = acc;
    }
  }
  up_store_bt(k, eb, 1.0, C, c, xc);
}

// Pullbacks of step n given its adjoint lam (lam^T R_n): the cotangent of
// c_n seen by R (through eps_p) plus cbar_n, pulled back through Phi onto
// c_{n-1} (cprev, written) and rho; R's explicit dependence on rho (rbar,
// accumulated); and the cotangent of the projected pressure gradient, the same
// 3-vector for every vertex of the cell (pib, component-major 3 per cell).
__global__ void k_upa_resid(const int32_t* __restrict__ cells, const double* __restrict__ coords, int64_t C, UpDev q,
                            J2Dev jd, const double* __restrict__ x, const double* __restrict__ prev,
                            const double* __restrict__ cur_loc, const double* __restrict__ pi,
                            const double* __restrict__ z, const double* __restrict__ lam,
                            const double* __restrict__ cbar, double* __restrict__ cprev, double* __restrict__ rbar,
                            double* __restrict__ pib) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= C) return;
  UpCell k;
  up_cell_load(cells, coords, x, z, c, k);
  double lu[12], lp[4], p[4], pic[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int a = 0; a < 4; ++a) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      lu[3 * a + i] = lam[4 * int64_t(k.v[a]) + i];
      pic[i] += 0.25 * pi[3 * int64_t(k.v[a]) + i];
    }
    lp[a] = lam[4 * int64_t(k.v[a]) + 3];
    p[a] = x[4 * int64_t(k.v[a]) + 3];
  }
  double el[6];
  tet_strain(k.g, lu, el);  // engineering strain of lam's displacement part
  const double pen = simp(k.rho, q.pe, q.pe_min);
  const double mu_g = pen * q.mu;
  // cotangent of c_n: cbar + (dR/d eps_p)^T lam = cbar - V D_dev eps(lam_u)
  double cb[kLocal];
#pragma unroll
  for (int i = 0; i < kLocal; ++i) cb[i] = cbar[kLocal * c + i];
  {
    const double tl = (el[0] + el[1] + el[2]) / 3.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) cb[2 + i] -= k.vol * 2.0 * mu_g * (el[i] - tl);
#pragma unroll
    for (int i = 3; i < 6; ++i) cb[2 + i] -= k.vol * mu_g * el[i];
  }
  // pull back through Phi onto c_{n-1} (entry 1 is not read by Phi) and rho
  double cp[kLocal], rb = 0.0;
  {
    D1 e[6], pv[kLocal], cur[kLocal];
#pragma unroll
    for (int i = 0; i < 6; ++i) e[i] = D1{k.eps[i], 0.0};
#pragma unroll 1
    for (int dir = 0; dir <= kLocal; ++dir) {  // dir < 14: c_{n-1} entry; dir == 14: rho
#pragma unroll
      for (int i = 0; i < kLocal; ++i) pv[i] = D1{prev[kLocal * c + i], i == dir ? 1.0 : 0.0};
      const D1 rho{k.rho, dir == kLocal ? 1.0 : 0.0};
      double acc = 0.0;
      if (dir != 1) {
        j2_phi(jd, rho, e, pv, cur);
#pragma unroll
        for (int i = 0; i < kLocal; ++i) acc += cb[i] * cur[i].d;
      }
      if (dir < kLocal)
        cp[dir] = acc;
      else
        rb = acc;
    }
  }
#pragma unroll
  for (int i = 0; i < kLocal; ++i) cprev[kLocal * c + i] = cp[i];
  // R's explicit dependence on the penalty of the u-p residual
  double e[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) e[i] = k.eps[i] - cur_loc[kLocal * c + 2 + i];
  const double tr3 = (e[0] + e[1] + e[2]) / 3.0;
  const double s1[6] = {2.0 * q.mu * (e[0] - tr3), 2.0 * q.mu * (e[1] - tr3), 2.0 * q.mu * (e[2] - tr3),
                        q.mu * e[3], q.mu * e[4], q.mu * e[5]};
  double gp[3] = {0.0, 0.0, 0.0}, gl[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      gp[d] += p[a] * k.g[a][d];
      gl[d] += lp[a] * k.g[a][d];
    }
  const double ps = q.ps;
  const double pc = ps * 0.25 * (p[0] + p[1] + p[2] + p[3]);
  const double cv = cbrt(k.vol);
  const double tau = cv * cv / (2.0 * q.mu);
  double dR = 0.0;  // lam . dR/dpen
#pragma unroll
  for (int i = 0; i < 6; ++i) dR += k.vol * s1[i] * el[i];
  double st1l = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) st1l += ps * tau * (ps * gp[d] - pic[d]) * gl[d];
  dR += -k.vol * st1l + k.vol * 0.25 * ps * pc / (pen * pen * q.kappa) * (lp[0] + lp[1] + lp[2] + lp[3]);
  rbar[c] += rb + dR * dsimp(k.rho, q.pe, q.pe_min);
  // projected pressure gradient: dR_p,a / dPi_b = V pen ps tau grad N_a / 4
#pragma unroll
  for (int d = 0; d < 3; ++d) pib[d * C + c] = 0.25 * k.vol * pen * ps * tau * gl[d];
}

// nodal sums of a 3-per-cell quantity (component-major) over the cells around each node
__global__ void k_upa_gather3(int64_t N, const int32_t* __restrict__ ptr, const int64_t* __restrict__ adj, int64_t C,
                              const double* __restrict__ v3, double* __restrict__ out) {
  const int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (n >= N) return;
  double r[3] = {0.0, 0.0, 0.0};
  for (int32_t e = ptr[n]; e < ptr[n + 1]; ++e) {
    const int64_t c = adj[e] >> 2;
#pragma unroll
    for (int d = 0; d < 3; ++d) r[d] += v3[d * C + c];
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) out[3 * n + d] = r[d];
}

// W_a = sum over the cells around node a of pen_c V_c (the projection's row sums)
__global__ void k_upa_weights(int64_t N, const int32_t* __restrict__ ptr, const int64_t* __restrict__ adj,
                              const int32_t* __restrict__ cells, const double* __restrict__ coords, UpDev q,
                              const double* __restrict__ z, double* __restrict__ W) {
  const int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (n >= N) return;
  double w = 0.0;
  for (int32_t e = ptr[n]; e < ptr[n + 1]; ++e) {
    const int64_t c = adj[e] >> 2;
    const int4 qv = reinterpret_cast<const int4*>(cells)[c];
    const int v[4] = {qv.x, qv.y, qv.z, qv.w};
    double x[4][3], g[4][3], vol, rho = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
      for (int d = 0; d < 3; ++d) x[k][d] = coords[3 * int64_t(v[k]) + d];
      rho += 0.25 * z[v[k]];
    }
    tet_geometry(x, g, vol);
    w += simp(rho, q.pe, q.pe_min) * vol;
  }
  W[n] = w;
}

// Pullback of the projection Pi_n = Q(p_{n-1}, z) (Pi_a = ps sum_c w_c grad p_c
// / W_a, w_c = pen_c V_c) given its cotangent pib (3N): onto the pressures of
// x_{n-1} (xc, per cell) and rho (rbar, accumulated).
__global__ void k_upa_proj(const int32_t* __restrict__ cells, const double* __restrict__ coords, int64_t C, UpDev q,
                           const double* __restrict__ x, const double* __restrict__ z, const double* __restrict__ pi,
                           const double* __restrict__ W, const double* __restrict__ pib, double* __restrict__ xc,
                           double* __restrict__ rbar) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= C) return;
  UpCell k;
  up_cell_load(cells, coords, x, z, c, k);
  double gp[3] = {0.0, 0.0, 0.0}, S[3] = {0.0, 0.0, 0.0}, rr = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const double pa = x[4 * int64_t(k.v[a]) + 3];
#pragma unroll
    for (int d = 0; d < 3; ++d) gp[d] += pa * k.g[a][d];
  }
  const double ps = q.ps, pen = simp(k.rho, q.pe, q.pe_min), w = pen * k.vol;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const double iw = 1.0 / W[k.v[a]];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double pb = pib[3 * int64_t(k.v[a]) + d];
      S[d] += pb * iw;
      rr += pb * (ps * gp[d] - pi[3 * int64_t(k.v[a]) + d]) * iw;
    }
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
#pragma unroll
    for (int i = 0; i < 3; ++i) xc[(4 * b + i) * C + c] = 0.0;
    xc[(4 * b + 3) * C + c] = ps * w * (k.g[b][0] * S[0] + k.g[b][1] * S[1] + k.g[b][2] * S[2]);
  }
  rbar[c] += rr * dsimp(k.rho, q.pe, q.pe_min) * k.vol;
}

// gradient of the criterion with respect to the nodal controls: rho_c is the
// mean of its four nodes' controls
__global__ void k_upa_nodal(int64_t N, const int32_t* __restrict__ ptr, const int64_t* __restrict__ adj,
                            const double* __restrict__ rbar, double* __restrict__ grad) {
  const int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (n >= N) return;
  double g = 0.0;
  for (int32_t e = ptr[n]; e < ptr[n + 1]; ++e) g += 0.25 * rbar[adj[e] >> 2];
  grad[n] = g;
}

// b = masked ? 0 : -xbar
__global__ void k_upa_rhs(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ xbar,
                          double* __restrict__ b) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    b[i] = up_masked(mask, i >> 2, int(i & 3)) ? 0.0 : -xbar[i];
}

__global__ void k_upa_sum(int64_t n, const double* __restrict__ a, double* __restrict__ partials) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += a[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

int blocks_of(int64_t n, int t) { return int(std::max<int64_t>(1, (n + t - 1) / t)); }
int grid_stride(int64_t n) { return int(std::min<int64_t>(std::max<int64_t>(1, (n + 255) / 256), 148 * 8)); }

struct UpSolver {
  Problem& P;
  cudaStream_t s;
  int64_t N, C, n;
  UpDev q;
  J2Full j;
  const double* z;
  DevBuf<int32_t> ptr, dofs4;
  DevBuf<int64_t> adj;
  DevBuf<uint8_t> mask;
  DevBuf<double> prev, rc, ke, R, ppg, dinv, b, dx, tv, y, partials, scal;
  // MINRES vectors
  DevBuf<double> r1, r2, v, w, w1, w2, yy;
  int64_t nbc = 0;

  UpSolver(Problem& P_, const pa_up_params& up, const pa_j2_params& jp, const double* z_)
      : P(P_), s(P_.stream), N(P_.N()), C(P_.C()), n(4 * P_.N()), q(updev(up)), z(z_) {
    j = J2Full{j2dev(jp), jp.youngs_modulus / (3.0 * (1.0 - 2.0 * jp.poissons_ratio)), 0.0};
    // node -> (cell, vertex) adjacency, cells in increasing order per node
    const Mesh& m = *P.mesh;
    std::vector<int32_t> hcells(size_t(4 * C));
    PA_CUDA(cudaMemcpyAsync(hcells.data(), m.d_cells.get(), sizeof(int32_t) * 4 * C, cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
    std::vector<int32_t> hp(size_t(N + 1), 0);
    for (int64_t k = 0; k < 4 * C; ++k) ++hp[size_t(hcells[size_t(k)]) + 1];
    for (int64_t i = 0; i < N; ++i) hp[size_t(i + 1)] += hp[size_t(i)];
    PA_CHECK(hp[size_t(N)] == 4 * C, "u-p adjacency size");
    std::vector<int64_t> ha(size_t(4 * C));
    std::vector<int32_t> fill(hp.begin(), hp.end() - 1);
    for (int64_t c = 0; c < C; ++c)
      for (int a = 0; a < 4; ++a) ha[size_t(fill[size_t(hcells[size_t(4 * c + a)])]++)] = 4 * c + a;
    ptr.upload(hp.data(), hp.size(), s);
    adj.upload(ha.data(), ha.size(), s);
    // Dirichlet dofs of the problem (3 per node) in the 4-dof numbering
    nbc = int64_t(P.bc_dofs.size());
    std::vector<uint8_t> hm(size_t(N), 0);
    std::vector<int32_t> d4(size_t(std::max<int64_t>(nbc, 1)), 0);
    for (int64_t k = 0; k < nbc; ++k) {
      const int32_t d = P.bc_dofs[size_t(k)];
      d4[size_t(k)] = 4 * (d / 3) + d % 3;
      hm[size_t(d / 3)] |= uint8_t(1u << (d % 3));
    }
    dofs4.upload(d4.data(), d4.size(), s);
    mask.upload(hm.data(), hm.size(), s);
    prev.resize(kLocal * C);
    rc.resize(16 * C);
    ke.resize(256 * C);
    for (DevBuf<double>* bf : {&R, &ppg, &dinv, &b, &dx, &tv, &y, &r1, &r2, &v, &w, &w1, &w2, &yy}) bf->resize(n);
    partials.resize(kRedBlocks);
    scal.resize(1);
  }

  double dot(const double* a, const double* bb, bool masked) {
    k_up_dot<<<kRedBlocks, 256, 0, s>>>(n, a, bb, masked ? mask.get() : nullptr, partials.get());
    k_up_sum<<<1, 256, 0, s>>>(kRedBlocks, partials.get(), scal.get());
    PA_LAUNCHED();
    double h = 0.0;
    PA_CUDA(cudaMemcpyAsync(&h, scal.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
    return h;
  }
  void lin3(double* out, double a, const double* x, double bb, const double* yv, double c, const double* wv) {
    k_up_lin3<<<grid_stride(n), 256, 0, s>>>(n, out, a, x, bb, yv, c, wv);
    PA_LAUNCHED();
  }
  void cells_eval(const double* state, double* cur, bool tangent) {
    k_up_cells<<<blocks_of(C, kUpT), kUpT, 0, s>>>(P.mesh->d_cells.get(), P.mesh->d_coords.get(), C, q, j, state,
                                                   prev.get(), ppg.get(), z, cur, rc.get(),
                                                   tangent ? ke.get() : nullptr);
    k_up_gather<<<blocks_of(N, 128), 128, 0, s>>>(N, ptr.get(), adj.get(), C, rc.get(), R.get());
    PA_LAUNCHED();
  }
  void apply(const double* x, double* yv, bool masked) {
    k_up_apply<<<blocks_of(N, 128), 128, 0, s>>>(N, ptr.get(), adj.get(), P.mesh->d_cells.get(), C, ke.get(),
                                                 masked ? mask.get() : nullptr, x, yv);
    PA_LAUNCHED();
  }
  // ||R|| over the free dofs at `state` (local states to cur)
  double residual(const double* state, double* cur) {
    cells_eval(state, cur, false);
    return std::sqrt(dot(R.get(), R.get(), true));
  }

  // MINRES on the masked tangent: K dx = b; returns iterations (negative: not converged)
  int64_t minres(double rel_tol, int64_t max_iters) {
    PA_CUDA(cudaMemsetAsync(dx.get(), 0, sizeof(double) * n, s));
    double* pr1 = r1.get();
    double* pr2 = r2.get();
    double* py = yy.get();
    double* pw = w.get();
    double* pw1 = w1.get();
    double* pw2 = w2.get();
    PA_CUDA(cudaMemcpyAsync(pr1, b.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    PA_CUDA(cudaMemcpyAsync(pr2, b.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_up_scale<<<grid_stride(n), 256, 0, s>>>(n, dinv.get(), pr1, py);
    PA_LAUNCHED();
    const double b1sq = dot(pr1, py, false);
    PA_CHECK(b1sq >= 0.0, "MINRES: preconditioner not positive definite");
    const double beta1 = std::sqrt(b1sq);
    if (beta1 == 0.0) return 0;
    PA_CUDA(cudaMemsetAsync(pw, 0, sizeof(double) * n, s));
    PA_CUDA(cudaMemsetAsync(pw2, 0, sizeof(double) * n, s));
    double oldb = 0.0, beta = beta1, dbar = 0.0, epsln = 0.0, phibar = beta1, cs = -1.0, sn = 0.0;
    for (int64_t it = 1; it <= max_iters; ++it) {
      const double sc = 1.0 / beta;
      lin3(v.get(), sc, py, 0.0, nullptr, 0.0, nullptr);  // v = y / beta
      apply(v.get(), py, true);                  // y = K v
      if (it >= 2) lin3(py, -beta / oldb, pr1, 1.0, py, 0.0, nullptr);
      const double alfa = dot(v.get(), py, false);
      lin3(py, -alfa / beta, pr2, 1.0, py, 0.0, nullptr);
      std::swap(pr1, pr2);  // r1 <- r2
      std::swap(pr2, py);   // r2 <- y; y takes the old r1's buffer
      k_up_scale<<<grid_stride(n), 256, 0, s>>>(n, dinv.get(), pr2, py);
      PA_LAUNCHED();
      oldb = beta;
      const double bsq = dot(pr2, py, false);
      PA_CHECK(bsq >= 0.0, "MINRES: preconditioner not positive definite");
      beta = std::sqrt(bsq);
      const double oldeps = epsln;
      const double delta = cs * dbar + sn * alfa;
      const double gbar = sn * dbar - cs * alfa;
      epsln = sn * beta;
      dbar = -cs * beta;
      const double gamma = std::max(std::hypot(gbar, beta), 1e-300);
      cs = gbar / gamma;
      sn = beta / gamma;
      const double phi = cs * phibar;
      phibar = sn * phibar;
      // w_new = (v - oldeps w1 - delta w2) / gamma with w1 <- w2, w2 <- w
      std::swap(pw1, pw2);  // w1 <- old w2
      std::swap(pw2, pw);   // w2 <- old w; pw takes the old w1's buffer
      lin3(pw, 1.0 / gamma, v.get(), -oldeps / gamma, pw1, -delta / gamma, pw2);
      lin3(dx.get(), phi, pw, 1.0, dx.get(), 0.0, nullptr);
      if (phibar <= rel_tol * beta1 || beta == 0.0) return it;
    }
    return -max_iters;
  }
};

}  // namespace

// Per-step states kept by the forward solve for the adjoint: state x_n (4N),
// local states c_n (C x 14) and the projected pressure gradient used in step
// n (3N), n = 0 .. steps-1.
struct UpHistory {
  std::vector<DevBuf<double>> x, c, pi;
};

pa_status up_forward(UpSolver& U, const pa_j2_solve_options& jo, const pa_solve_options& lo, double* state,
                     double* local, UpHistory* hist, pa_j2_stats* js) {
  Problem& P = U.P;
  const double* z = U.z;
  cudaStream_t s = U.s;
  const int64_t n = U.n, C = U.C;
  PA_CUDA(cudaMemsetAsync(state, 0, sizeof(double) * n, s));
  PA_CUDA(cudaMemsetAsync(U.prev.get(), 0, sizeof(double) * kLocal * C, s));
  PA_CUDA(cudaMemsetAsync(U.ppg.get(), 0, sizeof(double) * 3 * U.N, s));
  cudaEvent_t t0, t1;
  PA_CUDA(cudaEventCreate(&t0));
  PA_CUDA(cudaEventCreate(&t1));
  PA_CUDA(cudaEventRecord(t0, s));
  const double lin_tol = lo.rel_tol > 0 ? lo.rel_tol : 1e-12;
  const int64_t lin_max = lo.max_iters > 0 ? lo.max_iters : 100000;
  int newton_total = 0, linear_unconverged = 0, halvings = 0;
  int64_t lin_total = 0;
  bool all_converged = true;
  double worst_rel = 0.0;
  pa_status status = PA_OK;
  auto set_bc = [&](double scale, double* x) {
    if (U.nbc) {
      k_up_set<<<blocks_of(U.nbc, 256), 256, 0, s>>>(U.nbc, U.dofs4.get(), P.d_bc_vals.get(), scale, x);
      PA_LAUNCHED();
    }
  };
  // tangent at `state`, then K dx = -R with dx = inc x (Dirichlet values) on the constrained dofs
  auto tangent_solve = [&](double inc) {
    U.cells_eval(state, local, true);
    k_up_dinv<<<blocks_of(U.N, 128), 128, 0, s>>>(U.N, U.ptr.get(), U.adj.get(), C, U.ke.get(), U.mask.get(),
                                                   U.dinv.get());
    PA_CUDA(cudaMemsetAsync(U.tv.get(), 0, sizeof(double) * n, s));
    set_bc(inc, U.tv.get());
    if (inc != 0.0)
      U.apply(U.tv.get(), U.y.get(), false);
    else
      PA_CUDA(cudaMemsetAsync(U.y.get(), 0, sizeof(double) * n, s));
    k_up_rhs<<<grid_stride(n), 256, 0, s>>>(n, U.mask.get(), U.tv.get(), U.R.get(), U.y.get(), U.b.get());
    PA_LAUNCHED();
    const int64_t its = U.minres(lin_tol, lin_max);
    lin_total += its < 0 ? -its : its;
    if (its < 0) ++linear_unconverged;
    ++newton_total;
  };
  auto add_dx = [&](double a) { U.lin3(state, a, U.dx.get(), 1.0, state, 0.0, nullptr); };
  for (int step = 0; step < jo.steps && status == PA_OK; ++step) {
    const double s_old = double(step) / jo.steps, s_new = double(step + 1) / jo.steps;
    // reference norm: the residual with the new boundary values on the last converged field
    set_bc(s_new, state);
    const double r0 = U.residual(state, local);
    if (!std::isfinite(r0)) { status = PA_ERR_NONFINITE; break; }
    set_bc(s_old, state);
    // first iteration: tangent at the converged state, the Dirichlet increment imposed in the solve
    tangent_solve(s_new - s_old);
    add_dx(1.0);
    constexpr int kMaxHalvings = 5;
    bool converged = false;
    double rn = U.residual(state, local), last_rel = 0.0;
    for (int it = 0; it < jo.max_newton; ++it) {
      if (!std::isfinite(rn)) { status = PA_ERR_NONFINITE; break; }
      last_rel = r0 > 0.0 ? rn / r0 : 0.0;
      if (rn <= jo.newton_tol * r0 || rn == 0.0) { converged = true; break; }
      tangent_solve(0.0);
      double a = 1.0;
      add_dx(a);
      double rt = U.residual(state, local);
      for (int h = 0; h < kMaxHalvings && !(rt <= (1.0 - 1e-4 * a) * rn); ++h) {
        a *= 0.5;
        add_dx(-a);
        rt = U.residual(state, local);
        ++halvings;
      }
      rn = rt;
    }
    if (status != PA_OK) break;
    if (!converged) {
      all_converged = false;
      last_rel = r0 > 0.0 ? rn / r0 : 0.0;
    }
    worst_rel = std::max(worst_rel, last_rel);
    // the local states of the accepted iterate, then the next step's projection
    U.residual(state, local);
    PA_CUDA(cudaMemcpyAsync(U.prev.get(), local, sizeof(double) * kLocal * C, cudaMemcpyDeviceToDevice, s));
    if (hist) {
      hist->x.emplace_back();
      hist->c.emplace_back();
      hist->pi.emplace_back();
      hist->x.back().resize(n);
      hist->c.back().resize(kLocal * C);
      hist->pi.back().resize(3 * U.N);
      PA_CUDA(cudaMemcpyAsync(hist->x.back().get(), state, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      PA_CUDA(cudaMemcpyAsync(hist->c.back().get(), local, sizeof(double) * kLocal * C, cudaMemcpyDeviceToDevice, s));
      PA_CUDA(cudaMemcpyAsync(hist->pi.back().get(), U.ppg.get(), sizeof(double) * 3 * U.N, cudaMemcpyDeviceToDevice,
                              s));
    }
    if (step + 1 < jo.steps) {
      k_up_project<<<blocks_of(U.N, 128), 128, 0, s>>>(U.N, U.ptr.get(), U.adj.get(), P.mesh->d_cells.get(),
                                                      P.mesh->d_coords.get(), U.q, state, z, U.ppg.get());
      PA_LAUNCHED();
    }
  }
  PA_CUDA(cudaEventRecord(t1, s));
  PA_CUDA(cudaEventSynchronize(t1));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (js) {
    js->steps = jo.steps;
    js->newton_iterations = newton_total;
    js->cg_iterations = lin_total;
    js->seconds = ms * 1e-3;
    js->final_rel_residual = worst_rel;
    js->linear_unconverged = linear_unconverged;
    js->line_search_halvings = halvings;
    js->converged = all_converged ? 1 : 0;
  }
  if (status != PA_OK) return status;
  return all_converged ? PA_OK : PA_ERR_NOT_CONVERGED;
}

pa_status up_solve(Problem& P, const pa_up_params& up, const pa_j2_params& jp, const double* z,
                   const pa_j2_solve_options& jo, const pa_solve_options& lo, double* state, double* local,
                   double* ppg_out, pa_j2_stats* js) {
  PA_CHECK(jo.steps > 0 && jo.max_newton > 0 && jo.newton_tol > 0, "u-p solve options out of range");
  PA_CHECK(P.C() < (int64_t(1) << 29) && 4 * P.C() < (int64_t(1) << 31), "u-p solve: mesh too large");
  UpSolver U(P, up, jp, z);
  const pa_status st = up_forward(U, jo, lo, state, local, nullptr, js);
  if (ppg_out)
    PA_CUDA(cudaMemcpyAsync(ppg_out, U.ppg.get(), sizeof(double) * 3 * U.N, cudaMemcpyDeviceToDevice, U.s));
  PA_CUDA(cudaStreamSynchronize(U.s));
  return st;
}

// "Elastic Work" (ElasticWorkCriterion summed over the load steps by
// PlasticityProblem::evaluateCriterion, src/PlasticityProblem.hpp:929-953)
// and its gradient with respect to the nodal controls by the path-dependent
// adjoint (PathDependentAdjointSolver, src/PathDependentAdjointSolver.hpp:
// 154-940).  The steps' elastic work V (sigma_n + sigma_{n-1}) . (e_n -
// e_{n-1}) / 2 telescopes (sigma = C e, C symmetric) to the last step's
// stored energy V e_S . C e_S / 2.  The reverse sweep runs the steps
// backwards with the cotangents of x_n (xbar) and c_n (cbar):
//   c_n = Phi(eps(x_n), c_{n-1}, rho): xbar_n += B^T dPhi/deps^T cbar_n;
//   x_n solves R(x_n, Phi(..), Pi_n, rho) = 0: K_n lam_n = -xbar_n (free
//     dofs; K_n the condensed tangent, symmetric), then cbar_{n-1} =
//     dPhi/dc_{n-1}^T (cbar_n + dR/dc_n^T lam_n), rhobar += the rho parts,
//     Pibar_n = dR/dPi^T lam_n;
//   Pi_n = Q(p_{n-1}, rho) (n > 0): xbar_{n-1} = dQ/dp^T Pibar_n, rhobar +=.
// The reference solves the same reverse recurrence with the local adjoint
// kept as an unknown (its local residual H is zero at the returned state, so
// eliminating it through Phi gives the same gradient).
pa_status up_elastic_work(Problem& P, const pa_up_params& up, const pa_j2_params& jp, double fpe, double fpmin,
                          const double* z, const pa_j2_solve_options& jo, const pa_solve_options& lo, double* value,
                          double* grad, double* state, double* local, pa_j2_stats* js) {
  PA_CHECK(jo.steps > 0 && jo.max_newton > 0 && jo.newton_tol > 0, "u-p solve options out of range");
  PA_CHECK(P.C() < (int64_t(1) << 29) && 4 * P.C() < (int64_t(1) << 31), "u-p solve: mesh too large");
  PA_CHECK(fpmin >= 0.0 && fpmin < 1.0, "criterion penalty minimum out of range");
  UpSolver U(P, up, jp, z);
  UpHistory H;
  const pa_status fst = up_forward(U, jo, lo, state, local, &H, js);
  if (fst != PA_OK) return fst;
  cudaStream_t s = U.s;
  const int64_t N = U.N, C = U.C, n = U.n;
  const int S = int(H.x.size());
  const double lin_tol = lo.rel_tol > 0 ? lo.rel_tol : 1e-12;
  const int64_t lin_max = lo.max_iters > 0 ? lo.max_iters : 100000;
  const int32_t* cells = P.mesh->d_cells.get();
  const double* coords = P.mesh->d_coords.get();
  DevBuf<double> fcell(C), xc(16 * C), xbar(n), cb_cur(kLocal * C), cb_prev(kLocal * C), rbar(C), pib(3 * C),
      pibn(3 * N), W(N), zeros(kLocal * C), scratch(kLocal * C);
  PA_CUDA(cudaMemsetAsync(zeros.get(), 0, sizeof(double) * kLocal * C, s));
  const int cb = blocks_of(C, kUpT), nb = blocks_of(N, 128);
  // the criterion at the last step and its partials
  k_upa_final<<<cb, kUpT, 0, s>>>(cells, coords, C, U.q, fpe, fpmin, H.x[S - 1].get(), H.c[S - 1].get(), z,
                                  fcell.get(), xc.get(), cb_cur.get(), rbar.get());
  k_upa_sum<<<kRedBlocks, 256, 0, s>>>(C, fcell.get(), U.partials.get());
  k_up_sum<<<1, 256, 0, s>>>(kRedBlocks, U.partials.get(), U.scal.get());
  k_up_gather<<<nb, 128, 0, s>>>(N, U.ptr.get(), U.adj.get(), C, xc.get(), xbar.get(), 0);
  PA_LAUNCHED();
  PA_CUDA(cudaMemcpyAsync(value, U.scal.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
  k_upa_weights<<<nb, 128, 0, s>>>(N, U.ptr.get(), U.adj.get(), cells, coords, U.q, z, W.get());
  PA_LAUNCHED();
  int64_t lin_total = 0;
  int lin_unconverged = 0;
  for (int k = S - 1; k >= 0; --k) {
    const double* prevc = k > 0 ? H.c[k - 1].get() : zeros.get();
    // c_k = Phi(eps(x_k), c_{k-1}, rho): onto x_k
    k_upa_phi_eps<<<cb, kUpT, 0, s>>>(cells, coords, C, U.j.p, H.x[k].get(), prevc, z, cb_cur.get(), xc.get());
    k_up_gather<<<nb, 128, 0, s>>>(N, U.ptr.get(), U.adj.get(), C, xc.get(), xbar.get(), 1);
    PA_LAUNCHED();
    // adjoint of step k with its converged tangent
    PA_CUDA(cudaMemcpyAsync(U.prev.get(), prevc, sizeof(double) * kLocal * C, cudaMemcpyDeviceToDevice, s));
    PA_CUDA(cudaMemcpyAsync(U.ppg.get(), H.pi[k].get(), sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, s));
    U.cells_eval(H.x[k].get(), scratch.get(), true);
    k_up_dinv<<<nb, 128, 0, s>>>(N, U.ptr.get(), U.adj.get(), C, U.ke.get(), U.mask.get(), U.dinv.get());
    k_upa_rhs<<<grid_stride(n), 256, 0, s>>>(n, U.mask.get(), xbar.get(), U.b.get());
    PA_LAUNCHED();
    const int64_t its = U.minres(lin_tol, lin_max);
    lin_total += its < 0 ? -its : its;
    if (its < 0) ++lin_unconverged;
    k_upa_resid<<<cb, kUpT, 0, s>>>(cells, coords, C, U.q, U.j.p, H.x[k].get(), prevc, H.c[k].get(), H.pi[k].get(), z,
                                    U.dx.get(), cb_cur.get(), cb_prev.get(), rbar.get(), pib.get());
    PA_LAUNCHED();
    PA_CUDA(cudaMemsetAsync(xbar.get(), 0, sizeof(double) * n, s));
    if (k > 0) {  // Pi_k = Q(p_{k-1}): onto x_{k-1}
      k_upa_gather3<<<nb, 128, 0, s>>>(N, U.ptr.get(), U.adj.get(), C, pib.get(), pibn.get());
      k_upa_proj<<<cb, kUpT, 0, s>>>(cells, coords, C, U.q, H.x[k - 1].get(), z, H.pi[k].get(), W.get(), pibn.get(),
                                     xc.get(), rbar.get());
      k_up_gather<<<nb, 128, 0, s>>>(N, U.ptr.get(), U.adj.get(), C, xc.get(), xbar.get(), 0);
      PA_LAUNCHED();
    }
    std::swap(cb_cur.p, cb_prev.p);
  }
  k_upa_nodal<<<nb, 128, 0, s>>>(N, U.ptr.get(), U.adj.get(), rbar.get(), grad);
  PA_LAUNCHED();
  PA_CUDA(cudaStreamSynchronize(s));
  if (js) {
    js->cg_iterations += lin_total;
    js->linear_unconverged += lin_unconverged;
  }
  return lin_unconverged ? PA_ERR_NOT_CONVERGED : PA_OK;
}

}  // namespace pa
