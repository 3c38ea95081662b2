// pa_j2.cu -- per-cell J2 radial return (FP64).
//
// J2PlasticityLocalResidual::updateLocalState
// (src/J2PlasticityLocalResidual.hpp:421-523) for the displacement-only
// small-strain form: elastic trial state, yield check, closed-form plastic
// multiplier for linear isotropic/kinematic hardening, and the plastic strain
// and backstress updates.  The reference runs this as a Kokkos lambda with
// six DRAM work arrays per cell; here the whole update stays in registers and
// the 14-double local states are staged through shared memory so that both
// the load of the previous state and the store of the new one are coalesced.
#include "pa_problem.cuh"
#include <algorithm>
#include <cmath>

#include "pa_cell.cuh"
#include "pa_plastic.cuh"

namespace pa {

namespace {

constexpr int kJ2Threads = 128;

__global__ void __launch_bounds__(kJ2Threads) k_j2(const int32_t* __restrict__ cells, const double* __restrict__ coords,
                                                   int64_t C, J2Dev p, const double* __restrict__ u,
                                                   const double* __restrict__ z, const double* __restrict__ prev,
                                                   double* __restrict__ cur) {
  __shared__ double s_state[kJ2Threads * kLocal];
  const int64_t c0 = int64_t(blockIdx.x) * kJ2Threads;
  const int nloc = int((C - c0) < int64_t(kJ2Threads) ? (C - c0) : int64_t(kJ2Threads));
  // coalesced load of the block's previous local states
  for (int i = threadIdx.x; i < nloc * kLocal; i += kJ2Threads) s_state[i] = prev[c0 * kLocal + i];
  __syncthreads();
  if (threadIdx.x < nloc) {
    const int64_t c = c0 + threadIdx.x;
    const int4 q = reinterpret_cast<const int4*>(cells)[c];
    const int v[4] = {q.x, q.y, q.z, q.w};
    double x[4][3], ue[12], g[4][3], vol, e[6];
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        x[n][d] = __ldg(&coords[3 * int64_t(v[n]) + d]);
        ue[3 * n + d] = __ldg(&u[3 * int64_t(v[n]) + d]);
      }
    tet_geometry(x, g, vol);
    tet_strain(g, ue, e);
    double* st = s_state + threadIdx.x * kLocal;
    const double eqps_prev = st[0];
    // elastic strain = total - plastic (src/ThermoPlasticityUtilities.hpp:101-121)
    double ee[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) ee[i] = e[i] - st[2 + i];
    // cell density = mean of nodal controls (src/Plato_TopOptFunctors.hpp:52-63)
    const double rho = 0.25 * (__ldg(&z[v[0]]) + __ldg(&z[v[1]]) + __ldg(&z[v[2]]) + __ldg(&z[v[3]]));
    const double mu_p = simp(rho, p.pe, p.pe_min) * p.mu;
    // deviatoric stress (src/ComputeDeviatoricStress.hpp:110-130)
    const double tr3 = (ee[0] + ee[1] + ee[2]) / 3.0;
    double n[6] = {2.0 * mu_p * (ee[0] - tr3), 2.0 * mu_p * (ee[1] - tr3), 2.0 * mu_p * (ee[2] - tr3),
                   mu_p * ee[3], mu_p * ee[4], mu_p * ee[5]};
    // eta = s - backstress and its norm, shear terms counted twice
    // (src/J2PlasticityUtilities.hpp:378-407)
#pragma unroll
    for (int i = 0; i < 6; ++i) n[i] -= st[8 + i];
    const double norm =
        sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + 2.0 * (n[3] * n[3] + n[4] * n[4] + n[5] * n[5]));
    const double ppen = simp(rho, p.pp, p.pp_min);
    const double hi = ppen * p.hiso, hk = ppen * p.hkin;
    const double sy = ppen * p.sy0 + hi * eqps_prev;
    const double s32 = 1.2247448713915890491;   // sqrt(3/2)
    const double s23 = 0.81649658092772603273;  // sqrt(2/3)
    const double ftr = s32 * norm - sy;
    st[1] = 0.0;
    if (ftr > 1.0e-10) {  // plastic step (src/J2PlasticityLocalResidual.hpp:509-520)
      const double dg = ftr / (3.0 * mu_p + hi + hk);
      st[1] = dg;
      st[0] = eqps_prev + dg;
      const double inv = 1.0 / norm;
      const double m1 = dg * s32 * inv, m2 = dg * s23 * hk * inv;
      // plastic strain and backstress (src/J2PlasticityUtilities.hpp:250-273)
#pragma unroll
      for (int i = 0; i < 3; ++i) st[2 + i] += m1 * n[i];
#pragma unroll
      for (int i = 3; i < 6; ++i) st[2 + i] += 2.0 * m1 * n[i];
#pragma unroll
      for (int i = 0; i < 6; ++i) st[8 + i] += m2 * n[i];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nloc * kLocal; i += kJ2Threads) cur[c0 * kLocal + i] = s_state[i];
}

// Newton residual of the displacement form: R += vol B^T sigma(u) after the
// return mapping from `prev`; writes the new local states, the per-cell tangent
// records and elastic penalties in tile order (FP64 and FP32).
__global__ void __launch_bounds__(kJ2Threads) k_j2_newton(const int32_t* __restrict__ cells,
                                                          const double* __restrict__ coords, int64_t C, J2Full q,
                                                          const double* __restrict__ u, const double* __restrict__ z,
                                                          const double* __restrict__ prev, double* __restrict__ cur,
                                                          const int32_t* __restrict__ iperm, double* __restrict__ rec64,
                                                          float* __restrict__ rec32, double* __restrict__ w64,
                                                          float* __restrict__ w32, double* __restrict__ R) {
  __shared__ double s_state[kJ2Threads * kLocal];
  const int64_t c0 = int64_t(blockIdx.x) * kJ2Threads;
  const int nloc = int((C - c0) < int64_t(kJ2Threads) ? (C - c0) : int64_t(kJ2Threads));
  for (int i = threadIdx.x; i < nloc * kLocal; i += kJ2Threads) s_state[i] = prev[c0 * kLocal + i];
  __syncthreads();
  if (threadIdx.x < nloc) {
    const int64_t c = c0 + threadIdx.x;
    const int4 qv = reinterpret_cast<const int4*>(cells)[c];
    const int v[4] = {qv.x, qv.y, qv.z, qv.w};
    double x[4][3], ue[12], g[4][3], vol, e[6], sig[6], rec[8], pe, re[12];
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        x[n][d] = __ldg(&coords[3 * int64_t(v[n]) + d]);
        ue[3 * n + d] = __ldg(&u[3 * int64_t(v[n]) + d]);
      }
    tet_geometry(x, g, vol);
    tet_strain(g, ue, e);
    const double rho = 0.25 * (__ldg(&z[v[0]]) + __ldg(&z[v[1]]) + __ldg(&z[v[2]]) + __ldg(&z[v[3]]));
    j2_cell(q, rho, e, s_state + threadIdx.x * kLocal, sig, rec, pe);
#pragma unroll
    for (int i = 0; i < 6; ++i) sig[i] *= vol;
    tet_divergence(g, sig, re);
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int d = 0; d < 3; ++d) atomicAdd(&R[3 * int64_t(v[n]) + d], re[3 * n + d]);
    const int64_t ic = iperm[c];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      rec64[8 * ic + i] = rec[i];
      rec32[8 * ic + i] = float(rec[i]);
    }
    w64[ic] = pe;
    w32[ic] = float(pe);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nloc * kLocal; i += kJ2Threads) cur[c0 * kLocal + i] = s_state[i];
}

// Jacobi diagonal of the consistent tangent: for node a and direction i,
// vol * eps_ai^T C_ep eps_ai with eps_ai = B_a e_i.
__global__ void k_j2_diag(const int32_t* __restrict__ cells, const double* __restrict__ coords, int64_t C, J2Full q,
                          const int32_t* __restrict__ iperm, const double* __restrict__ rec64,
                          const double* __restrict__ w64, double* __restrict__ diag) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= C) return;
  const int4 qv = reinterpret_cast<const int4*>(cells)[c];
  const int v[4] = {qv.x, qv.y, qv.z, qv.w};
  double x[4][3], g[4][3], vol;
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int d = 0; d < 3; ++d) x[n][d] = __ldg(&coords[3 * int64_t(v[n]) + d]);
  tet_geometry(x, g, vol);
  const int64_t ic = iperm[c];
  const double* r = rec64 + 8 * ic;
  const double pe = w64[ic];
  const double mu = q.p.mu, k = q.kappa, t1 = r[6], t2 = r[7];
  for (int n = 0; n < 4; ++n)
    for (int i = 0; i < 3; ++i) {
      double e[6] = {0, 0, 0, 0, 0, 0};
      e[i] = g[n][i];
      if (i == 0) { e[4] = g[n][2]; e[5] = g[n][1]; }
      if (i == 1) { e[3] = g[n][2]; e[5] = g[n][0]; }
      if (i == 2) { e[3] = g[n][1]; e[4] = g[n][0]; }
      const double tr = e[0] + e[1] + e[2], m = tr / 3.0;
      const double ne = r[0] * e[0] + r[1] * e[1] + r[2] * e[2] + r[3] * e[3] + r[4] * e[4] + r[5] * e[5];
      const double ma = mu * (1.0 - t1), b = 2.0 * mu * (t2 - t1);
      double val = k * tr * tr;
      for (int j = 0; j < 3; ++j) val += (2.0 * ma * (e[j] - m) - b * ne * r[j]) * e[j];
      for (int j = 3; j < 6; ++j) val += (ma * e[j] - b * ne * r[j]) * e[j];
      atomicAdd(&diag[3 * int64_t(v[n]) + i], pe * vol * val);
    }
}

// J2PlasticityLocalResidual::evaluate (src/J2PlasticityLocalResidual.hpp:291-409):
// the 14 local residual equations of each cell at the given states.
__global__ void k_j2_local_residual(const int32_t* __restrict__ cells, const double* __restrict__ coords, int64_t C,
                                    J2Dev p, const double* __restrict__ u, const double* __restrict__ z,
                                    const double* __restrict__ loc, const double* __restrict__ prev,
                                    double* __restrict__ H) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= C) return;
  const int4 qv = reinterpret_cast<const int4*>(cells)[c];
  const int v[4] = {qv.x, qv.y, qv.z, qv.w};
  double x[4][3], ue[12], g[4][3], vol, e[6];
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      x[n][d] = coords[3 * int64_t(v[n]) + d];
      ue[3 * n + d] = u[3 * int64_t(v[n]) + d];
    }
  tet_geometry(x, g, vol);
  tet_strain(g, ue, e);
  const double* L = loc + 14 * c;
  const double* Pv = prev + 14 * c;
  double* h = H + 14 * c;
  const double rho = 0.25 * (z[v[0]] + z[v[1]] + z[v[2]] + z[v[3]]);
  const double mu_p = simp(rho, p.pe, p.pe_min) * p.mu;
  const double ppen = simp(rho, p.pp, p.pp_min);
  const double hi = ppen * p.hiso, hk = ppen * p.hkin;
  double ee[6];
  for (int i = 0; i < 6; ++i) ee[i] = e[i] - L[2 + i];
  const double tr3 = (ee[0] + ee[1] + ee[2]) / 3.0;
  double n[6] = {2.0 * mu_p * (ee[0] - tr3), 2.0 * mu_p * (ee[1] - tr3), 2.0 * mu_p * (ee[2] - tr3),
                 mu_p * ee[3], mu_p * ee[4], mu_p * ee[5]};
  for (int i = 0; i < 6; ++i) n[i] -= L[8 + i];
  const double norm = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + 2.0 * (n[3] * n[3] + n[4] * n[4] + n[5] * n[5]));
  const double s32 = 1.2247448713915890491, s23 = 0.81649658092772603273;
  h[0] = L[0] - Pv[0];
  h[1] = L[1];
  for (int i = 2; i < 14; ++i) h[i] = L[i] - Pv[i];
  if (L[1] > 0.0) {
    const double inv = 1.0 / norm;
    h[0] = L[0] - Pv[0] - L[1];
    h[1] = s32 * norm - (ppen * p.sy0 + hi * L[0]);
    for (int i = 0; i < 3; ++i) h[2 + i] = L[2 + i] - Pv[2 + i] - s32 * L[1] * n[i] * inv;
    for (int i = 3; i < 6; ++i) h[2 + i] = L[2 + i] - Pv[2 + i] - 2.0 * s32 * L[1] * n[i] * inv;
    for (int i = 0; i < 6; ++i) h[8 + i] = L[8 + i] - Pv[8 + i] - s23 * L[1] * hk * n[i] * inv;
  }
}

__global__ void k_set_dofs(int64_t n, const int32_t* __restrict__ dofs, const double* __restrict__ vals, double scale,
                           double* __restrict__ u) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) u[dofs[i]] = scale * vals[i];
}

__global__ void k_axpy_neg_masked(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ R,
                                  double* __restrict__ b, double* __restrict__ sumsq) {
  double acc = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const bool c = mask && ((mask[i / 3] >> (i % 3)) & 1);
    const double v = c ? 0.0 : -R[i];
    b[i] = v;
    acc += v * v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(sumsq, acc);
}

__global__ void k_add(int64_t n, const double* __restrict__ d, double* __restrict__ u, double a) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    u[i] += a * d[i];
}

}  // namespace

void launch_j2(const Problem& P, const pa_j2_params& jp, const double* u, const double* z, const double* prev,
               double* cur, cudaStream_t s) {
  const J2Dev p = j2dev(jp);
  const int64_t C = P.C();
  const int grid = int((C + kJ2Threads - 1) / kJ2Threads);
  k_j2<<<grid, kJ2Threads, 0, s>>>(P.mesh->d_cells.get(), P.mesh->d_coords.get(), C, p, u, z, prev, cur);
  PA_LAUNCHED();
}

// Stabilized u-p plasticity residual, InfinitesimalStrainPlasticityResidual::
// evaluate (src/InfinitesimalStrainPlasticityResidual.hpp:398-516): 4 dofs per
// node (u_x, u_y, u_z, p); elastic strain e = eps(u) - eps_p (local state
// 2..7); deviatoric stress s = 2 mu_p dev(e) (shears mu_p gamma); displacement
// rows V (s + ps p_c 1) grad N; pressure rows -V stab . grad N + V N theta with
// theta = ps (tr eps - ps p_c / kappa_p), stab = pen ps tau (ps grad p - Pi),
// tau = V^(2/3) / (2 mu) (src/ComputeStabilization.hpp:93-108); p_c and Pi
// (projected pressure gradient) interpolated with the one-point basis (1/4).
// Pi is per node (ppg_per_cell = 0: 3N) or per cell node (1: C x 12).  Output
// per cell (C x 16, node-major) or assembled (4N, atomics).
__global__ void k_up_residual(const int32_t* __restrict__ cells, const double* __restrict__ coords, int64_t C,
                              UpDev q, const double* __restrict__ state, const double* __restrict__ local,
                              const double* __restrict__ ppg, int ppg_per_cell, const double* __restrict__ z,
                              double* __restrict__ out, int assemble) {
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
      pi[d] += 0.25 * (ppg_per_cell ? ppg[12 * c + 3 * n + d] : ppg[3 * int64_t(v[n]) + d]);
    }
    p[n] = state[4 * int64_t(v[n]) + 3];
    rho += 0.25 * z[v[n]];
  }
  tet_geometry(x, g, vol);
  tet_strain(g, ue, eps);
  const double* L = local + 14 * c;
  double e[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) e[i] = eps[i] - L[2 + i];
  const double pen = simp(rho, q.pe, q.pe_min);
  const double mu_p = pen * q.mu, kappa_p = pen * q.kappa;
  const double tr3 = (e[0] + e[1] + e[2]) * (1.0 / 3.0);
  const double sv[6] = {2.0 * mu_p * (e[0] - tr3), 2.0 * mu_p * (e[1] - tr3), 2.0 * mu_p * (e[2] - tr3),
                        mu_p * e[3], mu_p * e[4], mu_p * e[5]};
  double gp[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int d = 0; d < 3; ++d) gp[d] += p[n] * g[n][d];
  const double pc = q.ps * 0.25 * (p[0] + p[1] + p[2] + p[3]);
  const double theta = q.ps * (eps[0] + eps[1] + eps[2] - pc / kappa_p);
  const double cv = cbrt(vol);
  const double tau = cv * cv / (2.0 * q.mu);
  double stab[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) stab[d] = pen * q.ps * tau * (q.ps * gp[d] - pi[d]);
  // stress rows: V (s + pc 1) grad N
  const double S[3][3] = {{sv[0] + pc, sv[5], sv[4]}, {sv[5], sv[1] + pc, sv[3]}, {sv[4], sv[3], sv[2] + pc}};
  double r[16];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
#pragma unroll
    for (int i = 0; i < 3; ++i) r[4 * n + i] = vol * (S[i][0] * g[n][0] + S[i][1] * g[n][1] + S[i][2] * g[n][2]);
    r[4 * n + 3] = -vol * (stab[0] * g[n][0] + stab[1] * g[n][1] + stab[2] * g[n][2]) + vol * 0.25 * theta;
  }
  if (assemble) {
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int k = 0; k < 4; ++k) atomicAdd(&out[4 * int64_t(v[n]) + k], r[4 * n + k]);
  } else {
#pragma unroll
    for (int k = 0; k < 16; ++k) out[16 * c + k] = r[k];
  }
}

void launch_up_residual(const Problem& P, const pa_up_params& up, const double* state, const double* local,
                        const double* ppg, int ppg_per_cell, const double* z, double* out, int assemble,
                        cudaStream_t s) {
  const int64_t C = P.C();
  const double mu = up.youngs_modulus / (2.0 * (1.0 + up.poissons_ratio));
  const double kappa = up.youngs_modulus / (3.0 * (1.0 - 2.0 * up.poissons_ratio));
  const UpDev q{mu, kappa, up.penalty_exponent, up.penalty_min, up.pressure_scaling};
  if (assemble) PA_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 4 * P.N(), s));
  k_up_residual<<<int((C + 127) / 128), 128, 0, s>>>(P.mesh->d_cells.get(), P.mesh->d_coords.get(), C, q, state,
                                                     local, ppg, ppg_per_cell, z, out, assemble);
  PA_LAUNCHED();
}

void launch_j2_local_residual(const Problem& P, const pa_j2_params& jp, const double* u, const double* z,
                              const double* loc, const double* prev, double* H, cudaStream_t s) {
  const int64_t C = P.C();
  k_j2_local_residual<<<int((C + 127) / 128), 128, 0, s>>>(P.mesh->d_cells.get(), P.mesh->d_coords.get(), C, j2dev(jp),
                                                           u, z, loc, prev, H);
  PA_LAUNCHED();
}

pa_status solve_operator(Problem& P, const SolveOperator& op, const double* b, double* x_out,
                         const pa_solve_options& o, pa_solve_stats* st, bool record_start);

// Displacement-form small-strain J2 problem by pseudo-time load stepping and
// Newton's method.  The reference's driver is NewtonRaphsonSolver::solve
// (src/NewtonRaphsonSolver.hpp:570-640) over PlasticityProblem's load steps
// (src/PlasticityProblem.hpp:791-846): Dirichlet values ramp linearly, each
// Newton iteration performs the radial return from the last converged local
// state, assembles the residual and solves with the consistent tangent.
// Here the tangent is applied matrix-free (tile kernel, J2 records) inside the
// problem's PCG (FP32 apply + FP64 true residual in mixed mode).
pa_status j2_solve(Problem& P, const pa_j2_params& jp, const double* z, const pa_j2_solve_options& jo,
                   const pa_solve_options& lo, double* u, double* local, pa_j2_stats* js) {
  cudaStream_t s = P.stream;
  const int64_t C = P.C(), n = P.ndof();
  const J2Full q{j2dev(jp), jp.youngs_modulus / (3.0 * (1.0 - 2.0 * jp.poissons_ratio)),
                 jp.youngs_modulus * jp.poissons_ratio / ((1.0 + jp.poissons_ratio) * (1.0 - 2.0 * jp.poissons_ratio))};
  PA_CHECK(jo.steps > 0 && jo.max_newton > 0 && jo.newton_tol > 0, "J2 solve options out of range");
  // tile kernel material: lambda, mu of the elastic law; penalties per cell
  ElasticParams saved = P.ep;
  P.ep.E = jp.youngs_modulus;
  P.ep.nu = jp.poissons_ratio;
  DevBuf<double> prev(14 * C), rec64(8 * C), w64(C), R(n), b(n), du(n), diag(n), sumsq(1);
  DevBuf<float> rec32(8 * C), w32(C);
  PA_CUDA(cudaMemsetAsync(u, 0, sizeof(double) * n, s));
  PA_CUDA(cudaMemsetAsync(prev.get(), 0, sizeof(double) * 14 * C, s));
  if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
  cudaEvent_t t0, t1;
  PA_CUDA(cudaEventCreate(&t0));
  PA_CUDA(cudaEventCreate(&t1));
  PA_CUDA(cudaEventRecord(t0, s));
  const int64_t nbc = int64_t(P.bc_dofs.size());
  const int grid = int((C + kJ2Threads - 1) / kJ2Threads);
  int newton_total = 0;
  int64_t cg_total = 0;
  bool all_converged = true;
  double last_rel = 0.0, worst_rel = 0.0;
  int linear_unconverged = 0, line_search_halvings = 0;
  pa_status status = PA_OK;
  // residual (and tangent records) at u; b = -R on the free dofs; returns ||R_free||
  auto residual = [&]() {
    PA_CUDA(cudaMemsetAsync(R.get(), 0, sizeof(double) * n, s));
    k_j2_newton<<<grid, kJ2Threads, 0, s>>>(P.mesh->d_cells.get(), P.mesh->d_coords.get(), C, q, u, z, prev.get(),
                                           local, P.mesh->d_cell_iperm.get(), rec64.get(), rec32.get(), w64.get(),
                                           w32.get(), R.get());
    PA_LAUNCHED();
    PA_CUDA(cudaMemsetAsync(sumsq.get(), 0, sizeof(double), s));
    k_axpy_neg_masked<<<int(std::min<int64_t>((n + 255) / 256, 148 * 8)), 256, 0, s>>>(
        n, P.d_node_mask.get(), R.get(), b.get(), sumsq.get());
    PA_LAUNCHED();
    double h = 0.0;
    PA_CUDA(cudaMemcpyAsync(&h, sumsq.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(h);
  };
  // K_T du = -R with the tangent of the last residual evaluation; Dirichlet
  // values of du: bc_scale x the problem's (0: homogeneous)
  auto tangent_solve = [&](double bc_scale, double eta) {
    PA_CUDA(cudaMemsetAsync(diag.get(), 0, sizeof(double) * n, s));
    k_j2_diag<<<int((C + 127) / 128), 128, 0, s>>>(P.mesh->d_cells.get(), P.mesh->d_coords.get(), C, q,
                                                  P.mesh->d_cell_iperm.get(), rec64.get(), w64.get(), diag.get());
    PA_LAUNCHED();
    SolveOperator op;
    op.w64 = w64.get();
    op.w32 = w32.get();
    op.plas64 = rec64.get();
    op.plas32 = rec32.get();
    op.diag_aos = diag.get();
    op.homogeneous_bc = bc_scale == 0.0;
    op.bc_scale = bc_scale;
    pa_solve_stats st{};
    pa_solve_options lo_k = lo;
    lo_k.rel_tol = std::max(lo.rel_tol, eta);
    const pa_status ls = lo.method == PA_SOLVER_PCG_MG ? solve_mg(P, op, b.get(), du.get(), lo_k, &st)
                                                       : solve_operator(P, op, b.get(), du.get(), lo_k, &st, true);
    cg_total += st.iterations;
    ++newton_total;
    if (ls == PA_ERR_NOT_CONVERGED) ++linear_unconverged;
    if (ls != PA_OK && ls != PA_ERR_NOT_CONVERGED) return ls;
    return PA_OK;
  };
  auto add_du = [&](double a) {
    k_add<<<int(std::min<int64_t>((n + 255) / 256, 148 * 8)), 256, 0, s>>>(n, du.get(), u, a);
    PA_LAUNCHED();
  };
  for (int step = 0; step < jo.steps && status == PA_OK; ++step) {
    const double s_old = double(step) / jo.steps, s_new = double(step + 1) / jo.steps;
    // reference norm of the step: the residual with the new boundary values
    // on the last converged field
    if (nbc)
      k_set_dofs<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), s_new, u);
    const double r0 = residual();
    if (!std::isfinite(r0)) { status = PA_ERR_NONFINITE; break; }
    if (nbc)
      k_set_dofs<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), s_old, u);
    // predictor (NewtonRaphsonSolver's first iteration, src/NewtonRaphsonSolver.hpp:127-131):
    // residual and tangent at the converged state, the Dirichlet increment imposed in the solve
    residual();
    // inexact Newton (Eisenstat-Walker, choice 2): tangent-solve tolerances
    // follow the observed reduction of ||R||, so that the early iterations of
    // a step do not oversolve; 0 keeps the caller's linear tolerance
    const bool ew = jo.adaptive_forcing != 0;
    constexpr double kEtaMax = 0.1, kGamma = 0.9;
    double eta = ew ? kEtaMax : 0.0;
    status = tangent_solve(s_new - s_old, eta);
    if (status != PA_OK) break;
    add_du(1.0);
    // Newton with a backtracking line search on ||R_free||: when thousands of
    // cells cross the yield surface in one step, full steps can overshoot
    // and cycle; halving until the residual norm decreases (at most
    // kMaxHalvings times, then the last trial is taken) restores descent.
    constexpr int kMaxHalvings = 5;
    bool converged = false;
    double rn = residual(), rn_prev = r0;
    for (int it = 0; it < jo.max_newton; ++it) {
      if (!std::isfinite(rn)) { status = PA_ERR_NONFINITE; break; }
      last_rel = r0 > 0.0 ? rn / r0 : 0.0;
      if (rn <= jo.newton_tol * r0 || rn == 0.0) { converged = true; break; }
      if (ew) {
        const double ratio = rn_prev > 0.0 ? rn / rn_prev : 1.0;
        double e = kGamma * ratio * ratio;
        const double guard = kGamma * eta * eta;  // do not tighten abruptly
        if (guard > 0.1) e = std::max(e, guard);
        e = std::min(e, kEtaMax);
        e = std::max(e, 0.5 * jo.newton_tol * r0 / rn);  // no finer than the remaining reduction
        eta = e;
      }
      status = tangent_solve(0.0, eta);
      if (status != PA_OK) break;
      double a = 1.0;
      add_du(a);
      double rt = residual();
      for (int h = 0; h < kMaxHalvings && !(rt <= (1.0 - 1e-4 * a) * rn); ++h) {
        a *= 0.5;
        add_du(-a);  // u_base + a du
        rt = residual();
        ++line_search_halvings;
      }
      rn_prev = rn;
      rn = rt;
    }
    if (status == PA_OK && !converged && std::isfinite(rn)) last_rel = r0 > 0.0 ? rn / r0 : 0.0;
    if (status != PA_OK) break;
    if (!converged) all_converged = false;
    worst_rel = std::max(worst_rel, last_rel);
    PA_CUDA(cudaMemcpyAsync(prev.get(), local, sizeof(double) * 14 * C, cudaMemcpyDeviceToDevice, s));
  }
  PA_CUDA(cudaEventRecord(t1, s));
  PA_CUDA(cudaEventSynchronize(t1));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  P.ep = saved;
  if (js) {
    js->steps = jo.steps;
    js->newton_iterations = newton_total;
    js->cg_iterations = cg_total;
    js->seconds = ms * 1e-3;
    js->final_rel_residual = worst_rel;
    js->linear_unconverged = linear_unconverged;
    js->line_search_halvings = line_search_halvings;
    js->converged = all_converged ? 1 : 0;
  }
  if (status != PA_OK) return status;
  return all_converged ? PA_OK : PA_ERR_NOT_CONVERGED;
}

}  // namespace pa
