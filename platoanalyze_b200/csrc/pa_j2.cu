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
#include "pa_cell.cuh"

namespace pa {

namespace {

constexpr int kJ2Threads = 128;
constexpr int kLocal = 14;

struct J2Dev {
  double mu, sy0, hiso, hkin, pe, pe_min, pp, pp_min;
};

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

}  // namespace

void launch_j2(const Problem& P, const pa_j2_params& jp, const double* u, const double* z, const double* prev,
               double* cur, cudaStream_t s) {
  J2Dev p{jp.youngs_modulus / (2.0 * (1.0 + jp.poissons_ratio)),
          jp.initial_yield_stress,
          jp.hardening_modulus_isotropic,
          jp.hardening_modulus_kinematic,
          jp.elastic_penalty_exponent,
          jp.elastic_min_ersatz,
          jp.plastic_penalty_exponent,
          jp.plastic_min_ersatz};
  const int64_t C = P.C();
  const int grid = int((C + kJ2Threads - 1) / kJ2Threads);
  k_j2<<<grid, kJ2Threads, 0, s>>>(P.mesh->d_cells.get(), P.mesh->d_coords.get(), C, p, u, z, prev, cur);
  PA_LAUNCHED();
}

}  // namespace pa
