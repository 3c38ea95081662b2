// pa_plastic.cuh -- device pieces shared by the J2 kernels (pa_j2.cu) and
// the stabilized u-p plasticity solve (pa_up.cu): the material records, the
// one-cell J2 return mapping with its tangent record, and their host makers.
// Each TU that includes this gets its own copy (anonymous namespace).
#pragma once

#include <cmath>

#include "pa_cell.cuh"
#include "pa_problem.cuh"

namespace pa {
namespace {

constexpr int kLocal = 14;  // local state entries per cell

struct J2Dev {
  double mu, sy0, hiso, hkin, pe, pe_min, pp, pp_min;
};

struct J2Full {
  J2Dev p;
  double kappa;  // bulk modulus E / (3 (1 - 2 nu))
  double lam;    // Lame lambda (for the tile kernel's iso parameters)
};

// One cell's return mapping from `st` (previous local state, updated in
// place) at total strain e; outputs the new stress (Voigt, tensor shears),
// the tangent record {n(6), theta1, theta2} and the elastic penalty.
__device__ __forceinline__ void j2_cell(const J2Full& q, double rho, const double e[6], double st[14],
                                        double sig[6], double rec[8], double& pe) {
  pe = simp(rho, q.p.pe, q.p.pe_min);
  const double mu_p = pe * q.p.mu;
  const double ppen = simp(rho, q.p.pp, q.p.pp_min);
  const double hi = ppen * q.p.hiso, hk = ppen * q.p.hkin;
  const double eqps_prev = st[0];
  double ee[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) ee[i] = e[i] - st[2 + i];
  double tr3 = (ee[0] + ee[1] + ee[2]) / 3.0;
  double n[6] = {2.0 * mu_p * (ee[0] - tr3), 2.0 * mu_p * (ee[1] - tr3), 2.0 * mu_p * (ee[2] - tr3),
                 mu_p * ee[3], mu_p * ee[4], mu_p * ee[5]};
#pragma unroll
  for (int i = 0; i < 6; ++i) n[i] -= st[8 + i];
  const double norm = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + 2.0 * (n[3] * n[3] + n[4] * n[4] + n[5] * n[5]));
  const double sy = ppen * q.p.sy0 + hi * eqps_prev;
  const double s32 = 1.2247448713915890491, s23 = 0.81649658092772603273;
  const double ftr = s32 * norm - sy;
  st[1] = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) rec[i] = 0.0;
  if (ftr > 1.0e-10) {
    const double dg = ftr / (3.0 * mu_p + hi + hk);
    st[1] = dg;
    st[0] = eqps_prev + dg;
    const double inv = 1.0 / norm;
    const double m1 = dg * s32 * inv, m2 = dg * s23 * hk * inv;
#pragma unroll
    for (int i = 0; i < 3; ++i) st[2 + i] += m1 * n[i];
#pragma unroll
    for (int i = 3; i < 6; ++i) st[2 + i] += 2.0 * m1 * n[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      st[8 + i] += m2 * n[i];
      rec[i] = n[i] * inv;
    }
    rec[6] = 2.449489742783178098 * mu_p * dg * inv;  // theta1 = sqrt(6) mu_p dgamma / |eta_trial|
    rec[7] = 3.0 * mu_p / (3.0 * mu_p + hi + hk);      // theta2
  }
  // stress at the returned state: kappa_p tr(e) 1 + 2 mu_p dev(e - eps_p)
#pragma unroll
  for (int i = 0; i < 6; ++i) ee[i] = e[i] - st[2 + i];
  tr3 = (ee[0] + ee[1] + ee[2]) / 3.0;
  const double ptr = pe * q.kappa * (e[0] + e[1] + e[2]);
  sig[0] = ptr + 2.0 * mu_p * (ee[0] - tr3);
  sig[1] = ptr + 2.0 * mu_p * (ee[1] - tr3);
  sig[2] = ptr + 2.0 * mu_p * (ee[2] - tr3);
  sig[3] = mu_p * ee[3];
  sig[4] = mu_p * ee[4];
  sig[5] = mu_p * ee[5];
}

inline J2Dev j2dev(const pa_j2_params& jp) {
  return J2Dev{jp.youngs_modulus / (2.0 * (1.0 + jp.poissons_ratio)),
               jp.initial_yield_stress,
               jp.hardening_modulus_isotropic,
               jp.hardening_modulus_kinematic,
               jp.elastic_penalty_exponent,
               jp.elastic_min_ersatz,
               jp.plastic_penalty_exponent,
               jp.plastic_min_ersatz};
}

// u-p residual material: shear and bulk moduli, SIMP penalty, pressure scaling
struct UpDev {
  double mu, kappa, pe, pe_min, ps;
};


inline UpDev updev(const pa_up_params& up) {
  return UpDev{up.youngs_modulus / (2.0 * (1.0 + up.poissons_ratio)),
               up.youngs_modulus / (3.0 * (1.0 - 2.0 * up.poissons_ratio)), up.penalty_exponent, up.penalty_min,
               up.pressure_scaling};
}

}  // namespace
}  // namespace pa
