"""NumPy restatement of the reference's stabilized u-p plasticity residual
(per cell, unassembled), for small meshes.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

InfinitesimalStrainPlasticityResidual::evaluate
(src/InfinitesimalStrainPlasticityResidual.hpp:398-516), 4 dofs per node
(u_x, u_y, u_z, p), one-point rule (weight 1/6, basis 1/4 each,
src/LinearTetCubRuleDegreeOne.hpp:84-111):

* elastic strain e = eps(u) - eps_p (local state entries 2..7,
  src/ThermoPlasticityUtilities.hpp computeElasticStrain)
* s = 2 mu_p dev(e), shears mu_p gamma (src/ComputeDeviatoricStress.hpp:110-130)
* pressure gradient grad p = sum_n p_n grad N_n (src/ScalarGrad.hpp), cell
  pressure and projected pressure gradient interpolated with the basis
  (src/InterpolateFromNodal.hpp:55-103)
* volume strain theta = ps (tr eps(u) - ps p / kappa_p) (StrainDivergence)
* stabilization tau = V^(2/3) / (2 mu), stab = ps tau (ps grad p - Pi),
  times the penalty (src/ComputeStabilization.hpp:93-108,
  src/Plato_TopOptFunctors.hpp:78-85)
* rows: displacement  += V s : grad N (src/StressDivergence.hpp)
                      += V ps p grad N (src/PressureDivergence.hpp:46-62)
        pressure      -= V stab . grad N (src/FluxDivergence.hpp:32-48)
                      += V N_n theta (src/ProjectToNode.hpp:61-74)
with mu_p = pen mu, kappa_p = pen kappa, pen = pmin + (1 - pmin) rho^p
(rho the mean nodal control, src/Simp.hpp:130-134), ps the pressure scaling.
"""
import numpy as np

from .np_ref import cell_gradients


def moduli(E, nu):
    """Shear and bulk moduli (src/IsotropicMaterialUtilities.hpp:23-45)."""
    return E / (2.0 * (1.0 + nu)), E / (3.0 * (1.0 - 2.0 * nu))


def up_residual_cells(cells, coords, state, local, ppg_cells, z, E, nu, pe=3.0, pe_min=1e-9, ps=1.0):
    """state: 4N nodal (u_x, u_y, u_z, p); local: C x 14; ppg_cells: C x 4 x 3
    projected pressure gradients at each cell's nodes; z: N nodal controls.
    Returns C x 16 (node-major, 4 dofs per node)."""
    cells = np.asarray(cells)
    st = np.asarray(state, dtype=np.float64).reshape(-1, 4)
    mu, kappa = moduli(E, nu)
    C = cells.shape[0]
    R = np.zeros((C, 16))
    ppg_cells = np.asarray(ppg_cells, dtype=np.float64).reshape(C, 4, 3)
    for c in range(C):
        v = cells[c]
        g, vol = cell_gradients(coords[v])
        u = st[v, :3]
        p = st[v, 3]
        # total strain, engineering shears (xx, yy, zz, yz, xz, xy)
        du = g.T @ u  # du[i, j] = d u_j / d x_i
        eps = np.array([du[0, 0], du[1, 1], du[2, 2], du[1, 2] + du[2, 1], du[0, 2] + du[2, 0],
                        du[0, 1] + du[1, 0]])
        e = eps - np.asarray(local[c][2:8])
        pen = pe_min + (1.0 - pe_min) * np.mean(np.asarray(z)[v]) ** pe
        mu_p, kappa_p = pen * mu, pen * kappa
        tr3 = (e[0] + e[1] + e[2]) / 3.0
        s = np.array([2 * mu_p * (e[0] - tr3), 2 * mu_p * (e[1] - tr3), 2 * mu_p * (e[2] - tr3),
                      mu_p * e[3], mu_p * e[4], mu_p * e[5]])
        gp = g.T @ p
        pc = ps * 0.25 * p.sum()
        pi = 0.25 * ppg_cells[c].sum(0)
        theta = ps * (eps[0] + eps[1] + eps[2] - pc / kappa_p)
        tau = vol ** (2.0 / 3.0) / (2.0 * mu)
        stab = pen * ps * tau * (ps * gp - pi)
        S = np.array([[s[0], s[5], s[4]], [s[5], s[1], s[3]], [s[4], s[3], s[2]]])
        for n in range(4):
            R[c, 4 * n:4 * n + 3] += vol * (S @ g[n]) + vol * pc * g[n]
            R[c, 4 * n + 3] += -vol * stab @ g[n] + vol * 0.25 * theta
    return R
