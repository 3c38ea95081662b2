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


def project_pressure_gradient(cells, coords, state, z, pe=3.0, pe_min=1e-9, ps=1.0):
    """Nodal projected pressure gradient by the row-summed (lumped) solve of
    the projection equation (PlasticityProblem::updateProjectedPressureGradient,
    src/PlasticityProblem.hpp:877-897; residual
    src/PressureGradientProjectionResidual.hpp): Pi_a = sum_c pen_c V_c ps
    grad p_c / sum_c pen_c V_c over the cells c around node a.  Returns N x 3."""
    st = np.asarray(state, dtype=np.float64).reshape(-1, 4)
    N = st.shape[0]
    num = np.zeros((N, 3))
    den = np.zeros(N)
    for c, v in enumerate(np.asarray(cells)):
        g, vol = cell_gradients(coords[v])
        pen = pe_min + (1.0 - pe_min) * np.mean(np.asarray(z)[v]) ** pe
        gp = ps * (g.T @ st[v, 3])
        for a in v:
            num[a] += pen * vol * gp
            den[a] += pen * vol
    return num / np.maximum(den, 1e-300)[:, None]


class UpProblem:
    """Stabilized u-p J2 plasticity (4 dofs per node: u_x, u_y, u_z, p) by
    pseudo-time load stepping and Newton's method, as PlasticityProblem
    drives it (src/PlasticityProblem.hpp:791-846 with
    NewtonRaphsonSolver::solve, src/NewtonRaphsonSolver.hpp:570-640): each
    Newton iterate returns the local states from the previous step's
    converged ones (np_j2.radial_return, the J2 local residual solved in
    closed form) and evaluates the global residual at them; the projected
    pressure gradient is lagged by one step (zero in the first step, the
    lumped projection of the converged pressure afterwards).  The tangent is
    the finite-difference Jacobian of the condensed residual, cell by cell
    (dense, small meshes only)."""

    def __init__(self, cells, coords, E, nu, j2prm, z=None, pe=3.0, pe_min=1e-9, ps=1.0):
        from .np_j2 import radial_return
        self._rr = radial_return
        self.cells = np.asarray(cells)
        self.coords = np.asarray(coords, float)
        self.N, self.C = self.coords.shape[0], self.cells.shape[0]
        self.E, self.nu, self.pe, self.pe_min, self.ps = E, nu, pe, pe_min, ps
        self.j2 = j2prm
        self.z = np.ones(self.N) if z is None else np.asarray(z, float)
        self.geo = [cell_gradients(self.coords[v]) for v in self.cells]

    def _idx(self, c):
        return np.array([4 * a + d for a in self.cells[c] for d in range(4)])

    def cell_residual(self, c, xc, prev_c, ppg_c):
        """16 residual entries of cell c at its dofs xc and the returned state."""
        v = self.cells[c]
        g = self.geo[c][0]
        u = xc.reshape(4, 4)[:, :3]
        du = g.T @ u
        eps = np.array([du[0, 0], du[1, 1], du[2, 2], du[1, 2] + du[2, 1], du[0, 2] + du[2, 0], du[0, 1] + du[1, 0]])
        cur, _ = self._rr(self.j2, self.z[v].mean(), eps, prev_c)
        loc = np.arange(4)
        R = up_residual_cells(loc[None, :], self.coords[v], xc, cur[None, :], ppg_c[None], self.z[v], self.E,
                              self.nu, self.pe, self.pe_min, self.ps)[0]
        return R, cur

    def residual(self, x, prev, ppg):
        R = np.zeros(4 * self.N)
        cur = np.empty_like(prev)
        for c in range(self.C):
            idx = self._idx(c)
            Rc, cur[c] = self.cell_residual(c, x[idx], prev[c], ppg[self.cells[c]])
            R[idx] += Rc
        return R, cur

    def cell_tangent(self, c, xc, prev_c):
        """Condensed 16 x 16 tangent of cell c: dR/dx at the returned local
        state, i.e. dR/du - dR/dc (dH/dc)^-1 dH/du of NewtonRaphsonSolver
        (src/NewtonRaphsonSolver.hpp:206-290) in closed form.  With
        eta = (s_trial - backstress) / |s_trial - backstress| and the return's
        theta1 = sqrt(6) mu_l dgamma / |eta_trial|, theta2 = 3 mu_l / (3 mu_l + H)
        (zero for an elastic cell), d eps_p = theta1 dev(d eps) + (theta2 -
        theta1) eta (eta : d eps), so ds/d eps = (1 - theta1) D_dev -
        2 mu_g (theta2 - theta1) eta eta^T; the pressure rows and columns do
        not depend on the local state."""
        from .np_j2 import deviatoric_stress, tensor_norm
        v = self.cells[c]
        g, vol = self.geo[c]
        rho = self.z[v].mean()
        mu, kappa = moduli(self.E, self.nu)
        pen = self.pe_min + (1.0 - self.pe_min) * rho ** self.pe
        mu_g, kappa_p = pen * mu, pen * kappa
        u = xc.reshape(4, 4)[:, :3]
        du = g.T @ u
        eps = np.array([du[0, 0], du[1, 1], du[2, 2], du[1, 2] + du[2, 1], du[0, 2] + du[2, 0], du[0, 1] + du[1, 0]])
        pe_l, pp_l = self.j2.penalties(rho)
        mu_l = pe_l * self.j2.mu
        hi, hk = pp_l * self.j2.h_iso, pp_l * self.j2.h_kin
        eta = deviatoric_stress(mu_l, eps - prev_c[2:8]) - prev_c[8:14]
        nrm = tensor_norm(eta)
        th1 = th2 = 0.0
        nh = np.zeros(6)
        if 1.2247448713915890491 * nrm - (pp_l * self.j2.sy0 + hi * prev_c[0]) > 1e-10:
            dg = (1.2247448713915890491 * nrm - (pp_l * self.j2.sy0 + hi * prev_c[0])) / (3 * mu_l + hi + hk)
            nh = eta / nrm
            th1 = np.sqrt(6.0) * mu_l * dg / nrm
            th2 = 3 * mu_l / (3 * mu_l + hi + hk)
        Dd = np.zeros((6, 6))
        Dd[:3, :3] = 2 * mu_g * (np.eye(3) - 1.0 / 3.0)
        Dd[3:, 3:] = mu_g * np.eye(3)
        D = (1 - th1) * Dd - 2 * mu_g * (th2 - th1) * np.outer(nh, nh)
        B = np.zeros((6, 12))
        for n in range(4):
            gx, gy, gz = g[n]
            B[:, 3 * n:3 * n + 3] = [[gx, 0, 0], [0, gy, 0], [0, 0, gz], [0, gz, gy], [gz, 0, gx], [gy, gx, 0]]
        Kuu = vol * B.T @ D @ B
        ps = self.ps
        tau = vol ** (2.0 / 3.0) / (2.0 * mu)
        K = np.zeros((16, 16))
        for a in range(4):
            for b in range(4):
                K[4 * a:4 * a + 3, 4 * b:4 * b + 3] = Kuu[3 * a:3 * a + 3, 3 * b:3 * b + 3]
                K[4 * a:4 * a + 3, 4 * b + 3] = vol * ps * 0.25 * g[a]
                K[4 * a + 3, 4 * b:4 * b + 3] = vol * ps * 0.25 * g[b]
                K[4 * a + 3, 4 * b + 3] = -vol * ps * ps / (16.0 * kappa_p) - vol * pen * ps * ps * tau * (g[a] @ g[b])
        return K

    def cell_tangent_fd(self, c, xc, prev_c, ppg_c):
        """Central finite differences of the condensed cell residual (checks
        cell_tangent)."""
        K = np.zeros((16, 16))
        for j in range(16):
            h = 1e-6 * max(1.0, abs(xc[j])) if j % 4 == 3 else 1e-7 * max(1e-3, abs(xc[j]))
            xp, xm = xc.copy(), xc.copy()
            xp[j] += h
            xm[j] -= h
            K[:, j] = (self.cell_residual(c, xp, prev_c, ppg_c)[0] - self.cell_residual(c, xm, prev_c, ppg_c)[0]) / (2 * h)
        return K

    def elastic_work(self, pe=3.0, pe_min=1e-9):
        """The "Elastic Work" criterion of the last solve: the steps' elastic
        work summed (PlasticityProblem::evaluateCriterion,
        src/PlasticityProblem.hpp:929-953)."""
        total, ps, pl = 0.0, np.zeros(4 * self.N), np.zeros((self.C, 14))
        for st, loc in self.history:
            total += elastic_work(self.cells, self.coords, st, loc, ps, pl, self.z, self.E, self.nu, pe, pe_min)
            ps, pl = st, loc
        return total

    def tangent(self, x, prev, ppg):
        n = 4 * self.N
        K = np.zeros((n, n))
        for c in range(self.C):
            idx = self._idx(c)
            K[np.ix_(idx, idx)] += self.cell_tangent(c, x[idx], prev[c])
        return K

    def solve(self, bc_dofs, bc_final, steps, tol=1e-11, max_newton=25):
        """bc_dofs in the 4-dof numbering (4 node + component).  Returns the
        state (4N), the local states (C x 14) and the projected pressure
        gradient of the last step (N x 3); self.converged tells whether every
        step met tol (||R_free|| <= tol max(1, ||R||)); self.history holds
        every step's state and local states."""
        x = np.zeros(4 * self.N)
        prev = np.zeros((self.C, 14))
        ppg = np.zeros((self.N, 3))
        free = np.setdiff1d(np.arange(4 * self.N), bc_dofs)
        self.converged = True
        self.history = []  # (state, local states) after every step
        for k in range(steps):
            x[bc_dofs] = np.asarray(bc_final) * (k + 1) / steps
            ok = False
            for it in range(max_newton):
                R, cur = self.residual(x, prev, ppg)
                rn = np.linalg.norm(R[free])
                if rn <= tol * max(1.0, np.linalg.norm(R)):
                    ok = True
                    break
                K = self.tangent(x, prev, ppg)
                dx = np.linalg.solve(K[np.ix_(free, free)], -R[free])
                a = 1.0
                for _ in range(30):
                    trial = x.copy()
                    trial[free] += a * dx
                    if np.linalg.norm(self.residual(trial, prev, ppg)[0][free]) < rn:
                        break
                    a *= 0.5
                x[free] += a * dx
            self.converged = self.converged and ok
            R, cur = self.residual(x, prev, ppg)
            prev = cur
            self.history.append((x.copy(), cur.copy()))
            if k + 1 < steps:
                ppg = project_pressure_gradient(self.cells, self.coords, x, self.z, self.pe, self.pe_min, self.ps)
        return x, prev, ppg


def elastic_work(cells, coords, state, local, prev_state, prev_local, z, E, nu, pe=3.0, pe_min=1e-9):
    """One step's elastic work, ElasticWorkCriterion::evaluate
    (src/ElasticWorkCriterion.hpp): per cell V (sigma_n + sigma_{n-1}) / 2 .
    (e_n - e_{n-1}) with e = eps(u) - eps_p and sigma the penalized isotropic
    Cauchy stress of e (shear strains engineering, so sigma . e counts them
    once).  PlasticityProblem::evaluateCriterion sums it over the steps."""
    mu, kappa = moduli(E, nu)
    total = 0.0
    for c, v in enumerate(np.asarray(cells)):
        g, vol = cell_gradients(coords[v])
        pen = pe_min + (1.0 - pe_min) * np.mean(np.asarray(z)[v]) ** pe
        es = []
        for st, loc in ((state, local), (prev_state, prev_local)):
            u = np.asarray(st).reshape(-1, 4)[v, :3]
            du = g.T @ u
            eps = np.array([du[0, 0], du[1, 1], du[2, 2], du[1, 2] + du[2, 1], du[0, 2] + du[2, 0],
                            du[0, 1] + du[1, 0]])
            es.append(eps - np.asarray(loc)[c, 2:8])
        sig = []
        for e in es:
            tr = e[:3].sum()
            sig.append(pen * np.concatenate([kappa * tr + 2 * mu * (e[:3] - tr / 3.0), mu * e[3:]]))
        total += vol * 0.5 * (sig[0] + sig[1]) @ (es[0] - es[1])
    return total
