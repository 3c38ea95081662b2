"""NumPy FP64 restatement of the J2 plasticity path (small meshes).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

* radial return and local residual: J2PlasticityLocalResidual::updateLocalState
  (src/J2PlasticityLocalResidual.hpp:421-523) and ::evaluate (:291-409), with
  the utilities of src/J2PlasticityUtilities.hpp (plastic-step updates
  :250-273, residual fills :514-616, normalisation :378-407).
* global problem: the displacement-only small-strain form (the reference's is
  the stabilized u-p form of src/InfinitesimalStrainPlasticityResidual.hpp;
  this build states that deviation): R(u) = sum_cells vol B^T sigma with
  sigma = kappa_p tr(eps) 1 + s, s the return-mapped deviatoric stress.
* consistent tangent: by central differences of the return-mapped stress in
  strain (independent of the closed form the CUDA kernels use).

Local state per cell (14): [eqps, dgamma, eps_p(6: xx,yy,zz,yz,xz,xy engineering
shears), backstress(6: tensor components)].
"""
import numpy as np

from . import np_ref

S32 = np.sqrt(1.5)
S23 = np.sqrt(2.0 / 3.0)


class J2Params:
    def __init__(self, E, nu, sy0, h_iso, h_kin, pe=1.0, pe_min=1e-9, pp=0.5, pp_min=1e-4):
        self.E, self.nu, self.sy0, self.h_iso, self.h_kin = E, nu, sy0, h_iso, h_kin
        self.pe, self.pe_min, self.pp, self.pp_min = pe, pe_min, pp, pp_min
        self.mu = E / (2 * (1 + nu))
        self.kappa = E / (3 * (1 - 2 * nu))

    def penalties(self, rho):
        return (self.pe_min + (1 - self.pe_min) * rho ** self.pe, self.pp_min + (1 - self.pp_min) * rho ** self.pp)


def deviatoric_stress(mu_p, ee):
    """ComputeDeviatoricStress<3> (src/ComputeDeviatoricStress.hpp:110-130)."""
    tr3 = ee[:3].sum() / 3.0
    return np.array([2 * mu_p * (ee[0] - tr3), 2 * mu_p * (ee[1] - tr3), 2 * mu_p * (ee[2] - tr3),
                     mu_p * ee[3], mu_p * ee[4], mu_p * ee[5]])


def tensor_norm(eta):
    return np.sqrt((eta[:3] ** 2).sum() + 2 * (eta[3:] ** 2).sum())


def radial_return(prm, rho, eps, prev):
    """New local state and stress (Voigt, tensor shear components)."""
    pe, pp = prm.penalties(rho)
    mu_p = pe * prm.mu
    hi, hk, sy0 = pp * prm.h_iso, pp * prm.h_kin, pp * prm.sy0
    cur = prev.copy()
    cur[1] = 0.0
    ee = eps - prev[2:8]
    s = deviatoric_stress(mu_p, ee)
    eta = s - prev[8:14]
    nrm = tensor_norm(eta)
    ftr = S32 * nrm - (sy0 + hi * prev[0])
    if ftr > 1e-10:
        dg = ftr / (3 * mu_p + hi + hk)
        n = eta / nrm
        cur[1] = dg
        cur[0] = prev[0] + dg
        cur[2:5] = prev[2:5] + S32 * dg * n[:3]
        cur[5:8] = prev[5:8] + 2 * S32 * dg * n[3:]
        cur[8:14] = prev[8:14] + S23 * dg * hk * n
    s_new = deviatoric_stress(mu_p, eps - cur[2:8])
    sig = s_new.copy()
    sig[:3] += pe * prm.kappa * eps[:3].sum()
    return cur, sig


def local_residual(prm, rho, eps, cur, prev):
    """J2PlasticityLocalResidual::evaluate for one cell (14 values)."""
    pe, pp = prm.penalties(rho)
    mu_p = pe * prm.mu
    hi, hk, sy0 = pp * prm.h_iso, pp * prm.h_kin, pp * prm.sy0
    s = deviatoric_stress(mu_p, eps - cur[2:8])
    eta = s - cur[8:14]
    nrm = tensor_norm(eta)
    n = eta / nrm
    ys = sy0 + hi * cur[0]
    H = np.zeros(14)
    H[0] = cur[0] - prev[0]
    H[1] = cur[1]
    H[2:14] = cur[2:14] - prev[2:14]
    if cur[1] > 0.0:
        H[0] = cur[0] - prev[0] - cur[1]
        H[1] = S32 * nrm - ys
        H[2:5] = cur[2:5] - prev[2:5] - S32 * cur[1] * n[:3]
        H[5:8] = cur[5:8] - prev[5:8] - 2 * S32 * cur[1] * n[3:]
        H[8:14] = cur[8:14] - prev[8:14] - S23 * cur[1] * hk * n
    return H


def stress_tangent_fd(prm, rho, eps, prev, h=1e-7):
    """d sigma / d eps (6x6, engineering strain columns) by central differences."""
    T = np.zeros((6, 6))
    scale = max(np.abs(eps).max(), 1e-3)
    for j in range(6):
        d = np.zeros(6)
        d[j] = h * scale
        _, sp = radial_return(prm, rho, eps + d, prev)
        _, sm = radial_return(prm, rho, eps - d, prev)
        T[:, j] = (sp - sm) / (2 * h * scale)
    return T


class J2Problem:
    """Displacement-form J2 problem on a linear-tet mesh (nodal densities)."""

    def __init__(self, cells, coords, prm, z=None):
        self.cells = np.asarray(cells)
        self.coords = np.asarray(coords, float)
        self.prm = prm
        self.N, self.C = self.coords.shape[0], self.cells.shape[0]
        self.z = np.ones(self.N) if z is None else np.asarray(z, float)
        self.geo = [np_ref.cell_gradients(self.coords[c]) for c in self.cells]
        self.B = [np_ref.bmatrix(g) for g, _ in self.geo]

    def rho(self, c):
        return self.z[self.cells[c]].mean()

    def dofs(self, c):
        return np.array([3 * a + d for a in self.cells[c] for d in range(3)])

    def residual(self, u, prev):
        """R(u) and the return-mapped local states."""
        R = np.zeros(3 * self.N)
        cur = np.empty_like(prev)
        for c in range(self.C):
            idx = self.dofs(c)
            eps = self.B[c] @ u[idx]
            cur[c], sig = radial_return(self.prm, self.rho(c), eps, prev[c])
            R[idx] += self.geo[c][1] * self.B[c].T @ sig
        return R, cur

    def tangent(self, u, prev):
        K = np.zeros((3 * self.N, 3 * self.N))
        for c in range(self.C):
            idx = self.dofs(c)
            eps = self.B[c] @ u[idx]
            D = stress_tangent_fd(self.prm, self.rho(c), eps, prev[c])
            K[np.ix_(idx, idx)] += self.geo[c][1] * self.B[c].T @ D @ self.B[c]
        return K

    def solve(self, bc_dofs, bc_final, steps, tol=1e-10, max_newton=25):
        """Pseudo-time load stepping, Dirichlet values ramped linearly; Newton
        with a dense solve of the constrained tangent and a backtracking line
        search on ||R_free|| (steps halved while the residual does not
        decrease; the converged increment does not depend on it).  Returns u
        and states; self.converged tells whether every step met tol."""
        u = np.zeros(3 * self.N)
        prev = np.zeros((self.C, 14))
        free = np.setdiff1d(np.arange(3 * self.N), bc_dofs)
        self.converged = True
        for k in range(steps):
            u[bc_dofs] = bc_final * (k + 1) / steps
            ok = False
            for it in range(max_newton):
                R, cur = self.residual(u, prev)
                rn = np.linalg.norm(R[free])
                if rn <= tol * max(1.0, np.linalg.norm(R)):
                    ok = True
                    break
                K = self.tangent(u, prev)
                du = np.linalg.solve(K[np.ix_(free, free)], -R[free])
                a = 1.0
                for _ in range(30):
                    trial = u.copy()
                    trial[free] += a * du
                    if np.linalg.norm(self.residual(trial, prev)[0][free]) < rn:
                        break
                    a *= 0.5
                u[free] += a * du
                if np.linalg.norm(a * du) <= 1e-14 * max(1.0, np.linalg.norm(u)):
                    ok = True
                    break
            self.converged = self.converged and ok
            R, cur = self.residual(u, prev)
            prev = cur
        return u, prev
