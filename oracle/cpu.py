"""ctypes wrapper over oracle/_build/libpa_oracle.so (FP64 C++/OpenMP oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
import ctypes as ct
import os
import time

import numpy as np

from . import build as _build

_lib = None
I64, I32, F64 = ct.c_int64, ct.c_int32, ct.c_double
P = ct.c_void_p


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        L = ct.CDLL(path)
        L.pao_box_mesh.argtypes = [ct.c_int] * 3 + [F64] * 3 + [P, P]
        L.pao_residual.argtypes = [I64, I64, P, P, P, P, ct.c_int, F64, F64, F64, F64, I64, P, P, P]
        L.pao_crs_graph.argtypes = [I64, I64, P, P, P]
        L.pao_crs_graph.restype = I64
        L.pao_jacobian.argtypes = [I64, I64, P, P, P, P, ct.c_int, F64, F64, F64, F64, P, P, P]
        L.pao_gradient_z.argtypes = [I64, I64, P, P, P, P, ct.c_int, F64, F64, F64, F64, P, P, P]
        L.pao_energy.argtypes = [I64, I64, P, P, P, P, ct.c_int, F64, F64, F64, F64, P, P]
        L.pao_energy.restype = F64
        L.pao_apply_block_constraints.argtypes = [I64, P, P, P, P, I64, P, P, F64]
        L.pao_block_spmv.argtypes = [I64, P, P, P, P, P]
        L.pao_pcg.argtypes = [I64, P, P, P, P, P, F64, ct.c_int, P]
        L.pao_pcg.restype = ct.c_int
        L.pao_pcg_run.argtypes = [I64, P, P, P, P, P, F64, F64, ct.c_int, P]
        L.pao_apply.argtypes = [I64, I64, P, P, P, P, ct.c_int, F64, F64, F64, F64, P]
        L.pao_j2_update.argtypes = [I64, P, P, P, P] + [F64] * 8 + [P, P]
        L.pao_j2_plastic_step.argtypes = [I64, P, P, F64, P]
        L.pao_gradient_x.argtypes = [I64, I64, P, P, P, P, ct.c_int, F64, F64, F64, F64, I64, P, P, P, P, P]
        L.pao_energy_grad_x.argtypes = [I64, I64, P, P, P, P, ct.c_int, F64, F64, F64, F64, P]
        L.pao_num_threads.restype = ct.c_int
        L.pao_set_threads.argtypes = [ct.c_int]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def num_threads():
    return lib().pao_num_threads()


def set_threads(n):
    lib().pao_set_threads(int(n))


def box_mesh(nx, ny, nz, lx, ly, lz):
    C, N = 6 * nx * ny * nz, (nx + 1) * (ny + 1) * (nz + 1)
    cells = np.empty((C, 4), np.int32)
    coords = np.empty((N, 3), np.float64)
    lib().pao_box_mesh(nx, ny, nz, lx, ly, lz, _p(cells), _p(coords))
    return cells, coords


class Oracle:
    """FP64 oracle bound to one mesh and one material (E, nu, SIMP p, pmin)."""

    def __init__(self, cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=0):
        self.cells = _c(cells, np.int32)
        self.coords = _c(coords, np.float64)
        self.C, self.N = self.cells.shape[0], self.coords.shape[0]
        self.mat = (float(E), float(nu), float(p), float(pmin))
        self.layout = int(layout)
        self._graph = None

    def graph(self):
        if self._graph is None:
            L = lib()
            rowmap = np.empty(self.N + 1, np.int32)
            nnz = L.pao_crs_graph(self.C, self.N, _p(self.cells), _p(rowmap), None)
            cols = np.empty(nnz, np.int32)
            L.pao_crs_graph(self.C, self.N, _p(self.cells), _p(rowmap), _p(cols))
            self._graph = (rowmap, cols)
        return self._graph

    def residual(self, u, z, faces=None, flux=(0.0, 0.0, 0.0)):
        u, z = _c(u, np.float64), _c(z, np.float64)
        r = np.empty(3 * self.N)
        nf = 0 if faces is None else len(faces)
        fa = _c(faces, np.int32) if nf else None
        fl = _c(flux, np.float64)
        lib().pao_residual(self.C, self.N, _p(self.cells), _p(self.coords), _p(u), _p(z), self.layout,
                           *self.mat, nf, _p(fa), _p(fl), _p(r))
        return r

    def apply(self, u, z):
        u, z = _c(u, np.float64), _c(z, np.float64)
        y = np.empty(3 * self.N)
        lib().pao_apply(self.C, self.N, _p(self.cells), _p(self.coords), _p(u), _p(z), self.layout, *self.mat, _p(y))
        return y

    def jacobian(self, u, z, graph=None):
        rowmap, cols = graph if graph is not None else self.graph()
        rowmap, cols = _c(rowmap, np.int32), _c(cols, np.int32)
        u, z = _c(u, np.float64), _c(z, np.float64)
        vals = np.empty(9 * len(cols))
        lib().pao_jacobian(self.C, self.N, _p(self.cells), _p(self.coords), _p(u), _p(z), self.layout, *self.mat,
                           _p(rowmap), _p(cols), _p(vals))
        return vals

    def gradient_z(self, u, z, graph=None):
        rowmap, cols = graph if graph is not None else self.graph()
        rowmap, cols = _c(rowmap, np.int32), _c(cols, np.int32)
        u, z = _c(u, np.float64), _c(z, np.float64)
        n = 12 * self.C if self.layout == 1 else 3 * len(cols)
        vals = np.empty(n)
        lib().pao_gradient_z(self.C, self.N, _p(self.cells), _p(self.coords), _p(u), _p(z), self.layout, *self.mat,
                             _p(rowmap), _p(cols), _p(vals))
        return vals

    def gradient_x(self, u, z, faces=None, flux=(0.0, 0.0, 0.0), graph=None):
        rowmap, cols = graph if graph is not None else self.graph()
        rowmap, cols = _c(rowmap, np.int32), _c(cols, np.int32)
        u, z = _c(u, np.float64), _c(z, np.float64)
        nf = 0 if faces is None else len(faces)
        fa = _c(faces, np.int32) if nf else None
        fl = _c(flux, np.float64)
        vals = np.empty(9 * len(cols))
        lib().pao_gradient_x(self.C, self.N, _p(self.cells), _p(self.coords), _p(u), _p(z), self.layout, *self.mat,
                             nf, _p(fa), _p(fl), _p(rowmap), _p(cols), _p(vals))
        return vals

    def energy_grad_x(self, u, z):
        u, z = _c(u, np.float64), _c(z, np.float64)
        gx = np.empty(3 * self.N)
        lib().pao_energy_grad_x(self.C, self.N, _p(self.cells), _p(self.coords), _p(u), _p(z), self.layout,
                                *self.mat, _p(gx))
        return gx

    def energy(self, u, z, grads=True):
        u, z = _c(u, np.float64), _c(z, np.float64)
        gu = np.empty(3 * self.N) if grads else None
        gz = np.empty(self.C if self.layout == 1 else self.N) if grads else None
        f = lib().pao_energy(self.C, self.N, _p(self.cells), _p(self.coords), _p(u), _p(z), self.layout, *self.mat,
                             _p(gu), _p(gz))
        return (f, gu, gz) if grads else f

    def solve(self, z, F, bc_dofs, bc_values=None, rel_tol=1e-10, max_iters=0, graph=None):
        """Elliptic::Problem::solution with one Newton step (src/elliptic/Problem.hpp:259-311):
        assemble K (dual numbers), constrain symmetrically, Jacobi-PCG."""
        rowmap, cols = graph if graph is not None else self.graph()
        z = _c(z, np.float64)
        u0 = np.zeros(3 * self.N)
        vals = self.jacobian(u0, z, (rowmap, cols))
        rhs = _c(F, np.float64).copy()
        bc_dofs = _c(bc_dofs, np.int32)
        bcv = np.zeros(len(bc_dofs)) if bc_values is None else _c(bc_values, np.float64)
        L = lib()
        L.pao_apply_block_constraints(self.N, _p(rowmap), _p(cols), _p(vals), _p(rhs), len(bc_dofs), _p(bc_dofs),
                                      _p(bcv), 1.0)
        x = np.zeros(3 * self.N)
        rel = ct.c_double(0)
        it = L.pao_pcg(self.N, _p(rowmap), _p(cols), _p(vals), _p(rhs), _p(x), rel_tol, max_iters, ct.byref(rel))
        return x, it, rel.value

    def constrained_system(self, z, F, bc_dofs, bc_values=None, graph=None):
        """The linear system of Elliptic::Problem::solution (src/elliptic/Problem.hpp:259-311):
        K assembled with dual numbers (gradient_u at u = 0) and constrained
        symmetrically (applyBlockConstraints, src/ApplyConstraints.hpp:11-79).
        Returns (rowmap, cols, vals, rhs) and the seconds of assembly and of
        elimination."""
        rowmap, cols = graph if graph is not None else self.graph()
        rowmap, cols = _c(rowmap, np.int32), _c(cols, np.int32)
        z = _c(z, np.float64)
        t0 = time.perf_counter()
        vals = self.jacobian(np.zeros(3 * self.N), z, (rowmap, cols))
        t1 = time.perf_counter()
        rhs = _c(F, np.float64).copy()
        bc_dofs = _c(bc_dofs, np.int32)
        bcv = np.zeros(len(bc_dofs)) if bc_values is None else _c(bc_values, np.float64)
        lib().pao_apply_block_constraints(self.N, _p(rowmap), _p(cols), _p(vals), _p(rhs), len(bc_dofs),
                                          _p(bc_dofs), _p(bcv), 1.0)
        t2 = time.perf_counter()
        return (rowmap, cols, vals, rhs), t1 - t0, t2 - t1

    def pcg_run(self, system, x=None, rel_tol=1e-8, report_tol=None, max_iters=0):
        """Jacobi-PCG on a constrained system from x (zero if None), to rel_tol,
        noting when the residual first reaches report_tol.  Returns x and a dict
        (iterations, seconds, relres and the checkpoint's iterations/seconds)."""
        rowmap, cols, vals, rhs = system
        x = np.zeros(3 * self.N) if x is None else _c(x, np.float64).copy()
        info = np.zeros(5)
        rt = rel_tol if report_tol is None else report_tol
        lib().pao_pcg_run(self.N, _p(rowmap), _p(cols), _p(vals), _p(rhs), _p(x), float(rt), float(rel_tol),
                          int(max_iters), _p(info))
        return x, {"report_iterations": int(info[0]), "report_seconds": float(info[1]), "iterations": int(info[2]),
                   "seconds": float(info[3]), "rel_residual": float(info[4])}

    def j2_update(self, u, z, prev, mu, sigma_y0, h_iso, h_kin, pe=3.0, pe_min=1e-9, pp=2.5, pp_min=1e-9):
        u, z, prev = _c(u, np.float64), _c(z, np.float64), _c(prev, np.float64)
        cur = np.empty_like(prev)
        lib().pao_j2_update(self.C, _p(self.cells), _p(self.coords), _p(u), _p(z), mu, sigma_y0, h_iso, h_kin,
                            pe, pe_min, pp, pp_min, _p(prev), _p(cur))
        return cur


def j2_plastic_step(prev, normal, cur_in, h_kin):
    prev, normal = _c(prev, np.float64), _c(normal, np.float64)
    cur = _c(cur_in, np.float64).copy()
    lib().pao_j2_plastic_step(prev.shape[0], _p(prev), _p(normal), float(h_kin), _p(cur))
    return cur
