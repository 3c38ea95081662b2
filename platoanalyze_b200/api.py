"""Host-side mirror of Plato Analyze's interfaces for the linear-tet hot path.

Class and method names follow the reference so that its callers and tests
translate line by line:

* ``Problem``               - Elliptic::Problem (src/elliptic/Problem.hpp:44-715):
                              solution(z), criterionValue, criterionGradient.
* ``VectorFunction``        - Elliptic::VectorFunction (src/elliptic/VectorFunction.hpp):
                              value / gradient_u / gradient_z.
* ``PhysicsScalarFunction`` - "Internal Elastic Energy"
                              (src/elliptic/PhysicsScalarFunction.hpp): value / gradient_u / gradient_z.

All arithmetic happens in libpa_b200.so through the C ABI (include/pa_b200.h).
Arrays may be NumPy arrays (host) or torch CUDA tensors (device); results
come back in the kind of array the first array argument was.
"""
import ctypes as ct
import os

import numpy as np

from . import _abi

_NP = {np.float64: "float64", np.float32: "float32", np.int32: "int32"}


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _ptr(a, dtype, count=None, name="array"):
    """Raw pointer of a contiguous array of `dtype` (NumPy or torch)."""
    if a is None:
        return None
    if _is_torch(a):
        import torch
        want = {np.float64: torch.float64, np.float32: torch.float32, np.int32: torch.int32}[dtype]
        if a.dtype != want or not a.is_contiguous():
            raise TypeError(f"{name}: need a contiguous torch tensor of {want}")
        if count is not None and a.numel() != count:
            raise ValueError(f"{name}: expected {count} entries, got {a.numel()}")
        return ct.c_void_p(a.data_ptr())
    if not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags.c_contiguous:
        raise TypeError(f"{name}: need a C-contiguous numpy array of {np.dtype(dtype)}")
    if count is not None and a.size != count:
        raise ValueError(f"{name}: expected {count} entries, got {a.size}")
    return ct.c_void_p(a.ctypes.data)


def _ptr_i64(a):
    if not isinstance(a, np.ndarray) or a.dtype != np.int64 or not a.flags.c_contiguous:
        raise TypeError("need a C-contiguous numpy array of int64")
    return ct.c_void_p(a.ctypes.data)


def _empty(like, n, dtype=np.float64):
    if like is not None and _is_torch(like):
        import torch
        t = {np.float64: torch.float64, np.float32: torch.float32}[dtype]
        return torch.empty(n, dtype=t, device=like.device)
    return np.empty(n, dtype=dtype)


def _as(a, dtype):
    if a is None or _is_torch(a):
        return a
    return np.ascontiguousarray(a, dtype=dtype)


class Mesh:
    """Linear-tet mesh: connectivity, coordinates, block-CRS graph, cell tiles."""

    def __init__(self, handle):
        self._lib = _abi.load()
        self._h = handle
        self.num_parts = 1
        C, N, B, T = (ct.c_int64() for _ in range(4))
        _abi.check(self._lib.pa_mesh_sizes(self._h, ct.byref(C), ct.byref(N), ct.byref(B), ct.byref(T)))
        self.num_cells, self.num_nodes, self.num_blocks, self.num_tiles = C.value, N.value, B.value, T.value

    @classmethod
    def box(cls, nx, ny, nz, lx=1.0, ly=1.0, lz=1.0):
        lib = _abi.load()
        h = ct.c_void_p()
        _abi.check(lib.pa_mesh_create_box(nx, ny, nz, lx, ly, lz, ct.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, cells, coords):
        lib = _abi.load()
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        h = ct.c_void_p()
        _abi.check(lib.pa_mesh_create(_ptr(cells, np.int32), cells.shape[0], _ptr(coords, np.float64),
                                      coords.shape[0], ct.byref(h)))
        return cls(h)

    @classmethod
    def from_exodus(cls, path):
        """The mesh of an Exodus II file (pa_exodus_*, then pa_mesh_create)
        and its node sets {name: node ids}."""
        cells, coords, sets = read_exodus(path)
        return cls.from_arrays(cells, coords), sets

    def arrays(self):
        cells = np.empty((self.num_cells, 4), np.int32)
        coords = np.empty((self.num_nodes, 3), np.float64)
        _abi.check(self._lib.pa_mesh_get(self._h, _ptr(cells, np.int32), _ptr(coords, np.float64)))
        return cells, coords

    def graph(self):
        rowmap = np.empty(self.num_nodes + 1, np.int32)
        cols = np.empty(self.num_blocks, np.int32)
        _abi.check(self._lib.pa_mesh_graph(self._h, _ptr(rowmap, np.int32), _ptr(cols, np.int32)))
        return rowmap, cols

    def set_graph(self, rowmap, cols):
        rowmap = np.ascontiguousarray(rowmap, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        _abi.check(self._lib.pa_mesh_set_graph(self._h, _ptr(rowmap, np.int32), _ptr(cols, np.int32), cols.size))

    def set_parts(self, node_offsets):
        """Declare the mesh a disjoint union of independent parts (node ranges);
        batched mixed solves then run one CG per part.  Before any Problem."""
        off = np.ascontiguousarray(node_offsets, np.int64)
        _abi.check(self._lib.pa_mesh_set_parts(self._h, off.size - 1, _ptr_i64(off)))
        self.num_parts = off.size - 1
        C, N, B, T = (ct.c_int64() for _ in range(4))
        _abi.check(self._lib.pa_mesh_sizes(self._h, ct.byref(C), ct.byref(N), ct.byref(B), ct.byref(T)))
        self.num_tiles = T.value

    def write_vtu(self, path, u=None, control=None, control_layout="nodal"):
        """Write the mesh with the displacement (3N) and the control (N nodal
        or C per-cell values) as a .vtu file (pa_write_vtu)."""
        lay = 1 if control_layout == "cell" else 0
        nz = self.num_cells if lay else self.num_nodes
        u = None if u is None else _as(u, np.float64)
        control = None if control is None else _as(control, np.float64)
        _abi.check(self._lib.pa_write_vtu(self._h, os.fsencode(str(path)),
                                          None if u is None else _ptr(u, np.float64, 3 * self.num_nodes, "u"),
                                          None if control is None else _ptr(control, np.float64, nz, "control"),
                                          lay))

    @property
    def uniform_geometry(self):
        """True when the FP32 kernels use the per-mesh hex geometry table
        (every hex a translate of the first)."""
        a = ct.c_int32()
        _abi.check(self._lib.pa_mesh_uniform_geometry(self._h, -1, ct.byref(a)))
        return bool(a.value)

    def set_uniform_geometry(self, enable):
        """Allow (True, the default) or forbid the hex geometry table; before
        any Problem on the mesh.  Returns whether the table is in use."""
        a = ct.c_int32()
        _abi.check(self._lib.pa_mesh_uniform_geometry(self._h, 1 if enable else 0, ct.byref(a)))
        return bool(a.value)

    @property
    def box_kernels(self):
        """True when pa_apply and the multigrid solve run on the box kernel."""
        a = ct.c_int32()
        _abi.check(self._lib.pa_mesh_box_kernels(self._h, -1, ct.byref(a)))
        return bool(a.value)

    def set_box_kernels(self, enable):
        """Use (True, the default) or bypass the box kernel on a structured box."""
        _abi.check(self._lib.pa_mesh_box_kernels(self._h, int(bool(enable)), None))

    def boundary_faces(self, axis, value):
        n = ct.c_int64()
        _abi.check(self._lib.pa_mesh_boundary_faces(self._h, axis, float(value), None, ct.byref(n)))
        faces = np.empty((n.value, 3), np.int32)
        _abi.check(self._lib.pa_mesh_boundary_faces(self._h, axis, float(value), _ptr(faces, np.int32), ct.byref(n)))
        return faces

    def close(self):
        if self._h:
            self._lib.pa_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolveOptions:
    def __init__(self, method="fp64", rel_tol=1e-10, max_iters=0, check_every=64, use_initial_guess=False,
                 mg_coarse="auto"):
        """mg_coarse (method "mg"): "auto" solves the coarsest level of an elastic
        solve with a dense inverse when it has at most 2048 dofs (J2 tangent
        solves iterate), "chebyshev" always iterates."""
        self.method, self.rel_tol, self.max_iters = method, rel_tol, max_iters
        self.check_every, self.use_initial_guess = check_every, use_initial_guess
        if mg_coarse not in ("auto", "chebyshev"):
            raise ValueError("mg_coarse must be 'auto' or 'chebyshev'")
        self.mg_coarse = mg_coarse

    def c(self):
        o = _abi.SolveOptions()
        _abi.load().pa_solve_options_default(ct.byref(o))
        o.method = {"fp64": _abi.PA_SOLVER_PCG_FP64, "mixed": _abi.PA_SOLVER_PCG_MIXED,
                    "learned": _abi.PA_SOLVER_FCG_LEARNED, "mg": _abi.PA_SOLVER_PCG_MG}[self.method]
        o.rel_tol = float(self.rel_tol)
        o.max_iters = int(self.max_iters)
        o.check_every = int(self.check_every)
        o.use_initial_guess = int(bool(self.use_initial_guess))
        o.mg_coarse_solver = _abi.PA_MG_COARSE_AUTO if self.mg_coarse == "auto" else _abi.PA_MG_COARSE_CHEBYSHEV
        return o


class Problem:
    """Elliptic mechanics problem (Elliptic::Problem<Mechanics<3>>)."""

    def __init__(self, mesh, youngs_modulus=1.0, poissons_ratio=0.3, simp_exponent=3.0, simp_min=1e-9,
                 control_layout="nodal", stream=None):
        self._lib = _abi.load()
        self.mesh = mesh
        self.control_layout = control_layout
        p = _abi.ElasticParams(youngs_modulus, poissons_ratio, simp_exponent, simp_min,
                               _abi.PA_CONTROL_CELL if control_layout == "cell" else _abi.PA_CONTROL_NODAL)
        h = ct.c_void_p()
        _abi.check(self._lib.pa_problem_create(mesh._h, ct.byref(p), ct.c_void_p(stream or 0), ct.byref(h)))
        self._h = h
        self.ndof = 3 * mesh.num_nodes
        self.nz = mesh.num_cells if control_layout == "cell" else mesh.num_nodes

    # -- boundary conditions -------------------------------------------------
    def add_traction(self, faces, flux):
        faces = np.ascontiguousarray(faces, np.int32)
        flux = np.ascontiguousarray(flux, np.float64)
        _abi.check(self._lib.pa_problem_add_traction(self._h, _ptr(faces, np.int32), faces.shape[0],
                                                     _ptr(flux, np.float64, 3)))

    def clear_tractions(self):
        _abi.check(self._lib.pa_problem_clear_tractions(self._h))

    def set_dirichlet(self, dofs, values=None):
        dofs = np.ascontiguousarray(dofs, np.int32)
        values = np.zeros(dofs.size) if values is None else np.ascontiguousarray(values, np.float64)
        _abi.check(self._lib.pa_problem_set_dirichlet(self._h, _ptr(dofs, np.int32), _ptr(values, np.float64),
                                                      dofs.size))

    # -- functions -------------------------------------------------------------
    def vector_function(self):
        return VectorFunction(self)

    def scalar_function(self, name="Internal Elastic Energy"):
        if name != "Internal Elastic Energy":
            raise NotImplementedError(f"criterion {name!r} is outside this build's scope")
        return PhysicsScalarFunction(self)

    def apply(self, z, x, y=None, constrained=False):
        """Matrix-free y = K(z) x in the precision of x (float64 or float32)."""
        z = _as(z, np.float64)
        fp32 = (x.dtype == np.float32) if not _is_torch(x) else (str(x.dtype) == "torch.float32")
        dt = np.float32 if fp32 else np.float64
        y = _empty(x, self.ndof, dt) if y is None else y
        _abi.check(self._lib.pa_apply(self._h, _ptr(z, np.float64, self.nz, "z"),
                                      _ptr(x, dt, self.ndof, "x"), _ptr(y, dt, self.ndof, "y"),
                                      _abi.PA_FP32 if fp32 else _abi.PA_FP64, int(bool(constrained))))
        return y

    def apply_block_constraints(self, entries, rhs, scale=1.0):
        _abi.check(self._lib.pa_apply_block_constraints(self._h, _ptr(entries, np.float64, 9 * self.mesh.num_blocks),
                                                        _ptr(rhs, np.float64, self.ndof), float(scale)))
        return entries, rhs

    # -- solves ------------------------------------------------------------------
    def solve(self, z, b, x=None, options=None, allow_not_converged=False):
        b = _as(b, np.float64)
        z = _as(z, np.float64)
        options = options or SolveOptions()
        x = _empty(b, self.ndof) if x is None else x
        st = _abi.SolveStats()
        o = options.c()
        s = self._lib.pa_solve(self._h, _ptr(z, np.float64, self.nz, "z"),
                               _ptr(b, np.float64, self.ndof, "b"), _ptr(x, np.float64, self.ndof, "x"),
                               ct.byref(o), ct.byref(st))
        _abi.check(s, allow=(3,) if allow_not_converged else ())
        return x, _stats(st)

    def solution(self, z, u=None, options=None, allow_not_converged=False):
        """Elliptic::Problem::solution: one Newton step from u = 0."""
        z = _as(z, np.float64)
        options = options or SolveOptions()
        u = _empty(z, self.ndof) if u is None else u
        st = _abi.SolveStats()
        o = options.c()
        s = self._lib.pa_problem_solution(self._h, _ptr(z, np.float64, self.nz, "z"),
                                          _ptr(u, np.float64, self.ndof, "u"), ct.byref(o), ct.byref(st))
        _abi.check(s, allow=(3,) if allow_not_converged else ())
        return u, _stats(st)

    def criterion_value(self, z, u):
        return self.scalar_function().value(u, z)

    def part_stats(self):
        """Per-part iterations and relative residuals of the last batched solve."""
        P = self.mesh.num_parts
        it = np.empty(P, np.int32)
        rr = np.empty(P, np.float64)
        _abi.check(self._lib.pa_problem_part_stats(self._h, _ptr(it, np.int32), _ptr(rr, np.float64)))
        return it, rr

    def autotune_tiles(self, z):
        """Pick the fastest tile size (64/128/256 clusters) for the fused CG kernel at density z."""
        z = _as(z, np.float64)
        k = ct.c_int32()
        ms = np.zeros(3)
        _abi.check(self._lib.pa_problem_autotune_tiles(self._h, _ptr(z, np.float64, self.nz, "z"), ct.byref(k),
                                                       _ptr(ms, np.float64, 3)))
        C, N, B, T = (ct.c_int64() for _ in range(4))
        _abi.check(self._lib.pa_mesh_sizes(self.mesh._h, ct.byref(C), ct.byref(N), ct.byref(B), ct.byref(T)))
        self.mesh.num_tiles = T.value
        return k.value, dict(zip((64, 128, 256), ms.tolist()))

    def coarse_grid(self):
        """Level-1 hex counts of the box multigrid (the coarse-weight network's grid)."""
        d = np.zeros(3, np.int32)
        _abi.check(self._lib.pa_boxmg_coarse_grid(self._h, _ptr(d, np.int32, 3)))
        return tuple(int(v) for v in d)

    def coarse_features(self, z, out=None):
        """The coarse-weight network's input features for control z (5 per level-1 hex)."""
        z = _as(z, np.float64)
        g = self.coarse_grid()
        n = 5 * g[0] * g[1] * g[2]
        out = _empty(z, n, np.float32) if out is None else out
        _abi.check(self._lib.pa_boxmg_coarse_features(self._h, _ptr(z, np.float64, self.nz, "z"),
                                                      _ptr(out, np.float32, n, "features")))
        return out

    def coarse_sensitivity(self, z, delta, residuals, energies, grad=None):
        """(loss, dloss/ddelta) of the V-cycle with level-1 weights mean * exp(delta)
        on residual/error pairs (residuals: k x 3N, energies: k)."""
        z = _as(z, np.float64)
        delta = _as(delta, np.float32)
        residuals = _as(residuals, np.float64)
        en = np.ascontiguousarray(np.asarray(energies, np.float64).ravel())
        k = en.size
        g = self.coarse_grid()
        H1 = g[0] * g[1] * g[2]
        grad = _empty(delta, H1, np.float32) if grad is None else grad
        loss = ct.c_double()
        _abi.check(self._lib.pa_boxmg_coarse_sensitivity(
            self._h, _ptr(z, np.float64, self.nz, "z"), _ptr(delta, np.float32, H1, "delta"), int(k),
            _ptr(residuals, np.float64, k * self.ndof, "residuals"), _ptr(en, np.float64, k), ct.byref(loss),
            _ptr(grad, np.float32, H1, "grad")))
        return loss.value, grad

    def set_coarse_network(self, net):
        """Network that corrects the box multigrid's level-1 weights (None detaches)."""
        h = net._h if net is not None else None
        _abi.check(self._lib.pa_problem_set_coarse_network(self._h, h))
        self._coarse_net = net

    def set_preconditioner(self, pc):
        """Network SolveOptions("learned") uses (None detaches); the mesh must be its grid."""
        _abi.check(self._lib.pa_problem_set_preconditioner(self._h, pc._h if pc is not None else None))
        self._pc = pc

    def criterion_gradient(self, z, u, self_adjoint=True, options=None):
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        options = options or SolveOptions()
        g = _empty(z, self.nz)
        o = options.c()
        _abi.check(self._lib.pa_problem_criterion_gradient(self._h, _ptr(z, np.float64, self.nz, "z"),
                                                           _ptr(u, np.float64, self.ndof, "u"),
                                                           _ptr(g, np.float64, self.nz, "grad"),
                                                           int(bool(self_adjoint)), ct.byref(o)))
        return g

    def j2_radial_return(self, params, u, z, prev_local, local=None):
        """J2PlasticityLocalResidual::updateLocalState for every cell (C x 14 states)."""
        prev_local = _as(prev_local, np.float64)
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        C = self.mesh.num_cells
        local = _empty(u, 14 * C) if local is None else local
        jp = self._j2_params(params)
        _abi.check(self._lib.pa_j2_radial_return(self._h, ct.byref(jp), _ptr(u, np.float64, self.ndof),
                                                 _ptr(z, np.float64, self.mesh.num_nodes),
                                                 _ptr(prev_local, np.float64, 14 * C, "prev_local"),
                                                 _ptr(local, np.float64, 14 * C, "local")))
        return local

    def up_residual(self, params, state, local, ppg, z, per_cell_ppg=False, assembled=True, out=None):
        """Stabilized u-p plasticity residual (InfinitesimalStrainPlasticityResidual::evaluate):
        per cell (C x 16) or assembled (4N)."""
        C, N = self.mesh.num_cells, self.mesh.num_nodes
        state, local, ppg, z = (_as(a, np.float64) for a in (state, local, ppg, z))
        n_out = 4 * N if assembled else 16 * C
        out = _empty(state, n_out) if out is None else out
        up = self._up_params(params)
        _abi.check(self._lib.pa_up_residual(self._h, ct.byref(up), _ptr(state, np.float64, 4 * N, "state"),
                                            _ptr(local, np.float64, 14 * C, "local"),
                                            _ptr(ppg, np.float64, 12 * C if per_cell_ppg else 3 * N, "ppg"),
                                            int(bool(per_cell_ppg)), _ptr(z, np.float64, N, "z"),
                                            _ptr(out, np.float64, n_out, "residual"), int(bool(assembled))))
        return out

    @staticmethod
    def _up_params(params):
        return _abi.UpParams(*[float(params.get(k, d)) for k, d in (
            ("youngs_modulus", None), ("poissons_ratio", None), ("penalty_exponent", 3.0), ("penalty_min", 1e-9),
            ("pressure_scaling", 1.0))])

    def up_solve(self, up_params, j2_params, z, steps=1, max_newton=20, newton_tol=1e-10, rel_tol=1e-12,
                 max_iters=0, state=None, local=None, ppg=None, allow_not_converged=False):
        """Stabilized u-p J2 plasticity solve (pa_up_solve): returns the state
        (u_x, u_y, u_z, p per node), the local states (C x 14), the projected
        pressure gradient of the last step (3N) and the solve statistics."""
        C, N = self.mesh.num_cells, self.mesh.num_nodes
        z = _as(z, np.float64)
        state = _empty(z, 4 * N) if state is None else state
        local = _empty(z, 14 * C) if local is None else local
        ppg = _empty(z, 3 * N) if ppg is None else ppg
        up = self._up_params(up_params)
        jp = self._j2_params(j2_params)
        jo = _abi.J2SolveOptions(int(steps), int(max_newton), float(newton_tol), 0)
        lo = SolveOptions("fp64", rel_tol=rel_tol, max_iters=max_iters).c()
        js = _abi.J2Stats()
        status = self._lib.pa_up_solve(self._h, ct.byref(up), ct.byref(jp), _ptr(z, np.float64, N, "z"), ct.byref(jo),
                                       ct.byref(lo), _ptr(state, np.float64, 4 * N, "state"),
                                       _ptr(local, np.float64, 14 * C, "local"), _ptr(ppg, np.float64, 3 * N, "ppg"),
                                       ct.byref(js))
        _abi.check(status, allow=(3,) if allow_not_converged else ())
        return state, local, ppg, {"steps": js.steps, "newton_iterations": js.newton_iterations,
                                   "minres_iterations": js.cg_iterations, "seconds": js.seconds,
                                   "final_rel_residual": js.final_rel_residual, "converged": bool(js.converged),
                                   "linear_unconverged": js.linear_unconverged,
                                   "line_search_halvings": js.line_search_halvings}

    def up_elastic_work(self, up_params, j2_params, z, steps=1, max_newton=20, newton_tol=1e-10, rel_tol=1e-12,
                        max_iters=0, penalty_exponent=3.0, penalty_min=1e-9, gradient=None, state=None, local=None):
        """"Elastic Work" of the u-p plasticity problem summed over the load
        steps and its gradient with respect to the nodal controls by the
        path-dependent adjoint (pa_up_elastic_work).  Returns (value,
        gradient, state, local states, statistics)."""
        C, N = self.mesh.num_cells, self.mesh.num_nodes
        z = _as(z, np.float64)
        gradient = _empty(z, N) if gradient is None else gradient
        state = _empty(z, 4 * N) if state is None else state
        local = _empty(z, 14 * C) if local is None else local
        up = self._up_params(up_params)
        jp = self._j2_params(j2_params)
        jo = _abi.J2SolveOptions(int(steps), int(max_newton), float(newton_tol), 0)
        lo = SolveOptions("fp64", rel_tol=rel_tol, max_iters=max_iters).c()
        js = _abi.J2Stats()
        value = ct.c_double()
        _abi.check(self._lib.pa_up_elastic_work(self._h, ct.byref(up), ct.byref(jp), float(penalty_exponent),
                                                float(penalty_min), _ptr(z, np.float64, N, "z"), ct.byref(jo),
                                                ct.byref(lo), ct.byref(value), _ptr(gradient, np.float64, N, "gradient"),
                                                _ptr(state, np.float64, 4 * N, "state"),
                                                _ptr(local, np.float64, 14 * C, "local"), ct.byref(js)))
        return value.value, gradient, state, local, {"newton_iterations": js.newton_iterations,
                                                     "minres_iterations": js.cg_iterations, "seconds": js.seconds,
                                                     "converged": bool(js.converged)}

    @staticmethod
    def _j2_params(params):
        return _abi.J2Params(*[float(params[k]) for k in (
            "youngs_modulus", "poissons_ratio", "initial_yield_stress", "hardening_modulus_isotropic",
            "hardening_modulus_kinematic", "elastic_penalty_exponent", "elastic_min_ersatz",
            "plastic_penalty_exponent", "plastic_min_ersatz")])

    def j2_local_residual(self, params, u, z, local, prev_local, out=None):
        """J2PlasticityLocalResidual::evaluate for every cell (C x 14)."""
        C = self.mesh.num_cells
        u, z = _as(u, np.float64), _as(z, np.float64)
        local, prev_local = _as(local, np.float64), _as(prev_local, np.float64)
        out = _empty(u, 14 * C) if out is None else out
        jp = self._j2_params(params)
        _abi.check(self._lib.pa_j2_local_residual(self._h, ct.byref(jp), _ptr(u, np.float64, self.ndof, "u"),
                                                  _ptr(z, np.float64, self.mesh.num_nodes, "z"),
                                                  _ptr(local, np.float64, 14 * C, "local"),
                                                  _ptr(prev_local, np.float64, 14 * C, "prev_local"),
                                                  _ptr(out, np.float64, 14 * C, "residual")))
        return out

    def j2_solve(self, params, z, steps=20, max_newton=25, newton_tol=1e-8, options=None, u=None, local=None,
                 allow_not_converged=False, adaptive_forcing=False):
        """Load-stepped Newton solve of the J2 problem (pa_j2_solve); the
        problem's Dirichlet values are the final prescribed displacements.
        adaptive_forcing: inexact Newton (Eisenstat-Walker tolerances for the
        tangent solves, options.rel_tol as their floor)."""
        C = self.mesh.num_cells
        z = _as(z, np.float64)
        u = _empty(z, self.ndof) if u is None else u
        local = _empty(z, 14 * C) if local is None else local
        jp = self._j2_params(params)
        jo = _abi.J2SolveOptions(int(steps), int(max_newton), float(newton_tol), 1 if adaptive_forcing else 0)
        lo = (options or SolveOptions("mixed", rel_tol=1e-8)).c()
        js = _abi.J2Stats()
        status = self._lib.pa_j2_solve(self._h, ct.byref(jp), _ptr(z, np.float64, self.mesh.num_nodes, "z"),
                                       ct.byref(jo), ct.byref(lo), _ptr(u, np.float64, self.ndof, "u"),
                                       _ptr(local, np.float64, 14 * C, "local"), ct.byref(js))
        _abi.check(status, allow=(3,) if allow_not_converged else ())
        return u, local, {"steps": js.steps, "newton_iterations": js.newton_iterations,
                          "cg_iterations": js.cg_iterations, "seconds": js.seconds,
                          "final_rel_residual": js.final_rel_residual, "converged": bool(js.converged),
                          "linear_unconverged": js.linear_unconverged,
                          "line_search_halvings": js.line_search_halvings}

    def close(self):
        if self._h:
            self._lib.pa_problem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_exodus(path):
    """(cells C x 4, coords N x 3, {node set name: node ids}) of an Exodus II
    file, read by the library's netCDF classic reader (host only)."""
    lib = _abi.load()
    h = ct.c_void_p()
    _abi.check(lib.pa_exodus_open(os.fsencode(path), ct.byref(h)))
    try:
        N, C, S = ct.c_int64(), ct.c_int64(), ct.c_int32()
        _abi.check(lib.pa_exodus_sizes(h, ct.byref(N), ct.byref(C), ct.byref(S)))
        coords = np.empty((N.value, 3), np.float64)
        cells = np.empty((C.value, 4), np.int32)
        _abi.check(lib.pa_exodus_mesh(h, _ptr(coords, np.float64), _ptr(cells, np.int32)))
        sets = {}
        for i in range(S.value):
            name = ct.create_string_buffer(256)
            n = ct.c_int64()
            _abi.check(lib.pa_exodus_node_set(h, i, name, 256, ct.byref(n), None))
            nodes = np.empty(n.value, np.int32)
            _abi.check(lib.pa_exodus_node_set(h, i, None, 0, None, _ptr(nodes, np.int32) if n.value else None))
            sets[name.value.decode()] = nodes
        return cells, coords, sets
    finally:
        lib.pa_exodus_close(h)


def _stats(st):
    return {"iterations": st.iterations, "replacements": st.replacements, "rel_residual": st.rel_residual,
            "seconds": st.seconds, "converged": bool(st.converged), "kernel_launches": st.kernel_launches,
            "fallback_iterations": st.fallback_iterations}


class VectorFunction:
    """Elliptic::VectorFunction for the elastostatics residual."""

    def __init__(self, problem):
        self.p = problem

    def value(self, u, z, out=None):
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        out = _empty(u, self.p.ndof) if out is None else out
        _abi.check(self.p._lib.pa_vf_value(self.p._h, _ptr(u, np.float64, self.p.ndof, "u"),
                                           _ptr(z, np.float64, self.p.nz, "z"),
                                           _ptr(out, np.float64, self.p.ndof, "r")))
        return out

    def gradient_u(self, u, z, out=None):
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        n = 9 * self.p.mesh.num_blocks
        out = _empty(u, n) if out is None else out
        _abi.check(self.p._lib.pa_vf_gradient_u(self.p._h, _ptr(u, np.float64, self.p.ndof, "u"),
                                                _ptr(z, np.float64, self.p.nz, "z"),
                                                _ptr(out, np.float64, n, "entries")))
        return out

    def gradient_z(self, u, z, out=None):
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        n = 12 * self.p.mesh.num_cells if self.p.control_layout == "cell" else 3 * self.p.mesh.num_blocks
        out = _empty(u, n) if out is None else out
        _abi.check(self.p._lib.pa_vf_gradient_z(self.p._h, _ptr(u, np.float64, self.p.ndof, "u"),
                                                _ptr(z, np.float64, self.p.nz, "z"),
                                                _ptr(out, np.float64, n, "entries")))
        return out


    def gradient_x(self, u, z, out=None):
        """dR/dx transposed into block-CRS entries (VectorFunction::gradient_x)."""
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        n = 9 * self.p.mesh.num_blocks
        out = _empty(u, n) if out is None else out
        _abi.check(self.p._lib.pa_vf_gradient_x(self.p._h, _ptr(u, np.float64, self.p.ndof, "u"),
                                                _ptr(z, np.float64, self.p.nz, "z"),
                                                _ptr(out, np.float64, n, "entries")))
        return out


class PhysicsScalarFunction:
    """PhysicsScalarFunction for the "Internal Elastic Energy" criterion."""

    def __init__(self, problem):
        self.p = problem

    def value(self, u, z):
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        v = ct.c_double()
        _abi.check(self.p._lib.pa_sf_value(self.p._h, _ptr(u, np.float64, self.p.ndof, "u"),
                                           _ptr(z, np.float64, self.p.nz, "z"), ct.byref(v)))
        return v.value

    def gradient_u(self, u, z, out=None):
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        out = _empty(u, self.p.ndof) if out is None else out
        _abi.check(self.p._lib.pa_sf_gradient_u(self.p._h, _ptr(u, np.float64, self.p.ndof, "u"),
                                                _ptr(z, np.float64, self.p.nz, "z"),
                                                _ptr(out, np.float64, self.p.ndof, "grad")))
        return out

    def gradient_z(self, u, z, out=None):
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        out = _empty(u, self.p.nz) if out is None else out
        _abi.check(self.p._lib.pa_sf_gradient_z(self.p._h, _ptr(u, np.float64, self.p.ndof, "u"),
                                                _ptr(z, np.float64, self.p.nz, "z"),
                                                _ptr(out, np.float64, self.p.nz, "grad")))
        return out

    def gradient_x(self, u, z, out=None):
        u = _as(u, np.float64)
        z = _as(z, np.float64)
        out = _empty(u, self.p.ndof) if out is None else out
        _abi.check(self.p._lib.pa_sf_gradient_x(self.p._h, _ptr(u, np.float64, self.p.ndof, "u"),
                                                _ptr(z, np.float64, self.p.nz, "z"),
                                                _ptr(out, np.float64, self.p.ndof, "grad")))
        return out


class LearnedPreconditioner:
    """Convolutional preconditioner on the nodal grid of a structured box
    (pa_pc_*): M r = D^-1 r + s D^-1/2 f(D^-1/2 r / s, stiffness, Dirichlet).
    No counterpart in the reference; used by SolveOptions("learned")."""

    def __init__(self, grid, seed=0):
        self._lib = _abi.load()
        self.grid = tuple(int(g) for g in grid)
        h = ct.c_void_p()
        _abi.check(self._lib.pa_pc_create(*self.grid, ct.c_uint64(seed), ct.byref(h)))
        self._h = h
        n = ct.c_int64()
        _abi.check(self._lib.pa_pc_num_params(self._h, ct.byref(n)))
        self.num_params = n.value
        self.num_points = self.grid[0] * self.grid[1] * self.grid[2]

    @classmethod
    def for_box(cls, nx, ny, nz, seed=0):
        return cls((nx + 1, ny + 1, nz + 1), seed)

    def get_params(self):
        out = np.empty(self.num_params, np.float32)
        _abi.check(self._lib.pa_pc_get_params(self._h, _ptr(out, np.float32, self.num_params)))
        return out

    def set_params(self, params):
        params = np.ascontiguousarray(params, np.float32)
        _abi.check(self._lib.pa_pc_set_params(self._h, _ptr(params, np.float32, self.num_params, "params")))

    def forward(self, features):
        f = _as(features, np.float32)
        out = _empty(f, 3 * self.num_points, np.float32)
        _abi.check(self._lib.pa_pc_forward(self._h, _ptr(f, np.float32, 5 * self.num_points, "features"),
                                           _ptr(out, np.float32, 3 * self.num_points, "out")))
        return out

    def backward(self, features, grad_out):
        f = _as(features, np.float32)
        g = _as(grad_out, np.float32)
        out = _empty(f, self.num_params, np.float32)
        _abi.check(self._lib.pa_pc_backward(self._h, _ptr(f, np.float32, 5 * self.num_points, "features"),
                                            _ptr(g, np.float32, 3 * self.num_points, "grad_out"),
                                            _ptr(out, np.float32, self.num_params, "grad_params")))
        return out

    def time_forward(self, reps=20):
        """(ms per forward of the four convolutions, algorithmic FLOPs) on the last input."""
        ms, fl = ct.c_double(), ct.c_int64()
        _abi.check(self._lib.pa_pc_time_forward(self._h, int(reps), ct.byref(ms), ct.byref(fl)))
        return ms.value, fl.value

    def apply(self, problem, z, r, out=None):
        z, r = _as(z, np.float64), _as(r, np.float64)
        out = _empty(r, problem.ndof) if out is None else out
        _abi.check(self._lib.pa_pc_apply(problem._h, self._h, _ptr(z, np.float64, problem.nz, "z"),
                                         _ptr(r, np.float64, problem.ndof, "r"),
                                         _ptr(out, np.float64, problem.ndof, "out")))
        return out

    def train(self, problem, densities, sample_density, residuals, energies, steps=200, batch=4,
              learning_rate=1e-3, seed=0):
        """Train on (residual, error) pairs: residuals[s] = K(densities[sample_density[s]]) e_s
        (zero on constrained dofs), energies[s] = e_s . residuals[s]."""
        densities = _as(densities, np.float64)
        residuals = _as(residuals, np.float64)
        sd = np.ascontiguousarray(sample_density, np.int32)
        en = np.ascontiguousarray(energies, np.float64)
        nd = (densities.numel() if _is_torch(densities) else densities.size) // problem.nz
        ns = sd.size
        o = _abi.PcTrainOptions(int(steps), int(batch), float(learning_rate), int(seed))
        st = _abi.PcTrainStats()
        _abi.check(self._lib.pa_pc_train(problem._h, self._h, nd, _ptr(densities, np.float64, nd * problem.nz,
                                                                          "densities"),
                                         ns, _ptr(sd, np.int32, ns), _ptr(residuals, np.float64, ns * problem.ndof,
                                                                          "residuals"),
                                         _ptr(en, np.float64, ns), ct.byref(o), ct.byref(st)))
        return {"initial_loss": st.initial_loss, "final_loss": st.final_loss, "seconds": st.seconds,
                "steps": st.steps, "kernel_launches": st.kernel_launches}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pa_pc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LearnedCoarsening:
    """Learned level-1 weights of the box multigrid (PA_SOLVER_PCG_MG): a
    convolutional network on the level-1 hex grid (the same four-layer BF16
    network as LearnedPreconditioner, tcgen05 forward, the library's backward
    kernels) maps 5 features per coarse hex to delta, and the coarse hex gets
    mean(child weights) * exp(0.5 tanh(delta)).  A new network (last layer
    zero) is the plain multigrid.  Trained on residual/error pairs (K e = r) of
    SIMP designs by Adam on the mean of ||e - V r||_K^2 / ||e||_K^2 (V the
    V-cycle), with dloss/ddelta from pa_boxmg_coarse_sensitivity; the plain
    multigrid decides: every `check_every` steps the CG iterations on a
    validation control are counted, and training keeps the parameters with
    the fewest (the untrained ones unless some beat them).  No counterpart in
    the reference."""

    def __init__(self, problem, seed=0):
        self.grid = problem.coarse_grid()
        self.net = LearnedPreconditioner(self.grid, seed)
        self.num_points = self.net.num_points

    def delta(self, problem, z):
        """The correction delta (one per level-1 hex) the network gives for control z."""
        return self.net.forward(problem.coarse_features(z))[0::3]

    def attach(self, problem):
        problem.set_coarse_network(self.net)

    def iterations(self, problem, z, rel_tol=1e-8):
        """CG iterations of the multigrid solve of control z with this network attached."""
        self.attach(problem)
        try:
            _, st = problem.solution(z, options=SolveOptions("mg", rel_tol=rel_tol), allow_not_converged=True)
        finally:
            problem.set_coarse_network(None)
        return st["iterations"]

    def train(self, problem, designs, residuals, energies, sample_design, steps=100, batch=4, learning_rate=3e-3,
              seed=0, log=None, validation=None, check_every=20):
        """designs: D x nz controls; residuals[s] (3N, zero on constrained dofs)
        with K(designs[sample_design[s]]) e_s = residuals[s], energies[s] = e_s . r_s.
        Each step takes one design and `batch` of its samples.  validation: a
        control whose multigrid CG iterations select the parameters kept
        (None: the last ones).  Returns {"loss": per-step loss before the
        update, "iterations": [(step, iterations)], "kept_step": step of the
        kept parameters (0: untrained)}."""
        import torch
        dev = residuals.device
        sd = np.asarray(sample_design, np.int64)
        en = np.asarray(energies, np.float64)
        rng = np.random.default_rng(seed)
        params = torch.tensor(self.net.get_params(), device=dev)
        m = torch.zeros_like(params)
        v = torch.zeros_like(params)
        b1, b2, eps = 0.9, 0.999, 1e-8
        feats = {}
        hist = []
        checks = []
        best = None
        if validation is not None:
            best = (self.iterations(problem, validation), 0, params.clone())
            checks.append((0, best[0]))
        for step in range(steps):
            d = int(sd[rng.integers(0, sd.size)])
            idx = np.flatnonzero(sd == d)
            pick = rng.choice(idx, size=min(batch, idx.size), replace=False)
            z = designs[d]
            if d not in feats:
                feats[d] = problem.coarse_features(z)
            f = feats[d]
            out = self.net.forward(f)
            delta = out[0::3].contiguous()
            loss, gd = problem.coarse_sensitivity(z, delta, residuals[torch.as_tensor(pick, device=dev)].contiguous(),
                                                  en[pick])
            gout = torch.zeros(3 * self.num_points, dtype=torch.float32, device=dev)
            gout[0::3] = gd
            g = self.net.backward(f, gout)
            hist.append(loss)
            if log:
                log(step, loss)
            m.mul_(b1).add_(g, alpha=1 - b1)
            v.mul_(b2).addcmul_(g, g, value=1 - b2)
            mh = m / (1 - b1 ** (step + 1))
            vh = v / (1 - b2 ** (step + 1))
            params.sub_(learning_rate * mh / (vh.sqrt() + eps))
            self._upload(params)
            if validation is not None and ((step + 1) % check_every == 0 or step + 1 == steps):
                it = self.iterations(problem, validation)
                checks.append((step + 1, it))
                if it < best[0]:
                    best = (it, step + 1, params.clone())
        kept = steps
        if best is not None:
            self._upload(best[2])
            kept = best[1]
        return {"loss": hist, "iterations": checks, "kept_step": kept}

    def _upload(self, params):
        _abi.check(self.net._lib.pa_pc_set_params(self.net._h, _ptr(params, np.float32, self.net.num_params,
                                                                     "params")))

    def close(self):
        self.net.close()
