"""J2 plasticity on the GPU through the C ABI: local residual (pinned on the
reference's J2Plasticity_Evaluate3D known answer) and the load-stepped
Newton solve (vs the NumPy J2 oracle with a finite-difference tangent)."""
import numpy as np
import pytest

from golden_util import floating_equality

pytestmark = pytest.mark.gpu


def test_j2_local_residual_evaluate_3d(pa):
    from test_oracle_golden import j2_evaluate_3d_case
    cells, X, u, prm, cur, prev, gold = j2_evaluate_3d_case()
    mesh = pa.Mesh.from_arrays(cells, X)
    prob = pa.Problem(mesh, 520.0, 0.3)
    params = dict(youngs_modulus=520.0, poissons_ratio=0.3, initial_yield_stress=3.0,
                  hardening_modulus_isotropic=20.0, hardening_modulus_kinematic=15.0,
                  elastic_penalty_exponent=3.0, elastic_min_ersatz=1e-9, plastic_penalty_exponent=2.5,
                  plastic_min_ersatz=1e-9)
    C = cells.shape[0]
    H = prob.j2_local_residual(params, u, np.full(X.shape[0], 0.9), np.tile(cur, C), np.tile(prev, C))
    for c in range(C):
        floating_equality(H[14 * c:14 * c + 14], gold, 1e-5)


def _bar(pa, nx, ny, nz, strain, E=200e3, nu=0.3, sy=250.0, hiso=1000.0, hkin=0.0):
    from oracle import np_ref
    L = float(nx)
    cells, coords = np_ref.box_mesh(nx, ny, nz, L, float(ny), float(nz))
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, E, nu)
    x0 = np.where(coords[:, 0] < 1e-9)[0]
    x1 = np.where(coords[:, 0] > L - 1e-9)[0]
    dofs = np.concatenate([3 * x0, 3 * x0 + 1, 3 * x0 + 2, 3 * x1])
    vals = np.concatenate([np.zeros(3 * x0.size), np.full(x1.size, strain * L)])
    order = np.argsort(dofs)
    prob.set_dirichlet(dofs[order].astype(np.int32), vals[order])
    params = dict(youngs_modulus=E, poissons_ratio=nu, initial_yield_stress=sy, hardening_modulus_isotropic=hiso,
                  hardening_modulus_kinematic=hkin, elastic_penalty_exponent=1.0, elastic_min_ersatz=1e-9,
                  plastic_penalty_exponent=0.5, plastic_min_ersatz=1e-4)
    return cells, coords, mesh, prob, params, dofs[order], vals[order]


@pytest.mark.parametrize("method,hkin,forcing", [("fp64", 0.0, False), ("mixed", 0.0, False), ("fp64", 400.0, False),
                                                ("mixed", 0.0, True), ("fp64", 400.0, True)])
def test_j2_newton_matches_oracle(pa, method, hkin, forcing):
    """forcing: inexact Newton (Eisenstat-Walker tangent tolerances); the
    converged solution is held to the same oracle tolerances."""
    from oracle import np_j2
    cells, coords, mesh, prob, params, dofs, vals = _bar(pa, 4, 1, 1, 0.02, hkin=hkin)
    z = np.ones(coords.shape[0])
    steps = 5
    u, local, st = prob.j2_solve(params, z, steps=steps, max_newton=30, newton_tol=1e-10,
                                 options=pa.SolveOptions(method, rel_tol=1e-12 if method == "fp64" else 1e-10),
                                 adaptive_forcing=forcing)
    assert st["converged"], st
    prm = np_j2.J2Params(200e3, 0.3, 250.0, 1000.0, hkin, pe=1.0, pe_min=1e-9, pp=0.5, pp_min=1e-4)
    J = np_j2.J2Problem(cells, coords, prm, z)
    u_ref, loc_ref = J.solve(dofs, vals, steps, tol=1e-12)
    loc = np.asarray(local).reshape(-1, 14)
    assert (loc_ref[:, 1] > 0).any()  # some cells yield in the last step
    assert np.abs(u - u_ref).max() <= 1e-7 * np.abs(u_ref).max()
    assert np.abs(loc - loc_ref).max() <= 1e-6 * max(np.abs(loc_ref).max(), 1e-12) + 1e-12
    # Newton with the consistent tangent converges in a handful of iterations per step
    assert st["newton_iterations"] <= (12 if forcing else 8) * steps


def test_j2_newton_on_a_shuffled_mesh(pa):
    """Cells and their vertex order shuffled (every tet a single cluster in the
    tile kernel, tangent records reached through the single-cell path): the
    same load-stepped solution as the structured numbering."""
    from oracle import np_ref
    rng = np.random.default_rng(8)
    cells, coords = np_ref.box_mesh(6, 2, 2, 6.0, 2.0, 2.0)
    perm = rng.permutation(cells.shape[0])
    shuffled = cells[perm].copy()
    for c in range(shuffled.shape[0]):  # any vertex order is valid: the volume uses |det|
        shuffled[c] = shuffled[c][rng.permutation(4)]
    results = []
    for cl in (cells, shuffled):
        mesh = pa.Mesh.from_arrays(cl, coords)
        prob = pa.Problem(mesh, 200e3, 0.3)
        x0 = np.where(coords[:, 0] < 1e-9)[0]
        x1 = np.where(coords[:, 0] > 6.0 - 1e-9)[0]
        dofs = np.concatenate([3 * x0, 3 * x0 + 1, 3 * x0 + 2, 3 * x1])
        vals = np.concatenate([np.zeros(3 * x0.size), np.full(x1.size, 0.02 * 6.0)])
        order = np.argsort(dofs)
        prob.set_dirichlet(dofs[order].astype(np.int32), vals[order])
        params = dict(youngs_modulus=200e3, poissons_ratio=0.3, initial_yield_stress=250.0,
                      hardening_modulus_isotropic=1000.0, hardening_modulus_kinematic=0.0,
                      elastic_penalty_exponent=3.0, elastic_min_ersatz=1e-9, plastic_penalty_exponent=2.5,
                      plastic_min_ersatz=1e-9)
        u, local, st = prob.j2_solve(params, np.ones(coords.shape[0]), steps=5, max_newton=30, newton_tol=1e-10,
                                     options=pa.SolveOptions("fp64", rel_tol=1e-12))
        assert st["converged"], st
        results.append((u, np.asarray(local).reshape(-1, 14), mesh.num_tiles))
    (u0, l0, _), (u1, l1, _) = results
    assert np.abs(u1 - u0).max() <= 1e-8 * np.abs(u0).max()
    # local states follow the user's cell order
    assert np.abs(l1 - l0[perm]).max() <= 1e-6 * max(np.abs(l0).max(), 1e-12) + 1e-12
    assert (l0[:, 0] > 0).any()


def test_inexact_newton_cuts_cg_work(pa):
    """A 12x4x4 bar yielding over 10 load steps: Eisenstat-Walker tangent
    tolerances reach the same converged field with fewer CG iterations."""
    res = {}
    for forcing in (False, True):
        cells, coords, mesh, prob, params, dofs, vals = _bar(pa, 12, 4, 4, 0.02)
        u, local, st = prob.j2_solve(params, np.ones(coords.shape[0]), steps=10, max_newton=30, newton_tol=1e-9,
                                     options=pa.SolveOptions("mixed", rel_tol=1e-9), adaptive_forcing=forcing)
        assert st["converged"], st
        res[forcing] = (u, np.asarray(local).reshape(-1, 14), st)
    (u0, l0, s0), (u1, l1, s1) = res[False], res[True]
    assert (l0[:, 0] > 0).any()
    assert np.abs(u1 - u0).max() <= 1e-6 * np.abs(u0).max()
    assert np.abs(l1 - l0).max() <= 1e-5 * max(np.abs(l0).max(), 1e-12)
    assert s1["cg_iterations"] < s0["cg_iterations"], (s0, s1)


@pytest.fixture(scope="module")
def bar_8x4x4_oracle():
    """The 8x4x4 bar (768 tets) to 2% axial strain in 4 steps, solved by the
    NumPy J2 oracle (dense Newton, finite-difference tangent, tolerance 1e-12)."""
    from oracle import np_j2
    from platoanalyze_b200.fields import box_arrays
    nx, ny, nz = 8, 4, 4
    cells, coords, _, _ = box_arrays(nx, ny, nz)  # the numbering of pa_mesh_create_box
    x0 = np.where(coords[:, 0] < 1e-9)[0]
    x1 = np.where(coords[:, 0] > nx - 1e-9)[0]
    dofs = np.concatenate([3 * x0, 3 * x0 + 1, 3 * x0 + 2, 3 * x1])
    vals = np.concatenate([np.zeros(3 * x0.size), np.full(x1.size, 0.02 * nx)])
    order = np.argsort(dofs)
    prm = np_j2.J2Params(200e3, 0.3, 250.0, 1000.0, 0.0, pe=1.0, pe_min=1e-9, pp=0.5, pp_min=1e-4)
    J = np_j2.J2Problem(cells, coords, prm, np.ones(coords.shape[0]))
    u_ref, loc_ref = J.solve(dofs[order], vals[order], 4, tol=1e-12)
    assert J.converged
    return u_ref, loc_ref


@pytest.mark.parametrize("method,forcing", [("mg", True), ("fp64", False)])
def test_j2_mid_size_bar_matches_oracle(pa, bar_8x4x4_oracle, method, forcing):
    """The benchmark's J2 setting (box mesh; multigrid tangent solves with
    Eisenstat-Walker tolerances, as bench.py --workload j2 runs it, and FP64
    Jacobi-PCG) on a bar where nearly every cell yields: displacements within
    1e-7 and local states within 1e-6 of the oracle."""
    u_ref, loc_ref = bar_8x4x4_oracle
    nx, ny, nz = 8, 4, 4
    mesh = pa.Mesh.box(nx, ny, nz, float(nx), float(ny), float(nz))
    prob = pa.Problem(mesh, 200e3, 0.3)
    cells, coords = mesh.arrays()
    x0 = np.where(coords[:, 0] < 1e-9)[0]
    x1 = np.where(coords[:, 0] > nx - 1e-9)[0]
    dofs = np.concatenate([3 * x0, 3 * x0 + 1, 3 * x0 + 2, 3 * x1])
    vals = np.concatenate([np.zeros(3 * x0.size), np.full(x1.size, 0.02 * nx)])
    order = np.argsort(dofs)
    prob.set_dirichlet(dofs[order].astype(np.int32), vals[order])
    params = dict(youngs_modulus=200e3, poissons_ratio=0.3, initial_yield_stress=250.0,
                  hardening_modulus_isotropic=1000.0, hardening_modulus_kinematic=0.0, elastic_penalty_exponent=1.0,
                  elastic_min_ersatz=1e-9, plastic_penalty_exponent=0.5, plastic_min_ersatz=1e-4)
    u, local, st = prob.j2_solve(params, np.ones(coords.shape[0]), steps=4, max_newton=30, newton_tol=1e-10,
                                 options=pa.SolveOptions(method, rel_tol=1e-12), adaptive_forcing=forcing)
    assert st["converged"], st
    loc = np.asarray(local).reshape(-1, 14)
    assert (loc_ref[:, 0] > 0).mean() > 0.95  # nearly every cell plastic at 2 %
    assert np.abs(u - u_ref).max() <= 1e-7 * np.abs(u_ref).max()
    assert np.abs(loc - loc_ref).max() <= 1e-6 * np.abs(loc_ref).max()
