"""Stabilized u-p plasticity residual on the GPU through the C ABI: the
reference's gold (ElastoPlasticity_Residual3D_Elastic) and FP64 parity with
the NumPy restatement on a jittered box with plastic local states."""
import numpy as np
import pytest

from oracle import np_ref, np_up

pytestmark = pytest.mark.gpu


def test_up_residual_reference_gold(pa):
    from test_oracle_up import up_case
    d, cells, coords, state, ppg = up_case()
    m = d["material"]
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, m["youngs_modulus"], m["poissons_ratio"])
    params = dict(youngs_modulus=m["youngs_modulus"], poissons_ratio=m["poissons_ratio"],
                  penalty_exponent=m["simp_exponent"], penalty_min=m["simp_min"],
                  pressure_scaling=m["pressure_scaling"])
    R = prob.up_residual(params, state, np.zeros(6 * 14), ppg.ravel(), np.ones(8), per_cell_ppg=True,
                         assembled=False).reshape(6, 16)
    gold = np.array(d["gold"])
    assert np.all(np.abs(R - gold) <= d["tolerance"] * np.abs(gold))
    ref = np_up.up_residual_cells(cells, coords, state, np.zeros((6, 14)), ppg.reshape(6, 4, 3), np.ones(8),
                                  m["youngs_modulus"], m["poissons_ratio"], m["simp_exponent"], m["simp_min"])
    assert np.abs(R - ref).max() <= 1e-10 * np.abs(ref).max()


def test_up_residual_parity_plastic_states(pa):
    rng = np.random.default_rng(21)
    nx, ny, nz = 5, 3, 3
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    coords = coords + rng.uniform(-0.15, 0.15, coords.shape)
    N, C = coords.shape[0], cells.shape[0]
    state = rng.normal(size=4 * N) * np.tile([1e-3, 1e-3, 1e-3, 10.0], N)
    local = np.zeros((C, 14))
    local[:, 2:8] = rng.normal(scale=1e-4, size=(C, 6))
    local[:, 0] = rng.uniform(0, 1e-3, C)
    ppg = rng.normal(size=3 * N)
    z = rng.uniform(0.2, 1.0, N)
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, 200e3, 0.3)
    params = dict(youngs_modulus=200e3, poissons_ratio=0.3, penalty_exponent=3.0, penalty_min=1e-9,
                  pressure_scaling=2.5)
    R = prob.up_residual(params, state, local.ravel(), ppg, z, assembled=True)
    ppg_cells = ppg.reshape(-1, 3)[cells]
    Rc = np_up.up_residual_cells(cells, coords, state, local, ppg_cells, z, 200e3, 0.3, 3.0, 1e-9, 2.5)
    ref = np.zeros((N, 4))
    for c in range(C):
        np.add.at(ref, cells[c], Rc[c].reshape(4, 4))
    ref = ref.ravel()
    assert np.abs(R - ref).max() <= 1e-10 * np.abs(ref).max()
    Rp = prob.up_residual(params, state, local.ravel(), ppg_cells.ravel(), z, per_cell_ppg=True,
                          assembled=False).reshape(C, 16)
    assert np.abs(Rp - Rc).max() <= 1e-10 * np.abs(Rc).max()


def _j2_dict(d):
    m, j = d["material"], d["j2"]
    return dict(youngs_modulus=m["youngs_modulus"], poissons_ratio=m["poissons_ratio"], **j)


def test_up_solve_reference_elastic_solution(pa):
    """pa_up_solve reproduces ElastoPlasticity_ElasticSolution3D
    (unit_tests/ElastoPlasticityTests.cpp:2101-2233) within the reference's
    tolerance, and the NumPy u-p Newton to 1e-9."""
    from test_oracle_up import elastic_solution_case, up_j2_params
    d, cells, coords, dofs4, vals = elastic_solution_case()
    m = d["material"]
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, m["youngs_modulus"], m["poissons_ratio"])
    dofs3 = 3 * (dofs4 // 4) + dofs4 % 4
    o = np.argsort(dofs3)
    prob.set_dirichlet(dofs3[o].astype(np.int32), vals[o])
    up = dict(youngs_modulus=m["youngs_modulus"], poissons_ratio=m["poissons_ratio"],
              penalty_exponent=m["simp_exponent"], penalty_min=m["simp_min"], pressure_scaling=m["pressure_scaling"])
    state, local, ppg, st = prob.up_solve(up, _j2_dict(d), np.ones(8), steps=d["steps"], newton_tol=1e-10)
    assert st["converged"], st
    gold = np.array(d["gold"])
    assert np.all(np.abs(state - gold) <= d["tolerance"] * np.abs(gold))
    assert np.all(state[gold == 0.0] == 0.0)
    P = np_up.UpProblem(cells, coords, m["youngs_modulus"], m["poissons_ratio"], up_j2_params(d),
                        pe=m["simp_exponent"], pe_min=m["simp_min"], ps=m["pressure_scaling"])
    x, loc, _ = P.solve(dofs4, vals, d["steps"])
    assert np.abs(state - x).max() <= 1e-9 * np.abs(x).max()
    assert np.all(ppg == 0.0)  # one step: the projection is never used


@pytest.mark.parametrize("hkin,ps", [(0.0, 1.0), (400.0, 1.7)])
def test_up_solve_plastic_bar_matches_oracle(pa, hkin, ps):
    """A jittered 6x2x2 bar with nodal SIMP densities stretched to 2 % in 4
    load steps: most cells yield; the state, the local states and the lagged
    projected pressure gradient match the NumPy u-p Newton."""
    from oracle import np_j2
    rng = np.random.default_rng(5)
    nx, ny, nz = 6, 2, 2
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    inner = (coords[:, 0] > 1e-9) & (coords[:, 0] < nx - 1e-9)
    coords = coords + np.where(inner[:, None], rng.uniform(-0.1, 0.1, coords.shape), 0.0)
    N = coords.shape[0]
    z = rng.uniform(0.6, 1.0, N)
    x0 = np.where(coords[:, 0] < 1e-9)[0]
    x1 = np.where(coords[:, 0] > nx - 1e-9)[0]
    dofs3 = np.concatenate([3 * x0, 3 * x0 + 1, 3 * x0 + 2, 3 * x1])
    vals = np.concatenate([np.zeros(3 * x0.size), np.full(x1.size, 0.02 * nx)])
    o = np.argsort(dofs3)
    dofs3, vals = dofs3[o], vals[o]
    E, nu = 200e3, 0.3
    j2 = dict(youngs_modulus=E, poissons_ratio=nu, initial_yield_stress=250.0, hardening_modulus_isotropic=1000.0,
              hardening_modulus_kinematic=hkin, elastic_penalty_exponent=3.0, elastic_min_ersatz=1e-9,
              plastic_penalty_exponent=2.5, plastic_min_ersatz=1e-4)
    up = dict(youngs_modulus=E, poissons_ratio=nu, penalty_exponent=3.0, penalty_min=1e-9, pressure_scaling=ps)
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, E, nu)
    prob.set_dirichlet(dofs3.astype(np.int32), vals)
    steps = 4
    state, local, ppg, st = prob.up_solve(up, j2, z, steps=steps, max_newton=30, newton_tol=1e-11)
    assert st["converged"], st
    prm = np_j2.J2Params(E, nu, 250.0, 1000.0, hkin, pe=3.0, pe_min=1e-9, pp=2.5, pp_min=1e-4)
    P = np_up.UpProblem(cells, coords, E, nu, prm, z=z, pe=3.0, pe_min=1e-9, ps=ps)
    dofs4 = 4 * (dofs3 // 3) + dofs3 % 3
    x, loc_ref, ppg_ref = P.solve(dofs4, vals, steps, tol=1e-12)
    assert P.converged
    loc = np.asarray(local).reshape(-1, 14)
    assert (loc_ref[:, 1] > 0).mean() > 0.5
    u, p = state.reshape(-1, 4)[:, :3], state.reshape(-1, 4)[:, 3]
    ur, pr = x.reshape(-1, 4)[:, :3], x.reshape(-1, 4)[:, 3]
    assert np.abs(u - ur).max() <= 1e-7 * np.abs(ur).max()
    assert np.abs(p - pr).max() <= 1e-7 * np.abs(pr).max()
    assert np.abs(loc - loc_ref).max() <= 1e-6 * np.abs(loc_ref).max()
    assert np.abs(ppg.reshape(-1, 3) - ppg_ref).max() <= 1e-7 * np.abs(ppg_ref).max()
    assert st["newton_iterations"] <= 15 * steps


@pytest.mark.parametrize("steps,strain", [(1, 1e-4), (3, 0.02)])
def test_up_elastic_work_gradient(pa, steps, strain):
    """The path-dependent adjoint gradient of the "Elastic Work" criterion
    (summed over the load steps) against central differences of the NumPy
    u-p Newton's criterion along random control directions; elastic (one
    step) and plastic (three steps, most cells yield, kinematic hardening,
    lagged projection active)."""
    from oracle import np_j2
    rng = np.random.default_rng(11)
    nx = 4
    cells, coords = np_ref.box_mesh(nx, 1, 1, float(nx), 1.0, 1.0)
    inner = (coords[:, 0] > 1e-9) & (coords[:, 0] < nx - 1e-9)
    coords = coords + np.where(inner[:, None], rng.uniform(-0.1, 0.1, coords.shape), 0.0)
    N = coords.shape[0]
    z = rng.uniform(0.6, 1.0, N)
    x0 = np.where(coords[:, 0] < 1e-9)[0]
    x1 = np.where(coords[:, 0] > nx - 1e-9)[0]
    dofs3 = np.concatenate([3 * x0, 3 * x0 + 1, 3 * x0 + 2, 3 * x1])
    vals = np.concatenate([np.zeros(3 * x0.size), np.full(x1.size, strain * nx)])
    o = np.argsort(dofs3)
    dofs3, vals = dofs3[o], vals[o]
    E, nu, ps, fpe = 200e3, 0.3, 1.3, 2.0
    j2 = dict(youngs_modulus=E, poissons_ratio=nu, initial_yield_stress=250.0, hardening_modulus_isotropic=1000.0,
              hardening_modulus_kinematic=400.0, elastic_penalty_exponent=3.0, elastic_min_ersatz=1e-9,
              plastic_penalty_exponent=2.5, plastic_min_ersatz=1e-4)
    up = dict(youngs_modulus=E, poissons_ratio=nu, penalty_exponent=3.0, penalty_min=1e-9, pressure_scaling=ps)
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, E, nu)
    prob.set_dirichlet(dofs3.astype(np.int32), vals)
    value, grad, state, local, st = prob.up_elastic_work(up, j2, z, steps=steps, max_newton=30, newton_tol=1e-12,
                                                         penalty_exponent=fpe)
    assert st["converged"], st
    prm = np_j2.J2Params(E, nu, 250.0, 1000.0, 400.0, pe=3.0, pe_min=1e-9, pp=2.5, pp_min=1e-4)
    dofs4 = 4 * (dofs3 // 3) + dofs3 % 3

    def oracle_value(zz):
        P = np_up.UpProblem(cells, coords, E, nu, prm, z=zz, pe=3.0, pe_min=1e-9, ps=ps)
        P.solve(dofs4, vals, steps, tol=1e-13)
        assert P.converged
        return P.elastic_work(fpe, 1e-9), P

    w0, P0 = oracle_value(z)
    assert abs(value - w0) <= 1e-9 * abs(w0)
    if steps > 1:
        assert (P0.history[-1][1][:, 1] > 0).mean() > 0.8
    h = 1e-5
    for _ in range(3):
        d = rng.normal(size=N)
        fd = (oracle_value(z + h * d)[0] - oracle_value(z - h * d)[0]) / (2 * h)
        assert abs(grad @ d - fd) <= 2e-6 * max(abs(fd), np.abs(grad).sum() * np.abs(d).max() * 1e-3)
