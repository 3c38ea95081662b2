"""CPU: the NumPy restatement of the stabilized u-p plasticity residual
(oracle/np_up.py) against the reference's gold values
(unit_tests/ElastoPlasticityTests.cpp:1967-2100, ElastoPlasticity_Residual3D_Elastic)."""
import json
import os

import numpy as np

from oracle import np_up

HERE = os.path.dirname(os.path.abspath(__file__))


def up_case():
    d = json.load(open(os.path.join(HERE, "golden", "up_residual_3d.json")))
    cells = np.array(d["cells"], np.int32)
    coords = np.array(d["coords"])
    ids = np.arange(coords.shape[0], dtype=np.float64)
    state = np.stack([1e-7 * ids, 2e-7 * ids, 3e-7 * ids, 4e-7 * ids], 1).ravel()
    ppg = np.array(d["projected_pressure_gradient"])
    return d, cells, coords, state, ppg


def test_up_residual_matches_reference_gold():
    d, cells, coords, state, ppg = up_case()
    m = d["material"]
    R = np_up.up_residual_cells(cells, coords, state, np.zeros((6, 14)), ppg.reshape(6, 4, 3), np.ones(8),
                                m["youngs_modulus"], m["poissons_ratio"], m["simp_exponent"], m["simp_min"],
                                m["pressure_scaling"])
    gold = np.array(d["gold"])
    assert d["numberings_matching"] == 1
    assert np.all(np.abs(R - gold) <= d["tolerance"] * np.abs(gold))


def elastic_solution_case():
    """The reference's ElastoPlasticity_ElasticSolution3D fixture and its
    Dirichlet dofs in the 4-dof numbering (x = 0: u fixed; x = 1: u_y = -1e-3)."""
    d = json.load(open(os.path.join(HERE, "golden", "up_elastic_solution_3d.json")))
    cells = np.array(d["cells"], np.int32)
    coords = np.array(d["coords"])
    x0 = np.where(coords[:, 0] < 1e-9)[0]
    x1 = np.where(coords[:, 0] > 1 - 1e-9)[0]
    dofs = np.concatenate([4 * x0, 4 * x0 + 1, 4 * x0 + 2, 4 * x1 + 1])
    vals = np.concatenate([np.zeros(3 * x0.size), np.full(x1.size, -1e-3)])
    o = np.argsort(dofs)
    return d, cells, coords, dofs[o], vals[o]


def up_j2_params(d):
    from oracle import np_j2
    m, j = d["material"], d["j2"]
    return np_j2.J2Params(m["youngs_modulus"], m["poissons_ratio"], j["initial_yield_stress"],
                          j["hardening_modulus_isotropic"], j["hardening_modulus_kinematic"],
                          pe=j["elastic_penalty_exponent"], pe_min=j["elastic_min_ersatz"],
                          pp=j["plastic_penalty_exponent"], pp_min=j["plastic_min_ersatz"])


def test_up_solve_oracle_matches_reference_elastic_solution():
    """The NumPy u-p Newton (one pseudo-time step, lagged projection = 0)
    reproduces ElastoPlasticity_ElasticSolution3D within the reference's own
    tolerance; the fixed dofs are exactly zero."""
    d, cells, coords, dofs, vals = elastic_solution_case()
    m = d["material"]
    P = np_up.UpProblem(cells, coords, m["youngs_modulus"], m["poissons_ratio"], up_j2_params(d),
                        pe=m["simp_exponent"], pe_min=m["simp_min"], ps=m["pressure_scaling"])
    x, loc, ppg = P.solve(dofs, vals, d["steps"])
    assert P.converged
    gold = np.array(d["gold"])
    assert np.all(np.abs(x - gold) <= d["tolerance"] * np.abs(gold))
    assert np.all(x[gold == 0.0] == 0.0)
    assert not (loc[:, 1] > 0).any()  # elastic: no cell yields


def test_up_cell_tangent_matches_finite_differences():
    """The closed-form condensed cell tangent (dR/du - dR/dc (dH/dc)^-1 dH/du)
    against central differences of the condensed residual, on cells that
    yield, with different global and local penalties, kinematic hardening
    and a pressure scaling."""
    from oracle import np_j2, np_ref
    rng = np.random.default_rng(1)
    cells, coords = np_ref.box_mesh(2, 1, 1, 2.0, 1.0, 1.0)
    coords = coords + rng.uniform(-0.1, 0.1, coords.shape)
    j2 = np_j2.J2Params(200e3, 0.3, 250.0, 1000.0, 400.0, pe=3.0, pe_min=1e-9, pp=2.5, pp_min=1e-4)
    z = rng.uniform(0.5, 1.0, coords.shape[0])
    P = np_up.UpProblem(cells, coords, 200e3, 0.3, j2, z=z, pe=2.0, pe_min=1e-6, ps=1.7)
    x = rng.normal(size=4 * P.N) * np.tile([3e-3, 3e-3, 3e-3, 100.0], P.N)
    prev = np.zeros((P.C, 14))
    prev[:, 2:8] = rng.normal(scale=1e-4, size=(P.C, 6))
    prev[:, 0] = 1e-3
    ppg = rng.normal(size=(P.N, 3))
    plastic = 0
    for c in range(P.C):
        idx = P._idx(c)
        Ka = P.cell_tangent(c, x[idx], prev[c])
        Kf = P.cell_tangent_fd(c, x[idx], prev[c], ppg[cells[c]])
        plastic += P.cell_residual(c, x[idx], prev[c], ppg[cells[c]])[1][1] > 0
        assert np.abs(Ka - Kf).max() <= 1e-6 * np.abs(Ka).max()
        assert np.abs(Ka - Ka.T).max() <= 1e-12 * np.abs(Ka).max()
    assert plastic >= 6
