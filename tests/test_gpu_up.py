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
