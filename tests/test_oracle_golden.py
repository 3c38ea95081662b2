"""The CPU oracle against the reference's own gold vectors (no GPU needed).

Mirrors unit_tests/DerivativeTests.cpp (ElastostaticResidual3D,
InternalElasticEnergy3D) and unit_tests/PlasticityTests.cpp
(J2PlasticityUtils_UpdatePlasticStep3D).
"""
import numpy as np
import pytest

from golden_util import derivative_case, floating_equality, load, star_graph


@pytest.fixture(scope="module")
def case(oracle_lib):
    d, cells, coords, u, z = derivative_case()
    m = d["material"]
    O = oracle_lib.Oracle(cells, coords, E=m["youngs_modulus"], nu=m["poissons_ratio"], p=m["simp_exponent"],
                          pmin=m["simp_min"])
    return d, O, u, z


def test_elastostatic_residual_3d_value(case):
    d, O, u, z = case
    floating_equality(O.residual(u, z), d["gold"]["residual"], d["tolerances"]["residual"])


def test_elastostatic_residual_3d_gradient_u(case):
    d, O, u, z = case
    graph = star_graph(*O.graph(), d["row0_star_order"])
    vals = O.jacobian(u, z, graph)
    gold = d["gold"]["jacobian_entries"]
    floating_equality(vals[:len(gold)], gold, d["tolerances"]["jacobian_entries"], zero_atol=1e-9)


def test_elastostatic_residual_3d_gradient_z(case):
    d, O, u, z = case
    graph = star_graph(*O.graph(), d["row0_star_order"])
    vals = O.gradient_z(u, z, graph)
    gold = d["gold"]["gradient_z_entries"]
    floating_equality(vals[:len(gold)], gold, d["tolerances"]["gradient_z_entries"])


def test_internal_elastic_energy_3d(case):
    d, O, u, z = case
    f, gu, gz = O.energy(u, z)
    floating_equality([f], [d["gold"]["energy_value"]], d["tolerances"]["energy_value"])
    floating_equality(gu, d["gold"]["energy_grad_u"], d["tolerances"]["energy_grad_u"])
    floating_equality(gz, d["gold"]["energy_grad_z"], d["tolerances"]["energy_grad_z"])


def test_numpy_restatement_matches_gold():
    from oracle import np_ref
    d, cells, coords, u, z = derivative_case()
    P = np_ref.Problem(cells, coords, E=1e6, nu=0.3, p=1.0, pmin=0.0)
    floating_equality(P.value(u, z), d["gold"]["residual"], 1e-13)
    f, gu, gz = P.energy(u, z)
    assert abs(f - 46.125) / 46.125 < 1e-13
    floating_equality(gz, d["gold"]["energy_grad_z"], 1e-13)


def test_j2_update_plastic_step_3d(oracle_lib):
    d = load("j2_plastic_step_3d.json")
    prev = np.array([[(i + 1.0) * (j + 1.0) for j in range(14)] for i in range(2)])
    normal = np.array([[(i + 1.0) * (j + 2.0) / 5.0 for j in range(6)] for i in range(2)])
    cur = oracle_lib.j2_plastic_step(prev, normal, prev, 3.0)
    floating_equality(cur, d["gold"], d["tolerance"])


def test_box_mesh_numbering_matches_numpy(oracle_lib):
    from oracle import np_ref
    for dims in [(1, 1, 1), (3, 2, 2), (5, 4, 3)]:
        c1, x1 = oracle_lib.box_mesh(*dims, float(dims[0]), float(dims[1]), float(dims[2]))
        c2, x2 = np_ref.box_mesh(*dims, float(dims[0]), float(dims[1]), float(dims[2]))
        assert (c1 == c2).all() and np.array_equal(x1, x2)


def test_oracle_cpp_matches_numpy_random(oracle_lib):
    from oracle import np_ref
    rng = np.random.default_rng(7)
    cells, coords = np_ref.box_mesh(3, 2, 2, 3.0, 2.0, 2.0)
    coords = coords + 0.05 * rng.standard_normal(coords.shape)  # unstructured geometry
    for layout in (0, 1):
        O = oracle_lib.Oracle(cells, coords, E=2.0, nu=0.27, p=3.0, pmin=1e-3, layout=layout)
        P = np_ref.Problem(cells, coords, E=2.0, nu=0.27, p=3.0, pmin=1e-3, layout=layout)
        u = rng.standard_normal(3 * O.N)
        z = rng.uniform(0.2, 1.0, O.C if layout else O.N)
        r = O.residual(u, z)
        assert np.allclose(r, P.value(u, z), rtol=0, atol=1e-13 * np.abs(r).max())
        f1, gu1, gz1 = O.energy(u, z)
        f2, gu2, gz2 = P.energy(u, z)
        assert abs(f1 - f2) <= 1e-13 * abs(f2)
        assert np.allclose(gz1, gz2, rtol=1e-12, atol=0)
        rowmap, cols = O.graph()
        K = P.stiffness_dense(z)
        assert np.allclose(O.jacobian(u, z), np_ref.block_entries(K, rowmap, cols), rtol=0, atol=1e-13 * np.abs(K).max())


def test_oracle_gradients_match_finite_differences(oracle_lib):
    """Central differences as in Plato_Diagnostics test_partial_control /
    test_partial_state (src/Plato_Diagnostics.hpp:111-575)."""
    from oracle import np_ref
    rng = np.random.default_rng(3)
    cells, coords = np_ref.box_mesh(2, 2, 1, 2.0, 2.0, 1.0)
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9)
    u = rng.standard_normal(3 * O.N)
    z = rng.uniform(0.3, 1.0, O.N)
    f, gu, gz = O.energy(u, z)
    dz = rng.standard_normal(O.N)
    h = 1e-6
    fd = (O.energy(u, z + h * dz, grads=False) - O.energy(u, z - h * dz, grads=False)) / (2 * h)
    assert abs(fd - gz @ dz) <= 1e-7 * abs(fd)
    du = rng.standard_normal(3 * O.N)
    fd = (O.energy(u + h * du, z, grads=False) - O.energy(u - h * du, z, grads=False)) / (2 * h)
    assert abs(fd - gu @ du) <= 1e-7 * abs(fd)


def test_elastostatic_residual_3d_gradient_x(case):
    d, O, u, z = case
    graph = star_graph(*O.graph(), d["row0_star_order"])
    vals = O.gradient_x(u, z, graph=graph)
    gold = d["gold"]["gradient_x_entries"]
    floating_equality(vals[:len(gold)], gold, d["tolerances"]["gradient_x_entries"])


def test_internal_elastic_energy_3d_gradient_x(case):
    d, O, u, z = case
    floating_equality(O.energy_grad_x(u, z), d["gold"]["energy_grad_x"], 1e-13)


def test_oracle_gradient_x_matches_finite_differences(oracle_lib):
    from oracle import np_ref
    rng = np.random.default_rng(11)
    cells, coords = np_ref.box_mesh(2, 1, 1, 2.0, 1.0, 1.0)
    coords = coords + 0.05 * rng.standard_normal(coords.shape)
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9)
    u = rng.standard_normal(3 * O.N)
    z = rng.uniform(0.3, 1.0, O.N)
    gx = O.energy_grad_x(u, z)
    dx = rng.standard_normal(coords.shape)
    h = 1e-6
    fp = oracle_lib.Oracle(cells, coords + h * dx, E=1.0, nu=0.3, p=3.0, pmin=1e-9).energy(u, z, grads=False)
    fm = oracle_lib.Oracle(cells, coords - h * dx, E=1.0, nu=0.3, p=3.0, pmin=1e-9).energy(u, z, grads=False)
    assert abs((fp - fm) / (2 * h) - gx @ dx.ravel()) <= 1e-6 * abs(gx @ dx.ravel())


def j2_evaluate_3d_case():
    """J2Plasticity_Evaluate3D (unit_tests/PlasticityTests.cpp:1749-1864): a
    1x1x1 box, u = 0.1 (y+z, x+z, x+y) (the test's boundary helper adds its
    values), control 0.9, the parameters of its tGenericParamList_Two."""
    from oracle import np_ref, np_j2
    cells, X = np_ref.box_mesh(1, 1, 1)
    u = 0.1 * np.stack([X[:, 1] + X[:, 2], X[:, 0] + X[:, 2], X[:, 0] + X[:, 1]], axis=1).ravel()
    prm = np_j2.J2Params(520.0, 0.3, 3.0, 20.0, 15.0, pe=3.0, pe_min=1e-9, pp=2.5, pp_min=1e-9)
    cur = np.array([0.3, 0.5, -0.1, 0.0, 0.1, 0.2, 0.2, 0.2, 12.0, -4.0, -8.0, 1.0, 1.0, 1.0])
    prev = np.array([0.2, 0.75, 0.0, -0.2, 0.2, 0.2, 0.2, 0.2, 2.0, 40.0, -42.0, 2.0, 2.0, 2.0])
    gold = [-0.400000, 26.941399, -0.480125, 0.111393, 0.368732, 0.0443036, 0.0443036, 0.0443036, 7.078994,
            -44.680887, 37.601894, -0.829778, -0.829778, -0.829778]
    return cells, X, u, prm, cur, prev, gold


def test_j2_local_residual_evaluate_3d():
    from oracle import np_ref, np_j2
    cells, X, u, prm, cur, prev, gold = j2_evaluate_3d_case()
    for c in cells:
        g, _ = np_ref.cell_gradients(X[c])
        eps = np_ref.bmatrix(g) @ u.reshape(-1, 3)[c].ravel()
        H = np_j2.local_residual(prm, 0.9, eps, cur, prev)
        floating_equality(H, gold, 1e-5)


def test_j2_radial_return_satisfies_local_residual():
    """After the return mapping the local residual vanishes (plastic and elastic cells)."""
    from oracle import np_j2
    rng = np.random.default_rng(5)
    prm = np_j2.J2Params(200e3, 0.3, 250.0, 1000.0, 300.0, pe=3.0, pp=2.5)
    for k in range(20):
        eps = 3e-3 * rng.standard_normal(6)
        prev = np.zeros(14)
        prev[0] = abs(1e-3 * rng.standard_normal())
        prev[2:14] = 1e-3 * rng.standard_normal(12)
        prev[8:14] *= 1e4
        prev[2:5] -= prev[2:5].mean()    # plastic strain and backstress are deviatoric
        prev[8:11] -= prev[8:11].mean()
        cur, _ = np_j2.radial_return(prm, 0.9, eps, prev)
        H = np_j2.local_residual(prm, 0.9, eps, cur, prev)
        assert np.abs(H).max() <= 1e-8 * max(1.0, np.abs(cur).max() * 1e3)
