"""The CUDA path through the C ABI against the reference's gold vectors.

GPU twins of unit_tests/DerivativeTests.cpp ElastostaticResidual3D /
InternalElasticEnergy3D and PlasticityTests.cpp radial-return pieces.
"""
import numpy as np
import pytest

from golden_util import derivative_case, floating_equality, star_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden(pa):
    d, cells, coords, u, z = derivative_case()
    mesh = pa.Mesh.from_arrays(cells, coords)
    m = d["material"]
    prob = pa.Problem(mesh, m["youngs_modulus"], m["poissons_ratio"], m["simp_exponent"], m["simp_min"])
    return d, mesh, prob, u, z


def test_elastostatic_residual_3d(golden):
    d, mesh, prob, u, z = golden
    vf = prob.vector_function()
    floating_equality(vf.value(u, z), d["gold"]["residual"], d["tolerances"]["residual"])


def test_elastostatic_jacobian_3d_reference_column_order(golden):
    d, mesh, prob, u, z = golden
    rowmap, cols = mesh.graph()
    mesh.set_graph(*star_graph(rowmap, cols, d["row0_star_order"]))
    try:
        vf = prob.vector_function()
        gold_j = d["gold"]["jacobian_entries"]
        floating_equality(vf.gradient_u(u, z)[:len(gold_j)], gold_j, d["tolerances"]["jacobian_entries"],
                          zero_atol=1e-9)
        gold_z = d["gold"]["gradient_z_entries"]
        floating_equality(vf.gradient_z(u, z)[:len(gold_z)], gold_z, d["tolerances"]["gradient_z_entries"])
    finally:
        mesh.set_graph(rowmap, cols)


def test_internal_elastic_energy_3d(golden):
    d, mesh, prob, u, z = golden
    sf = prob.scalar_function("Internal Elastic Energy")
    floating_equality([sf.value(u, z)], [46.125], d["tolerances"]["energy_value"])
    floating_equality(sf.gradient_u(u, z), d["gold"]["energy_grad_u"], d["tolerances"]["energy_grad_u"])
    floating_equality(sf.gradient_z(u, z), d["gold"]["energy_grad_z"], d["tolerances"]["energy_grad_z"])


def test_self_adjoint_criterion_gradient_is_minus_partial(golden):
    d, mesh, prob, u, z = golden
    g = prob.criterion_gradient(z, u, self_adjoint=True)
    floating_equality(-g, d["gold"]["energy_grad_z"], 1e-13)


def test_elastostatic_gradient_x_3d_reference_column_order(golden):
    d, mesh, prob, u, z = golden
    rowmap, cols = mesh.graph()
    mesh.set_graph(*star_graph(rowmap, cols, d["row0_star_order"]))
    try:
        gold = d["gold"]["gradient_x_entries"]
        floating_equality(prob.vector_function().gradient_x(u, z)[:len(gold)], gold,
                          d["tolerances"]["gradient_x_entries"])
    finally:
        mesh.set_graph(rowmap, cols)


def test_internal_elastic_energy_3d_gradient_x(golden):
    d, mesh, prob, u, z = golden
    floating_equality(prob.scalar_function().gradient_x(u, z), d["gold"]["energy_grad_x"], 1e-13)
