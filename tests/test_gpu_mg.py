"""Multigrid-preconditioned CG (PA_SOLVER_PCG_MG) on box meshes: the same
constrained system as the Jacobi-PCG solvers, checked by the oracle's own
operator and against the FP64 PCG solution; inhomogeneous Dirichlet values,
a changing density (hierarchy reuse), and the meshes it refuses."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_inf(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _cantilever(pa, dims, seed):
    from platoanalyze_b200.workloads import cantilever, cell_density
    mesh, prob, faces, dofs = cantilever(dims)
    z = cell_density(dims, seed, kind="smoothed", sigma=1.5, lo=0.01, hi=1.0)
    return mesh, prob, faces, dofs, z


@pytest.mark.parametrize("dims", [(16, 8, 8), (24, 8, 12), (8, 4, 4)])
def test_mg_matches_the_oracle_and_fp64_pcg(pa, oracle_lib, dims):
    from oracle import np_ref
    mesh, prob, faces, dofs, z = _cantilever(pa, dims, 3)
    u, st = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    assert st["converged"] and st["rel_residual"] <= 1e-10, st
    assert st["iterations"] <= 60, st
    u64, s64 = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-11))
    assert rel_inf(u, u64) <= 1e-7
    # residual of the constrained system measured by the oracle's operator
    nx, ny, nz = dims
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    flux = np.array([0.0, 0.0, -1.0 / (ny * nz)])
    F = -O.residual(np.zeros_like(u), z, faces, flux)
    res = F - O.apply(u, z)
    res[dofs] = 0.0
    assert np.linalg.norm(res) <= 1.01e-10 * np.linalg.norm(F)
    assert s64["iterations"] > 5 * st["iterations"]


@pytest.mark.parametrize("dims", [(16, 8, 8), (40, 20, 20)])
def test_mg_coarse_direct_matches_chebyshev(pa, dims):
    """The box multigrid with its dense Gauss-Jordan inverse on the coarsest
    level (4x2x2 hexes: 135 dofs; 5x3x3 as for 160x80x80: 288 dofs, 5
    elimination blocks) against the tile-kernel multigrid with the degree-40
    Chebyshev coarse solve: the same solution, no more outer iterations, far
    fewer launches."""
    mesh, prob, faces, dofs, z = _cantilever(pa, dims, 7)
    u_d, st_d = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    u_c, st_c = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10, mg_coarse="chebyshev"))
    assert st_d["converged"] and st_c["converged"], (st_d, st_c)
    assert rel_inf(u_d, u_c) <= 1e-7
    assert st_d["iterations"] <= st_c["iterations"], (st_d, st_c)
    # 80 launches of the Chebyshev coarse solve per V-cycle become one
    assert st_d["kernel_launches"] < st_c["kernel_launches"] - 40 * st_d["iterations"], (st_d, st_c)


def test_mg_inhomogeneous_dirichlet_and_reuse(pa):
    mesh, prob, faces, dofs, z = _cantilever(pa, (16, 8, 8), 5)
    vals = 0.01 * np.sin(np.arange(dofs.size))
    prob.set_dirichlet(dofs, vals)
    for seed in (5, 6):  # a second density reuses the hierarchy with new weights
        from platoanalyze_b200.workloads import cell_density
        zz = cell_density((16, 8, 8), seed, kind="smoothed", sigma=1.5, lo=0.01, hi=1.0)
        u, st = prob.solution(zz, options=pa.SolveOptions("mg", rel_tol=1e-10))
        u64, _ = prob.solution(zz, options=pa.SolveOptions("fp64", rel_tol=1e-11))
        assert st["converged"], st
        assert np.allclose(u[dofs], vals, rtol=0, atol=0)
        assert rel_inf(u, u64) <= 1e-7


def test_mg_accepts_array_boxes_and_refuses_unsupported_meshes(pa):
    """A box given as arrays is recognised as a lattice (the box kernels solve
    it); with the box kernels switched off the multigrid method refuses it,
    and an odd hex count, which the box multigrid solves."""
    from oracle import np_ref
    from platoanalyze_b200._abi import PaError
    cells, coords = np_ref.box_mesh(8, 4, 4, 8.0, 4.0, 4.0)
    m = pa.Mesh.from_arrays(cells, coords)
    assert m.box_kernels
    prob = pa.Problem(m, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
    clamp = np.where(coords[:, 0] == 0.0)[0]
    prob.set_dirichlet(np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32))
    prob.add_traction(m.boundary_faces(0, 8.0), np.array([0.0, 0.0, -1.0 / 16]))
    u, st = prob.solution(np.ones(m.num_cells), options=pa.SolveOptions("mg"))
    assert st["converged"], st
    m.set_box_kernels(False)
    with pytest.raises(PaError):
        prob.solution(np.ones(m.num_cells), options=pa.SolveOptions("mg"))
    m2, prob2, _, _, z2 = _cantilever(pa, (7, 4, 4), 3)  # odd hex count
    u3, st3 = prob2.solution(z2, options=pa.SolveOptions("mg"))
    assert st3["converged"], st3
    m2.set_box_kernels(False)
    with pytest.raises(PaError):
        prob2.solution(z2, options=pa.SolveOptions("mg"))


def test_mg_above_six_hundred_thousand_nodes(pa):
    """144x72x72 (773k fine nodes, above the 606k threads of a capped
    grid-stride launch): every fine node of the prolongation is reached; same
    compliance as the FP64 Jacobi-PCG."""
    mesh, prob, faces, dofs, z = _cantilever(pa, (144, 72, 72), 7)
    u, st = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-8))
    assert st["converged"] and st["iterations"] <= 60, st
    u64, _ = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-10))
    f = prob.scalar_function().value(u, z)
    f64 = prob.scalar_function().value(u64, z)
    assert abs(f - f64) <= 1e-7 * abs(f64)
    assert rel_inf(u, u64) <= 1e-5


@pytest.mark.parametrize("dims", [(7, 4, 4), (17, 9, 11), (33, 17, 15), (25, 5, 3)])
def test_mg_odd_boxes_against_the_oracle(pa, oracle_lib, dims):
    """Boxes with odd hex counts: each coarse level has ceil(n / 2) hexes per
    axis and a padding layer of weight zero.  The solution solves the oracle's
    constrained system to the requested tolerance and equals the FP64
    Jacobi-PCG solution; the iteration count stays that of a multigrid."""
    from oracle import np_ref
    mesh, prob, faces, dofs, z = _cantilever(pa, dims, 11)
    u, st = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    assert st["converged"] and st["rel_residual"] <= 1e-10, st
    assert st["iterations"] <= 60, st
    u64, s64 = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-11))
    assert rel_inf(u, u64) <= 1e-7
    nx, ny, nz = dims
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    flux = np.array([0.0, 0.0, -1.0 / (ny * nz)])
    F = -O.residual(np.zeros_like(u), z, faces, flux)
    res = F - O.apply(u, z)
    res[dofs] = 0.0
    assert np.linalg.norm(res) <= 1.01e-10 * np.linalg.norm(F)
