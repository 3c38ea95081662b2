"""CUDA path vs the FP64 CPU oracle on seeded inputs (through the C ABI).

Tolerances: FP64 kernels 1e-10 relative (infinity norm); FP32 apply 1e-5;
FP64 solve residual checked by the oracle's own operator; mixed-precision
compliance within 1e-6 of the FP64 oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL64 = 1e-10


def rel_inf(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def perturbed_box(nx, ny, nz, seed, amp=0.1, order="hex"):
    """Box mesh with jittered interior nodes.  order="hex": the generator's
    order (six tets of a hex consecutive: hex clusters); "mixed": the hexes in
    random order with a random vertex order inside each tet (still hex
    clusters) plus a shuffled tail of single cells; "shuffled": all cells
    shuffled (single-cell clusters)."""
    from oracle import np_ref
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    rng = np.random.default_rng(seed)
    inner = np.all((coords > 1e-9) & (coords < np.array([nx, ny, nz]) - 1e-9), axis=1)
    coords[inner] += amp * rng.uniform(-1, 1, (inner.sum(), 3))
    if order == "mixed":
        hexes = cells.reshape(-1, 6, 4)[rng.permutation(cells.shape[0] // 6)]
        cells = np.array([rng.permutation(c) for c in hexes.reshape(-1, 4)], dtype=np.int32)
        tail = cells.shape[0] // 3
        cells[-tail:] = cells[-tail:][rng.permutation(tail)]
    elif order == "shuffled":
        cells = cells[rng.permutation(cells.shape[0])]
    return np.ascontiguousarray(cells), coords


CASES = [((3, 2, 2), 0, "nodal", "hex"), ((7, 5, 4), 1, "cell", "mixed"), ((12, 9, 7), 2, "nodal", "hex"),
         ((1, 1, 1), 3, "cell", "hex"), ((6, 5, 4), 4, "nodal", "shuffled"), ((9, 7, 5), 5, "cell", "mixed")]


@pytest.fixture(scope="module", params=CASES, ids=lambda c: f"{c[0][0]}x{c[0][1]}x{c[0][2]}-{c[2]}-{c[3]}")
def setup(request, pa, oracle_lib):
    dims, seed, layout, order = request.param
    cells, coords = perturbed_box(*dims, seed, order=order)
    rng = np.random.default_rng(100 + seed)
    E, nu, p, pmin = 3.0, 0.27, 3.0, 1e-6
    lay = 1 if layout == "cell" else 0
    O = oracle_lib.Oracle(cells, coords, E=E, nu=nu, p=p, pmin=pmin, layout=lay)
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, E, nu, p, pmin, control_layout=layout)
    faces = mesh.boundary_faces(0, float(dims[0]))
    flux = np.array([0.1, -0.2, 0.7])
    prob.add_traction(faces, flux)
    u = rng.standard_normal(3 * O.N)
    z = rng.uniform(0.05, 1.0, O.C if lay else O.N)
    return dict(O=O, mesh=mesh, prob=prob, u=u, z=z, faces=faces, flux=flux, rng=rng, cells=cells, coords=coords)


def test_value(setup):
    s = setup
    r = s["prob"].vector_function().value(s["u"], s["z"])
    ref = s["O"].residual(s["u"], s["z"], s["faces"], s["flux"])
    assert rel_inf(r, ref) < RTOL64


def test_gradient_u(setup):
    s = setup
    K = s["prob"].vector_function().gradient_u(s["u"], s["z"])
    ref = s["O"].jacobian(s["u"], s["z"], s["mesh"].graph())
    assert rel_inf(K, ref) < RTOL64


def test_gradient_z(setup):
    s = setup
    G = s["prob"].vector_function().gradient_z(s["u"], s["z"])
    ref = s["O"].gradient_z(s["u"], s["z"], s["mesh"].graph())
    assert rel_inf(G, ref) < RTOL64


def test_gradient_x(setup):
    s = setup
    G = s["prob"].vector_function().gradient_x(s["u"], s["z"])
    ref = s["O"].gradient_x(s["u"], s["z"], s["faces"], s["flux"], s["mesh"].graph())
    assert rel_inf(G, ref) < RTOL64
    gx = s["prob"].scalar_function().gradient_x(s["u"], s["z"])
    assert rel_inf(gx, s["O"].energy_grad_x(s["u"], s["z"])) < RTOL64


def test_energy(setup):
    s = setup
    sf = s["prob"].scalar_function()
    f, gu, gz = s["O"].energy(s["u"], s["z"])
    assert abs(sf.value(s["u"], s["z"]) - f) <= RTOL64 * abs(f)
    assert rel_inf(sf.gradient_u(s["u"], s["z"]), gu) < RTOL64
    assert rel_inf(sf.gradient_z(s["u"], s["z"]), gz) < RTOL64


def test_apply_fp64_and_fp32(setup):
    s = setup
    ref = s["O"].apply(s["u"], s["z"])
    y = s["prob"].apply(s["z"], s["u"])
    assert rel_inf(y, ref) < RTOL64
    y32 = s["prob"].apply(s["z"], s["u"].astype(np.float32))
    assert y32.dtype == np.float32
    assert rel_inf(y32.astype(np.float64), ref) < 1e-5


def test_apply_with_device_tensors(setup):
    import torch
    s = setup
    u = torch.tensor(s["u"], device="cuda")
    z = torch.tensor(s["z"], device="cuda")
    y = s["prob"].apply(z, u)
    assert y.is_cuda
    assert rel_inf(y.cpu().numpy(), s["O"].apply(s["u"], s["z"])) < RTOL64


def test_apply_constrained_matches_eliminated_matrix(setup):
    s = setup
    prob, O = s["prob"], s["O"]
    N = O.N
    dofs = np.arange(0, 3 * N, 7, dtype=np.int32)
    vals = np.linspace(-1, 1, dofs.size)
    prob.set_dirichlet(dofs, vals)
    try:
        rowmap, cols = s["mesh"].graph()
        K = O.jacobian(s["u"], s["z"], (rowmap, cols))
        rhs = np.zeros(3 * N)
        from oracle import cpu
        lib = cpu.lib()
        lib.pao_apply_block_constraints(N, rowmap.ctypes.data, cols.ctypes.data, K.ctypes.data, rhs.ctypes.data,
                                       dofs.size, dofs.ctypes.data, vals.ctypes.data, 1.0)
        y_ref = np.empty(3 * N)
        lib.pao_block_spmv(N, rowmap.ctypes.data, cols.ctypes.data, K.ctypes.data, s["u"].ctypes.data,
                           y_ref.ctypes.data)
        y = prob.apply(s["z"], s["u"], constrained=True)
        assert rel_inf(y, y_ref) < RTOL64
        # assembled constraint imposition on the device
        K2 = prob.vector_function().gradient_u(s["u"], s["z"])
        rhs2 = np.zeros(3 * N)
        prob.apply_block_constraints(K2, rhs2)
        assert rel_inf(K2, K) < RTOL64
        assert rel_inf(rhs2, rhs) < RTOL64
    finally:
        prob.set_dirichlet(np.zeros(0, np.int32), np.zeros(0))


def test_nonself_adjoint_gradient_matches_self_adjoint(setup, pa):
    """criterionGradient through the adjoint solve equals -df/dz for compliance
    (src/elliptic/Problem.hpp:413-468)."""
    s = setup
    prob, O = s["prob"], s["O"]
    dims_x = s["coords"][:, 0].max()
    clamp = np.where(np.abs(s["coords"][:, 0]) < 1e-9)[0]
    dofs = np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32)
    prob.set_dirichlet(dofs, np.zeros(dofs.size))
    try:
        opts = pa.SolveOptions("fp64", rel_tol=1e-13)
        u, st = prob.solution(s["z"], options=opts)
        assert st["converged"]
        g_sa = prob.criterion_gradient(s["z"], u, self_adjoint=True)
        g_adj = prob.criterion_gradient(s["z"], u, self_adjoint=False, options=opts)
        assert rel_inf(g_adj, g_sa) < 1e-7
        f, gu, gz = O.energy(u, s["z"])
        assert rel_inf(g_sa, -gz) < RTOL64
        assert dims_x > 0
    finally:
        prob.set_dirichlet(np.zeros(0, np.int32), np.zeros(0))


def _cantilever(pa, oracle_lib, nx, ny, nz, seed, layout="cell"):
    """Box x=0 clamped, unit total traction -z on x=max; per-cell density U[0.3, 1]."""
    from oracle import np_ref
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    rng = np.random.default_rng(seed)
    lay = 1 if layout == "cell" else 0
    z = rng.uniform(0.3, 1.0, cells.shape[0] if lay else coords.shape[0])
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout=layout)
    faces = mesh.boundary_faces(0, float(nx))
    flux = np.array([0.0, 0.0, -1.0 / (ny * nz)])
    prob.add_traction(faces, flux)
    clamp = np.where(coords[:, 0] < 1e-9)[0]
    dofs = np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32)
    prob.set_dirichlet(dofs)
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=lay)
    F = -O.residual(np.zeros(3 * O.N), z, faces, flux)
    return mesh, prob, O, z, F, dofs


def _direct_solution(O, z, F, dofs):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    rowmap, cols = O.graph()
    vals = O.jacobian(np.zeros(3 * O.N), z)
    N = O.N
    rows = np.repeat(np.arange(N), np.diff(rowmap))
    I = (3 * rows[:, None, None] + np.arange(3)[None, :, None]).repeat(3, 2).ravel()
    J = (3 * cols[:, None, None] + np.arange(3)[None, None, :]).repeat(3, 1).ravel()
    K = sp.csr_matrix((vals, (I, J)), shape=(3 * N, 3 * N))
    free = np.setdiff1d(np.arange(3 * N), dofs)
    u = np.zeros(3 * N)
    u[free] = spla.spsolve(K[free][:, free].tocsc(), F[free])
    return u


def test_solution_fp64_config1_shape(pa, oracle_lib):
    """20x10x10 hexes x 6 tets (12,000 tets), per-cell density U[0.3,1]:
    Problem::solution with Jacobi-PCG to 1e-10 vs a sparse direct FP64 solve."""
    mesh, prob, O, z, F, dofs = _cantilever(pa, oracle_lib, 20, 10, 10, seed=11)
    u, st = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-10))
    assert st["converged"] and st["rel_residual"] <= 1e-10
    u_ref = _direct_solution(O, z, F, dofs)
    # residual of the GPU solution measured by the oracle's operator
    r = F - O.apply(u, z)
    r[dofs] = 0.0
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(F)
    f_gpu = prob.scalar_function().value(u, z)
    f_ref = O.energy(u_ref, z, grads=False)
    assert abs(f_gpu - f_ref) <= 1e-9 * f_ref
    assert rel_inf(u, u_ref) < 1e-6
    g = prob.criterion_gradient(z, u)
    _, _, gz_ref = O.energy(u_ref, z)
    assert rel_inf(g, -gz_ref) < 1e-6


def test_solution_mixed_precision(pa, oracle_lib):
    mesh, prob, O, z, F, dofs = _cantilever(pa, oracle_lib, 16, 8, 8, seed=5)
    u64, st64 = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-11))
    u, st = prob.solution(z, options=pa.SolveOptions("mixed", rel_tol=1e-8))
    assert st["converged"] and st["rel_residual"] <= 1e-8
    r = F - O.apply(u, z)
    r[dofs] = 0.0
    assert np.linalg.norm(r) <= 1.01e-8 * np.linalg.norm(F)
    f = prob.scalar_function().value(u, z)
    f64 = O.energy(u64, z, grads=False)
    assert abs(f - f64) <= 1e-6 * f64


def test_solution_inhomogeneous_dirichlet(pa, oracle_lib):
    """Nonzero prescribed displacements are lifted as applyBlockConstraints does."""
    mesh, prob, O, z, F, dofs = _cantilever(pa, oracle_lib, 6, 4, 3, seed=9)
    vals = 0.01 * np.sin(np.arange(dofs.size))
    prob.set_dirichlet(dofs, vals)
    x, st = prob.solve(z, F, options=pa.SolveOptions("fp64", rel_tol=1e-12))
    assert st["converged"]
    rowmap, cols = O.graph()
    x_ref, it, rel = O.solve(z, F, dofs, vals, rel_tol=1e-13)
    assert np.allclose(x[dofs], vals, rtol=0, atol=0)
    assert rel_inf(x, x_ref) < 1e-8


def test_j2_radial_return(pa, oracle_lib, setup):
    s = setup
    O, prob = s["O"], s["prob"]
    rng = np.random.default_rng(21)
    C, N = O.C, O.N
    u = 2e-3 * rng.standard_normal(3 * N)
    z = rng.uniform(0.5, 1.0, N)
    prev = 1e-4 * rng.standard_normal((C, 14))
    prev[:, 0] = np.abs(prev[:, 0])
    prev[:, 1] = 0.0
    params = dict(youngs_modulus=200e3, poissons_ratio=0.3, initial_yield_stress=250.0,
                  hardening_modulus_isotropic=1000.0, hardening_modulus_kinematic=500.0,
                  elastic_penalty_exponent=3.0, elastic_min_ersatz=1e-9, plastic_penalty_exponent=2.5,
                  plastic_min_ersatz=1e-9)
    mu = params["youngs_modulus"] / (2 * (1 + params["poissons_ratio"]))
    ref = O.j2_update(u, z, prev, mu, 250.0, 1000.0, 500.0, 3.0, 1e-9, 2.5, 1e-9).reshape(C, 14)
    got = np.asarray(prob.j2_radial_return(params, u, z, prev)).reshape(C, 14)
    plastic = ref[:, 1] > 0
    assert plastic.any()
    if C > 6:
        assert (~plastic).any()
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_library_stream_is_ordered_with_torchs_default_stream(pa, oracle_lib):
    """A problem created without a stream works on a blocking stream: device
    inputs that torch writes on its default stream just before a call are read
    after they land, and the results are complete when torch reads them."""
    import torch
    cells, coords = perturbed_box(8, 5, 4, 11)
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
    rng = np.random.default_rng(5)
    z = rng.uniform(0.1, 1.0, O.C)
    u = rng.standard_normal(3 * O.N)
    ref = O.apply(u, z)
    zt = torch.tensor(z, device="cuda")
    for _ in range(3):
        ut = torch.zeros(3 * O.N, dtype=torch.float64, device="cuda")
        big = torch.randn(4096, 4096, device="cuda")
        for _ in range(8):
            big = (big @ big) * 1e-4  # keeps the default stream busy
        ut.copy_(torch.tensor(u), non_blocking=False)
        y = prob.apply(zt, ut)
        assert rel_inf(y.cpu().numpy(), ref) < RTOL64
