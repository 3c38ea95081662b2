"""The box kernel (structured boxes of pa_mesh_create_box): K x through
pa_apply against the FP64 oracle and against the tile kernel, and the
multigrid solve whose every level runs on it against the oracle and the
tile-kernel multigrid.

Tolerances: FP64 apply 1e-12 relative (infinity norm) against the oracle;
FP32 apply 1e-5; solves to relres 1e-10 checked by the oracle's own
operator, and within 1e-7 of the FP64 Jacobi-PCG solution."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_inf(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


# (hexes, lengths, control layout, per-hex densities?) -- sizes cross the
# CTA brick edges (31 nodes along x, 7 along y, kz planes along z)
APPLY_CASES = [
    ((12, 8, 6), (12.0, 8.0, 6.0), "cell", True),
    ((40, 9, 17), (40.0, 9.0, 17.0), "cell", False),
    ((33, 15, 10), (1.0, 2.0, 3.0), "nodal", False),  # non-cubic hexes
    ((2, 2, 2), (2.0, 2.0, 2.0), "cell", False),
    ((64, 8, 8), (64.0, 8.0, 8.0), "cell", True),
]


@pytest.mark.parametrize("case", APPLY_CASES, ids=lambda c: f"{c[0][0]}x{c[0][1]}x{c[0][2]}-{c[2]}-{'hex' if c[3] else 'tet'}")
def test_box_apply_matches_oracle_and_tile_kernel(pa, oracle_lib, case):
    from oracle import np_ref
    (nx, ny, nz), (lx, ly, lz), layout, per_hex = case
    rng = np.random.default_rng(nx * 100 + nz)
    mesh = pa.Mesh.box(nx, ny, nz, lx, ly, lz)
    assert mesh.box_kernels
    E, nu, p, pmin = 2.5, 0.31, 3.0, 1e-6
    prob = pa.Problem(mesh, E, nu, p, pmin, control_layout=layout)
    cells, coords = np_ref.box_mesh(nx, ny, nz, lx, ly, lz)
    lay = 1 if layout == "cell" else 0
    O = oracle_lib.Oracle(cells, coords, E=E, nu=nu, p=p, pmin=pmin, layout=lay)
    if layout == "cell":
        z = np.repeat(rng.uniform(0.05, 1.0, nx * ny * nz), 6) if per_hex else rng.uniform(0.05, 1.0, O.C)
    else:
        z = rng.uniform(0.05, 1.0, O.N)
    x = rng.standard_normal(3 * O.N)
    y_ref = O.apply(x, z)
    y_box = prob.apply(z, x)
    assert rel_inf(y_box, y_ref) <= 1e-12
    # constrained: x = 0 face clamped (identity rows) and one more node's y dof
    clamp = np.where(coords[:, 0] == 0.0)[0]
    dofs = np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2, [3 * (O.N - 1) + 1]])).astype(np.int32)
    prob.set_dirichlet(dofs)
    yc_box = prob.apply(z, x, constrained=True)
    free = np.ones(3 * O.N, bool)
    free[dofs] = False
    yc_ref = O.apply(np.where(free, x, 0.0), z)
    yc_ref[~free] = x[~free]
    assert rel_inf(yc_box, yc_ref) <= 1e-12
    # FP32 box kernel, and the tile kernel on the same mesh
    y32 = prob.apply(z, x.astype(np.float32), constrained=True)
    assert rel_inf(y32, yc_ref) <= 1e-5
    mesh.set_box_kernels(False)
    assert not mesh.box_kernels
    yc_tile = prob.apply(z, x, constrained=True)
    assert rel_inf(yc_tile, yc_box) <= 1e-12


def _cantilever(dims, seed, lengths=None):
    from platoanalyze_b200.workloads import cantilever, cell_density
    mesh, prob, faces, dofs = cantilever(dims)
    z = cell_density(dims, seed, kind="smoothed", sigma=1.5, lo=0.01, hi=1.0)
    return mesh, prob, faces, dofs, z


@pytest.mark.parametrize("dims", [(16, 8, 8), (24, 12, 12), (64, 16, 16)])
def test_box_mg_matches_oracle_and_tile_mg(pa, oracle_lib, dims):
    from oracle import np_ref
    mesh, prob, faces, dofs, z = _cantilever(dims, 3)
    u, st = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    assert st["converged"] and st["rel_residual"] <= 1e-10, st
    nx, ny, nz = dims
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    flux = np.array([0.0, 0.0, -1.0 / (ny * nz)])
    F = -O.residual(np.zeros_like(u), z, faces, flux)
    res = F - O.apply(u, z)
    res[dofs] = 0.0
    assert np.linalg.norm(res) <= 1.01e-10 * np.linalg.norm(F)
    u64, _ = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-11))
    assert rel_inf(u, u64) <= 1e-7
    # the same method on the tile kernels: the same iteration count (to one)
    mesh.set_box_kernels(False)
    ut, stt = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    assert stt["converged"], stt
    assert abs(stt["iterations"] - st["iterations"]) <= 1, (st, stt)
    assert rel_inf(ut, u) <= 1e-7
    # deterministic (no atomics): a fresh problem's first solve gives the same
    # bits (a later solve on the same problem starts its spectral estimates
    # from the previous solve's vector)
    mesh.set_box_kernels(True)
    from platoanalyze_b200.workloads import cantilever
    _, prob2, _, _ = cantilever(dims)
    u2, st2 = prob2.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    assert st2["iterations"] == st["iterations"] and np.array_equal(u2, u)


def test_box_mg_nodal_per_tet_noncubic_inhomogeneous(pa, oracle_lib):
    """Nodal controls (per-tet weights), non-cubic hexes (lengths 2 x 1 x 1.5
    over 16 x 8 x 8) and prescribed nonzero Dirichlet values."""
    from oracle import np_ref
    nx, ny, nz = 16, 8, 8
    lx, ly, lz = 2.0, 1.0, 1.5
    mesh = pa.Mesh.box(nx, ny, nz, lx, ly, lz)
    prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="nodal")
    cells, coords = np_ref.box_mesh(nx, ny, nz, lx, ly, lz)
    faces = mesh.boundary_faces(0, lx)
    flux = np.array([0.0, 0.3, -1.0])
    prob.add_traction(faces, flux)
    clamp = np.where(coords[:, 0] == 0.0)[0]
    dofs = np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32)
    vals = 0.01 * np.cos(np.arange(dofs.size))
    prob.set_dirichlet(dofs, vals)
    rng = np.random.default_rng(9)
    z = rng.uniform(0.1, 1.0, coords.shape[0])
    u, st = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    assert st["converged"], st
    assert np.array_equal(u[dofs], vals)
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=0)
    F = -O.residual(np.zeros_like(u), z, faces, flux)
    res = F - O.apply(u, z)
    res[dofs] = 0.0
    ud = np.zeros_like(u)
    ud[dofs] = vals
    Fb = F - O.apply(ud, z)
    Fb[dofs] = 0.0
    assert np.linalg.norm(res) <= 1.01e-10 * np.linalg.norm(Fb)
    u64, _ = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-11))
    assert rel_inf(u, u64) <= 1e-7


def test_box_mg_density_change_reuses_hierarchy(pa):
    mesh, prob, faces, dofs, z = _cantilever((32, 16, 16), 11)
    from platoanalyze_b200.workloads import cell_density
    for seed in (11, 12, 13):
        zz = cell_density((32, 16, 16), seed, kind="smoothed", sigma=2.0, lo=0.01, hi=1.0)
        u, st = prob.solution(zz, options=pa.SolveOptions("mg", rel_tol=1e-10))
        u64, _ = prob.solution(zz, options=pa.SolveOptions("fp64", rel_tol=1e-11))
        assert st["converged"], st
        assert rel_inf(u, u64) <= 1e-7


def _scrambled(nx, ny, nz, seed, mirror_x=False):
    """The box of pa_mesh_create_box as caller arrays: nodes and cells in
    random order, each tet's vertices in random order, optionally mirrored in
    x (the split then runs along another cube diagonal).  Returns the arrays,
    the new node id of each box node, the box slot (6 h + t) of each cell, the
    load faces and the clamped nodes."""
    from platoanalyze_b200.fields import box_arrays
    cells, coords, faces, clamp = box_arrays(nx, ny, nz)
    rng = np.random.default_rng(seed)
    N, C = coords.shape[0], cells.shape[0]
    new_of_old = rng.permutation(N).astype(np.int32)
    X = np.empty_like(coords)
    X[new_of_old] = coords
    if mirror_x:
        X[:, 0] = nx - X[:, 0]
    order = rng.permutation(C)
    cl = new_of_old[cells][order]
    cl = np.array([row[rng.permutation(4)] for row in cl], dtype=np.int32)
    return cl, X, new_of_old, order, new_of_old[faces], new_of_old[clamp]


def test_box_kernels_on_reference_numbered_meshes(pa, oracle_lib):
    """The reference's own 2x2x2 Omega_h box (golden DerivativeTests mesh) and
    a scrambled, x-mirrored 12x8x6 box enter through pa_mesh_create, are
    recognised as lattices, and the box kernel's K x matches the oracle."""
    from golden_util import derivative_case
    d, cells, coords, u, z = derivative_case()
    m = pa.Mesh.from_arrays(cells, coords)
    assert m.box_kernels
    prob = pa.Problem(m, 1.0, 0.3, 3.0, 1e-9, control_layout="nodal")
    rng = np.random.default_rng(2)
    zz = rng.uniform(0.2, 1.0, coords.shape[0])
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=0)
    assert rel_inf(prob.apply(zz, u), O.apply(u, zz)) <= 1e-12
    cl, X, _, _, _, _ = _scrambled(12, 8, 6, 5, mirror_x=True)
    m2 = pa.Mesh.from_arrays(cl, X)
    assert m2.box_kernels
    p2 = pa.Problem(m2, 2.0, 0.25, 3.0, 1e-6, control_layout="cell")
    z2 = rng.uniform(0.05, 1.0, cl.shape[0])
    x2 = rng.standard_normal(3 * X.shape[0])
    O2 = oracle_lib.Oracle(cl, X, E=2.0, nu=0.25, p=3.0, pmin=1e-6, layout=1)
    assert rel_inf(p2.apply(z2, x2), O2.apply(x2, z2)) <= 1e-12
    assert rel_inf(p2.apply(z2, x2.astype(np.float32)), O2.apply(x2, z2)) <= 1e-5


def test_box_mg_through_pa_mesh_create_at_64x32x32(pa, oracle_lib):
    """The drop-in path: a 64x32x32 box handed over as scrambled arrays (node,
    cell and vertex order random) solves with the multigrid method on the box
    kernels, to the same solution and iteration count (within 10 %) as the
    pa_mesh_create_box mesh, with its residual checked by the oracle."""
    from platoanalyze_b200.workloads import cantilever, cell_density
    dims = (64, 32, 32)
    nx, ny, nz = dims
    mesh_b, prob_b, faces_b, dofs_b = cantilever(dims)
    z_box = cell_density(dims, 21, kind="smoothed", sigma=2.0, lo=0.01, hi=1.0)
    ub, stb = prob_b.solution(z_box, options=pa.SolveOptions("mg", rel_tol=1e-10))
    assert stb["converged"], stb
    cl, X, new_of_old, order, faces, clamp = _scrambled(nx, ny, nz, 8)
    m = pa.Mesh.from_arrays(cl, X)
    assert m.box_kernels
    prob = pa.Problem(m, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
    flux = np.array([0.0, 0.0, -1.0 / (ny * nz)])
    prob.add_traction(faces, flux)
    dofs = np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32)
    prob.set_dirichlet(dofs)
    z = z_box[order]
    u, st = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    assert st["converged"], st
    assert abs(st["iterations"] - stb["iterations"]) <= max(1, 0.1 * stb["iterations"]), (st, stb)
    ub_mapped = np.empty_like(ub)
    for dd in range(3):
        ub_mapped[3 * new_of_old + dd] = ub[dd::3]
    assert rel_inf(u, ub_mapped) <= 1e-9
    O = oracle_lib.Oracle(cl, X, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    F = -O.residual(np.zeros_like(u), z, faces, flux)
    res = F - O.apply(u, z)
    res[dofs] = 0.0
    assert np.linalg.norm(res) <= 1.01e-10 * np.linalg.norm(F)


def test_box_mg_mirrored_scrambled_with_dirichlet_values(pa):
    """A mirrored (split along another cube diagonal), scrambled 16x8x8 box
    with prescribed nonzero Dirichlet values: the multigrid solve on the box
    kernels equals the FP64 Jacobi-PCG solve on the caller's numbering."""
    nx, ny, nz = 16, 8, 8
    cl, X, new_of_old, order, faces, clamp = _scrambled(nx, ny, nz, 13, mirror_x=True)
    m = pa.Mesh.from_arrays(cl, X)
    assert m.box_kernels
    prob = pa.Problem(m, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
    prob.add_traction(faces, np.array([0.2, 0.0, -1.0 / (ny * nz)]))
    dofs = np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32)
    vals = 0.01 * np.sin(np.arange(dofs.size))
    prob.set_dirichlet(dofs, vals)
    rng = np.random.default_rng(4)
    z = rng.uniform(0.05, 1.0, cl.shape[0])
    u, st = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
    u64, _ = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-11))
    assert st["converged"], st
    assert np.array_equal(u[dofs], vals)
    assert rel_inf(u, u64) <= 1e-7


@pytest.mark.parametrize("dims,lengths,p", [((10, 6, 5), (10.0, 6.0, 5.0), 3.0), ((9, 7, 4), (4.5, 5.25, 1.0), 2.5)])
def test_box_entry_points_match_oracle(pa, oracle_lib, dims, lengths, p):
    """The per-cell entry points on a box mesh with per-cell controls (the
    box kernel with the penalty applied as the controls load, and the per-hex
    energy kernel): residual, internal energy, dF/du and dF/dz against the
    oracle, on cubic and non-cubic hexes, integer and fractional exponents."""
    mesh = pa.Mesh.box(*dims, *lengths)
    assert mesh.box_kernels
    cells, coords = mesh.arrays()
    E, nu, pmin = 3.0, 0.27, 1e-6
    prob = pa.Problem(mesh, E, nu, p, pmin, control_layout="cell")
    faces = mesh.boundary_faces(0, lengths[0])
    flux = np.array([0.1, -0.2, 0.7])
    prob.add_traction(faces, flux)
    rng = np.random.default_rng(17)
    u = rng.standard_normal(3 * coords.shape[0])
    z = rng.uniform(0.05, 1.0, cells.shape[0])
    O = oracle_lib.Oracle(cells, coords, E=E, nu=nu, p=p, pmin=pmin, layout=1)
    vf = prob.vector_function()
    assert rel_inf(vf.value(u, z), O.residual(u, z, faces, flux)) <= 1e-10
    f, gu, gz = O.energy(u, z)
    sf = prob.scalar_function()
    assert abs(sf.value(u, z) - f) <= 1e-10 * abs(f)
    assert rel_inf(sf.gradient_u(u, z), gu) <= 1e-10
    assert rel_inf(sf.gradient_z(u, z), gz) <= 1e-10
    assert rel_inf(vf.gradient_z(u, z), O.gradient_z(u, z)) <= 1e-10


def test_box_gradient_z_any_vertex_order(pa, oracle_lib):
    """dR/dz per cell on a box whose node and cell order is the lattice's but
    whose cells list their vertices in other orders: the box kernel reads each
    vertex slot's corner from the node ids.  Checked against the oracle and
    the per-cell kernel (box kernels off)."""
    from oracle import np_ref
    dims = (9, 6, 5)
    cells, coords = np_ref.box_mesh(*dims, 4.5, 3.0, 5.0)
    rng = np.random.default_rng(5)
    perms = np.array([[0, 1, 2, 3], [1, 2, 0, 3], [2, 0, 1, 3], [0, 2, 3, 1], [3, 1, 0, 2], [1, 0, 3, 2]])
    pick = perms[rng.integers(0, len(perms), cells.shape[0])]
    cells2 = np.take_along_axis(cells, pick, axis=1).astype(np.int32)
    mesh = pa.Mesh.from_arrays(cells2, coords)
    assert mesh.box_kernels
    prob = pa.Problem(mesh, 2.0, 0.25, 3.0, 1e-6, control_layout="cell")
    u = rng.standard_normal(3 * coords.shape[0])
    z = rng.uniform(0.05, 1.0, cells.shape[0])
    O = oracle_lib.Oracle(cells2, coords, E=2.0, nu=0.25, p=3.0, pmin=1e-6, layout=1)
    g = prob.vector_function().gradient_z(u, z)
    assert rel_inf(g, O.gradient_z(u, z)) <= 1e-10
    mesh.set_box_kernels(False)
    g_cell = prob.vector_function().gradient_z(u, z)
    assert rel_inf(g, g_cell) <= 1e-12


@pytest.mark.parametrize("dims", [(8, 5, 4), (37, 2, 3)])
@pytest.mark.parametrize("layout,lengths", [("cell", (8.0, 5.0, 4.0)), ("nodal", (4.0, 7.5, 2.0))])
def test_box_assembled_gradient_u(pa, oracle_lib, layout, lengths, dims):
    """VectorFunction::gradient_u on a box mesh: the per-block lattice
    assembly (no atomics) equals the oracle's block CRS matrix and, to
    rounding, the per-cell atomic assembly (box kernels switched off);
    reordered columns (pa_mesh_set_graph) fall back to the per-cell one.
    37x2x3: rows longer than a CTA's 32 nodes, CTAs across rows, and nearly
    every node on the boundary."""
    mesh = pa.Mesh.box(*dims, *lengths)
    assert mesh.box_kernels
    cells, coords = mesh.arrays()
    rng = np.random.default_rng(23)
    E, nu, p, pmin = 2.0, 0.3, 3.0, 1e-6
    z = rng.uniform(0.05, 1.0, cells.shape[0] if layout == "cell" else coords.shape[0])
    u = rng.standard_normal(3 * coords.shape[0])
    prob = pa.Problem(mesh, E, nu, p, pmin, control_layout=layout)
    K = prob.vector_function().gradient_u(u, z)
    O = oracle_lib.Oracle(cells, coords, E=E, nu=nu, p=p, pmin=pmin, layout=1 if layout == "cell" else 0)
    assert rel_inf(K, O.jacobian(u, z, mesh.graph())) <= 1e-12
    mesh.set_box_kernels(False)
    K_atomic = prob.vector_function().gradient_u(u, z)
    assert rel_inf(K, K_atomic) <= 1e-13
    mesh.set_box_kernels(True)
    # a graph with every row's columns reversed: the lattice path steps aside
    rowmap, cols = mesh.graph()
    rev = cols.copy()
    for v in range(coords.shape[0]):
        rev[rowmap[v]:rowmap[v + 1]] = cols[rowmap[v]:rowmap[v + 1]][::-1]
    mesh.set_graph(rowmap, rev)
    K_rev = prob.vector_function().gradient_u(u, z)
    assert rel_inf(K_rev, O.jacobian(u, z, mesh.graph())) <= 1e-12


@pytest.mark.parametrize("dims", [(24, 12, 12), (17, 9, 7)])
def test_box_fp64_jacobi_pcg_deterministic(pa, oracle_lib, dims):
    """PA_SOLVER_PCG_FP64 on a box runs the outer CG on the box kernel with
    the inverse diagonal (no atomics): two fresh problems give the same bits,
    the solution solves the oracle's constrained system, and it equals the
    tile kernel's FP64 Jacobi-PCG (box kernels off) to the tolerance."""
    from oracle import np_ref
    opts = pa.SolveOptions("fp64", rel_tol=1e-10)
    mesh, prob, faces, dofs, z = _cantilever(dims, 9)
    u, st = prob.solution(z, options=opts)
    assert st["converged"] and st["rel_residual"] <= 1e-10, st
    _, prob2, _, _, _ = _cantilever(dims, 9)
    u2, st2 = prob2.solution(z, options=opts)
    assert st2["iterations"] == st["iterations"] and np.array_equal(u2, u)
    nx, ny, nz = dims
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    flux = np.array([0.0, 0.0, -1.0 / (ny * nz)])
    F = -O.residual(np.zeros_like(u), z, faces, flux)
    res = F - O.apply(u, z)
    res[dofs] = 0.0
    assert np.linalg.norm(res) <= 1.01e-10 * np.linalg.norm(F)
    mesh.set_box_kernels(False)
    ut, stt = prob.solution(z, options=opts)
    assert stt["converged"], stt
    assert rel_inf(ut, u) <= 1e-8
    assert abs(stt["iterations"] - st["iterations"]) <= 0.05 * st["iterations"] + 2, (st, stt)


@pytest.mark.parametrize("dims", [(8, 5, 4), (37, 2, 3)])
@pytest.mark.parametrize("layout,lengths", [("cell", (8.0, 5.0, 4.0)), ("nodal", (4.0, 7.5, 2.0))])
def test_box_assembled_gradient_x(pa, oracle_lib, layout, lengths, dims):
    """VectorFunction::gradient_x on a box mesh: the per-block lattice
    assembly of the volume term (closed-form shape derivatives, no atomics)
    plus the surface loads equals the oracle's dR/dx and, to rounding, the
    per-cell dual-number kernel with atomics (box kernels switched off)."""
    mesh = pa.Mesh.box(*dims, *lengths)
    assert mesh.box_kernels
    cells, coords = mesh.arrays()
    rng = np.random.default_rng(29)
    E, nu, p, pmin = 2.0, 0.3, 3.0, 1e-6
    z = rng.uniform(0.05, 1.0, cells.shape[0] if layout == "cell" else coords.shape[0])
    u = rng.standard_normal(3 * coords.shape[0])
    prob = pa.Problem(mesh, E, nu, p, pmin, control_layout=layout)
    faces = mesh.boundary_faces(0, lengths[0])
    flux = np.array([0.2, -0.1, 0.5])
    prob.add_traction(faces, flux)
    G = prob.vector_function().gradient_x(u, z)
    O = oracle_lib.Oracle(cells, coords, E=E, nu=nu, p=p, pmin=pmin, layout=1 if layout == "cell" else 0)
    assert rel_inf(G, O.gradient_x(u, z, faces, flux, mesh.graph())) <= 1e-10
    mesh.set_box_kernels(False)
    G_cell = prob.vector_function().gradient_x(u, z)
    assert rel_inf(G, G_cell) <= 1e-12
