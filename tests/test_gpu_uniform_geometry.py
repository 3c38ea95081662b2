"""Uniform hex geometry (structured voxel meshes): the FP32 tile kernel takes
each template tet's rows of det * J^-1 and 1 / (6 |det|) from a per-mesh table
instead of recomputing them per tet.  Checked against the FP64 oracle and
against the per-tet geometry on the same mesh (pa_mesh_uniform_geometry(0)),
in the plain apply, the fused PCG, the batched PCG and the J2 tangent.

Tolerances: FP32 apply 1e-5 relative (infinity norm) against the FP64 oracle;
mixed solves: compliance within 1e-6 of FP64."""
import numpy as np
import pytest

from oracle import np_ref

pytestmark = pytest.mark.gpu


def rel_inf(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


SPACINGS = [(1.0, 1.0, 1.0), (1.3, 0.7, 2.1)]


def _meshes(pa, dims, spacing):
    nx, ny, nz = dims
    cells, coords = np_ref.box_mesh(nx, ny, nz, nx * spacing[0], ny * spacing[1], nz * spacing[2])
    table = pa.Mesh.from_arrays(cells, coords)
    per_tet = pa.Mesh.from_arrays(cells, coords)
    assert table.uniform_geometry
    assert not per_tet.set_uniform_geometry(False)
    return cells, coords, table, per_tet


def test_non_uniform_meshes_use_the_per_tet_geometry(pa):
    cells, coords = np_ref.box_mesh(4, 3, 2, 4.0, 3.0, 2.0)
    assert pa.Mesh.from_arrays(cells, coords).uniform_geometry
    jit = coords.copy()
    inner = np.all((coords > 1e-9) & (coords < np.array([4.0, 3.0, 2.0]) - 1e-9), axis=1)
    jit[inner] += 1e-3
    assert not pa.Mesh.from_arrays(cells, jit).uniform_geometry
    # a graded axis: hexes of two sizes
    graded = coords.copy()
    graded[:, 0] = graded[:, 0] ** 1.5
    assert not pa.Mesh.from_arrays(cells, graded).uniform_geometry
    # single-tet clusters (shuffled cells) never qualify
    rng = np.random.default_rng(0)
    assert not pa.Mesh.from_arrays(cells[rng.permutation(cells.shape[0])], coords).uniform_geometry
    # a duplicated hex has its twin's node in every slot of the same tile: the
    # table kernel's slot-by-slot (atomic-free) sums would collide, so the mesh
    # keeps the per-tet path, which still matches the oracle
    dup = np.concatenate([cells, cells[:6]])
    mdup = pa.Mesh.from_arrays(dup, coords)
    assert not mdup.uniform_geometry
    from oracle import cpu
    O = cpu.Oracle(dup, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    z = rng.uniform(0.1, 1.0, dup.shape[0])
    u = rng.standard_normal(3 * coords.shape[0])
    y = pa.Problem(mdup, 1.0, 0.3, 3.0, 1e-9, control_layout="cell").apply(z, u.astype(np.float32))
    assert rel_inf(y, O.apply(u, z)) < 1e-5
    # the box generator qualifies; switching back on re-detects it
    m = pa.Mesh.box(5, 4, 3, 2.5, 2.0, 1.5)
    assert m.uniform_geometry
    assert not m.set_uniform_geometry(False)
    assert m.set_uniform_geometry(True)


@pytest.mark.parametrize("spacing", SPACINGS)
@pytest.mark.parametrize("layout", ["nodal", "cell"])
def test_fp32_apply_with_the_geometry_table(pa, oracle_lib, spacing, layout):
    dims = (9, 7, 5)
    cells, coords, table, per_tet = _meshes(pa, dims, spacing)
    lay = 1 if layout == "cell" else 0
    O = oracle_lib.Oracle(cells, coords, E=3.0, nu=0.27, p=3.0, pmin=1e-6, layout=lay)
    rng = np.random.default_rng(7)
    z = rng.uniform(0.05, 1.0, O.C if lay else O.N)
    u = rng.standard_normal(3 * O.N)
    ref = O.apply(u, z)
    ys = []
    for mesh in (table, per_tet):
        prob = pa.Problem(mesh, 3.0, 0.27, 3.0, 1e-6, control_layout=layout)
        y = prob.apply(z, u.astype(np.float32))
        assert y.dtype == np.float32
        assert rel_inf(y, ref) < 1e-5
        ys.append(y)
    assert rel_inf(ys[0], ys[1]) < 1e-5
    # constrained apply: masked dofs drop out the same way
    dofs = np.arange(0, 3 * O.N, 5, dtype=np.int32)
    outs = []
    for mesh in (table, per_tet):
        prob = pa.Problem(mesh, 3.0, 0.27, 3.0, 1e-6, control_layout=layout)
        prob.set_dirichlet(dofs)
        outs.append(prob.apply(z, u.astype(np.float32), constrained=True))
    assert rel_inf(outs[0], outs[1]) < 1e-5


def _cantilever(pa, mesh, dims, spacing, seed):
    nx, ny, nz = dims
    lx, ly, lz = nx * spacing[0], ny * spacing[1], nz * spacing[2]
    prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
    faces = mesh.boundary_faces(0, lx)
    prob.add_traction(faces, np.array([0.0, 0.0, -1.0 / (ly * lz)]))
    _, coords = mesh.arrays()
    clamp = np.where(coords[:, 0] < 1e-9)[0]
    prob.set_dirichlet(np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32))
    z = np.random.default_rng(seed).uniform(0.05, 1.0, mesh.num_cells)
    return prob, z


@pytest.mark.parametrize("spacing", SPACINGS)
def test_mixed_solve_with_the_geometry_table(pa, spacing):
    dims = (16, 8, 6)
    cells, coords, table, per_tet = _meshes(pa, dims, spacing)
    res = []
    for mesh in (table, per_tet):
        prob, z = _cantilever(pa, mesh, dims, spacing, 3)
        u, st = prob.solution(z, options=pa.SolveOptions("mixed", rel_tol=1e-8))
        assert st["converged"] and st["rel_residual"] <= 1e-8, st
        res.append((prob.scalar_function().value(u, z), u, st["iterations"]))
    prob, z = _cantilever(pa, per_tet, dims, spacing, 3)
    u64, _ = prob.solution(z, options=pa.SolveOptions("fp64", rel_tol=1e-11))
    f64 = prob.scalar_function().value(u64, z)
    for f, u, its in res:
        assert abs(f - f64) <= 1e-6 * f64
        assert rel_inf(u, u64) <= 1e-5
    # the mixed solver's FP32 rounding plateau (atomic summation order) makes
    # its iteration count vary from run to run by a quarter or so
    assert abs(res[0][2] - res[1][2]) <= 0.35 * res[1][2] + 64


def test_batched_solve_with_the_geometry_table(pa):
    """Three boxes of unit hexes as parts of one mesh: the batched PCG on the
    table matches solving each box alone with the per-tet geometry."""
    dims = [(8, 4, 4), (6, 5, 3), (10, 3, 3)]
    cells_all, coords_all, offs = [], [], [0]
    shift = 0.0
    for (nx, ny, nz) in dims:
        c, x = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
        x = x + np.array([shift, 0.0, 0.0])
        shift += nx + 2.0
        cells_all.append(c + offs[-1])
        coords_all.append(x)
        offs.append(offs[-1] + x.shape[0])
    cells = np.concatenate(cells_all)
    coords = np.concatenate(coords_all)
    mesh = pa.Mesh.from_arrays(cells, coords)
    mesh.set_parts(np.array(offs))
    assert mesh.uniform_geometry
    prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
    rng = np.random.default_rng(4)
    z = rng.uniform(0.1, 1.0, mesh.num_cells)
    # clamp x = min of each box, unit -z traction on x = max of each box
    dofs = []
    shift = 0.0
    for p, (nx, ny, nz) in enumerate(dims):
        x = coords[offs[p]:offs[p + 1]]
        clamp = offs[p] + np.where(np.abs(x[:, 0] - shift) < 1e-9)[0]
        dofs += [3 * clamp, 3 * clamp + 1, 3 * clamp + 2]
        prob.add_traction(mesh.boundary_faces(0, shift + nx), np.array([0.0, 0.0, -1.0 / (ny * nz)]))
        shift += nx + 2.0
    prob.set_dirichlet(np.sort(np.concatenate(dofs)).astype(np.int32))
    u, st = prob.solution(z, options=pa.SolveOptions("mixed", rel_tol=1e-8))  # one CG per part
    assert st["converged"], st
    # the same boxes one at a time, per-tet geometry, FP64
    c0 = 0
    shift = 0.0
    for p, (nx, ny, nz) in enumerate(dims):
        c, x = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
        m1 = pa.Mesh.from_arrays(c, x)
        m1.set_uniform_geometry(False)
        p1 = pa.Problem(m1, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
        p1.add_traction(m1.boundary_faces(0, float(nx)), np.array([0.0, 0.0, -1.0 / (ny * nz)]))
        cl = np.where(x[:, 0] < 1e-9)[0]
        p1.set_dirichlet(np.sort(np.concatenate([3 * cl, 3 * cl + 1, 3 * cl + 2])).astype(np.int32))
        zc = z[c0:c0 + c.shape[0]]
        u1, s1 = p1.solution(zc, options=pa.SolveOptions("fp64", rel_tol=1e-11))
        up = u[3 * offs[p]:3 * offs[p + 1]]
        assert rel_inf(up, u1) <= 1e-5, p
        c0 += c.shape[0]
        shift += nx + 2.0


@pytest.mark.parametrize("spacing", SPACINGS)
def test_fp64_apply_and_solve_with_the_geometry_table(pa, oracle_lib, spacing):
    """FP64 takes the table only when every hex matches it to rounding level;
    then it keeps the 1e-10 parity of the per-tet FP64 arithmetic."""
    dims = (9, 7, 5)
    cells, coords, table, per_tet = _meshes(pa, dims, spacing)
    O = oracle_lib.Oracle(cells, coords, E=3.0, nu=0.27, p=3.0, pmin=1e-6, layout=1)
    rng = np.random.default_rng(9)
    z = rng.uniform(0.05, 1.0, O.C)
    u = rng.standard_normal(3 * O.N)
    ref = O.apply(u, z)
    for mesh in (table, per_tet):
        y = pa.Problem(mesh, 3.0, 0.27, 3.0, 1e-6, control_layout="cell").apply(z, u)
        assert rel_inf(y, ref) < 1e-10
    sols = []
    for mesh in (table, per_tet):
        prob, zc = _cantilever(pa, mesh, dims, spacing, 5)
        x, st = prob.solution(zc, options=pa.SolveOptions("fp64", rel_tol=1e-11))
        assert st["converged"], st
        sols.append(x)
    assert rel_inf(sols[0], sols[1]) < 1e-8


def test_fp64_keeps_the_per_tet_geometry_off_rounding_level(pa, oracle_lib):
    """Hexes that differ by up to 9.6e-10 of their size: FP32 still uses the table (its
    own rounding is far larger), FP64 does not, and stays within 1e-10."""
    cells, coords = np_ref.box_mesh(6, 5, 4, 6.0, 5.0, 4.0)
    rng = np.random.default_rng(3)
    jit = coords + 2.4e-10 * rng.uniform(-1.0, 1.0, coords.shape)  # edge vectors differ by <= 9.6e-10
    mesh = pa.Mesh.from_arrays(cells, jit)
    assert mesh.uniform_geometry
    O = oracle_lib.Oracle(cells, jit, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    z = rng.uniform(0.05, 1.0, O.C)
    u = rng.standard_normal(3 * O.N)
    ref = O.apply(u, z)
    prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
    assert rel_inf(prob.apply(z, u), ref) < 1e-10
    assert rel_inf(prob.apply(z, u.astype(np.float32)), ref) < 1e-5


@pytest.mark.parametrize("tile", [64, 128, 256])
def test_every_tile_size_with_the_geometry_table(pa, oracle_lib, monkeypatch, tile):
    """Each tile size is its own kernel instance (shared-memory layout, launch
    bounds): FP32 and FP64 applies against the oracle, mixed and FP64 solves
    against each other."""
    monkeypatch.setenv("PA_TILE_CLUSTERS", str(tile))
    dims = (12, 6, 5)
    cells, coords = np_ref.box_mesh(*dims, 12.0, 6.0, 5.0)
    mesh = pa.Mesh.from_arrays(cells, coords)
    assert mesh.uniform_geometry
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    rng = np.random.default_rng(tile)
    z = rng.uniform(0.05, 1.0, O.C)
    u = rng.standard_normal(3 * O.N)
    ref = O.apply(u, z)
    prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
    assert rel_inf(prob.apply(z, u), ref) < 1e-10
    assert rel_inf(prob.apply(z, u.astype(np.float32)), ref) < 1e-5
    prob, zc = _cantilever(pa, mesh, dims, (1.0, 1.0, 1.0), 7)
    x64, s64 = prob.solution(zc, options=pa.SolveOptions("fp64", rel_tol=1e-11))
    xm, sm = prob.solution(zc, options=pa.SolveOptions("mixed", rel_tol=1e-9))
    assert s64["converged"] and sm["converged"], (s64, sm)
    assert rel_inf(xm, x64) <= 1e-6
