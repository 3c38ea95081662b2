"""Visualisation output (pa_write_vtu): the .vtu file read back holds the
mesh, "Displacements" and "Control" exactly (the reference writes the same
vertex tags through Omega_h's VTK writer, src/AnalyzeOutput.hpp:469-482)."""
import base64
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}


def read_vtu(path):
    root = ET.parse(path).getroot()
    assert root.get("type") == "UnstructuredGrid" and root.get("header_type") == "UInt64"
    piece = root.find("UnstructuredGrid/Piece")
    out = {"N": int(piece.get("NumberOfPoints")), "C": int(piece.get("NumberOfCells"))}
    for sec in ("PointData", "CellData", "Points", "Cells"):
        for da in piece.find(sec).findall("DataArray"):
            raw = base64.b64decode(da.text.strip())
            nbytes = struct.unpack("<Q", raw[:8])[0]
            assert nbytes == len(raw) - 8
            a = np.frombuffer(raw[8:], dtype=DT[da.get("type")])
            out[(sec, da.get("Name"))] = a.reshape(-1, int(da.get("NumberOfComponents", "1")))
    return out


@pytest.mark.parametrize("layout", ["nodal", "cell"])
def test_vtu_round_trip(pa, tmp_path, layout):
    import torch
    mesh = pa.Mesh.box(5, 3, 2, 5.0, 3.0, 2.0)
    cells, coords = mesh.arrays()
    rng = np.random.default_rng(2)
    u = rng.standard_normal(3 * coords.shape[0])
    z = rng.uniform(0.0, 1.0, cells.shape[0] if layout == "cell" else coords.shape[0])
    path = tmp_path / "solution.vtu"
    mesh.write_vtu(path, u=torch.tensor(u, device="cuda"), control=z, control_layout=layout)  # device and host
    d = read_vtu(path)
    assert d["N"] == coords.shape[0] and d["C"] == cells.shape[0]
    assert np.array_equal(d[("Points", None)], coords)
    assert np.array_equal(d[("Cells", "connectivity")].ravel(), cells.ravel())
    assert np.array_equal(d[("Cells", "offsets")].ravel(), 4 * np.arange(1, cells.shape[0] + 1))
    assert (d[("Cells", "types")] == 10).all()
    assert np.array_equal(d[("PointData", "Displacements")], u.reshape(-1, 3))
    sec = "CellData" if layout == "cell" else "PointData"
    assert np.array_equal(d[(sec, "Control")].ravel(), z)


def test_vtu_without_fields_and_bad_path(pa, tmp_path):
    from platoanalyze_b200._abi import PaError
    mesh = pa.Mesh.box(2, 2, 2)
    mesh.write_vtu(tmp_path / "mesh.vtu")
    d = read_vtu(tmp_path / "mesh.vtu")
    assert d["C"] == 48 and ("PointData", "Displacements") not in d
    with pytest.raises(PaError):
        mesh.write_vtu(tmp_path / "no_such_dir" / "x.vtu")


def test_exodus_mesh_solves_on_the_box_multigrid(pa, tmp_path):
    """An Exodus II file of a scrambled, x-mirrored 24x12x12 box (two element
    blocks, named node sets) read with pa_exodus_*: the mesh is recognised as
    a lattice, the clamped face comes from its node set, and the multigrid
    solve equals the one of the same arrays handed to pa_mesh_create."""
    from exodus_writer import exodus_box
    from test_gpu_box import _scrambled
    nx, ny, nz = 24, 12, 12
    cl, X, _, order, faces, clamp = _scrambled(nx, ny, nz, 3, mirror_x=True)
    path = str(tmp_path / "box.exo")
    exodus_box(path, cl, X, {"ns_X1": clamp, "load": np.unique(faces)}, version=2)
    mesh, sets = pa.Mesh.from_exodus(path)
    assert mesh.box_kernels
    assert np.array_equal(sets["ns_X1"], clamp)
    rng = np.random.default_rng(4)
    z = rng.uniform(0.05, 1.0, cl.shape[0])
    flux = np.array([0.0, 0.0, -1.0 / (ny * nz)])
    out = []
    for m, ns in ((mesh, sets["ns_X1"]), (pa.Mesh.from_arrays(cl, X), clamp)):
        prob = pa.Problem(m, 1.0, 0.3, 3.0, 1e-9, control_layout="cell")
        prob.add_traction(faces, flux)
        prob.set_dirichlet(np.sort(np.concatenate([3 * ns, 3 * ns + 1, 3 * ns + 2])).astype(np.int32))
        u, st = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-10))
        assert st["converged"], st
        out.append(u)
    assert np.array_equal(out[0], out[1])
