"""Exodus II mesh input (pa_exodus_*, host only): files written by
tests/exodus_writer.py in the three netCDF classic variants, the writer
checked against scipy's netCDF reader, and the reader's refusals."""
import numpy as np
import pytest

from exodus_writer import exodus_box
from oracle import np_ref


def _box():
    cells, coords = np_ref.box_mesh(3, 2, 2, 3.0, 2.0, 2.0)
    sets = {"ns_X0": np.where(coords[:, 0] < 1e-9)[0], "ns_X1": np.where(coords[:, 0] > 3 - 1e-9)[0]}
    return cells, coords, sets


@pytest.mark.parametrize("version,kw", [
    (1, {}),
    (2, dict(combined_coord=True, coord_dtype=np.float32, names=False, blocks=3)),
    (5, dict(int_dtype=np.int64, blocks=1)),
])
def test_exodus_round_trip(tmp_path, version, kw):
    import platoanalyze_b200 as pa
    cells, coords, sets = _box()
    path = str(tmp_path / f"box_v{version}.exo")
    exodus_box(path, cells, coords, sets, version=version, **kw)
    c2, x2, s2 = pa.read_exodus(path)
    assert np.array_equal(c2, cells)
    want = coords.astype(kw.get("coord_dtype", np.float64)).astype(np.float64)
    assert np.array_equal(x2, want)
    names = list(sets) if kw.get("names", True) else ["ns_10", "ns_20"]
    assert list(s2) == names
    for a, b in zip(s2.values(), sets.values()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("version", [1, 2])
def test_writer_matches_scipy_reader(tmp_path, version):
    from scipy.io import netcdf_file
    cells, coords, sets = _box()
    path = str(tmp_path / "box.exo")
    exodus_box(path, cells, coords, sets, version=version)
    with netcdf_file(path, "r", mmap=False) as f:
        assert f.dimensions["num_nodes"] == coords.shape[0]
        assert np.array_equal(f.variables["coordy"][:], coords[:, 1])
        conn = np.concatenate([f.variables["connect1"][:], f.variables["connect2"][:]])
        assert np.array_equal(conn, cells + 1)
        assert f.variables["connect1"].elem_type == b"TETRA"
        assert np.array_equal(f.variables["node_ns2"][:], sets["ns_X1"] + 1)


def test_exodus_refusals(tmp_path):
    import platoanalyze_b200 as pa
    from platoanalyze_b200 import _abi
    cells, coords, sets = _box()
    hexes = str(tmp_path / "hex.exo")
    exodus_box(hexes, cells, coords, sets, elem_type="HEX8")
    with pytest.raises(_abi.PaError, match="only 4-node tetrahedra"):
        pa.read_exodus(hexes)
    h5 = tmp_path / "h5.exo"
    h5.write_bytes(b"\x89HDF\r\n\x1a\n" + b"\0" * 64)
    with pytest.raises(_abi.PaError, match="HDF5"):
        pa.read_exodus(str(h5))
    good = tmp_path / "good.exo"
    exodus_box(str(good), cells, coords, sets)
    cut = tmp_path / "cut.exo"
    cut.write_bytes(good.read_bytes()[:-200])
    with pytest.raises(_abi.PaError, match="truncated"):
        pa.read_exodus(str(cut))
    bad = cells.copy()
    bad[0, 0] = coords.shape[0]  # one past the last node
    oob = str(tmp_path / "oob.exo")
    exodus_box(oob, bad, coords, sets)
    with pytest.raises(_abi.PaError, match="out of range"):
        pa.read_exodus(oob)
    with pytest.raises(_abi.PaError, match="cannot open"):
        pa.read_exodus(str(tmp_path / "missing.exo"))
