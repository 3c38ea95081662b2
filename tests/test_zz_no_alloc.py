"""pa_sf_value_noalloc: the compliance value for callers that cannot allocate
device memory (the library uses only a fixed __device__ scratch array).

Checked through the C ABI against the existing entry point pa_sf_value on the
same device arrays, twice in a row (the scratch array keeps the previous
call's contents), for nodal and per-cell controls.  This file is collected
last so that a run stopping at the first failure has run every other test."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10


@pytest.mark.parametrize("layout", ["nodal", "cell"])
def test_noalloc_matches_sf_value_twice(pa, layout):
    import torch
    from oracle import np_ref
    from platoanalyze_b200 import _abi

    nx, ny, nz = 10, 8, 6
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    rng = np.random.default_rng(77 if layout == "nodal" else 78)
    coords = coords + 0.05 * rng.uniform(-1, 1, coords.shape)
    C, N = cells.shape[0], coords.shape[0]
    lay = _abi.PA_CONTROL_CELL if layout == "cell" else _abi.PA_CONTROL_NODAL
    params = _abi.ElasticParams(2.0, 0.28, 3.0, 1e-6, lay)

    d_cells = torch.tensor(cells, device="cuda")
    d_coords = torch.tensor(coords, device="cuda")
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda")

    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, 2.0, 0.28, 3.0, 1e-6, control_layout=layout)
    lib = _abi.load()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        u = torch.tensor(rng.standard_normal(3 * N), device="cuda")
        z = torch.tensor(rng.uniform(0.05, 1.0, C if layout == "cell" else N), device="cuda")
        expect = prob.scalar_function().value(u, z)
        status = lib.pa_sf_value_noalloc(ct.c_void_p(d_cells.data_ptr()), C, ct.c_void_p(d_coords.data_ptr()), N,
                                         ct.c_void_p(u.data_ptr()), ct.c_void_p(z.data_ptr()), ct.byref(params),
                                         ct.c_void_p(d_out.data_ptr()), ct.c_void_p(stream))
        assert status == _abi.PA_OK, lib.pa_last_error().decode()
        torch.cuda.synchronize()
        got = float(d_out.item())
        assert abs(got - expect) <= RTOL * abs(expect), (call, got, expect)


def test_noalloc_rejects_oversize_mesh(pa):
    import torch
    from platoanalyze_b200 import _abi
    lib = _abi.load()
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    ci = torch.zeros(16, dtype=torch.int32, device="cuda")
    params = _abi.ElasticParams(1.0, 0.3, 3.0, 1e-9, _abi.PA_CONTROL_NODAL)
    p = ct.c_void_p(d.data_ptr())
    status = lib.pa_sf_value_noalloc(ct.c_void_p(ci.data_ptr()), 8388609, p, 4, p, p, ct.byref(params), p, None)
    assert status == _abi.PA_ERR_INVALID_ARG
    assert b"8388608" in lib.pa_last_error()
