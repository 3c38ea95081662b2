"""pa_sf_value_noalloc: the compliance value for callers that cannot allocate
device memory (the library uses only a fixed __device__ scratch array).

Checked through the C ABI against the existing entry point pa_sf_value on the
same device arrays and against the FP64 CPU oracle, twice in a row (the
scratch array keeps the previous call's contents), for nodal and per-cell
controls; then a larger mesh followed by a smaller one on a side stream (the
smaller call launches fewer blocks than the leftovers in the scratch array),
and a node id out of range (NaN, no out-of-bounds read).  This file is
collected last so that a run stopping at the first failure has run every
other test."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _mesh(nx, ny, nz, seed):
    from oracle import np_ref
    cells, coords = np_ref.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    rng = np.random.default_rng(seed)
    return cells, coords + 0.05 * rng.uniform(-1, 1, coords.shape)


def _call(lib, _abi, d_cells, C, d_coords, N, u, z, params, d_out, stream):
    return lib.pa_sf_value_noalloc(ct.c_void_p(d_cells.data_ptr()), C, ct.c_void_p(d_coords.data_ptr()), N,
                                   ct.c_void_p(u.data_ptr()), ct.c_void_p(z.data_ptr()), ct.byref(params),
                                   ct.c_void_p(d_out.data_ptr()), ct.c_void_p(stream))


@pytest.mark.parametrize("layout", ["nodal", "cell"])
def test_noalloc_matches_sf_value_twice(pa, oracle_lib, layout):
    import torch
    from platoanalyze_b200 import _abi

    cells, coords = _mesh(10, 8, 6, 77 if layout == "nodal" else 78)
    rng = np.random.default_rng(5 if layout == "nodal" else 6)
    C, N = cells.shape[0], coords.shape[0]
    lay = _abi.PA_CONTROL_CELL if layout == "cell" else _abi.PA_CONTROL_NODAL
    params = _abi.ElasticParams(2.0, 0.28, 3.0, 1e-6, lay)

    d_cells = torch.tensor(cells, device="cuda")
    d_coords = torch.tensor(coords, device="cuda")
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda")

    mesh = pa.Mesh.from_arrays(cells, coords)
    prob = pa.Problem(mesh, 2.0, 0.28, 3.0, 1e-6, control_layout=layout)
    O = oracle_lib.Oracle(cells, coords, E=2.0, nu=0.28, p=3.0, pmin=1e-6, layout=1 if layout == "cell" else 0)
    lib = _abi.load()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        u_h = rng.standard_normal(3 * N)
        z_h = rng.uniform(0.05, 1.0, C if layout == "cell" else N)
        u, z = torch.tensor(u_h, device="cuda"), torch.tensor(z_h, device="cuda")
        expect = prob.scalar_function().value(u, z)
        f_oracle = O.energy(u_h, z_h, grads=False)
        status = _call(lib, _abi, d_cells, C, d_coords, N, u, z, params, d_out, stream)
        assert status == _abi.PA_OK, lib.pa_last_error().decode()
        torch.cuda.synchronize()
        got = float(d_out.item())
        assert abs(got - expect) <= RTOL * abs(expect), (call, got, expect)
        assert abs(got - f_oracle) <= RTOL * abs(f_oracle), (call, got, f_oracle)


def test_noalloc_larger_then_smaller_on_side_stream(pa, oracle_lib):
    """A 20x16x16 call (7680 tets, 30 blocks) then a 6x4x4 call (576 tets,
    3 blocks) on a non-default stream: the second call reads only the block
    sums it wrote, not the first call's leftovers."""
    import torch
    from platoanalyze_b200 import _abi

    lib = _abi.load()
    side = torch.cuda.Stream()
    params = _abi.ElasticParams(1.0, 0.3, 3.0, 1e-9, _abi.PA_CONTROL_CELL)
    with torch.cuda.stream(side):
        for dims, seed in (((20, 16, 16), 11), ((6, 4, 4), 12)):
            cells, coords = _mesh(*dims, seed)
            C, N = cells.shape[0], coords.shape[0]
            rng = np.random.default_rng(seed)
            u_h, z_h = rng.standard_normal(3 * N), rng.uniform(0.05, 1.0, C)
            d_cells, d_coords = torch.tensor(cells, device="cuda"), torch.tensor(coords, device="cuda")
            u, z = torch.tensor(u_h, device="cuda"), torch.tensor(z_h, device="cuda")
            d_out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
            mesh = pa.Mesh.from_arrays(cells, coords)
            prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="cell", stream=side.cuda_stream)
            expect = prob.scalar_function().value(u, z)
            status = _call(lib, _abi, d_cells, C, d_coords, N, u, z, params, d_out, side.cuda_stream)
            assert status == _abi.PA_OK, lib.pa_last_error().decode()
            side.synchronize()
            got = float(d_out.item())
            f_oracle = oracle_lib.Oracle(cells, coords, layout=1).energy(u_h, z_h, grads=False)
            assert abs(got - expect) <= RTOL * abs(expect), (dims, got, expect)
            assert abs(got - f_oracle) <= RTOL * abs(f_oracle), (dims, got, f_oracle)


def test_noalloc_out_of_range_node_is_nan(pa):
    """One node id equal to num_nodes: the kernel skips that cell's reads and
    the value is NaN; the context stays usable (a second, valid call works)."""
    import torch
    from platoanalyze_b200 import _abi

    lib = _abi.load()
    cells, coords = _mesh(4, 3, 2, 3)
    C, N = cells.shape[0], coords.shape[0]
    bad = cells.copy()
    bad[5, 2] = N
    params = _abi.ElasticParams(1.0, 0.3, 3.0, 1e-9, _abi.PA_CONTROL_NODAL)
    rng = np.random.default_rng(4)
    u = torch.tensor(rng.standard_normal(3 * N), device="cuda")
    z = torch.tensor(rng.uniform(0.1, 1.0, N), device="cuda")
    d_coords = torch.tensor(coords, device="cuda")
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    status = _call(lib, _abi, torch.tensor(bad, device="cuda"), C, d_coords, N, u, z, params, d_out, stream)
    assert status == _abi.PA_OK, lib.pa_last_error().decode()
    torch.cuda.synchronize()
    assert np.isnan(float(d_out.item()))
    status = _call(lib, _abi, torch.tensor(cells, device="cuda"), C, d_coords, N, u, z, params, d_out, stream)
    assert status == _abi.PA_OK
    torch.cuda.synchronize()
    assert np.isfinite(float(d_out.item()))


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


def test_noalloc_rejects_host_pointer(pa):
    import torch
    from platoanalyze_b200 import _abi
    lib = _abi.load()
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    ci = torch.zeros(16, dtype=torch.int32, device="cuda")
    host = np.zeros(16)
    params = _abi.ElasticParams(1.0, 0.3, 3.0, 1e-9, _abi.PA_CONTROL_NODAL)
    p = ct.c_void_p(d.data_ptr())
    status = lib.pa_sf_value_noalloc(ct.c_void_p(ci.data_ptr()), 4, ct.c_void_p(host.ctypes.data), 4, p, p,
                                     ct.byref(params), p, None)
    assert status == _abi.PA_ERR_INVALID_ARG
