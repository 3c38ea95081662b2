"""The C++ headers: include/pa_b200.hpp reproduces the reference's derivative
gold through libpa_b200.so, as a C++ caller of the reference would use it;
include/pa_b200_app.hpp (the MPMD_App-shaped application) matches the oracle."""
import os
import subprocess

import numpy as np
import pytest

from golden_util import derivative_case, floating_equality

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_derivative_tests(pa, tmp_path):
    d, cells, coords, u, z = derivative_case()
    inp = tmp_path / "mesh.txt"
    with open(inp, "w") as f:
        f.write(f"{cells.shape[0]} {coords.shape[0]}\n")
        f.write(" ".join(map(str, cells.ravel())) + "\n")
        f.write(" ".join(repr(float(x)) for x in coords.ravel()) + "\n")
    exe = tmp_path / "derivative_tests"
    libdir = os.path.join(ROOT, "platoanalyze_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "derivative_tests.cpp"), "-o", str(exe),
                           "-L", libdir, "-lpa_b200", "-Wl,-rpath," + libdir])
    out = subprocess.check_output([str(exe), str(inp)], text=True)
    vals = np.array([float(v) for v in out.split()])
    n = coords.shape[0]
    floating_equality(vals[:3 * n], d["gold"]["residual"], 1e-13)
    floating_equality([vals[3 * n]], [d["gold"]["energy_value"]], 1e-13)
    floating_equality(vals[3 * n + 1:], d["gold"]["energy_grad_z"], 1e-13)


def test_cpp_mpmd_app(pa, oracle_lib, tmp_path):
    """include/pa_b200_app.hpp, the MPMD_App-shaped application: named
    operations and shared data give the compliance, its self-adjoint control
    and configuration gradients (-df/dz, -df/dx) and the state, matching the
    FP64 oracle; unknown names and criteria are rejected."""
    nx, ny, nz = 6, 3, 3
    mesh = pa.Mesh.box(nx, ny, nz, nx, ny, nz)
    cells, coords = mesh.arrays()
    N = coords.shape[0]
    topo = np.random.default_rng(17).uniform(0.2, 1.0, N)
    inp = tmp_path / "topology.txt"
    inp.write_text(" ".join(repr(float(v)) for v in topo))
    exe = tmp_path / "mpmd_app_tests"
    libdir = os.path.join(ROOT, "platoanalyze_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "mpmd_app_tests.cpp"), "-o", str(exe),
                           "-L", libdir, "-lpa_b200", "-Wl,-rpath," + libdir])
    lines = subprocess.check_output([str(exe), str(inp)], text=True).splitlines()
    errs = [l for l in lines if l.startswith("ERR")]
    vals = np.array([float(l) for l in lines if not l.startswith("ERR") and l != "no error"])
    assert len(errs) == 2 and "No Such Value" in errs[0] and "Maximize Stiffness" in errs[1], lines[-2:]
    f, gz, gx = vals[0], vals[1:1 + N], vals[1 + N:1 + 4 * N]
    fs, sz = vals[1 + 4 * N], vals[2 + 4 * N:]
    assert sz.size == N
    # the same problem through the Python API (FP64 solve) and the oracle
    prob = pa.Problem(mesh, 1.0, 0.3, 3.0, 1e-9, control_layout="nodal")
    prob.add_traction(mesh.boundary_faces(0, float(nx)), np.array([0.0, 0.0, -1.0 / (ny * nz)]))
    clamp = np.where(coords[:, 0] < 1e-9)[0]
    prob.set_dirichlet(np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32))
    u, st = prob.solution(topo, options=pa.SolveOptions("fp64", rel_tol=1e-12))
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=0)
    f_ref, _, gz_ref = O.energy(u, topo)
    gx_ref = O.energy_grad_x(u, topo)
    assert abs(f - f_ref) <= 1e-10 * abs(f_ref)
    assert abs(fs - (f_ref - 0.25)) <= 1e-10 * abs(f_ref)
    assert np.abs(gz + gz_ref).max() <= 1e-8 * np.abs(gz_ref).max()
    assert np.abs(gx + gx_ref).max() <= 1e-8 * np.abs(gx_ref).max()
    assert np.abs(sz - u[2::3]).max() <= 1e-9 * np.abs(u).max()
