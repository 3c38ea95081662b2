"""The C++ header (include/pa_b200.hpp) reproduces the reference's derivative
gold through libpa_b200.so, as a C++ caller of the reference would use it."""
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
