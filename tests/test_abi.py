"""The C-ABI library loads and exports every symbol include/pa_b200.h declares
(no compute call: runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pa_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pa_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("pa_vf_value", "pa_vf_gradient_u", "pa_vf_gradient_z", "pa_sf_value", "pa_sf_gradient_u",
                 "pa_sf_gradient_z", "pa_apply", "pa_solve", "pa_problem_solution", "pa_j2_radial_return"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import importlib.util
    spec = importlib.util.spec_from_file_location("pa_build", os.path.join(ROOT, "platoanalyze_b200", "build.py"))
    builder = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(builder)
    lib = ctypes.CDLL(builder.build())
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from platoanalyze_b200 import _abi
    bound = {name for name, _, _ in _abi.SIGNATURES}
    assert set(declared_symbols()) == bound


def test_no_device_is_reported_not_crashed():
    """Without a visible GPU every entry point returns PA_ERR_NO_DEVICE or
    another error status -- it never falls back to a CPU path."""
    import torch
    if torch.cuda.is_available():
        return
    from platoanalyze_b200 import _abi
    lib = _abi.load()
    h = ctypes.c_void_p()
    status = lib.pa_mesh_create_box(2, 2, 2, 1.0, 1.0, 1.0, ctypes.byref(h))
    assert status != _abi.PA_OK
    assert lib.pa_last_error()


def test_python_structs_match_the_c_layout(tmp_path):
    """Every ctypes mirror in platoanalyze_b200/_abi.py has the size and the
    field offsets that a C compiler gives the header's struct (a field added
    on one side only would shift every later field)."""
    import subprocess
    from platoanalyze_b200 import _abi
    pairs = {"ElasticParams": "pa_elastic_params", "SolveOptions": "pa_solve_options",
             "SolveStats": "pa_solve_stats", "J2Params": "pa_j2_params", "J2SolveOptions": "pa_j2_solve_options",
             "J2Stats": "pa_j2_stats", "UpParams": "pa_up_params", "PcTrainOptions": "pa_pc_train_options",
             "PcTrainStats": "pa_pc_train_stats"}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "pa_b200.h"', "int main(void) {"]
    for py, c in pairs.items():
        lines.append(f'  printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(_abi, py)._fields_:
            lines.append(f'  printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                           "-o", str(exe)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        py, field, value = line.split()
        got[(py, field)] = int(value)
    for py in pairs:
        cls = getattr(_abi, py)
        assert got[(py, "size")] == ctypes.sizeof(cls), py
        for name, _ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)


def test_solve_option_defaults_and_coarse_solver_choice():
    """pa_solve_options_default (no GPU needed) picks the automatic coarsest
    multigrid solve; the Python options map the choice and refuse others."""
    import pytest
    from platoanalyze_b200 import _abi
    from platoanalyze_b200.api import SolveOptions
    o = _abi.SolveOptions()
    o.mg_coarse_solver = 7
    assert _abi.load().pa_solve_options_default(ctypes.byref(o)) == _abi.PA_OK
    assert o.mg_coarse_solver == _abi.PA_MG_COARSE_AUTO and o.method == _abi.PA_SOLVER_PCG_FP64
    assert SolveOptions("mg").c().mg_coarse_solver == _abi.PA_MG_COARSE_AUTO
    c = SolveOptions("mg", mg_coarse="chebyshev").c()
    assert c.method == _abi.PA_SOLVER_PCG_MG and c.mg_coarse_solver == _abi.PA_MG_COARSE_CHEBYSHEV
    with pytest.raises(ValueError):
        SolveOptions("mg", mg_coarse="direct")


def test_cpp_headers_compile_against_the_library(tmp_path):
    """The C++ views of the ABI (include/pa_b200.hpp, include/pa_b200_app.hpp)
    compile and link against libpa_b200.so without a GPU (running them needs
    one: tests/test_gpu_cpp_api.py)."""
    import subprocess
    libdir = os.path.join(ROOT, "platoanalyze_b200")
    for src in ("derivative_tests.cpp", "mpmd_app_tests.cpp"):
        exe = tmp_path / src.replace(".cpp", "")
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                               os.path.join(ROOT, "tests", "cpp", src), "-o", str(exe), "-L", libdir, "-lpa_b200",
                               "-Wl,-rpath," + libdir])
        assert exe.exists()
