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
