"""The CPU reference arm of bench.py runs the oracle on the benchmark's own
workload in a process that never maps libpa_b200.so or imports torch, and
its system is the one the GPU solves (same mesh, densities, clamp, load)."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_loads_no_product_code():
    code = (
        "import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--dims', '8x4x4', '--steps', '2', "
        "'--warmup', '1']\n"
        "import bench\n"
        "rc = bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'rc': rc, 'torch': 'torch' in sys.modules, 'pkg': 'platoanalyze_b200' in sys.modules,\n"
        "                  'so': 'libpa_b200' in maps, 'oracle_so': 'libpa_oracle' in maps}))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [json.loads(l) for l in out.stdout.strip().splitlines()]
    line, probe = lines[0], lines[-1]
    assert probe == {"rc": 0, "torch": False, "pkg": False, "so": False, "oracle_so": True}
    assert line["impl"] == "reference" and line["unit"] == "cells/s" and line["steps"] == 2
    assert line["config"]["cells"] == 6 * 8 * 4 * 4
    assert line["rel_residual"] <= 1.01e-8
    # the estimate from the timed samples and the directly measured full solve agree
    assert 0.5 < line["value"] / line["value_from_full_solve"] < 2.0


def test_cpu_cantilever_matches_gpu_workload_definition(oracle_lib):
    """CpuCantilever builds the mesh, densities, Dirichlet set and load of
    platoanalyze_b200.workloads.cantilever (the GPU benchmark's problem)."""
    sys.path.insert(0, ROOT)
    import bench
    fields = bench.load_fields()
    dims = (6, 4, 2)
    cc = bench.CpuCantilever(dims, 7, 2)
    cells, coords = oracle_lib.box_mesh(*dims, *map(float, dims))
    assert np.array_equal(cc.O.cells, cells) and np.array_equal(cc.O.coords, coords)
    assert np.array_equal(cc.z, np.repeat(fields.hex_density(dims, 7), 6))
    clamp = np.where(coords[:, 0] == 0.0)[0]
    assert np.array_equal(cc.dofs, np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])))
    # unit total traction in -z on x = nx
    fz = cc.F[2::3]
    assert abs(fz.sum() + 1.0) < 1e-12 and np.all(fz[coords[:, 0] < dims[0]] == 0.0)
    assert np.all(cc.F[0::3] == 0.0) and np.all(cc.F[1::3] == 0.0)
    cc.assemble()
    x, info = cc.solve(1e-10, report_tol=1e-8)
    # the stop is on the recursive residual; the reported (true) one may sit a
    # little above the tolerance, by an amount that depends on the host's
    # floating-point contraction and thread count
    assert 0 < info["report_iterations"] <= info["iterations"] and info["rel_residual"] < 2e-10
    res = cc.F - cc.O.apply(x, cc.z)
    res[cc.dofs] = 0.0
    assert np.linalg.norm(res) / np.linalg.norm(cc.F) < 2e-10
