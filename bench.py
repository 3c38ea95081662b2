#!/usr/bin/env python
"""Benchmark: SIMP cantilever solve on B200 through libpa_b200 (C ABI).

Workload (default): 160x80x80 unit hexes x 6 tets (6,144,000 tets, 1,056,321
nodes, 3,168,963 dofs), E=1, nu=0.3, SIMP p=3 / min 1e-9, per-cell density a
Gaussian-smoothed (sigma = 3 cells) random field clipped to [0.01, 1], x=0
face clamped, unit total traction -z on x=160; one step = one full
Problem::solution to relative residual 1e-8 (default --method mg: FP64 CG
preconditioned by a geometric multigrid V-cycle with FP32 Chebyshev smoothing
and a dense coarsest-level inverse; --method mixed / fp64: Jacobi-PCG).

Metric: cells/s = tets solved per second (C / solve time), whole job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one rank per GPU) every rank solves its own density
field (seed + rank): independent problems, weak scaling, no collective on
the data path; timing is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Solve s & cells/s, 1 B200: learned-PC mixed vs plain FP64 PCG @ relres 1e-8"
UNIT = "cells/s"
DIMS = (160, 80, 80)
SEED = 1234
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 100 for the multigrid cantilever solve, 20 otherwise)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dims", default="160x80x80")
    ap.add_argument("--method", default="mg", choices=["mg", "mixed", "fp64"],
                    help="mg: CG with a geometric multigrid V-cycle (FP32 smoothing); mixed: Jacobi-PCG, FP32 apply; "
                         "fp64: Jacobi-PCG in FP64")
    ap.add_argument("--rel-tol", type=float, default=1e-8)
    ap.add_argument("--check-every", type=int, default=64,
                    help="iterations between FP64 residual replacements (one captured graph chunk)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-kernel", action="store_true",
                    help="only build the workload and time the fused CG kernel (for ncu captures)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--per-tet-geometry", action="store_true",
                    help="FP32 kernels recompute the tet geometry instead of using the box's hex geometry table")
    ap.add_argument("--newton-tol", type=float, default=1e-8, help="J2: relative Newton tolerance per load step")
    ap.add_argument("--max-newton", type=int, default=25, help="J2: Newton iterations per load step")
    ap.add_argument("--forcing", default="adaptive", choices=["adaptive", "fixed"],
                    help="J2: tangent-solve tolerances (Eisenstat-Walker, or --rel-tol for every solve)")
    ap.add_argument("--mg-coarse", default="auto", choices=["auto", "chebyshev"],
                    help="multigrid coarsest level: dense inverse when small enough, or Chebyshev iteration")
    ap.add_argument("--boxes", type=int, default=64, help="batched: number of boxes")
    ap.add_argument("--workload", default="cantilever", choices=["cantilever", "j2", "learned", "batched", "kernels"],
                    help="cantilever: the SIMP solve (default); j2: the elasto-plastic bar; learned: the "
                         "learned-preconditioner solve on 64^3 after SIMP-pair training; kernels: every "
                         "per-cell entry point timed against its roofline")
    ap.add_argument("--simp-iterations", type=int, default=30)
    ap.add_argument("--train-steps", type=int, default=400)
    args = ap.parse_args()
    if args.steps is None:  # a timed region of about a second for the multigrid solve
        args.steps = 100 if args.workload == "cantilever" and args.method == "mg" and args.impl == "ours" else 20
    return args


def dims_of(s):
    return tuple(int(v) for v in s.lower().split("x"))


def counts(dims):
    nx, ny, nz = dims
    return 6 * nx * ny * nz, (nx + 1) * (ny + 1) * (nz + 1)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------- CPU side --
def load_fields():
    """platoanalyze_b200/fields.py (NumPy only), loaded by path: importing the
    package would map libpa_b200.so into a CPU-only process."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("pa_fields", os.path.join(ROOT, "platoanalyze_b200", "fields.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class CpuCantilever:
    """The benchmark's cantilever on the FP64 CPU restatement (oracle/): the
    same mesh, per-tet densities (seed), clamp and traction as the GPU run,
    and the linear system of Elliptic::Problem::solution
    (src/elliptic/Problem.hpp:259-311): K assembled with 12-partial dual
    numbers (the role of Sacado SFad in gradient_u), constrained symmetrically
    (applyBlockConstraints), solved by Jacobi-PCG in FP64 with all host
    threads.  The CRS graph (CreateBlockMatrix) is built once, untimed."""

    def __init__(self, dims, seed, threads):
        from oracle import cpu
        fields = load_fields()
        cpu.set_threads(threads)
        self.dims, self.threads = dims, threads
        nx, ny, nz = dims
        cells, coords, faces, clamp = fields.box_arrays(nx, ny, nz)
        self.z = fields.cell_density(dims, seed, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0)
        self.O = cpu.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
        self.flux = (0.0, 0.0, -1.0 / (ny * nz))
        self.faces = faces
        self.F = -self.O.residual(np.zeros(3 * self.O.N), self.z, faces, self.flux)
        self.dofs = fields.clamp_dofs(clamp)
        t0 = time.perf_counter()
        self.graph = self.O.graph()
        self.t_graph = time.perf_counter() - t0
        self.system = None

    def assemble(self):
        self.system, self.t_asm, self.t_bc = self.O.constrained_system(self.z, self.F, self.dofs, graph=self.graph)
        return self.t_asm + self.t_bc

    def solve(self, rel_tol, report_tol=None, max_iters=0):
        return self.O.pcg_run(self.system, rel_tol=rel_tol, report_tol=report_tol, max_iters=max_iters)


REF_SAMPLE_ITERS = 128  # Jacobi-PCG iterations per timed step of the CPU reference arm


def run_reference(args):
    """The reference arm: the FP64 CPU restatement of the path (the reference
    itself cannot be built here) on the same 160x80x80 cantilever, with all
    host threads, in a process that never loads libpa_b200.so or torch.

    Untimed prologue: assembly + elimination, then one full Jacobi-PCG solve
    to --rel-tol (its iteration count I and wall time are measured).  Each
    step (warm-up and timed) is a bounded sample of that solve: the PCG
    restarted on the same system for REF_SAMPLE_ITERS iterations.
    value = C / (t_assembly + I * t_iteration), t_iteration the median of the
    timed steps over REF_SAMPLE_ITERS; the directly measured full solve is
    reported beside it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    dims = dims_of(args.dims)
    threads = host_cores()
    C, N = counts(dims)
    t0 = time.perf_counter()
    cc = CpuCantilever(dims, SEED, threads)
    t_setup = time.perf_counter() - t0
    t_sys = cc.assemble()
    _, full = cc.solve(args.rel_tol)
    if full["rel_residual"] > 1.01 * args.rel_tol:
        raise RuntimeError(f"CPU reference solve did not reach {args.rel_tol}: {full}")
    t_full = t_sys + full["seconds"]
    step_s = []
    for k in range(args.warmup + args.steps):
        t = time.perf_counter()
        _, st = cc.solve(args.rel_tol, max_iters=REF_SAMPLE_ITERS)
        dt = time.perf_counter() - t
        if k >= args.warmup:
            step_s.append(dt)
    t_iter = float(np.median(step_s)) / REF_SAMPLE_ITERS
    t_est = t_sys + full["iterations"] * t_iter
    v = C / t_est
    sample = (f"oracle (C++/OpenMP FP64, g++ -O3 -march=native) on the full {dims[0]}x{dims[1]}x{dims[2]} "
              f"cantilever ({C} tets): dual-number assembly {cc.t_asm:.2f}s + elimination {cc.t_bc:.2f}s, "
              f"Jacobi-PCG to {args.rel_tol:g} in {full['iterations']} its measured once ({t_full:.1f}s); "
              f"each step = {REF_SAMPLE_ITERS} PCG iterations of that solve")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(step_s)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded smoothed density field)",
        "config": {"workload": f"SIMP cantilever {dims[0]}x{dims[1]}x{dims[2]} hex x 6 tets, "
                               f"Problem::solution to relres {args.rel_tol:g}",
                   "cells": C, "nodes": N, "dofs": 3 * N, "rel_tol": args.rel_tol, "method": "fp64 Jacobi-PCG (CPU)",
                   "parallelism": f"{threads} host threads", "step": f"{REF_SAMPLE_ITERS} Jacobi-PCG iterations"},
        "solve_s": t_est, "full_solve_measured_s": t_full, "value_from_full_solve": C / t_full,
        "iterations": full["iterations"], "rel_residual": full["rel_residual"],
        "t_assembly_s": cc.t_asm, "t_elimination_s": cc.t_bc, "t_iteration_s": t_iter, "setup_s": t_setup,
        "graph_s_untimed": cc.t_graph,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------- multi-rank helpers --
def max_over_ranks(value, world, device="cuda"):
    """Max of a per-rank float over all ranks (one all-reduce; identity at N=1)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, cells_per_rank, steps, max_ms):
    """Units all ranks processed divided by the slowest rank's time."""
    return world * cells_per_rank * steps / (max_ms * 1e-3)


# ----------------------------------------------------------------- GPU side --
def traffic_from_profiles(kernel_tag):
    """DRAM bytes per launch recorded by the ncu summary in profiles/, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel_tag)
    except Exception:
        return None


def profile_network(args):
    """The learned preconditioner's four tensor-core convolutions on the nodal
    grid of the 64^3 box (65^3 nodes), seeded weights and features: 1 + reps
    forwards, device time per forward and TFLOP/s (a short command for ncu)."""
    import torch
    import platoanalyze_b200 as pa
    dims = (64, 64, 64) if args.dims == "160x80x80" else dims_of(args.dims)
    torch.cuda.set_device(0)
    pc = pa.LearnedPreconditioner.for_box(*dims, seed=0)
    rng = np.random.default_rng(0)
    p = pc.get_params()
    p += rng.normal(0.0, 0.02, p.size).astype(np.float32)
    pc.set_params(p)
    G = pc.num_points
    f = torch.tensor(rng.normal(size=(G, 5)).astype(np.float32), device="cuda")
    pc.forward(f)
    ms, flops = pc.time_forward(args.reps)
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak, kind = float(json.load(fh)["bf16_tflops"]), "measured"
    except Exception:
        peak, kind = 1590.0, "fallback"
    tf = flops / (ms * 1e-3) / 1e12
    print(json.dumps({"dims": dims, "grid_nodes": G, "ms_per_forward": ms, "flops": flops, "TFLOP/s": tf,
                      "peak_bf16_tflops": peak, "peak_kind": kind, "frac": tf / peak}), flush=True)
    return 0


def profile_j2(args):
    """The FP64 radial return over the 80x40x40 bar at 2% axial strain from a
    zero local state: 1 + reps launches, device time and GB/s."""
    import torch
    import platoanalyze_b200 as pa
    dims = J2_DIMS if args.dims == "160x80x80" else dims_of(args.dims)
    C, N = counts(dims)
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    mesh, prob = j2_bar(pa, dims, stream=stream.cuda_stream)
    cells, coords = mesh.arrays()
    u = torch.zeros(3 * N, dtype=torch.float64, device="cuda")
    u[0::3] = 0.02 * torch.tensor(coords[:, 0], device="cuda")
    z = torch.ones(N, dtype=torch.float64, device="cuda")
    prev = torch.zeros(14 * C, dtype=torch.float64, device="cuda")
    out = torch.empty_like(prev)
    prob.j2_radial_return(J2_PARAMS, u, z, prev, out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.reps):
        prob.j2_radial_return(J2_PARAMS, u, z, prev, out)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    nb = j2_return_bytes(C, N)
    print(json.dumps({"dims": dims, "ms_per_launch": ms, "algorithmic_bytes": nb, "GB/s": nb / (ms * 1e-3) / 1e9}),
          flush=True)
    return 0


def profile_kernel(args):
    """Build the workload and launch the fused CG kernel 1 + reps times per
    precision (a short, self-contained command for ncu)."""
    if args.workload == "learned":
        return profile_network(args)
    if args.workload == "j2":
        return profile_j2(args)
    import ctypes as ct
    import torch
    import platoanalyze_b200 as pa  # noqa: F401
    from platoanalyze_b200 import _abi
    from platoanalyze_b200.workloads import cantilever, cell_density
    dims = dims_of(args.dims)
    torch.cuda.set_device(0)
    mesh, prob, faces, dofs = cantilever(dims, uniform_geometry=not args.per_tet_geometry)
    z = torch.tensor(cell_density(dims, SEED, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0), device="cuda")
    out = {"dims": dims, "tiles": mesh.num_tiles, "uniform_geometry": mesh.uniform_geometry}
    for prec, name in ((1, "fp32"), (0, "fp64")):
        ms, nb = ct.c_double(), ct.c_int64()
        _abi.check(_abi.load().pa_time_cg_apply(prob._h, ct.c_void_p(z.data_ptr()), prec, args.reps, ct.byref(ms),
                                                ct.byref(nb)))
        out[name] = {"ms_per_launch": ms.value, "GB/s": nb.value / (ms.value * 1e-3) / 1e9,
                     "algorithmic_bytes": nb.value}
    # the plain FP32 apply (multigrid smoothing) after the fused ones
    ms, nb = ct.c_double(), ct.c_int64()
    _abi.check(_abi.load().pa_time_apply(prob._h, ct.c_void_p(z.data_ptr()), 1, args.reps, ct.byref(ms),
                                         ct.byref(nb)))
    out["fp32_plain"] = {"ms_per_launch": ms.value, "GB/s": nb.value / (ms.value * 1e-3) / 1e9,
                         "algorithmic_bytes": nb.value}
    print(json.dumps(out), flush=True)
    return 0


def run_kernels(args):
    """Every per-cell entry point of the path on the 160x80x80 box (FP64,
    per-cell controls, device buffers through the C ABI), each timed with CUDA
    events on the problem's stream after an L2 flush (256 MB written, untimed):
    cells/s and GB/s of its algorithmic bytes (s = 8, index 4 B; B = CRS
    blocks), the fraction of the measured HBM bandwidth, and the CPU oracle's
    cells/s for the same function on an 80x40x40 sample with all host threads."""
    import torch
    import platoanalyze_b200 as pa
    from platoanalyze_b200.workloads import cantilever, cell_density

    torch.cuda.set_device(0)
    dims = dims_of(args.dims)
    C, N = counts(dims)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    mesh, prob, faces, dofs = cantilever(dims, stream=stream.cuda_stream)
    B = mesh.num_blocks
    z = torch.from_numpy(cell_density(dims, SEED, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0)).cuda()
    u, _ = prob.solution(z, options=pa.SolveOptions("mg", rel_tol=1e-8))
    vf, sf = prob.vector_function(), prob.scalar_function()
    r = torch.empty(3 * N, dtype=torch.float64, device="cuda")
    gz = torch.empty(C, dtype=torch.float64, device="cuda")
    gzc = torch.empty(12 * C, dtype=torch.float64, device="cuda")
    crs = torch.empty(9 * B, dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    cases = [  # name, call, algorithmic bytes, reference function
        ("vf_value (residual)", lambda: vf.value(u, z, r), C * 24 + N * 72,
         "Elliptic::VectorFunction::value, src/elliptic/VectorFunction.hpp:231"),
        ("sf_value (compliance)", lambda: sf.value(u, z), C * 24 + N * 48,
         "PhysicsScalarFunction::value, src/elliptic/PhysicsScalarFunction.hpp:225"),
        ("sf_gradient_u", lambda: sf.gradient_u(u, z, r), C * 24 + N * 72,
         "PhysicsScalarFunction::gradient_u, :365"),
        ("sf_gradient_z (self-adjoint dF/dz)", lambda: sf.gradient_z(u, z, gz), C * 32 + N * 48,
         "PhysicsScalarFunction::gradient_z, :432"),
        ("vf_gradient_z (dR/dz, 12 per cell)", lambda: vf.gradient_z(u, z, gzc), C * 120 + N * 48,
         "VectorFunction::gradient_z, src/elliptic/VectorFunction.hpp:598"),
        ("vf_gradient_u (assembled block CRS)", lambda: vf.gradient_u(u, z, crs), C * 88 + N * 24 + B * 76,
         "VectorFunction::gradient_u, :505"),
        ("vf_gradient_x (dR/dx, block CRS)", lambda: vf.gradient_x(u, z, crs), C * 88 + N * 48 + B * 76,
         "VectorFunction::gradient_x, :317"),
    ]
    peak, peak_kind = peaks()
    rows = []
    for name, fn, nbytes, ref in cases:
        for _ in range(max(args.warmup, 3)):
            fn()
        tot = 0.0
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        ms = tot / args.steps
        gbs = nbytes / (ms * 1e-3) / 1e9
        rows.append({"function": name, "reference": ref, "ms": ms, "cells_per_s": C / (ms * 1e-3),
                     "algorithmic_bytes": nbytes, "GB/s": gbs, "frac": gbs / peak})
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import cpu as ocpu
        threads = host_cores()
        ocpu.set_threads(threads)
        sd = (80, 40, 40)
        cells, coords = ocpu.box_mesh(*sd, float(sd[0]), float(sd[1]), float(sd[2]))
        O = ocpu.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
        zc = cell_density(sd, SEED, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0)
        uc = np.random.default_rng(SEED).standard_normal(3 * O.N) * 1e-3
        g = O.graph()
        cpu = {"cores": threads, "kind": "port", "sample": f"oracle (C++/OpenMP FP64) on {sd[0]}x{sd[1]}x{sd[2]}",
               "cells_per_s": {}}
        for name, fn in [("vf_value (residual)", lambda: O.residual(uc, zc)),
                         ("sf_value+gradients (compliance, dF/du, dF/dz)", lambda: O.energy(uc, zc)),
                         ("vf_gradient_z (dR/dz, 12 per cell)", lambda: O.gradient_z(uc, zc, g)),
                         ("vf_gradient_u (assembled block CRS)", lambda: O.jacobian(uc, zc, g)),
                         ("vf_gradient_x (dR/dx, block CRS)", lambda: O.gradient_x(uc, zc, graph=g))]:
            fn()
            t = time.perf_counter()
            reps = 0
            while reps < 3 or time.perf_counter() - t < 1.0:
                fn()
                reps += 1
            cpu["cells_per_s"][name] = O.C * reps / (time.perf_counter() - t)
    print(json.dumps({"workload": f"per-cell entry points, {dims[0]}x{dims[1]}x{dims[2]} box ({C} tets, {N} nodes, "
                                  f"{B} CRS blocks), FP64, per-cell control",
                      "steps": args.steps, "warmup": max(args.warmup, 3), "peak_gbs": peak, "peak_kind": peak_kind,
                      "l2": "256 MB buffer written before each timed call", "kernels": rows,
                      "cpu_baseline": cpu}), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    import platoanalyze_b200 as pa
    from platoanalyze_b200.workloads import cantilever, cell_density

    dims = dims_of(args.dims)
    C, N = counts(dims)
    ndof = 3 * N
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    mesh, prob, faces, dofs = cantilever(dims, stream=stream.cuda_stream, uniform_geometry=not args.per_tet_geometry)
    z_host = cell_density(dims, SEED + rank, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0)
    z = torch.tensor(z_host, device="cuda")
    tile, tile_ms = prob.autotune_tiles(z)  # tile size of the fused kernel, before any timing
    u = torch.empty(ndof, dtype=torch.float64, device="cuda")
    opts = pa.SolveOptions(args.method, rel_tol=args.rel_tol, check_every=args.check_every, mg_coarse=args.mg_coarse)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")  # 256 MB > 126 MB L2

    def solve_once():
        _, st = prob.solution(z, u, options=opts)
        if not st["converged"]:
            raise RuntimeError(f"solve did not converge: {st}")
        return st

    for _ in range(args.warmup):
        solve_once()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    total_ms, launches, iters = 0.0, 0, []
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        torch.cuda.nvtx.range_push("timed_step")  # ncu --nvtx --nvtx-include "timed_step/" lists these launches
        st = solve_once()
        torch.cuda.nvtx.range_pop()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        launches += st["kernel_launches"]
        iters.append(st["iterations"])
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    max_ms = max_over_ranks(total_ms, world)
    value = whole_job_rate(world, C, args.steps, max_ms)

    # end to end through the C ABI with host (pinned) buffers: z in, u out
    z_pin = torch.tensor(z_host, dtype=torch.float64).pin_memory()
    u_pin = torch.empty(ndof, dtype=torch.float64).pin_memory()
    e2e_ms = 0.0
    prob.solution(z_pin, u_pin, options=opts)  # warm the staging buffers
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, st = prob.solution(z_pin, u_pin, options=opts)
        e2e_ms += 1e3 * (time.perf_counter() - t0)
    e2e_value = whole_job_rate(world, C, args.steps, max_over_ranks(e2e_ms, world))
    rel_u = float(np.abs(u_pin.numpy() - u.cpu().numpy()).max() / max(np.abs(u.cpu().numpy()).max(), 1e-300))

    # plain FP64 Jacobi-PCG on the same system (the comparison the metric names),
    # and the mixed Jacobi-PCG when it is not the timed method
    fp64 = pa.SolveOptions("fp64", rel_tol=args.rel_tol)
    u64 = torch.empty_like(u)
    _, st64 = prob.solution(z, u64, options=fp64)
    f_mixed = prob.scalar_function().value(u, z)
    f_fp64 = prob.scalar_function().value(u64, z)
    st_jacobi = None
    if args.method == "mg":
        _, st_jacobi = prob.solution(z, u64, options=pa.SolveOptions("mixed", rel_tol=args.rel_tol,
                                                                     check_every=args.check_every))

    # roofline of the dominant kernel timed live on this stream: the plain
    # FP32 apply of the multigrid smoother (on a box: the box kernel, whose
    # fused variants run every level of the V-cycle), or the fused CG apply
    # of Jacobi-PCG.  `achieved` uses the per-cell/per-node algorithmic bytes
    # of the matrix-free apply (4 node ids + penalty per tet, coordinates, x
    # in and y out per node); the box kernel reads no ids and no coordinates
    # (the lattice implies them), so the bytes it must move are reported too.
    import ctypes as ct
    from platoanalyze_b200 import _abi
    ms_launch, nbytes = ct.c_double(), ct.c_int64()
    lattice_bytes = None
    if args.method == "mg":
        precision = 1
        _abi.check(_abi.load().pa_time_apply(prob._h, ct.c_void_p(z.data_ptr()), precision, 50, ct.byref(ms_launch),
                                             ct.byref(nbytes)))
        if mesh.box_kernels:
            kernel = "k_box (plain FP32 box apply; the multigrid levels run this kernel with fused epilogues)"
            lattice_bytes = nbytes.value
            nbytes.value = C * (16 + 4) + N * (3 * 4) * 3
            tag = f"k_box_plain_fp32_{dims[0]}x{dims[1]}x{dims[2]}"
        else:
            kernel = "k_apply_tiled (plain FP32 apply: multigrid smoothing and residuals)"
            tag = f"k_apply_tiled_plain_fp32_{dims[0]}x{dims[1]}x{dims[2]}"
    else:
        precision = 1 if args.method == "mixed" else 0
        kernel = "k_apply_tiled (fused CG: p update + K p + p.Kp)"
        _abi.check(_abi.load().pa_time_cg_apply(prob._h, ct.c_void_p(z.data_ptr()), precision, 50,
                                                ct.byref(ms_launch), ct.byref(nbytes)))
        tag = f"k_apply_tiled_{'fp32' if precision else 'fp64'}_{dims[0]}x{dims[1]}x{dims[2]}"
    peak, peak_kind = peaks()
    achieved = nbytes.value / (ms_launch.value * 1e-3) / 1e9
    traffic = traffic_from_profiles(f"{tag}_tile{tile}")
    if traffic is None:
        traffic = traffic_from_profiles(tag)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"mixed": "f32 apply / f64 dots+refinement", "fp64": "f64",
                  "mg": "f64 CG + apply / f32 multigrid smoothing"}[args.method],
        "data": "synthetic (seeded smoothed density field)",
        "config": {"workload": f"SIMP cantilever {dims[0]}x{dims[1]}x{dims[2]} hex x 6 tets, "
                               f"Problem::solution to relres {args.rel_tol:g}",
                   "cells": C, "nodes": N, "dofs": ndof, "method": args.method, "mg_coarse": args.mg_coarse, "parallelism": f"replicas x{world}",
                   "preconditioner": ("geometric multigrid V-cycle: box hierarchy of ceil(n/2) hexes per axis per level, "
                                      "Chebyshev(2) smoothing in D^-1 K before and after the coarse correction, "
                                      "trilinear transfers, dense FP64 inverse on the coarsest level")
                   if args.method == "mg" else "Jacobi",
                   "kernels": ("box kernels (lattice node ids, fused Chebyshev/residual/CG epilogues)"
                               if args.method == "mg" and mesh.box_kernels else
                               f"tile kernels, {tile} clusters per tile (autotuned: {tile_ms})"),
                   "geometry": "hex geometry table (uniform hexes)" if mesh.uniform_geometry else "per tet",
                   "l2": "256 MB buffer written between timed steps"},
        "solve_s": max_ms / args.steps * 1e-3, "iterations": iters, "fp64_solve_s": st64["seconds"],
        "fp64_iterations": st64["iterations"], "compliance_rel_err_vs_fp64": abs(f_mixed - f_fp64) / abs(f_fp64),
        "jacobi_mixed_solve_s": st_jacobi["seconds"] if st_jacobi else None,
        "jacobi_mixed_iterations": st_jacobi["iterations"] if st_jacobi else None,
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * C, "d2h_bytes_per_step": 8 * ndof,
                "max_rel_diff_u_vs_device_run": rel_u},
        "roofline": {"bound": "hbm", "kernel": kernel,
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": traffic, "algorithmic_bytes_per_launch": nbytes.value,
                     "ms_per_launch": ms_launch.value},
    }
    if lattice_bytes is not None:
        lat_gbs = lattice_bytes / (ms_launch.value * 1e-3) / 1e9
        line["roofline"]["lattice_bytes_per_launch"] = lattice_bytes
        line["roofline"]["lattice_bytes_frac"] = lat_gbs / peak
        line["roofline"]["note"] = ("achieved/frac on the apply's per-cell/per-node algorithmic bytes; the box "
                                    "kernel moves only weights, x, y and masks (lattice_bytes), and is bound by "
                                    "instruction issue, not HBM")
    if world == 1 and not args.no_cpu_baseline:
        line.update(cpu_leg(args, dims, prob, z, u, st64))
    print(json.dumps(line), flush=True)
    return 0


def cpu_leg(args, dims, prob, z, u, st64):
    """Rank 0 at N = 1, after the timed GPU work: the oracle's FP64 solve of
    the same cantilever on the host cores (assembly + Jacobi-PCG), timed to
    --rel-tol (cpu_baseline, the same algorithm as the GPU's plain FP64 PCG),
    then continued to 1e-10 as the reference solution: the GPU result's errors
    in displacement, compliance and gradient_z against it, and the GPU
    solution's residual measured with the oracle's own operator."""
    C, N = counts(dims)
    threads = host_cores()
    cc = CpuCantilever(dims, SEED, threads)
    t_sys = cc.assemble()
    ref_tol = min(1e-10, args.rel_tol)
    x_or, info = cc.solve(ref_tol, report_tol=args.rel_tol)
    t_cpu = t_sys + info["report_seconds"]
    u_h = u.cpu().numpy()
    f_or, _, gz_or = cc.O.energy(x_or, cc.z)
    f_gpu = prob.scalar_function().value(u, z)
    gz_gpu = prob.scalar_function().gradient_z(u, z).cpu().numpy()
    res = cc.F - cc.O.apply(u_h, cc.z)
    res[cc.dofs] = 0.0
    fnorm = np.linalg.norm(np.where(np.isin(np.arange(3 * N), cc.dofs), 0.0, cc.F))
    sample = (f"oracle (C++/OpenMP FP64, g++ -O3 -march=native) on the full {dims[0]}x{dims[1]}x{dims[2]} "
              f"cantilever ({C} tets): dual-number assembly {cc.t_asm:.2f}s + elimination {cc.t_bc:.2f}s + "
              f"Jacobi-PCG to {args.rel_tol:g} in {info['report_iterations']} its ({info['report_seconds']:.1f}s), "
              "measured once")
    return {
        "cpu_baseline": {"value": C / t_cpu, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "same_algorithm": {"what": "plain FP64 Jacobi-PCG to relres %g on the same system" % args.rel_tol,
                           "gpu_s": st64["seconds"], "gpu_iterations": st64["iterations"],
                           "cpu_s": t_cpu, "cpu_iterations": info["report_iterations"],
                           "cpu_over_gpu": t_cpu / st64["seconds"]},
        "vs_oracle": {"reference_solution": f"oracle Jacobi-PCG to relres {ref_tol:g} "
                                            f"({info['iterations']} its, true relres {info['rel_residual']:.2e})",
                      "err_u_vs_oracle": float(np.abs(u_h - x_or).max() / np.abs(x_or).max()),
                      "err_compliance_vs_oracle": abs(f_gpu - f_or) / abs(f_or),
                      "err_gradz_vs_oracle": float(np.abs(gz_gpu - gz_or).max() / np.abs(gz_or).max()),
                      "relres_of_gpu_u_by_oracle_operator": float(np.linalg.norm(res) / fnorm),
                      "norms": "max-norm relative (u, gradient_z); |f - f_oracle| / |f_oracle|"},
    }


J2_DIMS = (80, 40, 40)
J2_PARAMS = dict(youngs_modulus=200e3, poissons_ratio=0.3, initial_yield_stress=250.0,
                 hardening_modulus_isotropic=1000.0, hardening_modulus_kinematic=0.0, elastic_penalty_exponent=3.0,
                 elastic_min_ersatz=1e-9, plastic_penalty_exponent=2.5, plastic_min_ersatz=1e-9)


def j2_bar(pa, dims, strain=0.02, stream=None):
    """80x40x40 hex x 6 tet bar, x = 0 clamped, u_x = strain * L prescribed on
    x = L (the final value; pa_j2_solve ramps it over the load steps)."""
    nx, ny, nz = dims
    mesh = pa.Mesh.box(nx, ny, nz, float(nx), float(ny), float(nz))
    prob = pa.Problem(mesh, J2_PARAMS["youngs_modulus"], J2_PARAMS["poissons_ratio"], stream=stream)
    px, py = nx + 1, ny + 1
    jj, kk = np.meshgrid(np.arange(py), np.arange(nz + 1), indexing="ij")
    x0 = (px * (jj + py * kk)).ravel()
    x1 = x0 + nx
    dofs = np.concatenate([3 * x0, 3 * x0 + 1, 3 * x0 + 2, 3 * x1])
    vals = np.concatenate([np.zeros(3 * x0.size), np.full(x1.size, strain * nx)])
    order = np.argsort(dofs)
    prob.set_dirichlet(dofs[order].astype(np.int32), vals[order])
    return mesh, prob


def j2_return_bytes(C, N):
    """Algorithmic bytes of one radial return over the mesh: connectivity
    (16 B), 14 + 14 local-state doubles and the cell's density per cell;
    coordinates and displacements (3 + 3 doubles) per node."""
    return C * (16 + 14 * 8 * 2 + 8) + N * (3 * 8 + 3 * 8)


def cpu_j2_return_rate(dims, threads, reps=5):
    """Oracle (C++/OpenMP FP64) radial return over the full mesh at a
    plastic state: cells/s, median of `reps` after one warm-up."""
    from oracle import cpu
    cpu.set_threads(threads)
    nx, ny, nz = dims
    cells, coords = cpu.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    O = cpu.Oracle(cells, coords, E=J2_PARAMS["youngs_modulus"], nu=0.3, p=1.0, pmin=0.0)
    u = np.zeros(3 * O.N)
    u[0::3] = 0.02 * coords[:, 0]  # 2% axial strain: every cell past yield
    z = np.ones(O.N)
    prev = np.zeros(14 * O.C)
    mu = J2_PARAMS["youngs_modulus"] / (2 * (1 + J2_PARAMS["poissons_ratio"]))
    ts = []
    for k in range(reps + 1):
        t0 = time.perf_counter()
        O.j2_update(u, z, prev, mu, 250.0, 1000.0, 0.0)
        if k:
            ts.append(time.perf_counter() - t0)
    t = float(np.median(ts))
    return O.C / t, t


def run_j2(args):
    """cfg5: small-strain J2 bar, 20 load steps to 2% axial strain; one step
    of the benchmark = one whole load-stepped Newton solve (FP64 return
    mapping and residual, mixed-precision tangent solves)."""
    import torch
    import platoanalyze_b200 as pa

    dims = J2_DIMS if args.dims == "160x80x80" else dims_of(args.dims)
    C, N = counts(dims)
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    mesh, prob = j2_bar(pa, dims, stream=stream.cuda_stream)
    z = torch.ones(N, dtype=torch.float64, device="cuda")
    u = torch.empty(3 * N, dtype=torch.float64, device="cuda")
    local = torch.empty(14 * C, dtype=torch.float64, device="cuda")
    lin = pa.SolveOptions(args.method, rel_tol=args.rel_tol, mg_coarse=args.mg_coarse)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")

    def solve_once():
        _, _, st = prob.j2_solve(J2_PARAMS, z, steps=20, max_newton=args.max_newton, newton_tol=args.newton_tol,
                                 options=lin, u=u, local=local, allow_not_converged=True,
                                 adaptive_forcing=args.forcing == "adaptive")
        return st

    for _ in range(args.warmup):
        solve_once()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    total_ms, stats = 0.0, []
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        stats.append(solve_once())
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    clk = clocks.stop()
    loc = local.view(-1, 14)
    plastic_frac = float((loc[:, 0] > 0).double().mean().item())

    # the radial return alone (FP64), from the converged state: roofline
    prev = torch.zeros_like(local)
    out = torch.empty_like(local)
    for _ in range(3):
        prob.j2_radial_return(J2_PARAMS, u, z, prev, out)
    reps, ms = 20, 0.0
    for _ in range(reps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        prob.j2_radial_return(J2_PARAMS, u, z, prev, out)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= reps
    nbytes = j2_return_bytes(C, N)
    peak, peak_kind = peaks()
    achieved = nbytes / (ms * 1e-3) / 1e9

    # end to end with host buffers: z in, u and the local states out
    z_pin = torch.ones(N, dtype=torch.float64).pin_memory()
    u_pin = torch.empty(3 * N, dtype=torch.float64).pin_memory()
    l_pin = torch.empty(14 * C, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prob.j2_solve(J2_PARAMS, z_pin, steps=20, max_newton=args.max_newton, newton_tol=args.newton_tol, options=lin,
                  adaptive_forcing=args.forcing == "adaptive", u=u_pin,
                  local=l_pin, allow_not_converged=True)
    e2e_ms = 1e3 * (time.perf_counter() - t0)

    value = C * args.steps / (total_ms * 1e-3)
    line = {
        "metric": "J2 load-stepped solve cells/s, 1 B200", "value": value, "unit": "cells/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 return map + residual / " + ("f32 apply, f64 dots+refinement" if args.method == "mixed"
                                                   else "f64 tangent solves"),
        "data": "synthetic (uniform density 1)",
        "config": {"workload": f"J2 bar {dims[0]}x{dims[1]}x{dims[2]} hex x 6 tets, 20 load steps to 2% axial strain, "
                               "E=200e3 nu=0.3 sigma_y=250 H_iso=1000", "cells": C, "nodes": N,
                   "linear": args.method, "mg_coarse": args.mg_coarse, "linear_rel_tol": args.rel_tol,
                   "tangent_tolerance": "Eisenstat-Walker (floor linear_rel_tol)" if args.forcing == "adaptive"
                   else "linear_rel_tol for every tangent solve",
                   "l2": "256 MB buffer written between steps"},
        "newton_iterations": [s["newton_iterations"] for s in stats], "cg_iterations": [s["cg_iterations"] for s in stats],
        "newton_tol": args.newton_tol, "converged": all(s["converged"] for s in stats),
        "worst_step_rel_residual": max(s["final_rel_residual"] for s in stats),
        "linear_unconverged": [s["linear_unconverged"] for s in stats], "plastic_cell_fraction": plastic_frac,
        "clocks": clk,
        "e2e": {"value": C / (e2e_ms * 1e-3), "unit": "cells/s", "h2d_bytes_per_step": 8 * N,
                "d2h_bytes_per_step": 8 * (3 * N + 14 * C)},
        "roofline": {"bound": "hbm", "kernel": "k_j2 (radial return, FP64)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_launch": nbytes, "ms_per_launch": ms},
    }
    if not args.no_cpu_baseline:
        threads = host_cores()
        rate, t = cpu_j2_return_rate(dims, threads)
        line["cpu_baseline"] = {"value": rate, "unit": "cells/s (radial return)", "cores": threads, "kind": "port",
                                "sample": f"oracle radial return over the full {C}-cell mesh at 2% strain, "
                                          f"{t * 1e3:.1f} ms; the GPU return takes {ms:.3f} ms"}
    print(json.dumps(line), flush=True)
    return 0


def run_learned(args):
    """cfg4: 64x64x64 hexes x 6 tets cantilever; (residual, error) pairs from
    SIMP/OC design iterations (volume fraction 0.4, move 0.2) with plain
    solves, the network trained on the GPU, then the design after the last
    iteration (not seen in training) solved to relres 1e-8 by the learned
    flexible CG (mixed), the plain FP64 Jacobi-PCG and the mixed Jacobi-PCG."""
    import torch
    import platoanalyze_b200 as pa
    from platoanalyze_b200.workloads import cantilever, simp_training_pairs

    dims = (64, 64, 64) if args.dims == "160x80x80" else dims_of(args.dims)
    C, N = counts(dims)
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    mesh, prob, faces, dofs = cantilever(dims, stream=stream.cuda_stream)
    t0 = time.perf_counter()
    dens, sd, res, en, final, hist = simp_training_pairs(prob, dims, iterations=args.simp_iterations)
    torch.cuda.synchronize()
    t_pairs = time.perf_counter() - t0
    pc = pa.LearnedPreconditioner.for_box(*dims, seed=0)
    tr = pc.train(prob, dens, sd, res, en, steps=args.train_steps, batch=4, learning_rate=1e-3, seed=1)
    prob.set_preconditioner(pc)
    z = torch.tensor(final, device="cuda")
    u = torch.empty(3 * N, dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")
    opts = {"learned": pa.SolveOptions("learned", rel_tol=args.rel_tol),
            "mixed": pa.SolveOptions("mixed", rel_tol=args.rel_tol),
            "fp64": pa.SolveOptions("fp64", rel_tol=args.rel_tol),
            "mg": pa.SolveOptions("mg", rel_tol=args.rel_tol, mg_coarse=args.mg_coarse)}

    def timed(name, steps, warmup):
        for _ in range(warmup):
            prob.solution(z, u, options=opts[name])
        ms, st = [], None
        for _ in range(steps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, st = prob.solution(z, u, options=opts[name])
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms)), st, prob.scalar_function().value(u, z)

    clocks = ClockSampler(0)
    clocks.start()
    ms_l, st_l, f_l = timed("learned", args.steps, args.warmup)
    clk = clocks.stop()
    ms_m, st_m, f_m = timed("mixed", max(1, args.steps // 2), 1)
    ms_d, st_d, f_d = timed("fp64", max(1, args.steps // 2), 1)
    ms_g, st_g, f_g = timed("mg", max(1, args.steps // 2), 1)
    # learned level-1 weights of the box multigrid: pairs from multigrid
    # solves of the same design iterations, parameters selected by the CG
    # iterations on the last training design; the held-out final design
    # solved with the parameters kept
    from platoanalyze_b200.api import LearnedCoarsening
    t0 = time.perf_counter()
    dens_c, sd_c, res_c, en_c, _, _ = simp_training_pairs(prob, dims, iterations=args.simp_iterations,
                                                          snapshots=(2, 4, 8, 16), solver="mg", first=8)
    lc = LearnedCoarsening(prob, seed=0)
    tr_c = lc.train(prob, dens_c, res_c, en_c, sd_c, steps=args.train_steps // 2, batch=4, learning_rate=3e-3, seed=1,
                    validation=dens_c[-1], check_every=20)
    t_c = time.perf_counter() - t0
    lc.attach(prob)
    ms_c, st_c, f_c = timed("mg", max(1, args.steps // 2), 1)
    prob.set_coarse_network(None)
    coarse = {"solve_s": ms_c * 1e-3, **st_c, "compliance_rel_err_vs_fp64": abs(f_c - f_d) / abs(f_d),
              "validation_cg_iterations_by_step": tr_c["iterations"], "kept_step": tr_c["kept_step"],
              "loss_first_20": float(np.mean(tr_c["loss"][:20])), "loss_last_20": float(np.mean(tr_c["loss"][-20:])),
              "pairs": int(len(sd_c)), "pairs_and_training_s": t_c}
    lc.close()
    line = {
        "metric": METRIC, "value": C / (ms_l * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_l, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 network (f32 accumulate) / f32 apply / f64 dots+refinement",
        "data": "synthetic (SIMP/OC designs from a uniform 0.4 start)",
        "config": {"workload": f"learned-PC SIMP cantilever {dims[0]}x{dims[1]}x{dims[2]} hex x 6 tets, "
                               f"Problem::solution to relres {args.rel_tol:g}", "cells": C, "nodes": N,
                   "simp_iterations": args.simp_iterations, "pairs": int(len(sd)), "train_steps": args.train_steps,
                   "network_params": pc.num_params, "l2": "256 MB buffer written between timed steps"},
        "learned": {"solve_s": ms_l * 1e-3, **st_l, "compliance_rel_err_vs_fp64": abs(f_l - f_d) / abs(f_d)},
        "jacobi_mixed": {"solve_s": ms_m * 1e-3, **st_m, "compliance_rel_err_vs_fp64": abs(f_m - f_d) / abs(f_d)},
        "jacobi_fp64": {"solve_s": ms_d * 1e-3, **st_d},
        "multigrid": {"solve_s": ms_g * 1e-3, **st_g, "compliance_rel_err_vs_fp64": abs(f_g - f_d) / abs(f_d)},
        "multigrid_learned_coarse_weights": coarse,
        "speedup_learned_vs_fp64": ms_d / ms_l, "speedup_mixed_vs_fp64": ms_d / ms_m,
        "speedup_multigrid_vs_fp64": ms_d / ms_g,
        "training": tr, "pair_generation_s": t_pairs,
        "simp_history": [{k: h[k] for k in ("iteration", "compliance", "cg_iterations")} for h in hist],
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args):
    """cfg3: 64 independent cantilevers with edges U{16..48} hexes, each with
    its own smoothed density (seed + i) and unit traction direction, solved
    as one parted mesh (one CG per box, all boxes in the same kernels and
    one CUDA graph per chunk) to relres 1e-8 in mixed precision, after the
    tile-size autotuner.  Under torchrun the boxes are dealt to the ranks by
    estimated work (strong scaling; no collective on the data path)."""
    import torch
    import torch.distributed as dist
    import platoanalyze_b200 as pa
    from platoanalyze_b200.workloads import batch_specs, batched_boxes, _box

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    specs, dirs = batch_specs(args.boxes, SEED)
    mine = dealt_boxes(specs, world, rank)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    t0 = time.perf_counter()
    mesh, prob, z_host, offs = batched_boxes([specs[i] for i in mine], dirs[mine], seed=SEED, stream=stream.cuda_stream,
                                             box_ids=mine)
    t_build = time.perf_counter() - t0
    z = torch.tensor(z_host, device="cuda")
    tile, tile_ms = prob.autotune_tiles(z)
    C_mine, N_mine = mesh.num_cells, mesh.num_nodes
    u = torch.empty(3 * N_mine, dtype=torch.float64, device="cuda")
    opts = pa.SolveOptions("mixed", rel_tol=args.rel_tol)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")

    def solve_once():
        _, st = prob.solution(z, u, options=opts)
        if not st["converged"]:
            raise RuntimeError(f"batched solve did not converge: {st}")
        return st

    for _ in range(args.warmup):
        solve_once()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    total_ms, launches = 0.0, 0
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = solve_once()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        launches += st["kernel_launches"]
    clk = clocks.stop()
    its, rel = prob.part_stats()
    if world > 1:
        dist.barrier()
    max_ms = max_over_ranks(total_ms, world)
    C_all = sum(6 * a * b * c for a, b, c in specs)
    value = C_all * args.steps / (max_ms * 1e-3)
    # end to end with host arrays: densities in, displacements out
    z_pin = torch.tensor(z_host).pin_memory()
    u_pin = torch.empty(3 * N_mine, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    te = time.perf_counter()
    prob.solution(z_pin, u_pin, options=opts)
    e2e_ms = max_over_ranks(1e3 * (time.perf_counter() - te), world)
    # the same boxes one at a time (own mesh and problem each), rank 0 at N=1
    seq = None
    if world == 1:
        seq_ms, seq_its = 0.0, []
        for k, i in enumerate(mine[:args.boxes]):
            nx, ny, nz = specs[i]
            c, X, f, cl = _box(nx, ny, nz)
            m1 = pa.Mesh.from_arrays(c, X)
            p1 = pa.Problem(m1, 1.0, 0.3, 3.0, 1e-9, control_layout="cell", stream=stream.cuda_stream)
            p1.add_traction(f, dirs[i] / (ny * nz))
            p1.set_dirichlet(np.sort(np.concatenate([3 * cl, 3 * cl + 1, 3 * cl + 2])).astype(np.int32))
            zi = torch.tensor(z_host[offs_cells(offs, specs, mine, k)], device="cuda")
            p1.solution(zi, options=opts)  # warm
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, s1 = p1.solution(zi, options=opts)
            e1.record(stream)
            e1.synchronize()
            seq_ms += e0.elapsed_time(e1)
            seq_its.append(s1["iterations"])
            p1.close()
            m1.close()
        d = np.abs(np.array(seq_its) - its) / np.array(seq_its)
        seq = {"solve_s": seq_ms * 1e-3, "cells_per_s": C_all / (seq_ms * 1e-3),
               "iterations_rel_diff_vs_batched": {"median": float(np.median(d)), "max": float(d.max())}}
    # the same boxes one at a time by the box multigrid (any box size), each
    # box its own mesh (given as arrays, recognised as a lattice) and problem;
    # rank 0 at N=1
    seq_mg = None
    if world == 1:
        probs = []
        for k, i in enumerate(mine[:args.boxes]):
            nx, ny, nz = specs[i]
            c, X, f, cl = _box(nx, ny, nz)
            m1 = pa.Mesh.from_arrays(c, X)
            p1 = pa.Problem(m1, 1.0, 0.3, 3.0, 1e-9, control_layout="cell", stream=stream.cuda_stream)
            p1.add_traction(f, dirs[i] / (ny * nz))
            p1.set_dirichlet(np.sort(np.concatenate([3 * cl, 3 * cl + 1, 3 * cl + 2])).astype(np.int32))
            zi = torch.tensor(z_host[offs_cells(offs, specs, mine, k)], device="cuda")
            ui = torch.empty(3 * m1.num_nodes, dtype=torch.float64, device="cuda")
            probs.append((m1, p1, zi, ui))
        mg_opts = pa.SolveOptions("mg", rel_tol=args.rel_tol)
        for m1, p1, zi, ui in probs:  # warm: hierarchies, graphs
            p1.solution(zi, ui, options=mg_opts)
        mg_ms, mg_its, mg_rel = [], [], []
        for _ in range(max(1, args.steps)):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            its_k = []
            for m1, p1, zi, ui in probs:
                _, s1 = p1.solution(zi, ui, options=mg_opts)
                if not s1["converged"]:
                    raise RuntimeError(f"box multigrid solve did not converge: {s1}")
                its_k.append(s1["iterations"])
                mg_rel.append(s1["rel_residual"])
            e1.record(stream)
            e1.synchronize()
            mg_ms.append(e0.elapsed_time(e1))
            mg_its = its_k
        # the same problems from 8 host threads, each box on its own stream
        # (ctypes drops the GIL), largest boxes first, time from the host clock
        # around the batch.  Each problem's first solve (hierarchy and graph
        # capture) runs in this thread: concurrent first solves from several
        # threads failed inside a capture in one run
        import threading
        streams = [torch.cuda.Stream() for _ in probs]
        probs_t = []
        for (m1, p1, zi, ui), st_k in zip(probs, streams):
            p1.close()
            p2 = pa.Problem(m1, 1.0, 0.3, 3.0, 1e-9, control_layout="cell", stream=st_k.cuda_stream)
            i = mine[len(probs_t)]
            nx, ny, nz = specs[i]
            _, _, f, cl = _box(nx, ny, nz)
            p2.add_traction(f, dirs[i] / (ny * nz))
            p2.set_dirichlet(np.sort(np.concatenate([3 * cl, 3 * cl + 1, 3 * cl + 2])).astype(np.int32))
            probs_t.append((m1, p2, zi, ui))
        order = sorted(range(len(probs_t)), key=lambda k: -probs_t[k][0].num_cells)
        n_threads = 8
        groups = [order[t::n_threads] for t in range(n_threads)]
        errors = []

        def worker(idx):
            try:
                for k in idx:
                    _, p2, zi, ui = probs_t[k]
                    _, s2 = p2.solution(zi, ui, options=mg_opts)
                    if not s2["converged"]:
                        raise RuntimeError(f"box multigrid solve did not converge: {s2}")
            except Exception as ex:  # reported after the join
                errors.append(ex)

        for k in order:
            _, p2, zi, ui = probs_t[k]
            p2.solution(zi, ui, options=mg_opts)
        thr_ms = []
        for rep in range(1 + max(1, args.steps)):  # the first pass is a warm-up
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            th = [threading.Thread(target=worker, args=(g,)) for g in groups]
            for t in th:
                t.start()
            for t in th:
                t.join()
            torch.cuda.synchronize()
            if errors:
                raise errors[0]
            if rep:
                thr_ms.append(1e3 * (time.perf_counter() - t0))
        for m1, p2, zi, ui in probs_t:
            p2.close()
            m1.close()
        t_thr = float(np.median(thr_ms)) * 1e-3
        t_mg = float(np.median(mg_ms)) * 1e-3
        seq_mg = {"solve_s": t_mg, "cells_per_s": C_all / t_mg, "steps": len(mg_ms),
                  "per_box_iterations": {"min": int(min(mg_its)), "median": float(np.median(mg_its)),
                                         "max": int(max(mg_its))},
                  "max_rel_residual": float(max(mg_rel)),
                  "method": "box multigrid CG per box (FP64 CG, FP32 V-cycle), boxes in sequence on one stream",
                  "threads8": {"solve_s": t_thr, "cells_per_s": C_all / t_thr, "steps": len(thr_ms),
                               "method": "the same solves from 8 host threads, one stream per box, largest first; "
                                         "host clock around the batch"}}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": "Batched SIMP solves cells/s, 1 B200", "value": value, "unit": "cells/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32 apply / f64 dots+refinement",
        "data": "synthetic (seeded box sizes, smoothed densities, traction directions)",
        "config": {"workload": f"{args.boxes} cantilever boxes, edges U{{16..48}} hexes x 6 tets, one CG per box, "
                               f"relres {args.rel_tol:g}", "cells": C_all, "boxes": args.boxes,
                   "parallelism": f"boxes dealt over {world} rank(s)", "tile_clusters": tile,
                   "autotune_ms_per_apply": tile_ms, "l2": "256 MB buffer written between timed steps"},
        "per_box_iterations": {"min": int(its.min()), "median": float(np.median(its)), "max": int(its.max())},
        "max_rel_residual": float(rel.max()), "mesh_build_s": t_build, "gpu_launches": launches,
        "clocks": clk,
        "e2e": {"value": C_all / (e2e_ms * 1e-3), "unit": "cells/s", "h2d_bytes_per_step": 8 * C_mine,
                "d2h_bytes_per_step": 8 * 3 * N_mine},
        "one_box_at_a_time": seq,
        "one_box_at_a_time_multigrid": seq_mg,
    }
    print(json.dumps(line), flush=True)
    return 0


def dealt_boxes(specs, world, rank):
    """Boxes of this rank in the batched workload: dealt by estimated work
    (tets x longest edge), longest first, each to the least-loaded rank, so
    that every box is solved by exactly one rank and the largest rank load is
    within one box of the mean."""
    from platoanalyze_b200.partition import deal_boxes
    return deal_boxes(specs, world)[rank]


def offs_cells(offs, specs, mine, k):
    """Slice of the batched per-cell array that belongs to the k-th local box."""
    c0 = sum(6 * specs[i][0] * specs[i][1] * specs[i][2] for i in mine[:k])
    nx, ny, nz = specs[mine[k]]
    return slice(c0, c0 + 6 * nx * ny * nz)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_kernel:
        return profile_kernel(args)
    if args.workload == "j2":
        return run_j2(args)
    if args.workload == "learned":
        return run_learned(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "kernels":
        return run_kernels(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
