#!/usr/bin/env python
"""Benchmark: SIMP cantilever solve on B200 through libpa_b200 (C ABI).

Workload (default): 160x80x80 unit hexes x 6 tets (6,144,000 tets, 1,056,321
nodes, 3,168,963 dofs), E=1, nu=0.3, SIMP p=3 / min 1e-9, per-cell density a
Gaussian-smoothed (sigma = 3 cells) random field clipped to [0.01, 1], x=0
face clamped, unit total traction -z on x=160; one step = one full
Problem::solution (mixed precision Jacobi-PCG: FP32 matrix-free apply and
vectors, FP64 dots, FP64 true-residual replacement) to relative residual 1e-8.

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
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dims", default="160x80x80")
    ap.add_argument("--method", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--rel-tol", type=float, default=1e-8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-kernel", action="store_true",
                    help="only build the workload and time the fused CG kernel (for ncu captures)")
    ap.add_argument("--reps", type=int, default=3)
    return ap.parse_args()


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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
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
def cpu_solve_estimate(target_dims, threads, sample_dims=(80, 40, 40)):
    """FP64 CPU restatement (oracle) timed on a bounded sample of the same
    physics: dual-number assembly of the block CRS, symmetric Dirichlet
    elimination and Jacobi-PCG (the reference's structure: assemble, then
    Krylov).  Per-cell assembly cost and per-iteration cost are measured on
    `sample_dims`; the full solve of the sample runs to 1e-8 to get its
    iteration count, scaled to the target by the hex count along x (CG
    iterations grow like 1/h for this operator).  Returns cells/s for the
    target and a description."""
    from oracle import cpu
    from platoanalyze_b200.workloads import cell_density
    cpu.set_threads(threads)
    nx, ny, nz = sample_dims
    cells, coords = cpu.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    z = cell_density(sample_dims, SEED, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0)
    O = cpu.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    faces = []
    xs = coords[:, 0]
    for c in cells:
        for drop in range(4):
            f = [c[k] for k in range(4) if k != drop]
            if all(abs(xs[v] - nx) < 1e-9 for v in f):
                faces.append(f)
    faces = np.array(faces, np.int32)
    F = -O.residual(np.zeros(3 * O.N), z, faces, (0.0, 0.0, -1.0 / (ny * nz)))
    clamp = np.where(xs < 1e-9)[0]
    dofs = np.sort(np.concatenate([3 * clamp, 3 * clamp + 1, 3 * clamp + 2])).astype(np.int32)
    graph = O.graph()
    t0 = time.perf_counter()
    O.jacobian(np.zeros(3 * O.N), z, graph)
    t_asm = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, iters_sample, rel = O.solve(z, F, dofs, rel_tol=1e-8, graph=graph)
    t_full = time.perf_counter() - t0
    t_iter = max((t_full - t_asm) / max(iters_sample, 1), 1e-9)
    Ct, Nt = counts(target_dims)
    Cs, Ns = O.C, O.N
    iters_target = iters_sample * target_dims[0] / nx
    t_target = t_asm * Ct / Cs + iters_target * t_iter * Nt / Ns
    desc = (f"oracle (C++/OpenMP FP64) assembly + Jacobi-PCG to 1e-8 on a {nx}x{ny}x{nz} box "
            f"({Cs} tets, {iters_sample} its, {t_full:.2f}s); scaled to {target_dims[0]}x{target_dims[1]}x"
            f"{target_dims[2]} by cells/nodes and iterations x{target_dims[0] / nx:g} "
            f"(~{iters_target:.0f} its, {t_target:.1f}s per solve)")
    return Ct / t_target, desc, {"t_assembly_s": t_asm * Ct / Cs, "iters_est": iters_target, "t_iter_s": t_iter * Nt / Ns}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    dims = dims_of(args.dims)
    threads = host_cores()
    vals = []
    desc = ""
    for k in range(args.warmup + args.steps):
        v, desc, _ = cpu_solve_estimate(dims, threads)
        if k >= args.warmup:
            vals.append(v)
    v = float(np.median(vals))
    C, N = counts(dims)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * C / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"cantilever {dims[0]}x{dims[1]}x{dims[2]} hex x 6 tets", "cells": C, "nodes": N,
                   "rel_tol": args.rel_tol, "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc},
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


def profile_kernel(args):
    """Build the workload and launch the fused CG kernel 1 + reps times per
    precision (a short, self-contained command for ncu)."""
    import ctypes as ct
    import torch
    import platoanalyze_b200 as pa  # noqa: F401
    from platoanalyze_b200 import _abi
    from platoanalyze_b200.workloads import cantilever, cell_density
    dims = dims_of(args.dims)
    torch.cuda.set_device(0)
    mesh, prob, faces, dofs = cantilever(dims)
    z = torch.tensor(cell_density(dims, SEED, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0), device="cuda")
    out = {"dims": dims, "tiles": mesh.num_tiles}
    for prec, name in ((1, "fp32"), (0, "fp64")):
        ms, nb = ct.c_double(), ct.c_int64()
        _abi.check(_abi.load().pa_time_cg_apply(prob._h, ct.c_void_p(z.data_ptr()), prec, args.reps, ct.byref(ms),
                                                ct.byref(nb)))
        out[name] = {"ms_per_launch": ms.value, "GB/s": nb.value / (ms.value * 1e-3) / 1e9,
                     "algorithmic_bytes": nb.value}
    print(json.dumps(out), flush=True)
    return 0


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
    mesh, prob, faces, dofs = cantilever(dims, stream=stream.cuda_stream)
    z_host = cell_density(dims, SEED + rank, kind="smoothed", sigma=3.0, lo=0.01, hi=1.0)
    z = torch.tensor(z_host, device="cuda")
    u = torch.empty(ndof, dtype=torch.float64, device="cuda")
    opts = pa.SolveOptions(args.method, rel_tol=args.rel_tol)
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
        st = solve_once()
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

    # plain FP64 Jacobi-PCG on the same system (the comparison the metric names)
    fp64 = pa.SolveOptions("fp64", rel_tol=args.rel_tol)
    u64 = torch.empty_like(u)
    _, st64 = prob.solution(z, u64, options=fp64)
    f_mixed = prob.scalar_function().value(u, z)
    f_fp64 = prob.scalar_function().value(u64, z)

    # roofline of the dominant kernel (fused CG apply) timed live on this stream
    precision = 1 if args.method == "mixed" else 0
    import ctypes as ct
    from platoanalyze_b200 import _abi
    ms_launch, nbytes = ct.c_double(), ct.c_int64()
    _abi.check(_abi.load().pa_time_cg_apply(prob._h, ct.c_void_p(z.data_ptr()), precision, 50, ct.byref(ms_launch),
                                            ct.byref(nbytes)))
    peak, peak_kind = peaks()
    achieved = nbytes.value / (ms_launch.value * 1e-3) / 1e9
    tag = f"k_apply_tiled_{'fp32' if precision else 'fp64'}_{dims[0]}x{dims[1]}x{dims[2]}"
    traffic = traffic_from_profiles(tag)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 apply / f64 dots+refinement" if args.method == "mixed" else "f64",
        "data": "synthetic (seeded smoothed density field)",
        "config": {"workload": f"SIMP cantilever {dims[0]}x{dims[1]}x{dims[2]} hex x 6 tets, "
                               f"Problem::solution to relres {args.rel_tol:g}",
                   "cells": C, "nodes": N, "dofs": ndof, "method": args.method, "parallelism": f"replicas x{world}",
                   "l2": "256 MB buffer written between timed steps"},
        "solve_s": max_ms / args.steps * 1e-3, "iterations": iters, "fp64_solve_s": st64["seconds"],
        "fp64_iterations": st64["iterations"], "compliance_rel_err_vs_fp64": abs(f_mixed - f_fp64) / abs(f_fp64),
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * C, "d2h_bytes_per_step": 8 * ndof,
                "max_rel_diff_u_vs_device_run": rel_u},
        "roofline": {"bound": "hbm", "kernel": "k_apply_tiled (fused CG: p update + K p + p.Kp)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": traffic, "algorithmic_bytes_per_launch": nbytes.value,
                     "ms_per_launch": ms_launch.value},
    }
    if world == 1 and not args.no_cpu_baseline:
        threads = host_cores()
        v, desc, extra = cpu_solve_estimate(dims, threads)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_kernel:
        return profile_kernel(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
