"""The N > 1 host logic on CPU ranks (gloo, world size 2 and 3): the
benchmark's max-over-ranks timing and whole-job rate, the batched workload's
dealing of boxes to ranks by work, the reference arm's rank != 0 early exit,
and one box cut into slabs along x: the interface exchange of the
distributed K x reproduces the single-process operator, and the distributed
Jacobi-PCG (all-reduced dot products) the single-process solution."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mx = bench.max_over_ranks(10.0 * (rank + 1), world, device="cpu")
        rate = bench.whole_job_rate(world, 1000, 2, mx)
        # batched workload: the boxes dealt to the ranks cover every box once
        from platoanalyze_b200.workloads import batch_specs
        specs, _ = batch_specs(64, 1234)
        mine = bench.dealt_boxes(specs, world, rank)
        every = [None] * world
        dist.all_gather_object(every, mine)
        out.put((rank, mx, rate, sorted(b for lst in every for b in lst)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, mx, rate, boxes in res:
        assert mx == 20.0
        assert rate == pytest.approx(2 * 1000 * 2 / 0.020)
        assert boxes == list(range(64))


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")

    class Args:
        dims, warmup, steps, gpus, rel_tol = "4x2x2", 1, 1, 2, 1e-8

    called = []
    monkeypatch.setattr(bench, "CpuCantilever", lambda *a, **k: called.append(1))
    assert bench.run_reference(Args()) == 0
    assert not called


def test_deal_boxes_balances_work():
    from platoanalyze_b200.partition import box_work, deal_boxes
    from platoanalyze_b200.workloads import batch_specs
    specs, _ = batch_specs(64, 1234)
    w = [box_work(sp) for sp in specs]
    for world in (1, 2, 3, 4, 8):
        dealt = deal_boxes(specs, world)
        assert sorted(i for m in dealt for i in m) == list(range(64))
        loads = [sum(w[i] for i in m) for m in dealt]
        lower = max(sum(w) / world, max(w))
        assert max(loads) <= 4.0 / 3.0 * lower
        assert max(loads) <= sum(w) / world + max(w)
        assert deal_boxes(specs, world) == dealt  # deterministic
    # round-robin would leave one of two ranks far heavier on this batch
    rr = [sum(w[i] for i in range(r, 64, 2)) for r in range(2)]
    lpt = [sum(w[i] for i in m) for m in deal_boxes(specs, 2)]
    assert max(lpt) / min(lpt) <= max(rr) / min(rr)


def _slab_main(rank, world, port, dims, out):
    import sys
    import numpy as np
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from oracle import cpu
    from platoanalyze_b200.fields import box_arrays, clamp_dofs
    from platoanalyze_b200.partition import Slabs, SlabOperator, slab_pcg
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nx, ny, nz = dims
        rng = np.random.default_rng(5)
        zg = rng.uniform(0.05, 1.0, 6 * nx * ny * nz)   # per tet, global cell 6 h + t
        xg = rng.standard_normal(3 * (nx + 1) * (ny + 1) * (nz + 1))
        s = Slabs(dims, world, rank)
        cells, coords, _, _ = box_arrays(s.b - s.a, ny, nz)
        coords[:, 0] += s.a
        hexes = s.local_hexes()
        zl = zg.reshape(-1, 6)[hexes].ravel()
        O = cpu.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
        local_apply = lambda x: torch.from_numpy(O.apply(x.numpy(), zl))
        op = SlabOperator(s, local_apply, dist, torch)
        y = op(torch.from_numpy(s.scatter(xg)))
        # the assembled diagonal: the local diagonal, exchanged like K x
        e = np.zeros(3 * s.n_local)
        diag = np.empty(3 * s.n_local)
        for q in range(3 * s.n_local):  # small slabs: unit vectors
            e[q] = 1.0
            diag[q] = O.apply(e, zl)[q]
            e[q] = 0.0
        diag = op.exchange(torch.from_numpy(diag))
        # cantilever: x = 0 clamped, unit traction -z on x = nx (nodal loads from the oracle residual)
        cg, xcg, fg, clg = box_arrays(nx, ny, nz)
        Og = cpu.Oracle(cg, xcg, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
        F = -Og.residual(np.zeros(xg.size), zg, fg, (0.0, 0.0, -1.0 / (ny * nz)))
        dofs = clamp_dofs(clg)
        free_g = np.ones(xg.size)
        free_g[dofs] = 0.0
        free = torch.from_numpy(s.scatter(free_g))
        b = torch.from_numpy(s.scatter(F * free_g))
        u, its, rel = slab_pcg(s, op, diag, b, free, dist, torch, rel_tol=1e-10)
        out.put((rank, s.global_node, y.numpy(), u.numpy(), its, rel))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_decomposition_matches_single_process(oracle_lib, world):
    """A 9x3x2 box in 2 or 3 slabs along x: the exchanged slab K x equals the
    single-process oracle K x to FP64 rounding on every local node, and the
    distributed Jacobi-PCG solve equals the single-process one."""
    import numpy as np
    from platoanalyze_b200.fields import box_arrays, clamp_dofs
    dims = (9, 3, 2)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_main, args=(r, world, port, dims, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    nx, ny, nz = dims
    rng = np.random.default_rng(5)
    zg = rng.uniform(0.05, 1.0, 6 * nx * ny * nz)
    xg = rng.standard_normal(3 * (nx + 1) * (ny + 1) * (nz + 1))
    cells, coords, faces, clamp = box_arrays(nx, ny, nz)
    O = oracle_lib.Oracle(cells, coords, E=1.0, nu=0.3, p=3.0, pmin=1e-9, layout=1)
    y_ref = O.apply(xg, zg).reshape(-1, 3)
    F = -O.residual(np.zeros(xg.size), zg, faces, (0.0, 0.0, -1.0 / (ny * nz)))
    dofs = clamp_dofs(clamp)
    u_ref, _, _ = O.solve(zg, F, dofs, rel_tol=1e-12)
    u_ref = u_ref.reshape(-1, 3)
    scale = np.abs(y_ref).max()
    covered = np.zeros(coords.shape[0], bool)
    for rank, gnode, y, u, its, rel in res:
        assert np.abs(y.reshape(-1, 3) - y_ref[gnode]).max() <= 1e-13 * scale
        assert rel <= 1e-10 and its > 0
        assert np.abs(u.reshape(-1, 3) - u_ref[gnode]).max() <= 1e-8 * np.abs(u_ref).max()
        covered[gnode] = True
    assert covered.all()
