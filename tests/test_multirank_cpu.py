"""The benchmark's N > 1 host logic on CPU ranks (gloo, world size 2):
the max-over-ranks timing and the whole-job rate, the batched workload's
dealing of boxes to ranks, and the reference arm's rank != 0 early exit."""
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
        mine = bench.dealt_boxes(64, world, rank)
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
