"""The N-GPU bench runs independent replicas; its only collectives are a
barrier and the max over ranks of the step time.  Checked here with two gloo
ranks on the CPU: every rank sees the slowest rank's time and the whole-job
throughput counts every replica's bytes."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        local_ms = 2.0 + 1.5 * rank  # rank 1 is the slow one
        step = bench.max_over_ranks(local_ms, world, "cpu")
        e2e = bench.max_over_ranks(10.0 - rank, world, "cpu")
        dist.barrier()
        out.put((rank, step, e2e, bench.job_gbs(1_000_000_000, world, step)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_job_throughput():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, step, e2e, gbs in res:
        assert step == 3.5 and e2e == 10.0
        assert abs(gbs - 2 * 1e9 / 3.5e-3 / 1e9) < 1e-9


def test_single_rank_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(1.25, 1, "cpu") == 1.25
    assert abs(bench.job_gbs(6_538_000_000, 1, 1.0) - 6538.0) < 1e-9
