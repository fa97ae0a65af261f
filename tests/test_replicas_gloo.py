"""The N > 1 path of bench.py on CPU: world_size-2 gloo ranks run the same rendezvous and
max-over-ranks timing as the GPU replicas (one process per GPU over NCCL), with no device."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t_local = 0.25 + 0.5 * rank                  # rank 1 is the slow replica
        t_max = bench.max_over_ranks(t_local, world, "cpu")
        dist.barrier()
        q.put((rank, t_max, bench.whole_job_time_per_solve(t_max, world)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_max_over_ranks_with_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert [g[1] for g in got] == [0.75, 0.75]            # every rank sees the slowest rank's time
    assert [g[2] for g in got] == [0.375, 0.375]          # 2 solves in 0.75 s


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(0.5, 1, "cpu") == 0.5
    assert bench.whole_job_time_per_solve(0.5, 1) == 0.5
