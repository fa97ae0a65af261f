"""The host control flow of a slab solve spread over processes with a captured body of k
iterations (voxel_b200.slab.replay_until_done), on CPU: two gloo ranks whose bodies all-reduce
their slabs' residual sums, as the NCCL body does, decide identically when to stop -- converged,
or capped so that no body passes maxiter -- and so issue the same collectives."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, k, maxiter, rate, q):
    import datetime
    import torch.distributed as dist
    from voxel_b200.slab import replay_until_done
    from voxel_b200.solver import S_BREAK, S_DONE, S_IT, S_REL, S_TOL
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        S = torch.zeros(16, dtype=torch.float64)
        S[S_TOL] = 1e-8
        local = torch.tensor([1.0 + rank], dtype=torch.float64)     # this slab's share of |r|^2
        collectives = 0

        def replay():                      # k iterations; each shrinks the residual and all-reduces
            nonlocal collectives
            for _ in range(k):
                local.mul_(rate ** 2)
                tot = local.clone()
                dist.all_reduce(tot)
                collectives += 1
                S[S_IT] += 1
            S[S_REL] = float(tot.sqrt()) / np.sqrt(3.0)              # relative to the initial |r|
            S[S_DONE] = float(S[S_REL] <= S[S_TOL])

        s, bodies = replay_until_done(replay, lambda: S.numpy().copy(), k, maxiter, 0)
        q.put((rank, int(s[S_IT]), bool(s[S_DONE]), bool(s[S_BREAK]), bodies, collectives))
    finally:
        dist.destroy_process_group()


def _run(k, maxiter, rate):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, k, maxiter, rate, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    return sorted(q.get(timeout=10) for _ in range(world))


@pytest.mark.parametrize("k", [1, 5])
def test_ranks_stop_together_when_converged(k):
    got = _run(k, maxiter=200, rate=0.5)              # |r| halves per iteration: 1e-8 after 27
    assert got[0][1:] == got[1][1:]
    it, done, broke, bodies, coll = got[0][1:]
    assert done and not broke
    assert it == k * bodies and it >= 27 and it - k < 27
    assert coll == it


def test_no_body_passes_maxiter():
    got = _run(5, maxiter=23, rate=0.9)               # far from converged: stops at 20, 3 left for the tail
    assert got[0][1:] == got[1][1:]
    it, done, _, bodies, _ = got[0][1:]
    assert not done and it == 20 and bodies == 4
