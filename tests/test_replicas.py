"""Multi-rank host logic on CPU: two gloo ranks reduce the bench timings
(slowest rank) and shard a batch of RVEs without overlap or loss."""
import os
import socket

import pytest

from pigfem_assignment_b200.replicas import max_over_ranks, shard_rves, sum_over_ranks

torch = pytest.importorskip("torch")


def test_shards_cover_every_rve_once_and_balance():
    weights = [((k * 7919) % 97 + 1) * 1000 for k in range(512)]
    for world in (1, 2, 3, 8):
        shards = shard_rves(weights, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(weights)))
        loads = [sum(weights[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(weights)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t_max = max_over_ranks(0.5 + rank)
        total = sum_over_ranks(100 * (rank + 1))
        shards = shard_rves([5, 9, 2, 7, 7, 1, 3], world)
        out[rank] = (t_max, total, shards[rank])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_timings_and_share_rves():
    ctx = torch.multiprocessing.get_context("spawn")
    world = 2
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()  # both ranks rendezvous on it
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 1.5          # the slowest rank's time
    assert res[0][1] == res[1][1] == 300.0        # totals summed
    assert sorted(res[0][2] + res[1][2]) == list(range(7))
    assert not set(res[0][2]) & set(res[1][2])
