"""Serving sharded by request (serve.serve_sharded): each process serves its share of the
stream with no collective on the data path, and the statistics are combined once. Two gloo
ranks on CPU with the stand-in engine of tests/serve_fakes.py (no GPU)."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from mhd_gpu_solver_b200.serve import make_stream, shard_requests


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from mhd_gpu_solver_b200.serve import make_stream, serve_sharded, shard_requests
    from tests.serve_fakes import FakeEngine

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    stream = make_stream(12, rate=2000.0, seed=4, side=(64, 512), t_end=(0.01, 0.05))
    stats = serve_sharded(stream, keep_states=True,
                          engine_factory=lambda st: FakeEngine(st, rounds=2 + rank))
    mine = {r.rid for r in shard_requests(stream, world)[rank]}
    q.put((rank, [c.rid for c in stats.completions], stats.makespan, sorted(stats.states),
           sorted(mine), stats.chunks))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_serve_their_shares():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    (_, rids0, make0, kept0, mine0, chunks0), (_, rids1, make1, kept1, mine1, chunks1) = out
    # every process sees every completion once, and the slowest process's makespan
    assert rids0 == rids1 == list(range(12))
    assert make0 == make1 > 0.0 and chunks0 == chunks1
    # states stay where they were computed; the shares are disjoint and cover the stream
    assert kept0 == mine0 and kept1 == mine1
    assert not set(mine0) & set(mine1) and sorted(mine0 + mine1) == list(range(12))


def test_shard_requests_balances_estimated_work():
    stream = make_stream(200, rate=100.0, seed=9, side=(128, 1024), t_end=(0.1, 0.5))
    for world in (1, 2, 3, 8):
        parts = shard_requests(stream, world)
        assert parts == shard_requests(stream, world)  # deterministic
        assert sorted(r.rid for p in parts for r in p) == list(range(200))
        loads = [sum(r.work_estimate() for r in p) for p in parts]
        biggest = max(r.work_estimate() for r in stream)
        assert max(loads) - min(loads) <= biggest * (1 + 1e-12)
        for p in parts:
            assert [r.arrival for r in p] == sorted(r.arrival for r in p)
    with pytest.raises(ValueError):
        shard_requests(stream, 0)
