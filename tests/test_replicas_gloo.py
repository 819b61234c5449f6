"""The multi-GPU path of bench.py is replicas only: every rank runs the same workload and the
whole-job value is all ranks' units over the slowest rank's device time. This checks that
aggregation with two gloo ranks on CPU (no GPU, no data-path collective)."""

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

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    ms_local = 10.0 * (rank + 1)          # rank 1 is the slowest
    ms_max = bench.max_over_ranks(ms_local, dist)
    value = bench.replicas_value(1.0e9, ms_max, world)
    q.put((rank, ms_max, value))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_aggregate_replicas():
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
    for rank, ms_max, value in out:
        assert ms_max == 20.0
        assert abs(value - 2 * 1.0e9 / 0.020) < 1e-3 * value


def test_single_process_aggregation():
    import bench

    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.replicas_value(100.0, 1000.0, 1) == 100.0


def test_each_rank_sees_only_its_own_gpu():
    import bench

    assert bench.rank_device(1, 0, None) == (0, None, 0)
    assert bench.rank_device(4, 2, None) == (2, "2", 0)
    assert bench.rank_device(2, 1, "4,5") == (5, "5", 0)
