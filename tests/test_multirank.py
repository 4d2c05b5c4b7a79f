"""Host-side logic of the multi-GPU bench (independent replicas, one per rank),
exercised with 2 gloo ranks on the CPU: the job is timed by the slowest rank
and the throughput is summed over ranks."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    local_ms = [10.0, 25.0][rank]
    ms = bench.max_over_ranks(local_ms)
    out[rank] = (ms, bench.replica_throughput(1000, 4, ms, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replica_aggregation():
    import torch.multiprocessing as mp

    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    for r in (0, 1):
        ms, v = out[r]
        assert ms == 25.0
        assert v == pytest.approx(1000 * 3 * 4 / 0.025 * 2)


def test_single_process_identity():
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_throughput(10, 2, 1000.0, 1) == pytest.approx(60.0)
