"""The multi-GPU path is independent replicas (one rank per GPU, no
collective in the step): bench.py's barrier and its max/sum of timings and
cell counts over ranks, exercised with two gloo ranks on the CPU."""
import datetime
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, REPO)
    import bench
    dev = torch.device("cpu")
    ms = bench.max_over_ranks(10.0 + rank, dist, dev)        # slowest rank's time
    cells = bench.sum_over_ranks(1000.0 * (rank + 1), dist, dev)  # all ranks' cells
    bench.barrier(dist, dev)
    queue.put((rank, ms, cells))
    dist.destroy_process_group()


def test_replica_timing_reductions_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results == [(0, 11.0, 3000.0), (1, 11.0, 3000.0)]
