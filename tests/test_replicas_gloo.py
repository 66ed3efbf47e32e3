"""The multi-GPU path is replicas only (one independent render job per GPU): bench.py's
host-side rank logic, run as two gloo ranks on the CPU. A step's device time is the max
over the ranks, and the whole-job rate counts every rank's samples over that time."""
import os
import socket
import sys
from datetime import timedelta

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TIMES = [12.5, 17.25]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    ms = bench.max_over_ranks(TIMES[rank], dist, torch.device("cpu"))
    rate = bench.job_rate(world, 1000, 5, ms)
    q.put((rank, ms, rate))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_time_is_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate in results:
        assert ms == max(TIMES)
        assert rate == 2 * 1000 * 5 / (max(TIMES) / 1e3)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, None) == 3.5
    assert bench.job_rate(1, 100, 2, 1000.0) == 200.0
