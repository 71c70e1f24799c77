"""The multi-GPU path of bench.py is replicas only: every rank advances its own case and the job
is timed by its slowest rank.  This runs that host-side aggregation with two gloo ranks on CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # rank r's replica took (r + 1) * 100 ms of device time and 2 * that end to end
    ms = bench.max_over_ranks(dist, [100.0 * (rank + 1), 200.0 * (rank + 1)])
    rate = bench.whole_job_rate(world, 1_000_000, 2, ms[0])
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, rate))


def test_slowest_replica_times_the_job():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate in out:
        assert ms == [200.0, 400.0]
        assert rate == pytest.approx(2 * 1_000_000 * 2 / 0.2 / 1e6)
