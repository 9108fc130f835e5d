"""Replica aggregation of bench.py under torch.distributed (gloo, world size 2, CPU): each rank
reports its own device time; the job's time is the slowest rank's and the throughput counts every
rank's determinants."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [120.0, 150.0][rank]
    ms_max, value = bench.replica_throughput(dist, ms, 3_000_000_000, world)
    q.put((rank, ms_max, value))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_throughput_gloo_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, ms_max, value in out:
        assert ms_max == pytest.approx(150.0)  # the slowest replica
        assert value == pytest.approx(2 * 3.0 / 0.150)  # both ranks' determinants, GDets/s


def test_replica_throughput_single():
    sys.path.insert(0, ROOT)
    import bench
    ms_max, value = bench.replica_throughput(None, 200.0, 4_000_000_000, 1)
    assert ms_max == 200.0 and value == pytest.approx(20.0)
