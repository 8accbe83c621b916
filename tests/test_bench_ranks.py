"""The multi-rank host logic of bench.py on CPU: two gloo ranks (one per
process, as torchrun starts them), each with its own device time, must both
report the slowest rank's time and the whole-job rate built from it."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = [12.5, 20.25][rank]
        slowest = bench.max_over_ranks(ms, dist, device="cpu")
        out[rank] = (slowest, bench.job_rate(world, 1000, 10, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def free_port() -> int:
    """A TCP port on 127.0.0.1 that nothing listens on (the OS picks it)."""
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_report_the_slowest_time_and_the_job_rate():
    port = free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        got = dict(out)
    assert got[0] == got[1]
    slowest, rate = got[0]
    assert slowest == 20.25
    assert rate == pytest.approx(2 * 1000 * 10 / 0.02025 / 1e6)


def test_without_a_group_the_local_time_stands():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_rate(1, 56_623_104, 300, 1000.0) == pytest.approx(16986.93, rel=1e-6)
