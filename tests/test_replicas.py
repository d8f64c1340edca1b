"""CPU test of the multi-GPU (replicas) host logic of bench.py with two gloo
ranks: each rank times its own SVDs, the job's time is the slowest rank's,
and the reported value counts every rank's SVDs."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    my_ms = [120.0, 95.5][rank]
    mx = bench.max_over_ranks(my_ms, dist, device="cpu")
    q.put((rank, mx, bench.whole_job_value(world, 3, mx)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, val in out:
        assert mx == 120.0
        assert val == pytest.approx(2 * 3 / 0.120)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(42.0, None) == 42.0
    assert bench.whole_job_value(1, 5, 1000.0) == pytest.approx(5.0)
