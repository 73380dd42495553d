"""The N > 1 path of bench.py on CPU: replicas run the hot path independently
and the job's step time is the slowest rank's (max over ranks, every rank
taking the same collective steps).  Two gloo ranks as spawned processes on
127.0.0.1."""
import datetime
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    times = [bench.max_over_ranks(10.0 * (rank + 1) + step, dist, device="cpu")
             for step in range(3)]
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, times))


def test_single_process_time_is_its_own():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25) == 3.25


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert out[0] == out[1] == [20.0, 21.0, 22.0]
