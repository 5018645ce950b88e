"""The N > 1 path of bench.py (replicas only: one independent system per
rank, a barrier, and the MAX over ranks of the time) with two gloo ranks on
the CPU."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ranks = bench.Ranks(dist, None)
    ranks.barrier()
    local_seconds = 1.0 + rank  # rank 1 is the slowest
    mx = ranks.max(local_seconds)
    value = ranks.whole_job(1000.0, local_seconds)
    out.put((rank, mx, value, ranks.world))
    ranks.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, value, world in res:
        assert world == 2
        assert mx == 2.0
        assert value == pytest.approx(2 * 1000.0 / 2.0)
