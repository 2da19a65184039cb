"""The multi-rank path of bench.py on CPU: two gloo ranks (127.0.0.1) time
different amounts, the max over ranks is what every rank sees, and the
whole-job rate counts every rank's steps against that time."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t_local = 1.0 + rank          # rank 1 is the slow one
        dist.barrier()
        t_max = bench.reduce_max(dist, t_local, "cpu")
        out.put((rank, t_max, bench.aggregate_rate(world, 10, t_max)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [2.0, 2.0]          # both ranks see the slowest time
    assert [r[2] for r in res] == [10.0, 10.0]        # 2 ranks x 10 steps / 2 s
