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


def _shard_rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from tortoise_b200 import engine as E
    from tortoise_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        uid = shard.exchange_id()                      # made on rank 0, NCCL's own id format
        ranges = {n: E.shard_range(n, rank, world) for n in (0, 1, 127, 128, 129, 9_800_000, 3 * 2**31 + 5)}
        gathered = [None] * world
        dist.all_gather_object(gathered, (uid, ranges))
        out.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_one_id_and_split_every_tuple_list():
    """Host side of tuple sharding over two gloo ranks: both receive the
    same communicator id, and their tuple ranges are disjoint, in order,
    cover the whole list and start on 128-tuple tile boundaries."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    g = res[0]
    assert res[1] == g
    assert g[0][0] == g[1][0] and len(g[0][0]) == 128
    for n in g[0][1]:
        (b0, e0), (b1, e1) = g[0][1][n], g[1][1][n]
        assert (b0, e0, e1) == (0, b1, n), (n, g[0][1][n], g[1][1][n])
        assert b1 % 128 == 0 or b1 == n
        assert abs((e0 - b0) - (e1 - b1)) <= 128
