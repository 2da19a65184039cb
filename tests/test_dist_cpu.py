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


def _sharded_sum_rank(rank, world, port, out):
    """One gloo rank of a tuple-sharded run on the oracle: its part of every
    channel's tuple list (tb_shard_range), the partial operators all-reduced,
    and a replicated DP45 on the all-reduced right-hand side driven by the
    reference's own integrator (oracle/_ref)."""
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        mat = W.build_material(4, ("P", "D"), (0.2,), ee=True, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
        f0 = W.initial_status(mat, seed=5).vec
        o = oracle.Oracle(mat, nthreads=1)
        parts = [E.shard_range(o.num_tuples(ch), rank, world) for ch in range(len(mat.channels))]
        offs = [o.band_offset(b) for b in range(len(mat.bands))] + [o.ndofs]

        def rhs(y, drift=True):
            acc = np.zeros(o.ndofs)
            for ch, (b, e) in enumerate(parts):          # ScatteringChannel::propagate over this rank's tuples
                o.channel_propagate(ch, y, b, e, inverse_mass=True, out=acc)
            if drift and rank == 0:                      # the replicated drift term, added once
                for b in range(len(mat.bands)):
                    acc[offs[b]:offs[b + 1]] += o.vlasov(b, y[offs[b]:offs[b + 1]])
            t = torch.from_numpy(acc)
            dist.all_reduce(t)
            return t.numpy().copy()

        full = o.rhs(f0, drift=False)
        got = rhs(f0, drift=False)
        err_sum = float(np.linalg.norm(got - full) / np.linalg.norm(full))
        res = {"sum_rel_l2": err_sum, "n_tuples": [o.num_tuples(c) for c in range(len(mat.channels))],
               "parts": parts}
        ref_so = os.path.join(ROOT, "oracle", "_ref", "libref_dp54.so")
        if os.path.exists(ref_so):
            from test_oracle_ref_dp54 import reference_dp54
            r = reference_dp54(o, f0, 0.0, 0.3, 0.1, rhs_fn=rhs)
            res["dp"] = {k: r[k] for k in ("attempts", "accepted", "rejected", "rhs_evals", "n_dense")}
            res["dense"] = r["dense"].tobytes()
            if rank == 0:
                u = o.dp45(f0, 0.0, 0.3, 0.1, max_dense=64)
                res["unsharded"] = {k: u[k] for k in ("attempts", "accepted", "rejected", "rhs_evals", "n_dense")}
                res["unsharded_dense_rel"] = float(np.linalg.norm(u["dense"] - r["dense"]) / np.linalg.norm(u["dense"]))
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_ranks_partial_operators_sum_to_the_full_one_and_step_alike():
    """The data plane of tuple sharding on two gloo ranks, with the oracle as
    each rank's collision operator: every channel's tuple list split by
    tb_shard_range, the per-rank partial operators summed by an all-reduce
    (the reduce of ScatteringChannel.cpp:651-670 across processes) equal the
    full operator; and a DP45 run replicated on both ranks over the
    all-reduced right-hand side takes the same accept / reject decisions and
    the same dense outputs on both ranks, and those of the unsharded run."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_sum_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    r0, r1 = res[0], res[1]
    assert r0["sum_rel_l2"] < 1e-13 and r1["sum_rel_l2"] == r0["sum_rel_l2"]
    for n, (a, b) in zip(r0["n_tuples"], zip(r0["parts"], r1["parts"])):
        assert a[0] == 0 and a[1] == b[0] and b[1] == n
    assert sum(1 for a in r0["parts"] if a[1] > 0) >= 2   # both ranks hold work in several channels
    assert sum(1 for b in r1["parts"] if b[1] > b[0]) >= 2
    if "dp" in r0:
        assert r0["dp"] == r1["dp"] and r0["dense"] == r1["dense"]   # replicated controller: identical
        assert r0["dp"] == r0["unsharded"]
        assert r0["unsharded_dense_rel"] < 1e-10


def _item_sharded_rank(rank, world, port, out):
    """One gloo rank of a run whose four-leg channels are streamed and
    sharded by work item (the split of tb_shard_range over the items of
    the walk, not over stored tuples): the oracle enumerates and integrates
    exactly this rank's items, the partial operators are all-reduced."""
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import oracle
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        mat = W.build_material(4, ("P", "D"), (0.2,), ee=True, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
        f0 = W.initial_status(mat, seed=5).vec
        pk = mat.pack()
        part = oracle.Oracle(mat, enumerate_tuples=False, nthreads=1)
        acc = np.zeros(part.ndofs)
        res = {"items": [], "tuples": []}
        for ch, c in enumerate(mat.channels):
            if c.nlegs != 4:
                continue
            cd = pk.desc.channels[ch]
            n = cd.n_umklapp * 2 ** (cd.nlegs - 1)
            for l in range(cd.nlegs - 1):
                m = pk.desc.meshes[pk.desc.bands[cd.band[l]].mesh]
                n *= m.nsplit[0] * m.nsplit[1]
            b, e = E.shard_range(n, rank, world)
            part.enumerate_items(ch, b, e)
            part.channel_propagate(ch, f0, out=acc)
            res["items"].append((n, b, e))
            res["tuples"].append(part.num_tuples(ch))
        t = torch.from_numpy(acc)
        dist.all_reduce(t)
        full = oracle.Oracle(mat, nthreads=1)
        ref = np.zeros(full.ndofs)
        for ch, c in enumerate(mat.channels):
            if c.nlegs == 4:
                full.channel_propagate(ch, f0, out=ref)
        res["full_tuples"] = [full.num_tuples(ch) for ch, c in enumerate(mat.channels) if c.nlegs == 4]
        res["rel"] = float(np.linalg.norm(t.numpy() - ref) / np.linalg.norm(ref))
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_the_streamed_work_items():
    """Streamed four-leg channels sharded over two gloo ranks: the work items
    of the walk split by tb_shard_range hold every tuple of the full
    enumeration exactly once (the per-rank tuple counts add up), and the
    all-reduced partial operators equal the full one."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_item_sharded_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    r0, r1 = res[0], res[1]
    assert r0["items"] and len(r0["items"]) == len(r1["items"])
    for (n, b0, e0), (m, b1, e1) in zip(r0["items"], r1["items"]):
        assert n == m and b0 == 0 and e0 == b1 and e1 == n
    assert [a + b for a, b in zip(r0["tuples"], r1["tuples"])] == r0["full_tuples"]
    assert all(a > 0 for a in r0["tuples"]) and all(b > 0 for b in r1["tuples"])
    assert r0["rel"] < 1e-13 and r1["rel"] == r0["rel"]
