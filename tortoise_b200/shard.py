"""One run's tuples split over several processes (one GPU each).

The library does the work (tb_shard_* in include/tortoise_b200.h): a handle
created with ``shard=(rank, count)`` keeps its part of every tuple list and,
once connected, ends every collision evaluation with one NCCL all-reduce of
the collision accumulator, so that every rank holds the full operator and
the replicated integrator takes the same steps everywhere.  This module only
passes the communicator id from one rank to the others through an existing
torch.distributed process group (gloo or NCCL):

    dist.init_process_group("nccl", ...)
    eng = Engine(material, shard=(dist.get_rank(), dist.get_world_size()),
                 device=local_rank)
    shard.connect(eng)                  # collective over the group
    res = eng.dp45(f0, 0.0, t1, dense)  # the same result on every rank

It is the multi-GPU form of the TBB tuple reduce inside
ScatteringChannel<2,L>::propagate (src/Physics/Scattering/
ScatteringChannel.cpp:651-670).
"""
import torch.distributed as dist

from . import engine as E


def exchange_id(group=None, src=0, make_id=None):
    """The communicator id made on rank ``src`` of ``group``, on every rank."""
    make_id = make_id or E.shard_unique_id
    me = dist.get_rank(group)
    obj = [make_id() if me == src else None]
    dist.broadcast_object_list(obj, src=dist.get_global_rank(group, src) if group is not None else src, group=group)
    uid = obj[0]
    if not isinstance(uid, (bytes, bytearray)) or len(uid) != E.SHARD_ID_BYTES:
        raise RuntimeError("shard id exchange returned %r" % (type(uid),))
    return bytes(uid)


def connect(engine, timeout_s=60.0, group=None):
    """Connects ``engine`` (created with shard=(rank, count)) to the other
    ranks of ``group``; every rank calls it."""
    engine.shard_connect(exchange_id(group), timeout_s)
    return engine


__all__ = ["connect", "exchange_id"]
