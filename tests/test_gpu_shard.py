"""Tuple sharding on one GPU.

* The parts of R sharded handles (unconnected, so each returns its partial
  collision sum) add up to the full collision operator and the full
  scattering rates, and their tuple lists concatenate to the full list.
* A handle connected to a one-rank communicator runs the NCCL all-reduce in
  every collision evaluation -- inside the captured DP45 attempt graph and
  the adjoint sweeps too -- and gives the unsharded handle's results.
* A rank whose peer never joins gets TB_ERR_TIMEOUT from tb_shard_connect
  within its deadline (no kernel involved), and the handle refuses collision
  work afterwards.

Ranks that wait on one another are never run as several processes on one
GPU; the two-rank host logic runs on gloo in tests/test_dist_cpu.py."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT, rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W
from tests.golden.make_golden import cases

pytestmark = pytest.mark.gpu

CASES = list(cases().keys())


def _setup(name):
    build, seed, kT = cases()[name]
    mat = build()
    return mat, W.initial_status(mat, kT=kT, seed=seed).vec


@pytest.mark.parametrize("n_ranks", [2, 3])
@pytest.mark.parametrize("layout", [E.LAYOUT_MC64, E.LAYOUT_T64, E.LAYOUT_T40])
@pytest.mark.parametrize("name", CASES)
def test_parts_sum_to_the_full_operator(gpu_lib, name, layout, n_ranks, tmp_path):
    mat, f0 = _setup(name)
    full = E.Engine(mat, layout=layout)
    parts = [E.Engine(mat, layout=layout, shard=(r, n_ranks)) for r in range(n_ranks)]
    try:
        d = full.rhs(f0, drift=False)
        s = sum(p.rhs(f0, drift=False) for p in parts)
        assert rel_l2(s, d) < 1e-12
        rates = full.scattering_rates(f0)
        assert rel_l2(sum(p.scattering_rates(f0) for p in parts), rates) < 1e-12
        for ch in range(len(mat.channels)):
            ids, umk = full.tuples(ch)
            got = [p.tuples(ch) for p in parts]
            assert np.array_equal(np.concatenate([g[0] for g in got]), ids)
            assert np.array_equal(np.concatenate([g[1] for g in got]), umk)
            for r, p in enumerate(parts):
                b, n = p.shard_info(ch)
                assert n == len(umk) and b == E.shard_range(n, r, n_ranks)[0]
        with pytest.raises(E.TortoiseError):
            parts[0].write_scatt_indices(0, str(tmp_path / "x.scattIndices"))
    finally:
        for e in parts + [full]:
            e.close()


def test_one_rank_communicator_matches_the_unsharded_handle(gpu_lib):
    """Both handles in the deterministic mode: the one-rank all-reduce is an
    identity on the exactly accumulated sums, so every result is equal bit
    for bit -- operator, rates, a whole DP45 integration and the adjoint."""
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=True, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
    f0 = W.initial_status(mat, seed=5).vec
    ref = E.Engine(mat, deterministic=True)
    eng = E.Engine(mat, shard=(0, 1), deterministic=True)
    try:
        eng.shard_connect(E.shard_unique_id(), 60.0)
        assert np.array_equal(eng.rhs(f0), ref.rhs(f0))
        assert np.array_equal(eng.scattering_rates(f0), ref.scattering_rates(f0))
        a, b = eng.dp45(f0, 0.0, 0.2, 0.1, max_dense=4), ref.dp45(f0, 0.0, 0.2, 0.1, max_dense=4)
        assert a["attempts"] == b["attempts"] and a["accepted"] == b["accepted"]
        assert np.array_equal(a["y"], b["y"]) and np.array_equal(a["dense"], b["dense"])
        from tortoise_b200 import adjoint as A
        w = A.observable_weights(mat, 1, "energy")
        ga = A.gradient(eng, f0, [c.amplitude for c in mat.channels], w, 0.0, 0.1, 0.05, checkpoint_every=2)
        gb = A.gradient(ref, f0, [c.amplitude for c in mat.channels], w, 0.0, 0.1, 0.05, checkpoint_every=2)
        assert ga[0] == gb[0]
        assert np.array_equal(ga[1], gb[1]) and np.array_equal(ga[2], gb[2])
    finally:
        eng.close()
        ref.close()


_NO_PEER = textwrap.dedent("""
    import sys, time
    sys.path.insert(0, %r)
    from tortoise_b200 import engine as E
    from tortoise_b200 import workloads as W
    mat = W.build_material(4, ("P",), (), ee=True, eph=False, field=(0.0, 0.0), rtol=1e-6, atol=1e-9)
    f0 = W.initial_status(mat, seed=1).vec
    eng = E.Engine(mat, shard=(0, 2))
    t0 = time.time()
    try:
        eng.shard_connect(E.shard_unique_id(), 3.0)
        sys.exit("connected without a peer")
    except E.TortoiseError as e:
        assert e.rc == 6, e
    waited = time.time() - t0
    assert waited < 30, waited
    try:
        eng.rhs(f0)
        sys.exit("collision work ran on an aborted communicator")
    except E.TortoiseError:
        pass
    eng.close()
    print("ok %%.1f" %% waited)
""") % ROOT


def test_connect_without_a_peer_times_out(gpu_lib):
    r = subprocess.run([sys.executable, "-c", _NO_PEER], capture_output=True, text=True, timeout=120,
                       env=dict(os.environ, NCCL_NVLS_ENABLE="0"))
    lines = r.stdout.strip().splitlines()
    assert r.returncode == 0 and lines and lines[-1].startswith("ok"), (r.stdout[-2000:], r.stderr[-2000:])
