"""Streamed channels (tb_options.stream_legs, TB_LAYOUT_STREAM): no stored
tuple list, the candidates of precalculateIndices walked again in every
evaluation and integrated on the spot.

* In the deterministic mode the streamed operator, scattering rates and a
  whole DP45 integration equal the stored-list Monte-Carlo path (points
  inside the simplices) bit for bit: the same tuples, the same per-tuple sums,
  exact accumulation.
* The counts of the walk equal the stored enumeration's (prefilter,
  determinant, survivors, points inside).
* Sharded streamed handles (work items split over ranks) sum to the full
  operator.
* On a 32x32 four-leg e-e channel, far too large to store, a slice of the
  work items agrees with the oracle's enumeration and quadrature of the same
  items (1e-12) and has the same tuple count.
* The streamed VJP and a whole adjoint sweep equal the stored list's.
* A streamed channel refuses what needs a list (tuples, the .scattIndices
  cache, functAmplitude)."""
import numpy as np
import pytest

import oracle
from conftest import golden, rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W
from tests.golden.make_golden import cases

pytestmark = pytest.mark.gpu

CASES = list(cases().keys())


def _setup(name):
    build, seed, kT = cases()[name]
    mat = build()
    return mat, W.initial_status(mat, kT=kT, seed=seed).vec


def _n_items(mat, ch):
    pk = mat.pack()
    cd = pk.desc.channels[ch]
    n = cd.n_umklapp * 2 ** (cd.nlegs - 1)
    for l in range(cd.nlegs - 1):
        m = pk.desc.meshes[pk.desc.bands[cd.band[l]].mesh]
        n *= m.nsplit[0] * m.nsplit[1]
    return n


@pytest.mark.parametrize("name", CASES)
def test_streamed_equals_stored_list_bit_for_bit(gpu_lib, name):
    mat, f0 = _setup(name)
    stored = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True)
    streamed = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True, stream_legs=2)
    try:
        a, b = stored.rhs(f0), streamed.rhs(f0)
        assert np.array_equal(a, b)
        assert rel_l2(b, golden(name)["rhs"]) < 1e-12
        for ch in range(len(mat.channels)):
            si, ti = stored.channel_info(ch), streamed.channel_info(ch)
            assert ti["layout"] == "stream"
            assert [ti["n_tuples"], ti["n_prefilter"], ti["n_det"]] == [si["n_tuples"], si["n_prefilter"], si["n_det"]]
            if si["n_tuples"] > 0:   # an empty stored channel builds no list of inside points
                assert streamed.points_inside(ch) == stored.points_inside(ch)
            assert streamed.schedule(ch).get("streamed")
        assert np.array_equal(stored.scattering_rates(f0), streamed.scattering_rates(f0))
        for ch in range(len(mat.channels)):
            assert np.array_equal(stored.channel_propagate(ch, f0), streamed.channel_propagate(ch, f0))
    finally:
        stored.close()
        streamed.close()


@pytest.mark.parametrize("name", ["ee_n3", "eph_n4"])
def test_streamed_integration_equals_stored(gpu_lib, name):
    mat, f0 = _setup(name)
    stored = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True)
    streamed = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True, stream_legs=2)
    try:
        a, b = stored.dp45(f0, 0.0, 0.4, 0.1), streamed.dp45(f0, 0.0, 0.4, 0.1)
        assert b["status"] == 0
        assert [a[k] for k in ("attempts", "accepted", "rejected")] == [b[k] for k in ("attempts", "accepted", "rejected")]
        assert np.array_equal(a["dense"], b["dense"]) and np.array_equal(a["y"], b["y"])
    finally:
        stored.close()
        streamed.close()


def test_streamed_plain_mode_and_mixed_handles(gpu_lib):
    """FP64 atomics (not deterministic): within the summation noise of the
    stored path; only the four-leg channel streamed beside a moment-tensor
    e-ph channel."""
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=True, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
    f0 = W.initial_status(mat, seed=3).vec
    ref = oracle.Oracle(mat).rhs(f0)
    e = E.Engine(mat, stream_legs=4)
    try:
        layouts = [e.channel_info(ch)["layout"] for ch in range(len(mat.channels))]
        assert "stream" in layouts and any(x.startswith("t") for x in layouts)
        assert all((x == "stream") == (c.nlegs == 4) for x, c in zip(layouts, mat.channels))
        assert rel_l2(e.rhs(f0), ref) < 1e-12
        r = e.dp45(f0, 0.0, 0.05, 0.05)
        assert r["status"] == 0
    finally:
        e.close()


@pytest.mark.parametrize("n_ranks", [2, 5])
def test_streamed_parts_sum_to_the_full_operator(gpu_lib, n_ranks):
    mat, f0 = _setup("ee_n4")
    full = E.Engine(mat, stream_legs=2, deterministic=True)
    parts = [E.Engine(mat, stream_legs=2, deterministic=True, shard=(r, n_ranks)) for r in range(n_ranks)]
    try:
        d = full.rhs(f0, drift=False)
        s = sum(p.rhs(f0, drift=False) for p in parts)
        assert rel_l2(s, d) < 1e-14
        n = sum(p.channel_info(0)["n_tuples"] for p in parts)
        assert n == full.channel_info(0)["n_tuples"]
        for r, p in enumerate(parts):
            b, total = p.shard_info(0)
            assert total == _n_items(mat, 0) and b == E.shard_range(total, r, n_ranks)[0]
    finally:
        for e in parts + [full]:
            e.close()


def test_streamed_slice_of_a_32x32_ee_channel_matches_the_oracle(gpu_lib):
    """32x32 one-band e-e: about 2e9 surviving tuples, never stored.  Rank
    3000 of 8192 item slices (about a million work items around the middle of
    the leg-0 sections) against the oracle's own enumeration and quadrature of
    exactly those items."""
    mat = W.parabolic_ee(32)
    f0 = W.initial_status(mat, kT=0.1, seed=0).vec
    R, r = 8192, 3000
    e = E.Engine(mat, stream_legs=2, deterministic=True, shard=(r, R))
    try:
        b, total = e.shard_info(0)
        assert total == _n_items(mat, 0)
        end = E.shard_range(total, r, R)[1]
        got = e.rhs(f0, drift=False)
        info = e.channel_info(0)
    finally:
        e.close()
    o = oracle.Oracle(mat, enumerate_tuples=False)
    o.enumerate_items(0, b, end)
    assert o.num_tuples(0) == info["n_tuples"] > 10000
    assert list(o.enum_counts(0)) == [info["n_prefilter"], info["n_det"]]
    ref = o.channel_propagate(0, f0)
    assert rel_l2(got, ref) < 1e-12


def test_streamed_channel_refuses_what_needs_a_list(gpu_lib, tmp_path):
    mat, f0 = _setup("ee_n3")
    e = E.Engine(mat, stream_legs=2)
    try:
        with pytest.raises(E.TortoiseError):
            e.tuples(0)
        with pytest.raises(E.TortoiseError):
            e.write_scatt_indices(0, str(tmp_path / "x.scattIndices"))
        with pytest.raises(E.TortoiseError):
            e.set_channel_amplitude(0, lambda bary: np.ones(bary.shape[0]))
    finally:
        e.close()


@pytest.mark.parametrize("name", ["ee_n4", "eph_n4"])
def test_streamed_vjp_and_adjoint_equal_the_stored_list(gpu_lib, name):
    """The transposed operator over the walk: grad_f bit for bit in the
    deterministic mode (exact sums of the same per-tuple terms); the
    amplitude gradients sum each warp's tuples first, and the warps hold
    other tuples than in the stored list, so they agree to 1e-13.  Then a
    whole adjoint sweep."""
    from tortoise_b200 import adjoint as A
    mat, f0 = _setup(name)
    th = np.random.default_rng(2).standard_normal(f0.size)
    stored = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True)
    streamed = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True, stream_legs=2)
    try:
        ga, gb = stored.rhs_vjp(f0, th), streamed.rhs_vjp(f0, th)
        assert np.array_equal(ga[0], gb[0])
        assert rel_l2(gb[1], ga[1]) < 1e-13
        w = A.observable_weights(mat, 0, "energy")
        amps = [c.amplitude for c in mat.channels]
        xa = A.gradient(stored, f0, amps, w, 0.0, 0.1, 0.05, checkpoint_every=2)
        xb = A.gradient(streamed, f0, amps, w, 0.0, 0.1, 0.05, checkpoint_every=2)
        assert xa[0] == xb[0]
        assert rel_l2(xb[1], xa[1]) < 1e-12 and rel_l2(xb[2], xa[2]) < 1e-12
    finally:
        stored.close()
        streamed.close()
