"""The deterministic mode (tb_options.deterministic): exact fixed-point
accumulation of the per-tuple results instead of FP64 atomics.

* Bit-reproducibility: repeated evaluations and separate handles give equal
  bits for the collision operator (every layout, the Monte-Carlo quadrature
  over every point or over the inside points only), the scattering rates,
  whole DP45 integrations, batched ensembles and the VJP / adjoint.
* Independence of the contraction schedule: per-thread, instance pairs and
  every run-minor lane-group width give equal bits, because every schedule
  forms the same per-tuple values and their sum no longer depends on order.
* The values agree with the FP64-atomic mode to the FP64 summation noise
  (1e-12 relative L2) and with the oracle to the bounds of the parity tests.
* A non-finite contribution poisons the sum: the whole evaluation reads NaN.
"""
import numpy as np
import pytest

import oracle
from conftest import golden, rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W
from tests.golden.make_golden import cases

pytestmark = pytest.mark.gpu

CASES = list(cases().keys())
LAYOUTS = [E.LAYOUT_MC64, E.LAYOUT_T64, E.LAYOUT_T48, E.LAYOUT_T40, E.LAYOUT_T32]


def _setup(name):
    build, seed, kT = cases()[name]
    mat = build()
    return mat, W.initial_status(mat, kT=kT, seed=seed).vec


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("name", CASES)
def test_rhs_is_bit_reproducible(gpu_lib, name, layout):
    mat, f0 = _setup(name)
    a = E.Engine(mat, layout=layout, deterministic=True)
    b = E.Engine(mat, layout=layout, deterministic=True)
    plain = E.Engine(mat, layout=layout)
    try:
        r1, r2, r3 = a.rhs(f0), a.rhs(f0), b.rhs(f0)
        assert np.array_equal(r1, r2) and np.array_equal(r1, r3)
        assert rel_l2(r1, plain.rhs(f0)) < 1e-12
        s1, s2 = a.scattering_rates(f0), b.scattering_rates(f0)
        assert np.array_equal(s1, s2)
        assert rel_l2(s1, plain.scattering_rates(f0)) < 1e-12
        if layout == E.LAYOUT_MC64:
            g = golden(name)
            assert rel_l2(r1, g["rhs"]) < 1e-12
    finally:
        for e in (a, b, plain):
            e.close()


@pytest.mark.parametrize("name", ["ee_n4", "ee2_n3"])
def test_monte_carlo_visiting_modes_are_each_reproducible(gpu_lib, name):
    mat, f0 = _setup(name)
    e = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True)
    try:
        for inside in (True, False):
            for ch in range(len(mat.channels)):
                if e.points_inside(ch)[0] >= 0:   # channels without tuples have no list of inside points
                    e.set_schedule(ch, 0, inside_only=inside)
            r = [e.rhs(f0) for _ in range(3)]
            assert np.array_equal(r[0], r[1]) and np.array_equal(r[0], r[2])
    finally:
        e.close()


@pytest.mark.parametrize("layout", [E.LAYOUT_T64, E.LAYOUT_T40])
def test_every_schedule_gives_the_same_bits(gpu_lib, layout):
    """A 16-run batch of one structure: per-thread, paired and run-minor
    contractions (all lane-group widths, one and two pipeline stages)."""
    mats, states = W.ensemble_runs(16, seed=7, Ns=(4,))
    be = E.BatchEngine(mats, layout=layout, deterministic=True)
    try:
        f = np.concatenate(states)
        ref = None
        for stages in (1, 2):
            for kw in ({"pair": 0}, {"pair": 1}, {"runs": 4}, {"runs": 8}, {"runs": 16}, {"runs": 32}):
                for ch in range(len(mats[0].channels)):
                    be.set_schedule(ch, stages, **kw)
                got = be.rhs(f)
                if ref is None:
                    ref = got
                assert np.array_equal(got, ref), (stages, kw)
        # each run alone, deterministic too, gives the batch's bits
        for m, x, g in zip(mats[:3], states[:3], be.split(ref)):
            one = E.Engine(m, layout=layout, deterministic=True)
            try:
                assert np.array_equal(one.rhs(x), g)
            finally:
                one.close()
    finally:
        be.close()


@pytest.mark.parametrize("name", ["eph_n4", "eph_bath_n4", "ee_n3"])
def test_dp45_is_bit_reproducible_and_matches_the_oracle(gpu_lib, name):
    g = golden(name)
    mat, f0 = _setup(name)
    a = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True)
    b = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True)
    try:
        ra, rb = a.dp45(f0, 0.0, 0.4, 0.1), b.dp45(f0, 0.0, 0.4, 0.1)
        for k in ("attempts", "accepted", "rejected", "rhs_evals"):
            assert ra[k] == rb[k]
        assert np.array_equal(ra["dense"], rb["dense"]) and np.array_equal(ra["y"], rb["y"])
        assert ra["t"] == rb["t"]
        assert [ra["attempts"], ra["accepted"], ra["rejected"], ra["rhs_evals"]] == list(g["dp_stats"])
        assert rel_l2(ra["dense"], g["dp_dense"]) < 1e-11
    finally:
        a.close()
        b.close()


def test_batched_ensemble_is_bit_reproducible(gpu_lib):
    mats, states = W.ensemble_runs(12, seed=11, Ns=(4, 6))
    f = np.concatenate(states)
    out = []
    for _ in range(2):
        be = E.BatchEngine(mats, layout=E.LAYOUT_T64, deterministic=True)
        try:
            out.append(be.dp45(f, 0.0, 0.3, 0.1))
        finally:
            be.close()
    ra, rb = out
    assert ra["rc"] == 0 and rb["rc"] == 0
    assert np.array_equal(ra["y"], rb["y"])
    for a, b in zip(ra["runs"], rb["runs"]):
        assert (a["attempts"], a["accepted"], a["rejected"]) == (b["attempts"], b["accepted"], b["rejected"])
        assert np.array_equal(a["dense"], b["dense"]) and np.array_equal(a["dense_t"], b["dense_t"])


def test_vjp_and_adjoint_are_bit_reproducible(gpu_lib):
    from tortoise_b200 import adjoint as A
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=True, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
    f0 = W.initial_status(mat, seed=5).vec
    th = np.random.default_rng(4).standard_normal(f0.size)
    a = E.Engine(mat, deterministic=True)
    b = E.Engine(mat, deterministic=True)
    plain = E.Engine(mat)
    try:
        ga, gb, gp = a.rhs_vjp(f0, th), b.rhs_vjp(f0, th), plain.rhs_vjp(f0, th)
        assert np.array_equal(ga[0], gb[0]) and np.array_equal(ga[1], gb[1])
        assert rel_l2(ga[0], gp[0]) < 1e-12 and rel_l2(ga[1], gp[1]) < 1e-12
        w = A.observable_weights(mat, 1, "energy")
        amps = [c.amplitude for c in mat.channels]
        xa = A.gradient(a, f0, amps, w, 0.0, 0.1, 0.05, checkpoint_every=2)
        xb = A.gradient(b, f0, amps, w, 0.0, 0.1, 0.05, checkpoint_every=2)
        assert xa[0] == xb[0]
        assert np.array_equal(xa[1], xb[1]) and np.array_equal(xa[2], xb[2])
    finally:
        for e in (a, b, plain):
            e.close()


def test_rhs_matches_the_oracle_in_every_mode(gpu_lib):
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=True, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
    f0 = W.initial_status(mat, seed=3).vec
    ref = oracle.Oracle(mat).rhs(f0)
    for det in (False, True):
        e = E.Engine(mat, deterministic=det)
        try:
            assert rel_l2(e.rhs(f0), ref) < 1e-12
        finally:
            e.close()


def test_non_finite_input_poisons_the_whole_sum(gpu_lib):
    mat, f0 = _setup("eph_n4")
    e = E.Engine(mat, layout=E.LAYOUT_T64, deterministic=True)
    try:
        bad = f0.copy()
        bad[5] = np.nan
        assert np.all(np.isnan(e.rhs(bad, drift=False)))
        # the poison is cleared by the flush: the next evaluation is clean
        assert np.array_equal(e.rhs(f0), e.rhs(f0)) and np.all(np.isfinite(e.rhs(f0)))
    finally:
        e.close()


def test_out_of_range_contribution_is_clamped_and_reported(gpu_lib):
    """A finite contribution of magnitude 2^64 or more (here: a state scaled
    by 1e20, whose quadratic terms reach 1e40) is clamped to the exact
    accumulator's range: the operator reports TB_ERR_NONFINITE, the handle
    stays usable and its next evaluation has the bits of a fresh one.  The
    FP64-atomic mode returns the finite huge values."""
    mat, f0 = _setup("eph_n4")
    e = E.Engine(mat, layout=E.LAYOUT_T64, deterministic=True)
    plain = E.Engine(mat, layout=E.LAYOUT_T64)
    try:
        ref = e.rhs(f0)
        with pytest.raises(E.TortoiseError, match="2\\^64"):
            e.rhs(f0 * 1e20)
        assert np.array_equal(e.rhs(f0), ref)
        big = plain.rhs(f0 * 1e20)
        assert np.all(np.isfinite(big)) and np.max(np.abs(big)) > 1e30
    finally:
        e.close()
        plain.close()


def test_ensemble_with_an_oversized_first_step(gpu_lib):
    """Dense step 2 on the ensemble: the first attempts take steps far too
    large, whose trial stages blow up past 2^64 before the error norm
    rejects them.  In the deterministic mode the clamped stages are rejected
    like the FP64 ones: every run reaches t = 4, two batches agree bit for
    bit, and the FP64-atomic batch's dense outputs (t = 2, 4) agree to its
    own tolerance (the final states lie at each run's last step, past t = 4
    by different amounts)."""
    mats, states = W.ensemble_runs(16, seed=5, Ns=(16,))
    f = np.concatenate(states)
    out = []
    for det in (True, True, False):
        be = E.BatchEngine(mats, layout=E.LAYOUT_T64, deterministic=det)
        try:
            out.append(be.dp45(f, 0.0, 4.0, 2.0, max_dense=4))
        finally:
            be.close()
    a, b, p = out
    for r in (a, b, p):
        assert r["rc"] == 0 and all(x["status"] == 0 and x["t"] >= 4.0 for x in r["runs"])
    assert np.array_equal(a["y"], b["y"])
    for x, y in zip(a["runs"], p["runs"]):
        assert len(x["dense"]) == len(y["dense"]) >= 2
        assert rel_l2(x["dense"], y["dense"]) < 1e-6
