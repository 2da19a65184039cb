"""Batched ensembles: one handle, several runs.  Every run of a batch must
give what it gives alone (RHS to 1e-12; DP45 with its own accept/reject
sequence and dense outputs to 1e-10), whether it shares structure with other
runs (shared tuple lists / moment tensors) or not."""
import numpy as np
import pytest

from conftest import rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _runs():
    """Three e-ph runs of equal structure (4x4) with different coupling and
    temperature, plus one run of another structure (3x3, two phonon baths)."""
    mats, states = [], []
    for k, (amp, kT) in enumerate([(1.0, 0.1), (0.5, 0.05), (2.0, 0.2)]):
        m = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9,
                             eph_amplitude=amp)
        mats.append(m)
        states.append(W.initial_status(m, kT=kT, seed=10 + k).vec)
    m = W.build_material(3, ("P",), (0.15, 0.25), ee=False, eph=True, field=(0.0, 0.05), rtol=1e-6, atol=1e-9,
                         phonon_bath=True)
    mats.append(m)
    states.append(W.initial_status(m, kT=0.1, seed=20).vec)
    return mats, states


@pytest.mark.parametrize("layout", [E.LAYOUT_MC64, E.LAYOUT_T64])
def test_batch_rhs_equals_individual_runs(gpu_lib, layout):
    mats, states = _runs()
    be = E.BatchEngine(mats, layout=layout)
    got = be.split(be.rhs(np.concatenate(states)))
    for m, f, g in zip(mats, states, got):
        ref = E.Engine(m, layout=layout).rhs(f)
        assert rel_l2(g, ref) < 1e-12
    # equal-structure runs share one tuple list
    n0 = be.channel_info(be.chan0[0])["n_tuples"]
    assert be.channel_info(be.chan0[1])["n_tuples"] == n0


def test_batch_amplitude_update(gpu_lib):
    mats, states = _runs()
    be = E.BatchEngine(mats, layout=E.LAYOUT_T64)
    f = np.concatenate(states)
    base = be.split(be.rhs(f, drift=False))
    for c in range(len(mats[1].channels)):
        be.set_amplitude(be.chan0[1] + c, 0.0)
    after = be.split(be.rhs(f, drift=False))
    assert np.linalg.norm(after[1]) == 0.0
    assert rel_l2(after[0], base[0]) < 1e-14 and rel_l2(after[2], base[2]) < 1e-14


def test_batch_dp45_equals_individual_runs(gpu_lib):
    mats, states = _runs()
    be = E.BatchEngine(mats, layout=E.LAYOUT_MC64)
    tf = [0.4, 0.3, 0.2, 0.4]
    res = be.dp45(np.concatenate(states), 0.0, tf, 0.1)
    for r, (m, f) in enumerate(zip(mats, states)):
        ref = E.Engine(m, layout=E.LAYOUT_MC64).dp45(f, 0.0, tf[r], 0.1)
        got = res["runs"][r]
        assert got["status"] == 0
        assert [got["attempts"], got["accepted"], got["rejected"]] == [ref["attempts"], ref["accepted"], ref["rejected"]]
        assert np.allclose(got["dense_t"], ref["dense_t"], rtol=0, atol=1e-14)
        assert rel_l2(got["dense"], ref["dense"]) < 1e-10


def test_mixed_precision_trajectory_within_1e8(gpu_lib):
    """Mixed-precision moment storage (FP64 products, accumulation,
    gain - loss, error norm, controller) against the FP64 path on the two-band
    e-ph + drift workload at 16x16, rtol 1e-8, to t = 1, every dense output:
    40-bit storage (T40: upper 40 bits of FP64, 2^-29) within 5e-9 relative L2
    (measured ~1e-9), 48-bit storage (T48, 2^-37) within 1e-10, plain FP32
    storage (T32) within 3e-8 (measured ~1e-8).
    A batch of three runs of that structure in T40 gives every run's FP64
    trajectory to 5e-9 as well."""
    mats, states = [], []
    for k, (amp, kT) in enumerate([(1.0, 0.1), (0.6, 0.05), (1.7, 0.2)]):
        m = W.two_band_eph_drift(16, eph_amplitude=amp)
        mats.append(m)
        states.append(W.initial_status(m, kT=kT, seed=40 + k).vec)
    r64 = E.Engine(mats[0], layout=E.LAYOUT_T64).dp45(states[0], 0.0, 1.0, 0.25)
    r40 = E.Engine(mats[0], layout=E.LAYOUT_T40).dp45(states[0], 0.0, 1.0, 0.25)
    r32 = E.Engine(mats[0], layout=E.LAYOUT_T32).dp45(states[0], 0.0, 1.0, 0.25)
    r48 = E.Engine(mats[0], layout=E.LAYOUT_T48).dp45(states[0], 0.0, 1.0, 0.25)
    assert r64["status"] == 0 and r40["status"] == 0 and r32["status"] == 0 and r48["status"] == 0
    e48 = [rel_l2(a, b) for a, b in zip(r48["dense"], r64["dense"])]
    assert len(e48) == 4 and max(e48) < 1e-10, e48
    e40 = [rel_l2(a, b) for a, b in zip(r40["dense"], r64["dense"])]
    e32 = [rel_l2(a, b) for a, b in zip(r32["dense"], r64["dense"])]
    assert len(e40) == 4 and max(e40) < 5e-9, e40
    assert max(e32) < 3e-8, e32
    be = E.BatchEngine(mats, layout=E.LAYOUT_AUTO, allow_fp32=2)
    assert {be.channel_info(c)["layout"] for c in range(be.channel_count())} == {"t40"}
    res = be.dp45(np.concatenate(states), 0.0, 1.0, 0.25)
    for r, (m, f) in enumerate(zip(mats, states)):
        ref = E.Engine(m, layout=E.LAYOUT_T64).dp45(f, 0.0, 1.0, 0.25)
        got = res["runs"][r]
        assert got["status"] == 0
        assert max(rel_l2(a, b) for a, b in zip(got["dense"], ref["dense"])) < 5e-9


def test_autotuned_schedule_gives_the_same_operator(gpu_lib):
    """tb_options.autotune times the contraction schedules (bulk-copy stages
    1 / 2, instance pairs off / on) and keeps the fastest; the operator must
    not change (1e-12), and the chosen schedule is reported."""
    mats, states = _runs()
    f = np.concatenate(states)
    for layout in (E.LAYOUT_T64, E.LAYOUT_T40):
        plain = E.BatchEngine(mats, layout=layout)
        tuned = E.BatchEngine(mats, layout=layout, autotune=True)
        assert rel_l2(tuned.rhs(f), plain.rhs(f)) < 1e-12
        s = tuned.schedule(0)
        assert s["stages"] in (1, 2) and s["pair"] in (0, 1) and s["tuned_seconds"] > 0.0
        assert plain.schedule(0)["tuned_seconds"] == 0.0
    mc = E.BatchEngine(mats, layout=E.LAYOUT_MC64, autotune=True)
    assert mc.schedule(0) == {"stages": 0, "pair": 0, "runs": 0, "tuned_seconds": 0.0, "inside_only": True}


@pytest.mark.parametrize("layout", [E.LAYOUT_T64, E.LAYOUT_T40, E.LAYOUT_T48, E.LAYOUT_T32])
def test_run_minor_contraction_equals_individual_runs(gpu_lib, layout):
    """Groups shared by 16 runs or more take the run-minor contraction (one
    lane per run, lane groups of 8 runs by default, f and the results staged
    run-minor); every other schedule, pinned with tb_set_channel_schedule,
    gives the same operator.
    40 runs of two structures (4x4 and 6x6, about 20 runs each, so the second
    chunk of 32 lanes is partly idle): every run's RHS equals its RHS alone to
    1e-12, and a short DP45 integration reproduces every run's own
    accept/reject sequence and dense outputs to 1e-10.  With one run switched
    off (amplitudes 0), its lane emits nothing."""
    mats, states = W.ensemble_runs(40, seed=7, Ns=(4, 6))
    be = E.BatchEngine(mats, layout=layout)
    assert all(be.schedule(c)["runs"] == 8 for c in range(be.channel_count()))
    f = np.concatenate(states)
    singles = [E.Engine(m, layout=layout) for m in mats]
    refs = [e1.rhs(x) for e1, x in zip(singles, states)]
    # every pinned schedule: lane groups of 32 / 16 / 8 / 4 runs, the per-thread
    # paths, one or two bulk-copy stages
    for stages in (1, 2):
        for kw in ({"runs": 32}, {"runs": 16}, {"runs": 8}, {"runs": 4}, {"pair": 0}, {"pair": 1}):
            for c in range(be.channel_count()):
                be.set_schedule(c, stages, **kw)
            got = be.split(be.rhs(f))
            for g, ref in zip(got, refs):
                assert rel_l2(g, ref) < 1e-12, (stages, kw)
    for c in range(be.channel_count()):
        be.set_schedule(c, 1, runs=8)
    res = be.dp45(f, 0.0, 0.05, 0.025)
    for r in (0, 1, 17, 39):
        ref = singles[r].dp45(states[r], 0.0, 0.05, 0.025)
        run = res["runs"][r]
        assert run["status"] == 0
        assert [run["attempts"], run["accepted"], run["rejected"]] == [ref["attempts"], ref["accepted"], ref["rejected"]]
        assert rel_l2(run["dense"], ref["dense"]) < 1e-10
    for c in range(len(mats[5].channels)):
        be.set_amplitude(be.chan0[5] + c, 0.0)
    after = be.split(be.rhs(f, drift=False))
    assert np.linalg.norm(after[5]) == 0.0
    assert rel_l2(after[6], singles[6].rhs(states[6], drift=False)) < 1e-12


def test_points_inside_only_beyond_the_shared_accumulator(gpu_lib):
    """256 runs of one 4x4 two-band structure with e-e channels: the
    Monte-Carlo kernel's shared-memory copy of the accumulator (one block per
    run) would exceed its limit, so it adds straight into the global
    accumulator.  Against the same handle pinned to every Monte-Carlo point,
    and against a batch of the first 8 runs (shared-memory copies), the
    operator must not change (1e-12, the FP64 parity bar)."""
    mats, states = W.ensemble_runs(256, seed=9, Ns=(4,), ee=True)
    f = np.concatenate(states)
    be = E.BatchEngine(mats, layout=E.LAYOUT_MC64)
    per_run = len(mats[0].channels)
    live = [c for c in range(per_run) if be.channel_info(c)["n_tuples"]]
    assert live and all(be.schedule(c).get("inside_only") for c in live)
    a = be.rhs(f)
    small = E.BatchEngine(mats[:8], layout=E.LAYOUT_MC64)
    s = small.rhs(np.concatenate(states[:8]))
    assert rel_l2(a[:s.size], s) < 1e-12
    for c in live:
        be.set_schedule(c, 0, inside_only=False)
    assert rel_l2(a, be.rhs(f)) < 1e-12
