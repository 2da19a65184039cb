"""Time-dependent constrained populations (Band::constrainedPopulation as a
callback, tb_set_constraint_fn) in the device integrator, against the
oracle's restatement of DormandPrince54 with enforceValue at every stage,
y5, y4 and dense-output time and MaterialTimeStatus::timeStepVetoer at the
start and after every accepted step.

The workload is the two-band e-ph + drift material whose optical-phonon bath
follows a Gaussian temperature pulse in time (workloads.pulsed_bath): the
vetoer cuts steps that straddle the pulse, and the bath's values reach the
electrons through the e-ph channels."""
import numpy as np
import pytest

import oracle
from conftest import rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dense", [0.01, 0.1])
def test_pulsed_bath_trajectory_matches_the_oracle(gpu_lib, dense):
    mat = W.pulsed_bath(6)
    f0 = W.initial_status(mat, seed=2).vec
    r = E.Engine(mat).dp45(f0, 0.0, 0.3, dense)
    rr = oracle.Oracle(mat).dp45(f0, 0.0, 0.3, dense)
    assert r["rc"] == 0 and rr["rc"] == 0
    assert [r["attempts"], r["accepted"], r["rejected"]] == [rr["attempts"], rr["accepted"], rr["rejected"]]
    assert np.allclose(r["dense_t"], rr["dense_t"], rtol=0, atol=1e-14)
    assert rel_l2(r["dense"], rr["dense"]) < 1e-11
    ph = mat.bands[2]
    off = mat.band_offsets()[0][2]
    for t, y in zip(r["dense_t"], r["dense"]):
        assert np.array_equal(y[off:off + ph.mesh.ne * 3], ph.population_at(t))


def test_the_pulse_costs_attempts(gpu_lib):
    """The same integration with the bath held at its t = 0 value takes far
    fewer attempts: the pulse is what the controller and the vetoer react to."""
    mat = W.pulsed_bath(6)
    f0 = W.initial_status(mat, seed=2).vec
    eng = E.Engine(mat)
    pulsed = eng.dp45(f0, 0.0, 0.3, 0.05)
    ph = mat.bands[2]
    eng.set_constraint(lambda b, t: ph.population_at(0.0))
    flat = eng.dp45(f0, 0.0, 0.3, 0.05)
    eng.set_constraint(None)
    const = eng.dp45(f0, 0.0, 0.3, 0.05)   # the description's placeholder populations
    assert pulsed["rc"] == 0 and flat["rc"] == 0 and const["rc"] == 0
    assert pulsed["attempts"] > 2 * flat["attempts"], (pulsed["attempts"], flat["attempts"])


def test_apply_constraints_at_matches_the_oracle(gpu_lib):
    mat = W.pulsed_bath(6)
    f = W.initial_status(mat, seed=3).vec
    eng, o = E.Engine(mat), oracle.Oracle(mat)
    for t in (0.0, 0.11, 0.12, 0.2):
        assert np.array_equal(eng.apply_constraints_at(f, t), o.apply_constraints_at(f, t))
    with pytest.raises(E.TortoiseError):
        from tortoise_b200.engine import lib, PTR_HOST
        g = np.ascontiguousarray(f).copy()
        E._check(lib().tb_apply_constraints(eng.h, E._hp(g), PTR_HOST), "tb_apply_constraints")


def test_batch_runs_keep_their_own_constraint_histories(gpu_lib):
    """Runs with pulses at different times and one with a fixed bath, in one
    handle: every run reproduces its single-run integration (its own veto,
    accept/reject sequence and dense outputs)."""
    mats = [W.pulsed_bath(4, t_pulse=0.1), W.pulsed_bath(4, t_pulse=0.2),
            W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9,
                             phonon_bath=True)]
    states = [W.initial_status(m, seed=5 + i).vec for i, m in enumerate(mats)]
    be = E.BatchEngine(mats)
    res = be.dp45(np.concatenate(states), 0.0, 0.3, 0.02)
    for r, (m, f) in enumerate(zip(mats, states)):
        ref = E.Engine(m).dp45(f, 0.0, 0.3, 0.02)
        got = res["runs"][r]
        assert got["status"] == 0 and ref["rc"] == 0
        assert [got["attempts"], got["accepted"], got["rejected"]] == [ref["attempts"], ref["accepted"], ref["rejected"]]
        assert rel_l2(got["dense"], ref["dense"]) < 1e-10


def test_a_failing_callback_ends_the_integration(gpu_lib):
    """A callback that fails (here: raises after t = 0.1) stops the
    integration with TB_ERR_ARG on the host side of the attempt graph; the
    handle stays usable."""
    mat = W.pulsed_bath(4)
    f0 = W.initial_status(mat, seed=2).vec
    eng = E.Engine(mat)
    ph = mat.bands[2]

    def bad(b, t):
        if t > 0.1:
            raise ValueError("no population after t = 0.1")
        return ph.population_at(t)
    eng.set_constraint(bad)
    r = eng.dp45(f0, 0.0, 0.3, 0.05)
    assert r["rc"] == 8 and r["t"] < 0.3
    assert isinstance(eng.constraint_error, ValueError)
    eng.set_constraint(lambda b, t: ph.population_at(t))
    assert eng.dp45(f0, 0.0, 0.3, 0.05)["rc"] == 0


def test_the_adjoint_refuses_time_dependent_constraints(gpu_lib):
    mat = W.pulsed_bath(4)
    f0 = W.initial_status(mat, seed=2).vec
    eng = E.Engine(mat)
    with pytest.raises(E.TortoiseError):
        eng.adjoint_forward(f0, 0.0, 0.1, 0.05)
