"""A k-dependent matrix element: ScatteringChannel::functAmplitude evaluated
once per tuple at the barycentres of its elements (tb_set_channel_amplitude_fn),
against the oracle's restatement of constructAmplitude.  The function is a
Froehlich-like coupling 1 / (|k_in - k_out|^2 + 0.1) of the electron legs of
the e-ph channels (legs el, pn, el)."""
import numpy as np
import pytest

import oracle
from conftest import rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W

pytestmark = pytest.mark.gpu


def froehlich(b):
    q = b[:, 0, :] - b[:, 2, :]
    return 1.0 / ((q * q).sum(axis=1) + 0.1)


def _material(N=6):
    mat = W.build_material(N, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
    for c in mat.channels:
        c.functAmplitude = froehlich
    return mat


@pytest.mark.parametrize("layout,tol", [(E.LAYOUT_MC64, 1e-12), (E.LAYOUT_T64, 1e-12), (E.LAYOUT_T40, 2e-8)])
def test_rhs_and_rates_match_the_oracle(gpu_lib, layout, tol):
    mat = _material()
    f = W.initial_status(mat, seed=6).vec
    eng, o = E.Engine(mat, layout=layout), oracle.Oracle(mat)
    assert rel_l2(eng.rhs(f), o.rhs(f)) < tol
    assert rel_l2(eng.scattering_rates(f), o.scattering_rates(f)) < tol
    # the factors matter: without them the operator is another one
    plain = E.Engine(W.build_material(6, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.1, 0.0), rtol=1e-6,
                                      atol=1e-9), layout=layout)
    assert rel_l2(plain.rhs(f), eng.rhs(f)) > 1e-2
    # back to 1 on the same handle
    for c in range(len(mat.channels)):
        eng.set_channel_amplitude(c, None)
    assert rel_l2(eng.rhs(f), plain.rhs(f)) < tol


def test_dp45_matches_the_oracle(gpu_lib):
    mat = _material()
    f0 = W.initial_status(mat, seed=6).vec
    r = E.Engine(mat).dp45(f0, 0.0, 0.2, 0.1)
    rr = oracle.Oracle(mat).dp45(f0, 0.0, 0.2, 0.1)
    assert r["rc"] == 0 and rr["rc"] == 0
    assert [r["attempts"], r["accepted"], r["rejected"]] == [rr["attempts"], rr["accepted"], rr["rejected"]]
    assert rel_l2(r["dense"], rr["dense"]) < 1e-11


@pytest.mark.parametrize("layout", [E.LAYOUT_MC64, E.LAYOUT_T64])
def test_vjp_matches_central_differences(gpu_lib, layout):
    """The transposed operator carries the factors too: <w, J d> from
    tb_adjoint_rhs_vjp against a central difference of the RHS."""
    mat = _material()
    f = W.initial_status(mat, seed=6).vec
    eng = E.Engine(mat, layout=layout)
    rng = np.random.default_rng(1)
    w, d = rng.standard_normal(f.size), rng.standard_normal(f.size)
    g, _ = eng.rhs_vjp(f, w)
    h = 1e-6
    fd = (w @ eng.rhs(f + h * d) - w @ eng.rhs(f - h * d)) / (2 * h)
    assert abs(fd - g @ d) <= 1e-6 * abs(fd)


def test_batch_shares_the_factors_of_its_structure(gpu_lib):
    mats = [_material(4), _material(4)]
    mats[1].channels[0].amplitude = 0.5
    states = [W.initial_status(m, seed=8 + i).vec for i, m in enumerate(mats)]
    be = E.BatchEngine(mats, layout=E.LAYOUT_T64)
    got = be.split(be.rhs(np.concatenate(states)))
    for m, x, g in zip(mats, states, got):
        assert rel_l2(g, oracle.Oracle(m).rhs(x)) < 1e-12
