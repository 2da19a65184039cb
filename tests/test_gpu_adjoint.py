"""GPU: transposed right-hand side and the discrete Dormand-Prince adjoint.

Checks, all in FP64 (the T32 layout also has its own, exactly transposed
FP32-moment operator):
  * <theta, F'(f) v> from central differences of tb_rhs equals
    <F'(f)^T theta, v> from tb_adjoint_rhs_vjp (relative 1e-8; F is a
    polynomial of degree <= 4 in f, so h = 1e-5 leaves ~1e-10);
  * amplitude gradients of the VJP equal <theta, C_c(f)> / amplitude_c;
  * the adjoint gradient of J = <w, f(t_obs)> equals central differences
    (h = 1e-6) of the same map (fixed-step replay of the logged steps) to 1e-6
    relative, for the initial state and for the coupling constants;
  * the replay reproduces the adaptive run, and the oracle's replay (CPU
    restatement, at perturbed couplings) gives the same finite differences;
  * the result does not depend on the checkpoint spacing;
  * the torch.autograd harness returns the same gradients.
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from tortoise_b200 import adjoint as A
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _mat(N=4, ee=True, bath=False):
    if bath:
        return W.build_material(N, ("P",), (0.15, 0.25), ee=ee, eph=True, field=(0.0, 0.05), rtol=1e-8, atol=1e-9,
                                phonon_bath=True)
    return W.build_material(N, ("P", "D"), (0.2,), ee=ee, eph=True, field=(0.1, 0.0), rtol=1e-8, atol=1e-9)


def _dir_err(fd, ad, scale):
    return abs(fd - ad) / max(abs(ad), 1e-3 * scale)


@pytest.mark.parametrize("layout", [E.LAYOUT_MC64, E.LAYOUT_T64, E.LAYOUT_T32, E.LAYOUT_T40, E.LAYOUT_T48])
@pytest.mark.parametrize("bath", [False, True])
def test_rhs_vjp_is_the_transpose(gpu_lib, layout, bath):
    mat = _mat(4, ee=True, bath=bath)
    f = W.initial_status(mat, kT=0.1, seed=11).vec
    eng = E.Engine(mat, layout=layout)
    rng = np.random.default_rng(7)
    n = eng.ndofs
    for drift in (True, False):
        for _ in range(3):
            th = rng.standard_normal(n)
            v = rng.standard_normal(n)
            g, ga = eng.rhs_vjp(f, th, drift=drift)
            h = 1e-5
            jv = (eng.rhs(f + h * v, drift=drift) - eng.rhs(f - h * v, drift=drift)) / (2 * h)
            lhs, rhs = float(th @ jv), float(g @ v)
            assert abs(lhs - rhs) <= 1e-8 * (abs(lhs) + np.linalg.norm(th) * np.linalg.norm(jv) * 1e-6)
    th = rng.standard_normal(n)
    g, ga = eng.rhs_vjp(f, th, drift=False)
    for c, ch in enumerate(mat.channels):
        want = float(th @ eng.channel_propagate(c, f)) / ch.amplitude
        assert abs(ga[c] - want) <= 1e-11 * (abs(want) + 1e-300) + 1e-14


def test_rhs_vjp_zero_amplitude_still_has_amplitude_gradient(gpu_lib):
    mat = _mat(4, ee=False)
    f = W.initial_status(mat, kT=0.1, seed=3).vec
    eng = E.Engine(mat, layout=E.LAYOUT_T64)
    th = np.random.default_rng(1).standard_normal(eng.ndofs)
    ref = [float(th @ eng.channel_propagate(c, f)) / ch.amplitude for c, ch in enumerate(mat.channels)]
    eng.set_amplitude(0, 0.0)
    g0, ga = eng.rhs_vjp(f, th, drift=False)
    assert abs(ga[0] - ref[0]) <= 1e-11 * abs(ref[0])
    assert all(abs(ga[c] - ref[c]) <= 1e-11 * abs(ref[c]) for c in range(1, len(ref)))


def _forward(eng, f0, t1=0.5, dense=0.25, K=2):
    fo, st = eng.adjoint_forward(f0, 0.0, t1, dense, checkpoint_every=K, max_steps=4096)
    dts, s = eng.adjoint_steps()
    return fo, st, dts, s


@pytest.mark.parametrize("layout", [E.LAYOUT_AUTO, E.LAYOUT_MC64])
def test_replay_reproduces_the_adaptive_run(gpu_lib, layout):
    mat = _mat(4, ee=True)
    f0 = W.initial_status(mat, kT=0.1, seed=5).vec
    eng = E.Engine(mat, layout=layout)
    fo, st, dts, s = _forward(eng, f0)
    ref = eng.dp45(f0, 0.0, 0.5, 0.25)
    assert st["steps"] >= 2 and abs(st["t_obs"] - 0.5) < 1e-12
    assert rel_l2(fo, ref["dense"][-1]) < 1e-13
    assert rel_l2(eng.dp45_replay(f0, dts, s), fo) < 1e-13
    # the oracle replays the same steps (CPU restatement)
    o = oracle.Oracle(mat)
    assert rel_l2(o.dp45_replay(f0, dts, s), fo) < 1e-11


@pytest.mark.parametrize("bath", [False, True])
def test_adjoint_matches_finite_differences(gpu_lib, bath):
    mat = _mat(4, ee=True, bath=bath)
    f0 = W.initial_status(mat, kT=0.1, seed=9).vec
    eng = E.Engine(mat)
    band = 0 if bath else 1
    w = A.observable_weights(mat, band, "energy")
    fo, st, dts, s = _forward(eng, f0)
    g, ga, bst = eng.adjoint_backward(w)
    assert bst["vjp_evals"] == 6 * st["steps"] + 1
    J = lambda f, d=dts: float(w @ eng.dp45_replay(f, d, s))
    rng = np.random.default_rng(21)
    h = 1e-6
    for _ in range(8):
        d = rng.standard_normal(eng.ndofs)
        fd = (J(f0 + h * d) - J(f0 - h * d)) / (2 * h)
        ad = float(g @ d)
        assert _dir_err(fd, ad, np.linalg.norm(g) * np.linalg.norm(d)) < 1e-6, (fd, ad)
    if bath:   # constrained (phonon) bands carry no gradient
        offs, _ = mat.band_offsets()
        assert np.all(g[offs[1]:] == 0.0)
    # amplitudes: channels whose gradient is ~1e-3 of the largest sit at the
    # rounding floor of J for any h, so the check is normwise over channels
    amps = np.array([c.amplitude for c in mat.channels])
    fds = np.zeros_like(amps)
    for c in range(len(amps)):
        hc = 1e-6 * amps[c]
        a = amps.copy()
        a[c] += hc
        A.set_amplitudes(eng, a)
        jp = J(f0)
        a[c] -= 2 * hc
        A.set_amplitudes(eng, a)
        jm = J(f0)
        A.set_amplitudes(eng, amps)
        fds[c] = (jp - jm) / (2 * hc)
    assert rel_l2(ga, fds) < 1e-6, (ga, fds)
    assert np.all(np.abs(ga - fds) <= 1e-6 * np.max(np.abs(ga))), (ga, fds)


def test_coupling_gradients_against_the_oracle(gpu_lib):
    """Finite differences of the oracle's replay at perturbed coupling
    constants (e-e and e-ph, each scaling its channels) against the GPU
    adjoint."""
    mat = W.build_material(4, ("P",), (0.2,), ee=True, eph=True, field=(0.1, 0.0), rtol=1e-8, atol=1e-9)
    f0 = W.initial_status(mat, kT=0.1, seed=13).vec
    eng = E.Engine(mat, layout=E.LAYOUT_MC64)
    w = A.observable_weights(mat, 0, "energy")
    fo, st, dts, s = _forward(eng, f0)
    g, ga, _ = eng.adjoint_backward(w)
    o = oracle.Oracle(mat)
    amps = np.array([c.amplitude for c in mat.channels])
    groups = {"ee": [i for i, c in enumerate(mat.channels) if c.nlegs == 4],
              "eph": [i for i, c in enumerate(mat.channels) if c.nlegs == 3]}
    assert groups["ee"] and groups["eph"]
    for name, chans in groups.items():
        ad = float(sum(amps[c] * ga[c] for c in chans))   # dJ/dg at g = 1 for amp_c = g * a_c
        h = 1e-6
        vals = []
        for sgn in (1, -1):
            for c in chans:
                o.set_amplitude(c, amps[c] * (1 + sgn * h))
            vals.append(float(w @ o.dp45_replay(f0, dts, s)))
            for c in chans:
                o.set_amplitude(c, amps[c])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert _dir_err(fd, ad, abs(ad)) < 1e-6, (name, fd, ad)


def test_checkpoint_spacing_does_not_change_the_gradient(gpu_lib):
    mat = _mat(4, ee=False)
    f0 = W.initial_status(mat, kT=0.1, seed=17).vec
    eng = E.Engine(mat)
    w = A.observable_weights(mat, 0, "density") + A.observable_weights(mat, 1, "current")
    out = []
    for K in (1, 3, 16):
        _, st = eng.adjoint_forward(f0, 0.0, 0.5, 0.125, checkpoint_every=K, max_steps=4096)
        g, ga, bst = eng.adjoint_backward(w)
        assert bst["checkpoint_every"] == K
        out.append((g, ga))
    for g, ga in out[1:]:
        assert rel_l2(g, out[0][0]) < 1e-12
        assert rel_l2(ga, out[0][1]) < 1e-12


def test_capacity_and_argument_errors(gpu_lib):
    mat = _mat(4, ee=False)
    f0 = W.initial_status(mat, kT=0.1, seed=1).vec
    eng = E.Engine(mat)
    with pytest.raises(E.TortoiseError) as ei:
        eng.adjoint_forward(f0, 0.0, 0.5, 0.25, checkpoint_every=2, max_steps=1)
    assert ei.value.rc == 9
    with pytest.raises(E.TortoiseError):
        eng.adjoint_backward(np.zeros(eng.ndofs))   # the failed forward left nothing to reverse
    with pytest.raises(E.TortoiseError):
        eng.adjoint_forward(f0, 0.0, 0.5, 1.0)
    # a plain integration after an adjoint forward records nothing and still matches
    eng.adjoint_forward(f0, 0.0, 0.5, 0.25)
    r = eng.dp45(f0, 0.0, 0.5, 0.25)
    fo, _ = eng.adjoint_forward(f0, 0.0, 0.5, 0.25)
    assert rel_l2(r["dense"][-1], fo) < 1e-13


def test_torch_autograd_harness(gpu_lib):
    mat = _mat(4, ee=False)
    f0n = W.initial_status(mat, kT=0.1, seed=19).vec
    eng = E.Engine(mat)
    w = A.observable_weights(mat, 1, "energy")
    amps_n = np.array([c.amplitude for c in mat.channels])
    J0, g_ref, ga_ref, _ = A.gradient(eng, f0n, amps_n, w, 0.0, 0.5, 0.25, checkpoint_every=4)
    dev = torch.device("cuda:0")
    f0 = torch.tensor(f0n, dtype=torch.float64, device=dev, requires_grad=True)
    coupling = torch.tensor(1.0, dtype=torch.float64, device=dev, requires_grad=True)
    amps = coupling * torch.tensor(amps_n, dtype=torch.float64, device=dev)
    fo = A.DP45Solve.apply(f0, amps, eng, 0.0, 0.5, 0.25, 4)
    J = (torch.tensor(w, dtype=torch.float64, device=dev) * fo).sum()
    J.backward()
    assert abs(J.item() - J0) <= 1e-13 * abs(J0)
    assert rel_l2(f0.grad.cpu().numpy(), g_ref) < 1e-12
    assert abs(coupling.grad.item() - float(amps_n @ ga_ref)) <= 1e-12 * abs(float(amps_n @ ga_ref))
    # the right-hand side as an autograd function
    f = torch.tensor(f0n, dtype=torch.float64, device=dev, requires_grad=True)
    a = torch.tensor(amps_n, dtype=torch.float64, device=dev, requires_grad=True)
    th = torch.tensor(np.random.default_rng(2).standard_normal(eng.ndofs), dtype=torch.float64, device=dev)
    (A.RHS.apply(f, a, eng) * th).sum().backward()
    g, ga = eng.rhs_vjp(f0n, th.cpu().numpy())
    assert rel_l2(f.grad.cpu().numpy(), g) < 1e-14
    assert rel_l2(a.grad.cpu().numpy(), ga) < 1e-14
