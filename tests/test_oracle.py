"""CPU tests of the oracle: identities the reference algorithm obeys, the
DP54 documentation example, and regression against the golden fixtures."""
import numpy as np
import pytest

import oracle
from conftest import golden, rel_l2
from tortoise_b200 import workloads as W
from tortoise_b200.model import linform_to_nodal
from tests.golden.make_golden import cases, tuple_hash


def test_mass_matrix_identities():
    mat = W.parabolic_ee(4)
    o = oracle.Oracle(mat)
    M, Mi = o.mass_matrix(0)
    vol = mat.bands[0].mesh.elemVolume
    # exact P1 mass matrix on the reference triangle scaled by |T|/|T_ref|
    exact = vol * np.array([[1, 1 / 3, 1 / 3], [1 / 3, 1 / 6, 1 / 12], [1 / 3, 1 / 12, 1 / 6]])
    assert np.allclose(M, exact, rtol=1e-12)
    assert np.allclose(M @ Mi, np.eye(3), atol=1e-12)


def _integral(o, band, coeffs, weight=None):
    mat = o.material
    ne = mat.bands[band].mesh.ne
    w = np.tile([1.0, 0.0, 0.0], ne) if weight is None else weight
    return o.integrate(band, coeffs, w)


@pytest.mark.parametrize("name", ["ee_n4", "eph_n4"])
def test_conservation_laws(name):
    """Particle number (e-e), energy and crystal momentum are conserved by
    every tuple: the delta constraint makes sum_l dir_l E_l(p_l) = 0 exactly
    for the P1 energy (IntegratorCore.hpp:298-320)."""
    build, seed, kT = cases()[name]
    mat = build()
    o = oracle.Oracle(mat)
    f0 = W.initial_status(mat, kT=kT, seed=seed).vec
    d = o.rhs(f0, drift=False)
    offs, _ = mat.band_offsets()
    tot_e = 0.0
    scale_e = 0.0
    tot_n = 0.0
    scale_n = 0.0
    for b, band in enumerate(mat.bands):
        sl = slice(offs[b], offs[b] + band.mesh.ne * 3)
        tot_e += o.integrate(b, d[sl], band.dispersion_coeffs)
        scale_e += abs(o.integrate(b, np.abs(d[sl]), np.abs(band.dispersion_coeffs)))
        if band.statistics == -1:
            one = np.tile([1.0, 0.0, 0.0], band.mesh.ne)
            tot_n += o.integrate(b, d[sl], one)
            scale_n += o.integrate(b, np.abs(d[sl]), one)
    assert abs(tot_e) <= 1e-12 * scale_e
    if name.startswith("ee"):
        assert abs(tot_n) <= 1e-12 * scale_n


def test_equilibrium_is_nearly_stationary():
    """Fermi-Dirac at common T and mu: gain and loss balance up to the P1
    interpolation of f along the energy shell, so the residual is small when
    the mesh resolves kT and shrinks under refinement."""
    ratios = []
    for N in (4, 6):
        mat = W.parabolic_ee(N)
        o = oracle.Oracle(mat)
        eq = W.initial_status(mat, kT=3.0, seed=0, bump_amplitude=0.0).vec
        neq = W.initial_status(mat, kT=3.0, seed=0, bump_amplitude=0.3).vec
        ratios.append(np.linalg.norm(o.rhs(eq, drift=False)) / np.linalg.norm(o.rhs(neq, drift=False)))
    assert ratios[0] < 1e-2 and ratios[1] < ratios[0]


def test_dp54_documentation_example():
    """DormandPrince54.hpp:80-106: y' = cos t from 0 to 10, dense step 1."""
    d, t, st = oracle.scalar_example()
    assert len(t) == 10
    assert np.allclose(t, np.arange(1, 11))
    assert np.max(np.abs(d - np.sin(t))) < 5e-6
    g = golden("dp54_scalar")
    assert np.array_equal(d, g["dense"]) and np.array_equal(st, g["stats"])


@pytest.mark.parametrize("name", list(cases().keys()))
def test_oracle_matches_golden(name):
    g = golden(name)
    build, seed, kT = cases()[name]
    mat = build()
    o = oracle.Oracle(mat)
    f0 = W.initial_status(mat, kT=kT, seed=seed).vec
    assert np.array_equal(f0, g["f0"])
    for ch in range(len(mat.channels)):
        ids, umk = o.tuples(ch)
        pre, det = o.enum_counts(ch)
        assert [len(umk), pre, det] == list(g["ch%d_counts" % ch])
        assert tuple_hash(ids, umk) == str(g["ch%d_hash" % ch])
        assert rel_l2(o.channel_propagate(ch, f0), g["ch%d_prop" % ch]) < 1e-14
    assert rel_l2(o.rhs(f0, drift=True), g["rhs"]) < 1e-14
    assert abs(o.relative_error(g["err"], f0) - float(g["relerr"])) <= 1e-14 * float(g["relerr"])
    if "dp_y" in g:
        r = o.dp45(f0, 0.0, 0.4, 0.1)
        assert [r["attempts"], r["accepted"], r["rejected"], r["rhs_evals"]] == list(g["dp_stats"])
        assert rel_l2(r["y"], g["dp_y"]) < 1e-13


def test_tuples_are_valid_and_ordered():
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True)
    o = oracle.Oracle(mat)
    for ch, c in enumerate(mat.channels):
        ids, umk = o.tuples(ch)
        ne = [mat.bands[b].mesh.ne for b in c.legBandNumber]
        for l in range(c.nlegs):
            assert ids[:, l].min() >= 0 and ids[:, l].max() < ne[l]
        # reference loop order: sections of legs 0..L-2, then elements
        sec = ids[:, :-1] // 2
        key = np.lexsort(tuple([ids[:, -1]] + [ids[:, l] % 2 for l in reversed(range(c.nlegs - 1))]
                               + [sec[:, l] for l in reversed(range(c.nlegs - 1))]))
        assert np.array_equal(key, np.arange(len(key)))


def test_single_tuple_partition_additivity():
    """propagate over a tuple range is additive (the TBB reduction split)."""
    mat = W.parabolic_ee(4)
    o = oracle.Oracle(mat)
    f0 = W.initial_status(mat, seed=2).vec
    n = o.num_tuples(0)
    full = o.channel_propagate(0, f0)
    a = o.channel_propagate(0, f0, 0, n // 3)
    b = o.channel_propagate(0, f0, n // 3, n)
    assert rel_l2(a + b, full) < 1e-13


def test_scattering_rates_are_twice_the_affine_slope():
    """The oracle's ScatteringChannel::scatteringRates (ScatteringChannel.cpp:
    544-612) against its propagate: each leg's gain / loss forms are affine in
    that leg's coefficients with half the slope of the rate's unit forms, so
    for a leg whose band no other leg of the channel uses, the rate equals -2
    times the change of the channel's output on that band when c0 of every
    element of the band rises by 1 (exact up to rounding)."""
    import oracle
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.1, 0.0))
    f = W.initial_status(mat, kT=0.1, seed=4).vec
    o = oracle.Oracle(mat)
    offs, n = mat.band_offsets()
    checked = 0
    for ch, c in enumerate(mat.channels):
        for leg, b in enumerate(c.legBandNumber):
            if list(c.legBandNumber).count(b) != 1:
                continue
            sl = slice(offs[b], offs[b] + mat.bands[b].mesh.ne * 3)
            u = np.zeros(n)
            u[sl][0::3] = 1.0
            slope = o.channel_propagate(ch, f + u)[sl] - o.channel_propagate(ch, f)[sl]
            rate = o.scattering_rates(f, ch, leg)[sl]
            assert np.linalg.norm(rate + 2.0 * slope) <= 1e-12 * np.linalg.norm(rate)
            checked += 1
    assert checked >= 6
    # the whole-status sum is the sum over channels and legs
    tot = sum(o.scattering_rates(f, ch) for ch in range(len(mat.channels)))
    assert np.allclose(o.scattering_rates(f), tot, rtol=1e-13, atol=0)


def test_time_step_veto_of_a_pulsed_bath():
    """MaterialTimeStatus::timeStepVetoer, restated: a constant or linear
    constrained history never shortens the step; a Gaussian pulse inside the
    tested step cuts it at the first dense-step probe that leaves the
    tolerance band, a whole number of dense steps after t; and a
    DP45 integration through the pulse takes more attempts than one with the
    bath held fixed."""
    import numpy as np
    from tortoise_b200 import workloads as W
    from tortoise_b200.model import nodal_to_linform
    mat = W.pulsed_bath(4)
    o = oracle.Oracle(mat)
    ph = mat.bands[2]
    # well before the pulse: flat history, no veto
    assert o.veto_step(0.0, 0.01, 0.001) == (0.0 + 0.01) - 0.0
    # a linear history: the probes sit within half the interval change
    base = ph.population_at(0.0)
    o.set_constraint(lambda b, t: base * (1.0 + t))
    assert o.veto_step(0.05, 0.1, 0.001) == (0.05 + 0.1) - 0.05
    # the pulse (t 0.12, width 0.02) inside the stage interval [0.09, 0.24]
    # of a step of 0.3 from 0: the first probe beyond 1.3 |left - right|
    # (+ tolerances) from the interval average cuts the step there
    o.set_constraint(lambda b, t: ph.population_at(t))
    v = o.veto_step(0.0, 0.3, 0.001)
    assert 0.09 < v < 0.12, v
    k = v / 0.001
    assert abs(k - round(k)) < 1e-6, k
    f0 = W.initial_status(mat, seed=2).vec
    pulsed = o.dp45(f0, 0.0, 0.3, 0.01)
    o.set_constraint(lambda b, t: ph.population_at(0.0))
    flat = o.dp45(f0, 0.0, 0.3, 0.01)
    assert pulsed["rc"] == 0 and flat["rc"] == 0
    assert pulsed["attempts"] > flat["attempts"], (pulsed["attempts"], flat["attempts"])
    # the bath follows the pulse in the dense outputs
    off = o.band_offset(2)
    for t, y in zip(pulsed["dense_t"], pulsed["dense"]):
        assert np.array_equal(y[off:off + ph.mesh.ne * 3], ph.population_at(t))


def test_funct_amplitude_scales_each_tuple():
    """ScatteringChannel::functAmplitude, restated: a factor of 1 per tuple
    leaves the operator bit for bit, 2 doubles it exactly, and the
    barycentres handed to the function are the element centroids of
    Mesh<2>::elemCentre (reference point 0.333333333 each way)."""
    import numpy as np
    from tortoise_b200 import workloads as W
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True, rtol=1e-6, atol=1e-9)
    f = W.initial_status(mat, seed=4).vec
    o = oracle.Oracle(mat)
    base = o.rhs(f, drift=False)
    o.set_channel_amplitude(0, lambda b: np.ones(len(b)))
    assert np.array_equal(o.rhs(f, drift=False), base)
    seen = []

    def two(b):
        seen.append(b.copy())
        return np.full(len(b), 2.0)
    o.set_channel_amplitude(0, two)
    only0 = o.channel_propagate(0, f)
    o.set_channel_amplitude(0, None)
    assert np.array_equal(only0, 2.0 * o.channel_propagate(0, f))
    ids, _ = o.tuples(0)
    mesh = mat.bands[mat.channels[0].legBandNumber[0]].mesh
    cent = mesh.vertices().mean(axis=1)            # (ne, 2) element centroids
    assert np.abs(seen[0][:, 0, :] - cent[ids[:, 0]]).max() < 1e-8


@pytest.mark.parametrize("name", ["ee_n4", "eph_n4"])
def test_tuples_without_points_inside_contribute_exactly_zero(name):
    """The device quadrature visits only the Monte-Carlo points whose
    ThetapC * ThetaFC is 1 and drops the tuples that have none.  On the
    oracle, one thread, reference order: the dropped tuples give exactly zero
    and the list without them gives the same operator bit for bit."""
    build, seed, kT = cases()[name]
    mat = build()
    f0 = W.initial_status(mat, kT=kT, seed=seed).vec
    o = oracle.Oracle(mat, nthreads=1)
    for ch, c in enumerate(mat.channels):
        n_in, p_in, cnt = o.points_inside(ch, per_tuple=True)
        assert n_in == np.count_nonzero(cnt) and p_in == cnt.sum()
        assert 0 < p_in < cnt.size * c.numMCPoints
        ids, umk = o.tuples(ch)
        full = o.channel_propagate(ch, f0)
        sub = oracle.Oracle(mat, enumerate_tuples=False, nthreads=1)
        if n_in < cnt.size:
            sub.set_tuples(ch, ids[cnt == 0], umk[cnt == 0])
            assert not np.any(sub.channel_propagate(ch, f0))
        sub.set_tuples(ch, ids[cnt > 0], umk[cnt > 0])
        assert np.array_equal(sub.channel_propagate(ch, f0), full)


@pytest.mark.parametrize("name", ["ee_n4", "ee2_n3", "eph_n4"])
def test_item_ranges_concatenate_to_the_full_enumeration(name):
    """The work-item index of the streamed walk (umklapp, sections of legs
    0..L-2, element choice; the reference's loop order): enumerating item
    ranges and concatenating them gives the full list, in order."""
    build, _, _ = cases()[name]
    mat = build()
    full = oracle.Oracle(mat)
    part = oracle.Oracle(mat, enumerate_tuples=False)
    pk = mat.pack()
    for ch in range(len(mat.channels)):
        cd = pk.desc.channels[ch]
        n_items = cd.n_umklapp * 2 ** (cd.nlegs - 1)
        for l in range(cd.nlegs - 1):
            m = pk.desc.meshes[pk.desc.bands[cd.band[l]].mesh]
            n_items *= m.nsplit[0] * m.nsplit[1]
        ids, umk = full.tuples(ch)
        cuts = [0, n_items // 7, n_items // 2, n_items - 1, n_items]
        got_ids, got_umk = [], []
        for a, b in zip(cuts[:-1], cuts[1:]):
            part.enumerate_items(ch, a, b)
            i, u = part.tuples(ch)
            got_ids.append(i)
            got_umk.append(u)
        assert np.array_equal(np.concatenate(got_ids), ids)
        assert np.array_equal(np.concatenate(got_umk), umk)
