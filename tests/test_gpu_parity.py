"""GPU parity: the CUDA library against the oracle and the golden fixtures.

Tolerances: tuple lists bit-exact (integer work); FP64 collision / drift /
RHS within 1e-12 relative L2 (only the summation order differs: FP64 atomics
and fused multiply-adds on the device); error norm within 1e-13 relative;
DP45: identical accept/reject sequences, dense outputs (fixed times) within
1e-11 relative L2.  The embedded error y5 - y4 is a difference of nearly
equal vectors, so a 1e-16 rounding difference of the RHS reaches the error
norm amplified by ~1/rtol; step sizes, and with them the time and state of
the last accepted step, therefore agree to ~1e-10 relative.
"""
import numpy as np
import pytest

import oracle
from conftest import golden, rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W
from tests.golden.make_golden import cases, tuple_hash

pytestmark = pytest.mark.gpu

CASES = list(cases().keys())


def _setup(name):
    build, seed, kT = cases()[name]
    mat = build()
    f0 = W.initial_status(mat, kT=kT, seed=seed).vec
    return mat, f0


@pytest.mark.parametrize("name", CASES)
def test_enumeration_bit_exact(gpu_lib, name):
    g = golden(name)
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=E.LAYOUT_MC64)
    for ch in range(len(mat.channels)):
        ids, umk = eng.tuples(ch)
        info = eng.channel_info(ch)
        assert [info["n_tuples"], info["n_prefilter"], info["n_det"]] == list(g["ch%d_counts" % ch])
        assert tuple_hash(ids, umk) == str(g["ch%d_hash" % ch])


@pytest.mark.parametrize("name", CASES)
def test_channel_and_rhs_parity_fp64(gpu_lib, name):
    g = golden(name)
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=E.LAYOUT_MC64)
    for ch in range(len(mat.channels)):
        assert rel_l2(eng.channel_propagate(ch, f0), g["ch%d_prop" % ch]) < 1e-12
    assert rel_l2(eng.rhs(f0, drift=True), g["rhs"]) < 1e-12
    assert rel_l2(eng.rhs(f0, drift=False), g["rhs_nodrift"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_relative_error_parity(gpu_lib, name):
    g = golden(name)
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=E.LAYOUT_MC64)
    r = eng.relative_error(g["err"], f0)
    assert abs(r - float(g["relerr"])) <= 1e-13 * float(g["relerr"])


@pytest.mark.parametrize("name", ["eph_n4", "eph_bath_n4", "ee_n3"])
def test_dp45_trajectory_parity(gpu_lib, name):
    """In the deterministic mode: the device trajectory is the same on every
    run, so the comparison with the oracle is decided once and for all."""
    g = golden(name)
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=E.LAYOUT_MC64, deterministic=True)
    r = eng.dp45(f0, 0.0, 0.4, 0.1)
    assert r["status"] == 0 and r["done"] == 1
    assert [r["attempts"], r["accepted"], r["rejected"], r["rhs_evals"]] == list(g["dp_stats"])
    assert np.allclose(r["dense_t"], g["dp_dense_t"], rtol=0, atol=1e-14)
    assert rel_l2(r["dense"], g["dp_dense"]) < 1e-11
    assert rel_l2(r["y"], g["dp_y"]) < 1e-9
    assert abs(r["t"] - float(g["dp_t"][0])) < 1e-9 * float(g["dp_t"][0])


def test_caller_supplied_tuples_match(gpu_lib):
    """A tuple list handed in (the .scattIndices path) gives the same operator."""
    name = "eph_n4"
    g = golden(name)
    mat, f0 = _setup(name)
    o = oracle.Oracle(mat)
    for ch, c in enumerate(mat.channels):
        c.tuples, c.tuple_umklapp = o.tuples(ch)
    eng = E.Engine(mat, layout=E.LAYOUT_MC64)
    assert rel_l2(eng.rhs(f0), g["rhs"]) < 1e-12
    assert eng.channel_info(0)["n_prefilter"] == -1


def test_larger_ee_against_live_oracle(gpu_lib):
    """1.7 M four-leg tuples at N=8."""
    mat = W.parabolic_ee(8)
    f0 = W.initial_status(mat, kT=0.1, seed=11).vec
    o = oracle.Oracle(mat)
    eng = E.Engine(mat, layout=E.LAYOUT_MC64)
    ids_o, umk_o = o.tuples(0)
    ids_g, umk_g = eng.tuples(0)
    assert np.array_equal(ids_o, ids_g) and np.array_equal(umk_o, umk_g)
    assert rel_l2(eng.rhs(f0), o.rhs(f0)) < 1e-12


@pytest.mark.parametrize("name", CASES + ["ee_n8"])
def test_points_inside_only_equal_the_full_quadrature(gpu_lib, name):
    """Monte-Carlo channels visit only the points whose ThetapC * ThetaFC is 1
    (decided once per handle, kept as a 64-bit mask per tuple, tuples without
    such a point dropped); the kept tuples and points are exactly the
    oracle's.  Pinned back to every point of every tuple, the operator and
    the scattering rates must not change: the skipped terms are the
    integrand times 0 (1e-12, the FP64 parity bar: FP64 atomics order,
    shared-memory partial sums, and fused rather than reference-order
    coordinates for points near a simplex edge)."""
    if name == "ee_n8":
        mat = W.parabolic_ee(8)
        f0 = W.initial_status(mat, kT=0.1, seed=11).vec
    else:
        mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=E.LAYOUT_MC64)
    chans = [c for c in range(len(mat.channels)) if eng.channel_info(c)["n_tuples"] > 0]
    assert chans and all(eng.schedule(c).get("inside_only") for c in chans)
    o = oracle.Oracle(mat)
    for c in chans:
        assert eng.points_inside(c) == o.points_inside(c)
    a, ra = eng.rhs(f0), eng.scattering_rates(f0)
    for c in chans:
        eng.set_schedule(c, 0, inside_only=False)
        assert "inside_only" not in eng.schedule(c)
    b, rb = eng.rhs(f0), eng.scattering_rates(f0)
    assert rel_l2(a, b) < 1e-12
    assert rel_l2(ra, rb) < 1e-12
    with pytest.raises(E.TortoiseError):
        eng.set_schedule(chans[0], 1)


@pytest.mark.parametrize("variant", ["umklapp", "nonsquare", "partial_mesh", "empty_channel", "zero_amplitude"])
def test_edge_cases(gpu_lib, variant):
    from tortoise_b200.model import Material, Mesh, Region, IN, OUT, FERMION, BOSON
    region = Region((-1.0, -1.0), ((2.0, 0.0), (0.0, 2.0)))
    if variant == "umklapp":
        mat = W.build_material(3, ("P",), (0.2,), ee=False, eph=False)
        for c in mat.addScatteringChannelsWildcards(["el:*", "pn:*", "el:*"], [IN, IN, OUT], 1):
            pass
        assert mat.channels[0].umklappUnitVectors.shape == (9, 2)
    elif variant == "nonsquare":
        mat = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.05, -0.02), mesh_nsplit=(5, 3))
    elif variant == "partial_mesh":
        mat = Material("partial", region)
        full = Mesh(region, (0.0, 0.0), (1.0, 1.0), (6, 6))
        part = Mesh(region, (0.2, 0.25), (0.5, 0.4), (4, 3))
        mat.addBand("pn:ac", 0, BOSON, full, lambda x, y: 0.05 + 0.1 * np.sqrt(x * x + y * y))
        mat.addBand("el:C", -1, FERMION, part, lambda x, y: 0.5 * (x * x + y * y))
        mat.addScatteringChannelsWildcards(["el:*", "pn:*", "el:*"], [IN, IN, OUT], 0)
    elif variant == "empty_channel":
        mat = W.build_material(3, ("P",), (50.0,), ee=False, eph=True)
    else:
        mat = W.build_material(3, ("P", "D"), (0.2,), ee=False, eph=True)
        mat.channels[1].amplitude = 0.0
    f0 = W.initial_status(mat, seed=7).vec
    o = oracle.Oracle(mat)
    eng = E.Engine(mat, layout=E.LAYOUT_MC64)
    for ch in range(len(mat.channels)):
        a, ua = o.tuples(ch)
        b, ub = eng.tuples(ch)
        assert np.array_equal(a, b) and np.array_equal(ua, ub)
    ref = o.rhs(f0)
    got = eng.rhs(f0)
    if np.linalg.norm(ref) == 0.0:
        assert np.linalg.norm(got) == 0.0
    else:
        assert rel_l2(got, ref) < 1e-12


def test_bad_descriptions_are_rejected(gpu_lib):
    mat = W.parabolic_ee(3)
    mat.channels[0].tuples = np.array([[0, 1, 2, 99999]], dtype=np.int32)
    mat.channels[0].tuple_umklapp = np.array([0], dtype=np.int32)
    with pytest.raises(E.TortoiseError) as ei:
        E.Engine(mat)
    assert ei.value.rc == 1


@pytest.mark.parametrize("name", ["ee_n3", "ee2_n3", "eph_n4", "eph_bath_n4"])
def test_tensor_layout_fp64_parity(gpu_lib, name):
    """Precomputed moment tensor, FP64 storage: same operator as the MC
    quadrature up to summation order."""
    g = golden(name)
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=E.LAYOUT_T64)
    assert all(eng.channel_info(c)["layout"] == "t64" for c in range(len(mat.channels))
               if eng.channel_info(c)["n_tuples"] > 0)
    for ch in range(len(mat.channels)):
        assert rel_l2(eng.channel_propagate(ch, f0), g["ch%d_prop" % ch]) < 1e-12
    assert rel_l2(eng.rhs(f0, drift=True), g["rhs"]) < 1e-12


@pytest.mark.parametrize("name", ["eph_n4", "ee_n3"])
def test_tensor_layout_fp32_error_bound(gpu_lib, name):
    """FP32 moment storage with FP64 accumulation: relative error against
    the FP64 oracle stays below 1e-6 on the collision term (measured: about
    1e-7)."""
    g = golden(name)
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=E.LAYOUT_T32, allow_fp32=True)
    assert rel_l2(eng.rhs(f0, drift=False), g["rhs_nodrift"]) < 1e-6


@pytest.mark.parametrize("layout,name_l,tol", [(E.LAYOUT_T40, "t40", 2e-8), (E.LAYOUT_T48, "t48", 2e-10)])
@pytest.mark.parametrize("name", ["eph_n4", "ee_n3", "ee2_n3", "eph_bath_n4"])
def test_tensor_layout_40_and_48bit_error_bound(gpu_lib, name, layout, name_l, tol):
    """Moments stored as the upper 40 bits of FP64 (sign, exponent, 28
    mantissa bits, rounded: 2^-29 relative) or the upper 48 bits (2^-37),
    rebuilt into FP64 registers: every channel and the RHS within 2e-8
    (40-bit) or 2e-10 (48-bit) relative L2 of the FP64 oracle (FP32 storage
    gives ~1.2e-7; 40 bits are 32x finer, 48 bits 8192x)."""
    g = golden(name)
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=layout)
    for ch in range(len(mat.channels)):
        if eng.channel_info(ch)["n_tuples"] > 0:
            assert eng.channel_info(ch)["layout"] == name_l
        assert rel_l2(eng.channel_propagate(ch, f0), g["ch%d_prop" % ch]) < tol
    assert rel_l2(eng.rhs(f0, drift=False), g["rhs_nodrift"]) < tol


@pytest.mark.parametrize("layout,tol", [(E.LAYOUT_MC64, 1e-12), (E.LAYOUT_T64, 1e-12), (E.LAYOUT_T40, 2e-8),
                                        (E.LAYOUT_T48, 2e-10), (E.LAYOUT_T32, 1e-6)])
@pytest.mark.parametrize("name", CASES)
def test_scattering_rates_parity(gpu_lib, name, layout, tol):
    """tb_scattering_rates (ScatteringChannel::scatteringRates /
    MaterialStatus::scatteringRates) against the oracle's golden rates, per
    channel and for the whole status; FP64 layouts to 1e-12, reduced-precision
    storage to its stated bound."""
    g = golden(name)
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=layout)
    assert rel_l2(eng.scattering_rates(f0), g["rates"]) < tol
    for ch in range(len(mat.channels)):
        ref = g["ch%d_rates" % ch]
        got = eng.scattering_rates(f0, ch)
        if np.linalg.norm(ref) == 0.0:
            assert np.linalg.norm(got) == 0.0
        else:
            assert rel_l2(got, ref) < tol


def test_scattering_rates_per_leg_and_errors(gpu_lib):
    """Single legs against the live oracle, the reference-shaped Material API,
    and argument checks."""
    mat, f0 = _setup("eph_n4")
    o = oracle.Oracle(mat)
    eng = mat.engine()
    for ch, c in enumerate(mat.channels):
        for leg in range(c.nlegs):
            assert rel_l2(eng.scattering_rates(f0, ch, leg), o.scattering_rates(f0, ch, leg)) < 1e-12
    from tortoise_b200.model import IN, OUT, MaterialStatus
    st = MaterialStatus(mat, f0)
    offs, _ = mat.band_offsets()
    b = mat.id("el:P")
    want = sum(o.scattering_rates(f0, ch, leg) for ch, c in enumerate(mat.channels)
               if mat.band_names[c.legBandNumber[0]] in ("el:P", "el:D")
               for leg in range(c.nlegs) if c.legBandNumber[leg] == b)
    got = mat.scatteringRates(["el:*", "pn:*", "el:*"], [IN, IN, OUT], st, "el:P")
    assert rel_l2(got, want[offs[b]:offs[b] + got.size]) < 1e-12
    assert rel_l2(st.scatteringRates().vec, o.scattering_rates(f0)) < 1e-12
    with pytest.raises(E.TortoiseError):
        eng.scattering_rates(f0, len(mat.channels), -1)
    with pytest.raises(E.TortoiseError):
        eng.scattering_rates(f0, 0, 3)


def test_tuple_cache_round_trip(gpu_lib, tmp_path):
    """Tuple lists enumerated on the device, written in the reference's
    .scattIndices format, read back into a fresh material: the second handle
    skips enumeration and gives the same operator; a channel whose inputs
    changed (other survival points) is not taken from the cache."""
    from tortoise_b200.model import read_scatt_indices
    mat, f0 = _setup("eph_n4")
    eng = E.Engine(mat, layout=E.LAYOUT_T64)
    ref = eng.rhs(f0)
    mat.save_tuple_cache(str(tmp_path), eng)
    for ch, c in enumerate(mat.channels):
        path = mat.cache_path(str(tmp_path), ch)
        ids, umk = eng.tuples(ch)
        n = ids.shape[0]
        assert (tmp_path / path.split("/")[-1]).stat().st_size == 8 * c.nlegs + 8 + 4 * n * (c.nlegs + 1)
        rid, rumk = read_scatt_indices(path, c.nlegs)
        assert np.array_equal(rid, ids) and np.array_equal(rumk, umk)
    mat2, _ = _setup("eph_n4")
    mat2.channels[2].constructMCPoints(seed=999)      # its cached list is stale now
    loaded = mat2.load_tuple_cache(str(tmp_path))
    assert loaded == [0, 1, 3]
    mat2.channels[2].constructMCPoints(seed=mat.channels[2].mc_seed)
    eng2 = E.Engine(mat2, layout=E.LAYOUT_T64)
    for ch in (0, 1, 3):
        assert eng2.channel_info(ch)["n_prefilter"] == -1          # supplied, not enumerated
    assert eng2.channel_info(2)["n_prefilter"] > 0
    assert rel_l2(eng2.rhs(f0), ref) < 1e-13


@pytest.mark.parametrize("layout,etol", [(E.LAYOUT_MC64, 1e-12), (E.LAYOUT_T64, 1e-12), (E.LAYOUT_T40, 1e-8),
                                         (E.LAYOUT_T48, 1e-10), (E.LAYOUT_T32, 1e-6)])
@pytest.mark.parametrize("name", CASES)
def test_device_operator_conserves(gpu_lib, name, layout, etol):
    """Collision term of the device operator.  Electron number: every channel
    here pairs each electron in leg with an electron out leg, and the
    zeroth-moment output of a tuple is one number shared by all its legs, so
    number is conserved to 1e-12 of the sum of magnitudes for every storage
    layout.  Energy: the P1 delta makes sum_l dir_l E_l = 0 at every
    Monte-Carlo point, which the FP64 layouts keep to 1e-12; reduced-precision
    moments round the moments of that identity one by one, so it holds to
    their precision (1e-8 for 40-bit, 1e-6 for FP32 storage)."""
    from tortoise_b200.adjoint import observable_weights
    mat, f0 = _setup(name)
    eng = E.Engine(mat, layout=layout)
    d = eng.rhs(f0, drift=False)
    tot_n = scale_n = tot_e = scale_e = 0.0
    for b, band in enumerate(mat.bands):
        if band.constrained:
            continue
        we = observable_weights(mat, b, "energy")
        tot_e += float(we @ d)
        scale_e += float(np.abs(we) @ np.abs(d))
        if band.statistics == -1:
            wn = observable_weights(mat, b, "density")
            tot_n += float(wn @ d)
            scale_n += float(np.abs(wn) @ np.abs(d))
    assert abs(tot_n) <= 1e-12 * scale_n, (tot_n, scale_n)
    if not any(b.constrained for b in mat.bands):
        assert abs(tot_e) <= etol * scale_e, (tot_e, scale_e)
