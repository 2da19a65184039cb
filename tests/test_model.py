"""Host-side model: wildcard matching, channel deduplication, mesh geometry."""
import numpy as np
import pytest

from tortoise_b200 import IN, OUT, workloads as W
from tortoise_b200.model import Mesh, Region, match_string, random_points_reference


def test_match_string_semantics():
    assert match_string("el:*", "el:P")
    assert match_string("*", "")
    assert match_string("e?:*", "el:D")
    assert not match_string("pn:*", "el:P")
    assert match_string("*P", "el:P") and not match_string("*P", "el:D")


def test_wildcard_channel_dedup_counts():
    # {in,in,out,out} over 2 bands: unordered pairs of (in multiset, out multiset) = 6
    mat = W.build_material(3, ("P", "D"), (), ee=True, eph=False)
    assert len(mat.channels) == 6
    # e-ph {el:*, pn:*, el:*} {in,in,out}: 2 x 1 x 2 = 4 distinct channels
    mat = W.build_material(3, ("P", "D"), (0.2,), ee=False, eph=True)
    assert len(mat.channels) == 4
    names = sorted(c.scatteringName() for c in mat.channels)
    assert names[0] == "[(el:D)(pn:0)]-[(el:D)]"


def test_mesh_geometry():
    r = Region((-1.0, -1.0), ((2.0, 0.0), (0.0, 2.0)))
    m = Mesh(r, (0.0, 0.0), (1.0, 1.0), (4, 4))
    v = m.vertices()
    assert v.shape == (32, 3, 2)
    assert np.allclose(v[0], [[-1, -1], [-0.5, -1], [-0.5, -0.5]])
    assert np.allclose(v[1], [[-1, -1], [-1, -0.5], [-0.5, -0.5]])
    assert np.isclose(m.elemVolume, 0.125)
    c = m.function(lambda x, y: x + 2 * y)
    assert np.allclose(c[:3], [-3.0, 0.5, 1.5])


def test_mc_points_in_reference_simplex():
    rng = np.random.default_rng(0)
    p = random_points_reference(rng, 2, 1000)
    assert (p >= 0).all() and (p.sum(axis=1) <= 1.0).all()
    mat = W.parabolic_ee(3)
    c = mat.channels[0]
    assert c.mc_points.shape == (50, 5) and c.mc_points_precalc.shape == (50, 5)
    assert not np.array_equal(c.mc_points, c.mc_points_precalc)


def test_observable_weights_against_the_oracle_integral():
    """J = w . f of tortoise_b200.adjoint equals the oracle's mass-matrix
    integral of f times the weight function (1, E, or dE/dk)."""
    import oracle
    from tortoise_b200 import adjoint as A
    from tortoise_b200 import workloads as W
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True)
    f = W.initial_status(mat, kT=0.1, seed=2).vec
    o = oracle.Oracle(mat, enumerate_tuples=False)
    offs, _ = mat.band_offsets()
    for b, band in enumerate(mat.bands):
        n = band.mesh.ne * 3
        fb = f[offs[b]:offs[b] + n]
        one = np.tile([1.0, 0.0, 0.0], band.mesh.ne)
        assert abs(A.observable_weights(mat, b, "density") @ f - o.integrate(b, fb, one)) < 1e-14
        want = o.integrate(b, fb, band.dispersion_coeffs)
        assert abs(A.observable_weights(mat, b, "energy") @ f - want) <= 1e-13 * abs(want)


def test_current_weights_of_a_linear_dispersion():
    """For E = a kx + b ky the band velocity is (a, b) on every element, so
    the current of f = 1 is (a, b) times the k-space area."""
    from tortoise_b200 import adjoint as A
    from tortoise_b200.model import FERMION, Material, Mesh, Region
    region = Region((-1.0, -1.0), ((2.0, 0.0), (0.0, 2.0)))
    mesh = Mesh(region, (0.0, 0.0), (1.0, 1.0), (5, 3))
    mat = Material("lin", region)
    mat.addBand("el:L", -1.0, FERMION, mesh, lambda kx, ky: 0.7 * kx - 0.2 * ky)
    f = np.tile([1.0, 0.0, 0.0], mesh.ne)
    jx = A.observable_weights(mat, 0, "current", 0) @ f
    jy = A.observable_weights(mat, 0, "current", 1) @ f
    assert abs(jx - 0.7 * 4.0) < 1e-12 and abs(jy + 0.2 * 4.0) < 1e-12


def test_scatt_indices_reader_follows_the_reference_layout(tmp_path):
    """A file laid out as ScatteringChannel::precalculateIndices writes it
    (int32 mesh splits per leg, uint64 count, int32 ids + umklapp per tuple)
    is read back by the Python reader and by the C ABI (no device needed);
    other mesh splits are refused, as the reference refuses them."""
    import ctypes as C
    import struct
    from tortoise_b200 import engine
    from tortoise_b200.model import read_scatt_indices
    ids = np.array([[1, 2, 3], [4, 5, 6], [7, 8, 9], [10, 11, 12]], dtype=np.int32)
    umk = np.array([0, 3, 1, 2], dtype=np.int32)
    path = tmp_path / "[(el:P)(pn:0)]-[(el:P)].scattIndices"
    with open(path, "wb") as fh:
        fh.write(struct.pack("<6i", 4, 4, 4, 4, 4, 4))
        fh.write(struct.pack("<Q", 4))
        for r, u in zip(ids, umk):
            fh.write(struct.pack("<4i", *r, u))
    got_ids, got_umk = read_scatt_indices(str(path), 3, [4] * 6)
    assert np.array_equal(got_ids, ids) and np.array_equal(got_umk, umk)
    assert read_scatt_indices(str(path), 3, [8] * 6) == (None, None)
    L = engine.lib()
    n = C.c_int64()
    ns = (C.c_int32 * 6)(*([4] * 6))
    assert L.tb_read_scatt_indices(str(path).encode(), 3, ns, C.byref(n), None, None, 0) == 0 and n.value == 4
    cids, cumk = np.zeros(12, dtype=np.int32), np.zeros(4, dtype=np.int32)
    ip = C.POINTER(C.c_int32)
    assert L.tb_read_scatt_indices(str(path).encode(), 3, ns, C.byref(n), cids.ctypes.data_as(ip),
                                   cumk.ctypes.data_as(ip), 4) == 0
    assert np.array_equal(cids.reshape(4, 3), ids) and np.array_equal(cumk, umk)
    bad = (C.c_int32 * 6)(*([8] * 6))
    assert L.tb_read_scatt_indices(str(path).encode(), 3, bad, C.byref(n), None, None, 0) == 1   # TB_ERR_BAD_DESC
    assert L.tb_read_scatt_indices(str(path).encode(), 3, ns, C.byref(n), cids.ctypes.data_as(ip),
                                   cumk.ctypes.data_as(ip), 2) == 9                              # TB_ERR_CAPACITY


def test_tuple_cache_content_hash():
    """Equal inputs give equal digests; a changed survival table, threshold or
    dispersion changes the channel's digest."""
    a = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True)
    b = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True)
    assert [c.content_hash() for c in a.channels] == [c.content_hash() for c in b.channels]
    h0 = b.channels[0].content_hash()
    b.channels[0].constructMCPoints(seed=12345)
    assert b.channels[0].content_hash() != h0
    c = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True)
    c.channels[1].scattElemeThreshold *= 2
    assert c.channels[1].content_hash() != a.channels[1].content_hash()
    d = W.build_material(4, ("P", "H"), (0.2,), ee=False, eph=True)
    assert d.channels[3].content_hash() != a.channels[3].content_hash()


def test_material_status_save_load(tmp_path):
    """MaterialStatus::save / load (declared in the reference, defined here):
    round trip bit-exact; a status of another material is refused."""
    from tortoise_b200.model import MaterialStatus
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True)
    st = W.initial_status(mat, kT=0.1, seed=3)
    st.save(str(tmp_path / "s.bin"))
    back = MaterialStatus(mat).load(str(tmp_path / "s.bin"))
    assert np.array_equal(back.vec, st.vec)
    other = W.build_material(3, ("P", "D"), (0.2,), ee=False, eph=True)
    with pytest.raises(ValueError):
        MaterialStatus(other).load(str(tmp_path / "s.bin"))
