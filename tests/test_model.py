"""Host-side model: wildcard matching, channel deduplication, mesh geometry."""
import numpy as np

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
    mat = W.config0(3)
    c = mat.channels[0]
    assert c.mc_points.shape == (50, 5) and c.mc_points_precalc.shape == (50, 5)
    assert not np.array_equal(c.mc_points, c.mc_points_precalc)
