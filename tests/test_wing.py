"""The seeded swept-wing cloud generator, checked on the host at a small
size (the same construction as the 4.2M-point workload with a 80 x 24 wall
grid and 60,000 target points)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def small_wing():
    from mfcfd import wing
    return wing.swept_wing(points=60_000, nc=80, ns=24, name="wing-60k")


def test_wing_lists_are_usable(small_wing):
    """Every interior and wall point's six split lists have at least three
    members and a non-singular 3x3 least-squares system."""
    c = small_wing
    assert c.bad_lists == 0 and c.bad_wall_lists == 0
    counts = c.counts()
    assert counts["wall"] == 80 * 24 + 3 * 20     # surface grid and tip face
    assert counts["interior"] > 0.7 * c.n and counts["outer"] > 0
    # no list overflows the reference's 22-entry storage, and the library's
    # set-up takes the cloud
    from mfcfd.solver import Solver
    s = Solver(c, 0.84, 3.06, device=-1)
    info = s.info()
    s.close()
    assert info["split_overflows"] == 0
    assert info["n_wall"] == counts["wall"]


def test_wing_geometry(small_wing):
    from mfcfd import wing
    from mfcfd.cloud import STATUS_WALL
    c = small_wing
    pts = np.stack([c.x, c.y, c.z], axis=1)
    vol = c.status != STATUS_WALL
    assert not wing.inside_wing(pts[vol]).any()
    # frames: unit, orthogonal, right-handed
    for a in (c.tan1, c.tan2, c.nor):
        np.testing.assert_allclose(np.linalg.norm(a, axis=1), 1.0, atol=1e-12)
    np.testing.assert_allclose(np.einsum("ij,ij->i", c.tan1, c.nor), 0.0, atol=1e-12)
    np.testing.assert_allclose(np.cross(c.tan1, c.tan2), c.nor, atol=1e-12)
    # wall normals point out of the wing: a short step along them leaves it
    w = c.status == STATUS_WALL
    assert not wing.inside_wing(pts[w] + 1e-4 * c.nor[w]).any()
    assert wing.inside_wing(pts[w] - 1e-4 * c.nor[w]).mean() > 0.95
    # no neighbour is seen through the wing
    for i in np.nonzero(w)[0][::7]:
        k = c.conn[i, :c.nbhs[i]] - 1
        mid = 0.5 * (pts[k] + pts[i])
        assert not wing._deep_inside(mid).any()
    # per-point areas add up to the surface area of both sides and the tip
    assert c.wall_areas is not None
    s = np.sum(c.wall_areas)
    assert 1.5 < s < 1.7 and abs(s - c.wall_area) < 1e-12


def test_wing_is_seeded():
    from mfcfd import wing
    a = wing.swept_wing(points=20_000, nc=40, ns=12, seed=9)
    b = wing.swept_wing(points=20_000, nc=40, ns=12, seed=9)
    assert a.n == b.n and np.array_equal(a.x, b.x) and np.array_equal(a.conn, b.conn)
