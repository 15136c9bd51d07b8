"""Synthetic cloud generator: deterministic, valid connectivity and frames."""
import numpy as np


def test_deterministic_and_valid():
    from mfcfd import cloud
    a = cloud.small_sphere()
    b = cloud.small_sphere()
    for k in ("x", "y", "z", "conn", "nor", "min_dist"):
        assert np.array_equal(getattr(a, k), getattr(b, k))
    n = a.n
    assert a.counts()["wall"] == 150 and a.counts()["outer"] == 150
    assert np.all(a.nbhs == 26)
    assert a.conn[:, :26].min() >= 1 and a.conn[:, :26].max() <= n
    assert np.all(a.conn[:, 26] == 0)
    assert np.all(a.conn[np.arange(n), 0] != np.arange(1, n + 1))
    for f in (a.tan1, a.tan2, a.nor):
        assert np.allclose(np.linalg.norm(f, axis=1), 1.0)
    assert np.allclose(np.sum(a.tan1 * a.nor, axis=1), 0.0, atol=1e-12)
    assert np.allclose(np.cross(a.tan1, a.tan2), a.nor, atol=1e-12)
    r = np.sqrt(a.x ** 2 + a.y ** 2 + a.z ** 2)
    assert np.allclose(r[a.status == 1], 0.5)
    w = a.status == 1
    assert np.allclose(a.nor[w] * r[w, None], np.stack([a.x, a.y, a.z], 1)[w])


def test_initial_state_has_no_wall_penetration():
    from mfcfd import cloud
    c = cloud.small_sphere()
    p = cloud.initial_state(c, 0.8, 2.0)
    w = c.status == 1
    assert np.allclose(np.sum(p[w, 1:4] * c.nor[w], axis=1), 0.0, atol=1e-15)
    assert np.all(p[~w] == np.array(cloud.freestream(0.8, 2.0)))
