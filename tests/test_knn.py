"""Connectivity from raw points (mfcfd_knn), on the host's threads.

The answer is defined exactly -- the k points j != i of smallest (d2, j),
d2 = dx*dx + dy*dy + dz*dz with dx = x[j] - x[i] -- so it is checked against
a k-d tree query (scipy's cKDTree, which orders by the same distances) on
the generator's clouds, and against a brute-force numpy evaluation of the
definition on a small cloud with exact ties.
"""
import numpy as np
import pytest


def _kdtree(pts, k):
    from scipy.spatial import cKDTree
    dist, idx = cKDTree(pts).query(pts, k=k + 1)
    return idx[:, 1:] + 1


@pytest.mark.parametrize("name", ["small", "ellipsoid", "62k"])
def test_knn_host_matches_kdtree(mfcfd_lib, name):
    from mfcfd import cloud
    c = {"small": cloud.small_sphere, "62k": cloud.sphere_62k,
         "ellipsoid": lambda: cloud.shell_cloud(14, 900, r1=3.0, seed=77, aspect=(1.0, 1.8, 2.6))}[name]()
    pts = np.stack([c.x, c.y, c.z], 1)
    nbhs, conn, md = cloud.knn(c.x, c.y, c.z, 26, device=-1)
    assert np.all(nbhs == 26)
    assert np.array_equal(conn[:, :26], _kdtree(pts, 26))
    assert np.all(conn[:, 26:] == 0)
    k = conn[:, 0] - 1
    d = pts[k] - pts
    assert np.array_equal(md, np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]))


def test_knn_ties_by_index(mfcfd_lib):
    """A lattice has many equal distances: the order is (d2, index)."""
    from mfcfd import cloud
    g = np.arange(6, dtype=np.float64)
    x, y, z = (a.ravel() for a in np.meshgrid(g, g, g, indexing="ij"))
    n = x.shape[0]
    for k in (6, 18, 26):
        nbhs, conn, md = cloud.knn(x, y, z, k, device=-1)
        for i in range(n):
            d2 = (x - x[i]) * (x - x[i]) + (y - y[i]) * (y - y[i]) + (z - z[i]) * (z - z[i])
            order = sorted((d2[j], j) for j in range(n) if j != i)[:k]
            assert list(conn[i, :k] - 1) == [j for _, j in order]
            assert md[i] == np.sqrt(order[0][0])


def test_knn_rejects_duplicates_and_tiny_clouds(mfcfd_lib):
    from mfcfd import cloud
    from mfcfd._lib import MfcfdError
    x = np.array([0.0, 1.0, 1.0, 2.0])
    y = np.zeros(4)
    z = np.zeros(4)
    with pytest.raises(MfcfdError, match="coincide"):
        cloud.knn(x, y, z, 2, device=-1)
    with pytest.raises(MfcfdError, match="no more than k"):
        cloud.knn(np.arange(3.0), np.zeros(3), np.zeros(3), 3, device=-1)
    with pytest.raises(MfcfdError):
        cloud.knn(np.arange(30.0), np.zeros(30), np.zeros(30), 28, device=-1)
