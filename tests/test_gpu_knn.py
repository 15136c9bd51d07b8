"""mfcfd_knn on the GPU gives the host's arrays exactly (the answer is
defined by (d2, index); see tests/test_knn.py), on shell clouds, a lattice
full of equal distances, and the 1,104,000-point benchmark sphere."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _both(x, y, z, k):
    from mfcfd import cloud
    return cloud.knn(x, y, z, k, device=-1), cloud.knn(x, y, z, k, device=0)


@pytest.mark.parametrize("name", ["62k", "ellipsoid", "lattice", "1.1M"])
def test_knn_device_equals_host(mfcfd_lib, name):
    from mfcfd import cloud
    if name == "lattice":
        g = np.arange(9, dtype=np.float64)
        x, y, z = (a.ravel().copy() for a in np.meshgrid(g, g, g, indexing="ij"))
    else:
        c = {"62k": cloud.sphere_62k, "1.1M": cloud.sphere_1m,
             "ellipsoid": lambda: cloud.shell_cloud(14, 900, r1=3.0, seed=77, aspect=(1.0, 1.8, 2.6))}[name]()
        x, y, z = c.x, c.y, c.z
    for k in (26, 27) if name != "1.1M" else (26,):
        h, d = _both(x, y, z, k)
        for a, b in zip(h, d):
            assert np.array_equal(a, b), name
        if name == "1.1M":
            assert np.array_equal(d[1], c.conn) and np.array_equal(d[2], c.min_dist)


def test_knn_device_rejects_duplicates(mfcfd_lib):
    from mfcfd import cloud
    from mfcfd._lib import MfcfdError
    x = np.array([0.0, 1.0, 1.0, 2.0, 3.0])
    with pytest.raises(MfcfdError, match="coincide"):
        cloud.knn(x, np.zeros(5), np.zeros(5), 2, device=0)
