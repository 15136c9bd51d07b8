"""The 62,400-point sphere fixture on the host.

The fixture holds the reference's own routines (translated to C) run for
500 iterations with glibc's exp/log/erf and with the solver's own.  The two
differ only in the last bits of the transcendentals; over the 500
iterations their density residuals stay within 1e-10 relative of each other
(limiter branches do not flip apart) and their forces agree to 1e-10 of the
force scale.  That is what lets the GPU, which computes the mfmath build's
bits, meet the 1e-10 bound against the glibc build.  The cloud regenerates
to the same bytes from its seed.
"""
import hashlib
import json
import os

import numpy as np

FIX = os.path.join(os.path.dirname(__file__), "golden", "sphere_62k_500.npz")


def test_fixture_cloud_regenerates():
    from mfcfd import cloud
    with np.load(FIX) as z:
        meta = json.loads(str(z["meta"]))
    c = cloud.sphere_62k()
    h = hashlib.sha256()
    for a in (c.status, c.x, c.y, c.z, c.tan1, c.tan2, c.nor, c.nbhs, c.conn, c.min_dist):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == meta["cloud_sha256"]
    assert c.n == meta["n"]


def test_glibc_and_mfmath_builds_stay_within_tolerance():
    with np.load(FIX) as z:
        g, m = z["glibc_res"], z["mfmath_res"]
        cl = (z["glibc_cl"], z["mfmath_cl"])
        cd = (z["glibc_cd"], z["mfmath_cd"])
    assert g.shape == (500, 2)
    np.testing.assert_allclose(m[:, 0], g[:, 0], rtol=1e-10, atol=0)
    scale = np.maximum(np.abs(cl[0]), np.abs(cd[0]))
    assert np.all(np.abs(cl[0] - cl[1]) <= 1e-10 * scale)
    assert np.all(np.abs(cd[0] - cd[1]) <= 1e-10 * scale)
