"""500 FP64 iterations of the 62,400-point sphere against the reference.

The fixture (tests/golden/sphere_62k_500.npz, made by make_sphere62k.py)
holds the reference's own routines (translated to C) run on this cloud at
Mach 0.4, alpha 0 from the impulsive start, twice: with glibc's exp/log/erf,
as the Fortran program calls them, and with the solver's own (mfmath).

Tolerances:
  - against the mfmath build, prim is the same bits at iterations 1, 10, 100
    and 500 (SHA-256 of the (N, 5) array), and res_new agrees within 1e-13
    relative at every iteration (the GPU's reduction sums in another order);
  - against the glibc build, res_new agrees within 1e-10 relative at every
    iteration, and CL and CD within 1e-10 of the force scale max(|CL|, |CD|)
    at the snapshots (CL of a sphere at alpha 0 is near zero, so a relative
    bound on CL alone would measure cancellation, not the solver).
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(__file__), "golden", "sphere_62k_500.npz")


@pytest.fixture(scope="module")
def fixture():
    with np.load(FIX) as z:
        return {k: z[k] for k in z.files}


def _cloud_sha256(c):
    h = hashlib.sha256()
    for a in (c.status, c.x, c.y, c.z, c.tan1, c.tan2, c.nor, c.nbhs, c.conn, c.min_dist):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_sphere62k_500_iterations(fixture, mfcfd_lib):
    from mfcfd import cloud
    from mfcfd.solver import Solver
    meta = json.loads(str(fixture["meta"]))
    c = cloud.sphere_62k()
    assert _cloud_sha256(c) == meta["cloud_sha256"], "the regenerated cloud differs from the fixture's"
    s = Solver(c, meta["mach"], meta["aoa"])
    s.initial_conditions(cloud.initial_state(c, meta["mach"], meta["aoa"]))
    hist, t = [], 1
    for k, snap in enumerate(meta["snaps"]):
        hist.append(s.q_lskum(snap - t + 1, t0=t))
        t = snap + 1
        prim = s.get(mfcfd_lib.FIELD_PRIM)
        sha = hashlib.sha256(np.ascontiguousarray(prim).tobytes()).hexdigest()
        assert sha == str(fixture["mfmath_prim_sha256"][k]), f"prim differs from the mfmath build at t={snap}"
        cl_, cd_, _ = s.forces()
        ref_cl, ref_cd = float(fixture["glibc_cl"][k]), float(fixture["glibc_cd"][k])
        scale = max(abs(ref_cl), abs(ref_cd))
        assert abs(cl_ - ref_cl) <= 1e-10 * scale, (snap, cl_, ref_cl)
        assert abs(cd_ - ref_cd) <= 1e-10 * scale, (snap, cd_, ref_cd)
    hist = np.vstack(hist)
    np.testing.assert_allclose(hist[:, 0], fixture["mfmath_res"][:, 0], rtol=1e-13, atol=0)
    np.testing.assert_allclose(hist[:, 0], fixture["glibc_res"][:, 0], rtol=1e-10, atol=0)
    s.close()
