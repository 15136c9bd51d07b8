"""Known answers of the scheme, checked on the oracle (reference algorithm)."""
import numpy as np


def test_uniform_freestream_is_a_fixed_point(oracle_lib, small_cloud):
    from mfcfd import cloud
    o = oracle_lib.Oracle(small_cloud, 0.6, 3.0)
    o.set_prim(cloud.freestream_prim(small_cloud.n, 0.6, 3.0))
    o.step(1)
    assert np.all(o.get(oracle_lib.FIELD_DQ) == 0.0)
    assert np.all(o.get(oracle_lib.FIELD_FLUX_RES) == 0.0)


def test_lsq_gradient_of_linear_field(oracle_lib, small_cloud):
    """q-derivatives of prim with ln(rho) linear in x: exact gradient in q1."""
    c = small_cloud
    prim = np.tile(np.array([1.0, 0.0, 0.0, 0.0, 1 / 1.4]), (c.n, 1))
    prim[:, 0] = np.exp(0.01 * c.x)
    prim[:, 4] = prim[:, 0] / 1.4            # beta constant -> q1 = ln rho + const
    o = oracle_lib.Oracle(c, 0.0, 0.0)
    o.set_prim(prim)
    o.step(1)
    dq = o.get(oracle_lib.FIELD_DQ).reshape(c.n, 5, 3)
    np.testing.assert_allclose(dq[:, 0, 0], 0.01, rtol=1e-9)
    np.testing.assert_allclose(dq[:, 0, 1:], 0.0, atol=1e-11)


def test_dinv_positive_and_residual_finite(oracle_lib, small_cloud):
    from mfcfd import cloud
    o = oracle_lib.Oracle(small_cloud, 0.4, 0.0)
    o.set_prim(cloud.initial_state(small_cloud, 0.4, 0.0))
    r = [o.step(t)[0] for t in range(1, 6)]
    assert np.all(np.isfinite(r)) and r[0] > 0
    dinv = o.get(oracle_lib.FIELD_DINV)
    swept = dinv != 0
    assert swept.sum() > 0.9 * small_cloud.n * 0.7 and np.all(dinv[swept] > 0)
