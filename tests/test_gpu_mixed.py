"""Mixed precision (MFCFD_PRECISION_MIXED) against the FP64 CPU oracle.

The mixed path evaluates the reconstruction, limiter and every flux of the
flux residual and of both sweeps in FP32; the least-squares sums and 3x3
solves, D_inv, the increments, the state update, the residual norm and the
forces stay FP64.  It is not bit-matched: each result is stated as its error
against the FP64 oracle on the same cloud, with the bounds written here.

Tolerances: |dCL|, |dCD| <= 1e-4 (absolute, the serving target) and the
pressure field within 1e-4 relative after the stated iteration counts; the
density residual history within 1e-3 relative.  Measured on B200 for these
cases the errors are near 1e-7, far inside the bounds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CL_TOL = 1e-4
PRESSURE_TOL = 1e-4
RES_TOL = 1e-3


def _mixed_vs_oracle(c, mach, aoa, iters, oracle_lib, precision=1):
    from mfcfd.cloud import initial_state
    from mfcfd.solver import Solver
    s = Solver(c, mach, aoa, precision=precision)
    o = oracle_lib.Oracle(c, mach, aoa, libm=oracle_lib.LIBM_MFMATH)
    prim0 = initial_state(c, mach, aoa)
    s.initial_conditions(prim0)
    o.set_prim(prim0)
    hist = s.q_lskum(iters)
    ref = np.array([o.step(t) for t in range(1, iters + 1)])
    return s, o, hist, ref


@pytest.mark.parametrize("mach,aoa,iters", [(0.8, 2.0, 60), (0.4, 0.0, 30)])
def test_mixed_precision_error_against_fp64_oracle(small_cloud, oracle_lib, mfcfd_lib, mach, aoa, iters):
    s, o, hist, ref = _mixed_vs_oracle(small_cloud, mach, aoa, iters, oracle_lib)
    np.testing.assert_allclose(hist[:, 0], ref[:, 0], rtol=RES_TOL)
    prim, prim_o = s.get(mfcfd_lib.FIELD_PRIM), o.get(oracle_lib.FIELD_PRIM)
    assert np.isfinite(prim).all()
    p_err = np.max(np.abs(prim[:, 4] - prim_o[:, 4]) / np.abs(prim_o[:, 4]))
    assert p_err <= PRESSURE_TOL, p_err
    cl, cd, _ = s.forces()
    clo, cdo, _ = oracle_lib.forces(small_cloud, prim_o, mach, aoa)
    assert abs(cl - clo) <= CL_TOL and abs(cd - cdo) <= CL_TOL, (cl - clo, cd - cdo)
    # the FP32 arithmetic really ran: the state is close to, not equal to, FP64
    assert not np.array_equal(prim, prim_o)
    s.close()


def test_mixed_precision_supersonic_and_inner_iterations(oracle_lib, mfcfd_lib):
    """Copies of supersonic points and second-order q-derivatives under mixed
    precision, against the FP64 oracle with the same options."""
    from mfcfd import _lib, cloud
    from mfcfd.cloud import initial_state
    from mfcfd.solver import Solver
    c = cloud.with_supersonic_boundary(cloud.small_sphere(7, 120, r1=1.6, seed=5))
    s = Solver(c, 0.6, 1.0, precision=_lib.PRECISION_MIXED, inner_iterations=1)
    o = oracle_lib.Oracle(c, 0.6, 1.0, libm=oracle_lib.LIBM_MFMATH, inner_iterations=1)
    prim0 = initial_state(c, 0.6, 1.0)
    s.initial_conditions(prim0)
    o.set_prim(prim0)
    hist = s.q_lskum(20)
    ref = np.array([o.step(t) for t in range(1, 21)])
    np.testing.assert_allclose(hist[:, 0], ref[:, 0], rtol=RES_TOL)
    prim_o = o.get(oracle_lib.FIELD_PRIM)
    p_err = np.max(np.abs(s.get(mfcfd_lib.FIELD_PRIM)[:, 4] - prim_o[:, 4]) / np.abs(prim_o[:, 4]))
    assert p_err <= PRESSURE_TOL, p_err
    s.close()


def test_mixed_precision_is_deterministic_alone_and_in_a_batch(mfcfd_lib):
    """The mixed path's arithmetic does not depend on scheduling: a repeated
    run, and the same cloud inside a batch, give identical bits."""
    from mfcfd import _lib, batch, cloud
    from mfcfd.solver import Solver
    clouds = [cloud.small_sphere(8, 150, seed=4), cloud.small_sphere(6, 100, r1=1.5, seed=3)]
    alone = []
    for rep in range(2):
        s = Solver(clouds[0], 0.8, 2.0, precision=_lib.PRECISION_MIXED)
        s.initial_conditions()
        s.q_lskum(8)
        alone.append(s.get(mfcfd_lib.FIELD_PRIM))
        s.close()
    assert np.array_equal(alone[0], alone[1])
    solvers = []
    for c, prec in zip(clouds, (_lib.PRECISION_MIXED, _lib.PRECISION_FP64)):
        s = Solver(c, 0.8, 2.0, precision=prec)
        s.initial_conditions()
        solvers.append(s)
    batch.run_batch(solvers, 8)
    assert np.array_equal(solvers[0].get(mfcfd_lib.FIELD_PRIM), alone[0])
    for s in solvers:
        s.close()


@pytest.mark.parametrize("mach,aoa,iters", [(0.8, 2.0, 60), (0.4, 0.0, 30)])
def test_defect_correction_error_against_fp64_oracle(small_cloud, oracle_lib, mfcfd_lib, mach, aoa, iters):
    """MFCFD_PRECISION_MIXED_DC: the flux residual in FP64, the sweeps in
    FP32; same bounds as the mixed form."""
    from mfcfd import _lib
    from oracle.oracle import forces
    s, o, hist, ref = _mixed_vs_oracle(small_cloud, mach, aoa, iters, oracle_lib, _lib.PRECISION_MIXED_DC)
    np.testing.assert_allclose(hist[:, 0], ref[:, 0], rtol=RES_TOL)
    pm = s.get(mfcfd_lib.FIELD_PRIM)
    po = o.get(oracle_lib.FIELD_PRIM)
    assert np.max(np.abs(pm[:, 4] - po[:, 4]) / np.abs(po[:, 4])) <= PRESSURE_TOL
    clm, cdm, _ = s.forces()
    clo, cdo, _ = forces(small_cloud, po, mach, aoa)
    assert abs(clm - clo) <= CL_TOL and abs(cdm - cdo) <= CL_TOL


def test_defect_correction_with_polish_converges_like_fp64(mfcfd_lib):
    """MIXED_DC tracks FP64 down to about a 1e-5 drop of the density
    residual; switched to FP64 there (mfcfd_set_precision), it reaches the
    1e-6 drop (residue -6) within a few per cent of FP64's iterations, and
    its forces agree with FP64's converged ones to 1e-4."""
    from mfcfd import _lib, batch, cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere()
    res = {}
    for prec, polish in ((_lib.PRECISION_FP64, None), (_lib.PRECISION_MIXED_DC, -5.0)):
        s = Solver(c, 0.8, 2.0, precision=prec)
        s.initial_conditions()
        r = batch.solve_batch([s], max_iters=12000, chunk=100, polish=polish)[0]
        res[prec] = (r, s.forces()[:2])
        s.close()
    r64, rdc = res[_lib.PRECISION_FP64][0], res[_lib.PRECISION_MIXED_DC][0]
    assert r64["converged"] and rdc["converged"], res
    assert rdc["polished"]
    assert rdc["iters"] <= 1.05 * r64["iters"] + 100, res
    (cl64, cd64), (cldc, cddc) = res[_lib.PRECISION_FP64][1], res[_lib.PRECISION_MIXED_DC][1]
    assert abs(cldc - cl64) <= CL_TOL and abs(cddc - cd64) <= CL_TOL


def test_precision_switch(mfcfd_lib):
    """FP64 and MIXED_DC handles switch either way between iterations: a
    MIXED_DC handle sweeps with folded weights and keeps the unfolded ones,
    which the switch to FP64 puts back bit for bit.  A MIXED handle (folded
    weights only) refuses; switching to FP64 before the first iteration gives
    the plain FP64 bits."""
    from mfcfd import _lib, cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere()
    a = Solver(c, 0.8, 2.0)
    a.initial_conditions()
    ha = a.q_lskum(5)
    b = Solver(c, 0.8, 2.0, precision=_lib.PRECISION_MIXED_DC)
    b.initial_conditions()
    assert b.digest("fwd_ent") != a.digest("fwd_ent")          # folded weights
    b.set_precision(_lib.PRECISION_FP64)
    assert b.digest("fwd_ent") == a.digest("fwd_ent") and b.digest("bwd_ent") == a.digest("bwd_ent")
    hb = b.q_lskum(5)
    assert np.array_equal(ha, hb)
    assert np.array_equal(a.get(mfcfd_lib.FIELD_PRIM), b.get(mfcfd_lib.FIELD_PRIM))
    b.set_precision(_lib.PRECISION_MIXED_DC)
    d = Solver(c, 0.8, 2.0, precision=_lib.PRECISION_MIXED_DC)
    assert b.digest("fwd_ent") == d.digest("fwd_ent") and b.digest("bwd_ent") == d.digest("bwd_ent")
    d.close()
    assert np.all(np.isfinite(b.q_lskum(5, t0=6)[:, 0]))
    m = Solver(c, 0.8, 2.0, precision=_lib.PRECISION_MIXED)
    with pytest.raises(_lib.MfcfdError):
        m.set_precision(_lib.PRECISION_FP64)
    for s in (a, b, m):
        s.close()
