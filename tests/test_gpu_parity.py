"""GPU iteration vs the CPU oracle on the same seeded clouds.

The oracle runs with the solver's own exp/log/erf (libm mode 1), so every
field must match bit for bit: the GPU path rounds every operation exactly as
the reference's FP64 build does.  Against the oracle with glibc's exp/log/erf
(what the Fortran reference calls) the fields agree to a few ulp per call;
the density residual is checked to 1e-10 relative, the tolerance the FP64 path is held to.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["PRIM", "U", "Q", "QM", "DQ", "DELT", "FLUX_RES", "DELUP", "DELUN"]


def _pair(cloud, mach, aoa, libm, oracle_lib, sweep_mode=0, inner_iterations=0, power=0.0,
          update_variant=0, sweep_variant=0):
    from mfcfd.solver import Solver
    from mfcfd.cloud import initial_state
    s = Solver(cloud, mach, aoa, sweep_mode=sweep_mode, inner_iterations=inner_iterations, power=power,
               update_variant=update_variant, sweep_variant=sweep_variant)
    o = oracle_lib.Oracle(cloud, mach, aoa, libm=libm, inner_iterations=inner_iterations, power=power,
                          update_variant=update_variant, sweep_variant=sweep_variant)
    prim0 = initial_state(cloud, mach, aoa)
    s.initial_conditions(prim0)
    o.set_prim(prim0)
    return s, o


def _field_ids(oracle_lib):
    from mfcfd import _lib
    return [(name, getattr(_lib, "FIELD_" + name), getattr(oracle_lib, "FIELD_" + name))
            for name in FIELDS]


@pytest.mark.parametrize("sweep_mode", [0, 1, 2])
@pytest.mark.parametrize("mach,aoa", [(0.4, 0.0), (0.8, 2.0)])
def test_one_iteration_bitexact(small_cloud, oracle_lib, mfcfd_lib, mach, aoa, sweep_mode):
    s, o = _pair(small_cloud, mach, aoa, oracle_lib.LIBM_MFMATH, oracle_lib, sweep_mode)
    r_gpu = s.fpi_solver(1)
    r_cpu = o.step(1)
    for name, fg, fo in _field_ids(oracle_lib):
        a, b = s.get(fg), o.get(fo)
        bad = np.argwhere(a.view(np.uint64) != b.view(np.uint64))
        assert bad.size == 0, f"{name}: {len(bad)} values differ, first {bad[:3]}"
    dinv_g = s.get(mfcfd_lib.FIELD_DINV)
    dinv_o = o.get(oracle_lib.FIELD_DINV)
    swept = dinv_o != 0
    assert np.array_equal(dinv_g[swept], dinv_o[swept])
    assert abs(r_gpu[0] - r_cpu[0]) <= 1e-13 * abs(r_cpu[0])


@pytest.mark.parametrize("sweep_mode", [0, 1, 2])
def test_twenty_iterations_bitexact(small_cloud, oracle_lib, mfcfd_lib, sweep_mode):
    s, o = _pair(small_cloud, 0.4, 0.0, oracle_lib.LIBM_MFMATH, oracle_lib, sweep_mode)
    if sweep_mode == 2:
        # the wall points' neighbour fluxes come from the kernel run before
        # the sweeps (k_g0), and still give the oracle's bits
        assert s.info()["g0_points"] > 0
    hist = s.q_lskum(20)
    for t in range(1, 21):
        rc = o.step(t)
        assert abs(hist[t - 1, 0] - rc[0]) <= 1e-12 * abs(rc[0])
    a, b = s.get(mfcfd_lib.FIELD_PRIM), o.get(oracle_lib.FIELD_PRIM)
    assert np.array_equal(a, b)


def test_against_glibc_oracle(small_cloud, oracle_lib, mfcfd_lib):
    s, o = _pair(small_cloud, 0.4, 0.0, oracle_lib.LIBM_GLIBC, oracle_lib)
    hist = s.q_lskum(50)
    for t in range(1, 51):
        rc = o.step(t)
        assert abs(hist[t - 1, 0] - rc[0]) <= 1e-10 * abs(rc[0]), t
    a, b = s.get(mfcfd_lib.FIELD_PRIM), o.get(oracle_lib.FIELD_PRIM)
    np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-14)


@pytest.mark.parametrize("inner", [1, 3])
def test_inner_iterations_bitexact(small_cloud, oracle_lib, mfcfd_lib, inner):
    """Second-order q-derivatives (q_derivatives.f90:116-201), every field."""
    s, o = _pair(small_cloud, 0.8, 2.0, oracle_lib.LIBM_MFMATH, oracle_lib, inner_iterations=inner)
    s.q_lskum(3)
    for t in range(1, 4):
        o.step(t)
    for name, fg, fo in _field_ids(oracle_lib):
        a, b = s.get(fg), o.get(fo)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("sweep_mode", [0, 1, 2])
def test_supersonic_boundary_bitexact(oracle_lib, mfcfd_lib, sweep_mode):
    """Status 5/6 points (nearest-neighbour copies in the sweeps and the state
    update, implicit_forward_and_reverse_sweeps.f90:38-51,
    state_update_implicit.f90:63-94), every field after 5 iterations."""
    from mfcfd import cloud
    c = cloud.with_supersonic_boundary(cloud.small_sphere(6, 100, r1=1.5))
    s, o = _pair(c, 0.8, 2.0, oracle_lib.LIBM_MFMATH, oracle_lib, sweep_mode)
    hist = s.q_lskum(5)
    for t in range(1, 6):
        rc = o.step(t)
        assert abs(hist[t - 1, 0] - rc[0]) <= 1e-13 * abs(rc[0])
    for name, fg, fo in _field_ids(oracle_lib):
        a, b = s.get(fg), o.get(fo)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("power,inner", [(2.0, 0), (0.5, 2)])
def test_weighted_least_squares_bitexact(small_cloud, oracle_lib, mfcfd_lib, power, inner):
    """power != 0: weights 1/dist**power in the q-derivative, flux, D_inv and
    sweep least squares (glibc pow on the host, as the oracle), every field."""
    s, o = _pair(small_cloud, 0.8, 2.0, oracle_lib.LIBM_MFMATH, oracle_lib, inner_iterations=inner, power=power)
    s.q_lskum(3)
    for t in range(1, 4):
        o.step(t)
    for name, fg, fo in _field_ids(oracle_lib):
        a, b = s.get(fg), o.get(fo)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("supersonic", [False, True])
def test_explicit_update_variant_bitexact(oracle_lib, mfcfd_lib, supersonic):
    """MFCFD_UPDATE_EXPLICIT (state_update.f90), every field after 4 iterations."""
    from mfcfd import cloud
    c = cloud.small_sphere(6, 100, r1=1.5)
    if supersonic:
        c = cloud.with_supersonic_boundary(c)
    s, o = _pair(c, 0.8, 2.0, oracle_lib.LIBM_MFMATH, oracle_lib, update_variant=1)
    hist = s.q_lskum(4)
    for t in range(1, 5):
        rc = o.step(t)
        assert abs(hist[t - 1, 0] - rc[0]) <= 1e-13 * abs(rc[0])
    for name, fg, fo in _field_ids(oracle_lib):
        a, b = s.get(fg), o.get(fo)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("sweep_mode", [0, 1, 2])
@pytest.mark.parametrize("supersonic,iters", [(False, 2), (True, 3)])
def test_backup_sweep_driver_bitexact(oracle_lib, mfcfd_lib, sweep_mode, supersonic, iters):
    """MFCFD_SWEEPS_BACKUP (implicit_forward_and_reverse_sweeps_backup.f90):
    index-order sweeps with outer points, terms from before the sweep where
    the producer comes later; every field, including D_inv of outer points.
    (The driver diverges at outer points after a few iterations in the
    reference too, so the runs are short.)"""
    from mfcfd import cloud
    c = cloud.small_sphere(6, 100, r1=1.5)
    if supersonic:
        c = cloud.with_supersonic_boundary(c)
    s, o = _pair(c, 0.8, 2.0, oracle_lib.LIBM_MFMATH, oracle_lib, sweep_mode, sweep_variant=1)
    hist = s.q_lskum(iters)
    for t in range(1, iters + 1):
        rc = o.step(t)
        assert abs(hist[t - 1, 0] - rc[0]) <= 1e-13 * abs(rc[0])
    for name, fg, fo in _field_ids(oracle_lib):
        a, b = s.get(fg), o.get(fo)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name
    dinv_g, dinv_o = s.get(mfcfd_lib.FIELD_DINV), o.get(oracle_lib.FIELD_DINV)
    assert np.array_equal(dinv_g[dinv_o != 0], dinv_o[dinv_o != 0])


def test_forces_match_oracle(small_cloud, oracle_lib, mfcfd_lib):
    """CL/CD of the state after 10 iterations against the oracle's state and a
    sequential wall sum: within 1e-10 relative (the sums' order differs)."""
    s, o = _pair(small_cloud, 0.8, 2.0, oracle_lib.LIBM_MFMATH, oracle_lib)
    s.q_lskum(10)
    for t in range(1, 11):
        o.step(t)
    cl, cd, f = s.forces()
    clo, cdo, fo = oracle_lib.forces(small_cloud, o.get(oracle_lib.FIELD_PRIM), 0.8, 2.0)
    assert abs(cl - clo) <= 1e-10 * abs(clo) and abs(cd - cdo) <= 1e-10 * abs(cdo)
    np.testing.assert_allclose(f, fo, rtol=1e-10)


@pytest.mark.parametrize("chain_warps", [0, 400])
def test_batch_equals_separate_runs(oracle_lib, mfcfd_lib, chain_warps):
    """mfcfd_run_batch over clouds of different sizes and flows gives each
    cloud exactly its separate run (400 warps per cloud forces waves)."""
    from mfcfd import batch, cloud
    from mfcfd.solver import Solver
    clouds = [cloud.small_sphere(6, 100, r1=1.5, seed=3), cloud.small_sphere(8, 150, seed=4),
              cloud.with_supersonic_boundary(cloud.small_sphere(7, 120, r1=1.6, seed=5))]
    flows = [(0.4, 0.0), (0.8, 2.0), (0.6, 1.0)]
    sep, hsep = [], []
    for c, (m, a) in zip(clouds, flows):
        s = Solver(c, m, a, chain_warps=chain_warps)
        s.initial_conditions()
        hsep.append(s.q_lskum(5))
        sep.append(s.get(mfcfd_lib.FIELD_PRIM))
        s.close()
    solvers = []
    for c, (m, a) in zip(clouds, flows):
        s = Solver(c, m, a, chain_warps=chain_warps)
        s.initial_conditions()
        solvers.append(s)
    hist = batch.run_batch(solvers, 5)
    for i, s in enumerate(solvers):
        assert np.array_equal(hist[i], hsep[i])
        assert np.array_equal(s.get(mfcfd_lib.FIELD_PRIM), sep[i])
        s.close()
