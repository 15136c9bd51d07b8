"""The allocation-free residual entry point against the iteration's own value.

mfcfd_residual_noalloc is for callers that must not allocate device memory
(their device memory belongs to another allocator, or allocation is not
allowed where they need the number).  It recomputes res_new of the last
iteration with scratch that lives in a fixed device array inside the library.
Called through the C ABI after two consecutive iterations, it must give the
res_new that mfcfd_fpi_step returned, within the residual tolerance the
parity tests use.  This file is collected last on purpose.
"""
import pytest

pytestmark = pytest.mark.gpu


def test_residual_noalloc_matches_fpi_step(mfcfd_lib):
    from mfcfd import cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere()
    s = Solver(c, 0.4, 0.0)
    s.initial_conditions()
    for t in (1, 2):
        res_new, _ = s.fpi_solver(t)
        again = s.residual_noalloc()
        assert res_new > 0.0
        assert abs(again - res_new) <= 1e-13 * abs(res_new), (t, again, res_new)
    s.close()


def test_residual_noalloc_without_a_completed_iteration(mfcfd_lib):
    """Before the first iteration and after the state is set again there is
    no residual to recompute: the call says so instead of returning a stale
    or zero value."""
    from mfcfd import _lib, cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere()
    s = Solver(c, 0.4, 0.0)
    s.initial_conditions()
    with pytest.raises(_lib.MfcfdError) as e:
        s.residual_noalloc()
    assert e.value.code == 1
    res_new, _ = s.fpi_solver(1)
    assert abs(s.residual_noalloc() - res_new) <= 1e-13 * abs(res_new)
    s.initial_conditions()
    with pytest.raises(_lib.MfcfdError) as e:
        s.residual_noalloc()
    assert e.value.code == 1
    s.close()
