"""Checkpoint / restart through mfcfd_get_state / mfcfd_set_state: a run
stopped after 5 iterations, its state (prim, delUn, res_old) saved into the
caller's buffers and restored into a new handle, continues to the same bits
as an uninterrupted run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kw", [{}, {"precision": 1}, {"sweep_mode": 0}])
def test_restart_continues_bit_for_bit(mfcfd_lib, small_cloud, kw):
    from mfcfd import _lib
    from mfcfd.solver import Solver
    full = Solver(small_cloud, 0.8, 2.0, **kw)
    full.initial_conditions()
    h_full = full.q_lskum(10)
    a = Solver(small_cloud, 0.8, 2.0, **kw)
    a.initial_conditions()
    h_a = a.q_lskum(5)
    prim, delu = np.empty((small_cloud.n, 5)), np.empty((small_cloud.n, 5))
    _, _, ro = a.get_state(out=(prim, delu))
    a.close()
    b = Solver(small_cloud, 0.8, 2.0, **kw)
    b.set_state(prim, delu, ro)
    h_b = b.q_lskum(5, t0=6)
    assert np.array_equal(np.vstack([h_a, h_b]), h_full)
    assert np.array_equal(b.get(_lib.FIELD_PRIM), full.get(_lib.FIELD_PRIM))
    b.close()
    full.close()
