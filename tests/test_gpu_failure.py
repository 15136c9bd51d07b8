"""Failure detection on the GPU without a fault.

Every wait of the sweeps is bounded.  mfcfd_set_fault_hook makes one point
publish none of its sweep increments, so the points that read them poll until
their (here shortened) bound runs out: the kernel sets its error word and
returns, the step reports MFCFD_ERR_TIMEOUT, and the handle stays usable --
with the hook off and the state set again, the next step gives the same bits
as a handle that never saw the fault.  Nothing traps or waits without bound.

The dataflow schedule is used because every consumer there polls the
producer's words in global memory (the chain schedule may hand an increment
over in a warp's shared-memory ring, where nothing waits).
"""
import numpy as np
import pytest

from mfcfd import _lib

pytestmark = pytest.mark.gpu

TIMEOUT = 8      # MFCFD_ERR_TIMEOUT
ARG = 1          # MFCFD_ERR_ARG


def test_sweep_wait_times_out_and_handle_recovers(mfcfd_lib):
    from mfcfd import cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere()
    ref = Solver(c, 0.4, 0.0, sweep_mode=0)
    ref.initial_conditions()
    want = ref.fpi_solver(1)
    want_prim = ref.get(_lib.FIELD_PRIM)
    ref.close()

    s = Solver(c, 0.4, 0.0, sweep_mode=0)
    s.initial_conditions()
    _, pwa = s.alias()
    first = int(pwa[0])              # the first swept point: later points read it
    s.set_fault_hook(first, wait_limit=1 << 12)
    with pytest.raises(_lib.MfcfdError) as e:
        s.fpi_solver(1)
    assert e.value.code == TIMEOUT
    # the timed-out iteration left no valid residual behind
    with pytest.raises(_lib.MfcfdError) as e:
        s.residual_noalloc()
    assert e.value.code == ARG
    # the error word was cleared: with the hook off and the state set again,
    # the same handle reproduces the clean run bit for bit
    s.set_fault_hook(0, 0)
    s.initial_conditions()
    got = s.fpi_solver(1)
    assert got[0] == want[0]
    assert np.array_equal(s.get(_lib.FIELD_PRIM), want_prim)
    # and a second fault on the same handle is reported again
    s.set_fault_hook(first, wait_limit=1 << 12)
    with pytest.raises(_lib.MfcfdError) as e:
        s.fpi_solver(2)
    assert e.value.code == TIMEOUT
    s.close()


def test_fault_hook_arguments(mfcfd_lib):
    from mfcfd import cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere()
    s = Solver(c, 0.4, 0.0)
    for point, limit in ((-1, 0), (c.n + 1, 0), (1, -5)):
        with pytest.raises(_lib.MfcfdError) as e:
            s.set_fault_hook(point, limit)
        assert e.value.code == ARG
    s.close()
