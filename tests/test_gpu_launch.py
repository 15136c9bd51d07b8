"""mfcfd_launch / mfcfd_complete: iterations queued without waiting, then
polled or waited for, give exactly what mfcfd_run gives; one launch may be
pending per handle; the slot figures of mfcfd_info bound what may run at
once."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_launch_complete_equals_run(mfcfd_lib, small_cloud):
    from mfcfd import _lib
    from mfcfd._lib import MfcfdError
    from mfcfd.solver import Solver
    ref = Solver(small_cloud, 0.8, 2.0)
    ref.initial_conditions()
    h_ref = ref.q_lskum(17)
    s = Solver(small_cloud, 0.8, 2.0)
    s.initial_conditions()
    with pytest.raises(MfcfdError):          # nothing pending
        s._pending = (1, 1)
        s.complete()
    s.launch(1, 10)
    with pytest.raises(MfcfdError):          # one launch at a time
        s.launch(11, 7)
    h1 = None
    deadline = time.time() + 60
    while h1 is None and time.time() < deadline:
        h1 = s.complete(wait=False)
    s.launch(11, 7)
    h2 = s.complete(wait=True)
    assert np.array_equal(np.vstack([h1, h2]), h_ref)
    assert np.array_equal(s.get(_lib.FIELD_PRIM), ref.get(_lib.FIELD_PRIM))
    info = s.info()
    assert 0 < info["chain_slots"] <= info["chain_slot_capacity"]
    s.close()
    ref.close()
