"""Autotuner of the chain schedule (mfcfd_tune_chain).

Tuning times candidate warp counts from the current state and keeps the
fastest: the state must come back unchanged, the kept schedule must be one
of the candidates, and later iterations must give the same bits as an
untuned handle (the schedule orders the work, not the arithmetic).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tuning_keeps_state_and_results(mfcfd_lib):
    from mfcfd import _lib, cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere(8, 150, seed=4)
    ref = Solver(c, 0.8, 2.0)
    ref.initial_conditions()
    h_ref = ref.q_lskum(12)
    s = Solver(c, 0.8, 2.0)
    s.initial_conditions()
    h1 = s.q_lskum(4)
    before = s.get_state()
    chosen, ms = s.tune_chain(iters=2)
    after = s.get_state()
    assert all(np.array_equal(a, b) for a, b in zip(before[:2], after[:2])) and before[2] == after[2]
    width = s.info()["max_level_width"]
    assert s.info()["chain_warps"] == chosen and np.all(ms > 0)
    assert chosen >= width      # every default candidate is at least 1.5x the widest level
    h2 = s.q_lskum(8, t0=5)
    assert np.array_equal(np.vstack([h1, h2]), h_ref)
    assert np.array_equal(s.get(_lib.FIELD_PRIM), ref.get(_lib.FIELD_PRIM))
    s.close()
    ref.close()


def test_tuning_explicit_candidates_and_mixed(mfcfd_lib):
    from mfcfd import _lib, batch, cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere(10, 160, r1=1.9, seed=9)
    s = Solver(c, 0.6, -3.0, precision=_lib.PRECISION_MIXED)
    s.initial_conditions()
    chosen, ms = s.tune_chain([32, 64, 96], iters=2)
    assert chosen in (32, 64, 96) and ms.shape == (3,)
    t = Solver(c, 0.6, -3.0, precision=_lib.PRECISION_MIXED)
    t.initial_conditions()
    assert batch.tune_all([t]) == [t.info()["chain_warps"]]
    assert np.array_equal(s.q_lskum(6), t.q_lskum(6))
    s.close()
    t.close()


def test_tuning_needs_the_chain_schedule(mfcfd_lib):
    from mfcfd import cloud
    from mfcfd._lib import MfcfdError
    from mfcfd.solver import Solver
    s = Solver(cloud.small_sphere(), 0.4, 0.0, sweep_mode=0)
    s.initial_conditions()
    with pytest.raises(MfcfdError) as e:
        s.tune_chain()
    assert e.value.code == 1
    s.close()
