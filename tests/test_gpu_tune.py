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


def test_batch_tuning_and_set_warps(mfcfd_lib):
    """tune_batch restores states and histories; schedules set by
    set_chain_warps (attached handles) iterate to the same bits."""
    from mfcfd import _lib, batch, cloud
    from mfcfd.solver import Solver
    clouds = [cloud.small_sphere(6, 100, r1=1.5, seed=3), cloud.small_sphere(8, 150, seed=4),
              cloud.small_sphere(10, 160, r1=1.9, seed=9)]
    ref, tuned = [], []
    for c in clouds:
        for lst in (ref, tuned):
            s = Solver(c, 0.7, 1.0)
            s.initial_conditions()
            lst.append(s)
    h_ref = batch.run_batch(ref, 9)
    batch.run_batch(tuned, 3)
    before = [s.get_state() for s in tuned]
    pc, times = batch.tune_batch(tuned, percents=(75, 100, 200), iters=2)
    assert pc in (75, 100, 200) and set(times) == {75, 100, 200}
    assert all(len(s.history) == 3 for s in tuned)
    for s, b in zip(tuned, before):
        a = s.get_state()
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    h = batch.run_batch(tuned, 6)
    assert np.array_equal(h, h_ref[:, 3:])
    w = tuned[0].set_chain_warps(8)
    assert w == 8 and tuned[0].info()["chain_warps"] == 8
    assert np.array_equal(tuned[0].q_lskum(2, t0=10), ref[0].q_lskum(2, t0=10))
    for s in ref + tuned:
        s.close()


def test_server_chain_percent_keeps_results(mfcfd_lib):
    from mfcfd import cloud, serve
    c = cloud.small_sphere(8, 150, seed=4)
    out = []
    for pc in (0, 100):
        with serve.Server(chunk=10, chain_percent=pc) as srv:
            out.append(srv.wait(srv.submit(c, 0.8, 2.0, max_iters=30, residue_target=-9.0), timeout=120))
    assert out[0]["status"] == 0 and out[1]["status"] == 0
    assert np.array_equal(out[0]["prim"], out[1]["prim"]) and out[0]["res_new"] == out[1]["res_new"]
