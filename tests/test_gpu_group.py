"""Group launches (mfcfd_run_group): the chain sweeps of several clouds in
one kernel launch per direction, the clouds in lockstep.

Each cloud of a group must get exactly the bits of its own run -- every
field, every residual -- in FP64 (against the oracle-pinned single-cloud
path) and in both mixed forms, with and without captured graphs, with phase-A
(k_g0) points and supersonic copies in the mix.  Groups the kernel cannot run
are refused as a whole before anything is launched, and a bounded sweep wait
that runs out in one cloud of a group is that cloud's error alone.
"""
import ctypes

import numpy as np
import pytest

from mfcfd import _lib

pytestmark = pytest.mark.gpu

ARG, UNSUPPORTED, TIMEOUT = 1, 6, 8
FIELDS = ("PRIM", "U", "Q", "DQ", "FLUX_RES", "DELUP", "DELUN", "DINV")


def _clouds():
    from mfcfd import cloud
    return [cloud.small_sphere(6, 100, r1=1.5, seed=3), cloud.small_sphere(8, 150, seed=4),
            cloud.with_supersonic_boundary(cloud.small_sphere(7, 120, r1=1.6, seed=5)),
            cloud.shell_cloud(10, 400, r1=3.0, seed=77, aspect=(1.0, 1.8, 2.6))]


FLOWS = [(0.4, 0.0), (0.8, 2.0), (0.6, 1.0), (0.85, 5.0)]


def _solvers(clouds, **kw):
    from mfcfd.solver import Solver
    out = []
    for c, (m, a) in zip(clouds, FLOWS):
        s = Solver(c, m, a, **kw)
        s.initial_conditions()
        out.append(s)
    return out


def _fields(s):
    return {f: s.get(getattr(_lib, "FIELD_" + f)) for f in FIELDS}


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("graphs", [0, 1])
def test_group_equals_separate_runs(mfcfd_lib, precision, graphs):
    from mfcfd import batch
    clouds = _clouds()
    want = []
    for s in _solvers(clouds, precision=precision):
        h = s.q_lskum(7)
        want.append((h, _fields(s)))
        s.close()
    ss = _solvers(clouds, precision=precision, graphs=graphs)
    try:
        assert len({s.info()["chain_warps_per_block"] for s in ss}) == 1
        hist = batch.run_group(ss, 4)
        hist2 = batch.run_group(ss, 3)       # a second call continues the same states
        for i, s in enumerate(ss):
            got = np.concatenate([hist[i], hist2[i]])
            assert np.array_equal(got.view(np.uint64), want[i][0].view(np.uint64)), i
            f = _fields(s)
            for k in FIELDS:
                assert np.array_equal(f[k].view(np.uint64), want[i][1][k].view(np.uint64)), (i, k)
            assert [t for t, _, _ in s.history] == list(range(1, 8))
    finally:
        for s in ss:
            s.close()


def test_run_grouped_equals_run_batch(mfcfd_lib):
    """plan_groups + run_grouped over clouds of both block shapes against
    mfcfd_run_batch (continuous scheduling): the same bits per cloud."""
    from mfcfd import batch
    clouds = _clouds()
    a = _solvers(clouds, chain_warps=0)
    b = _solvers(clouds, chain_warps=0)
    try:
        # one cloud on 8-warp blocks: its own group
        for s in (a[3], b[3]):
            s.set_chain_warps(4 * (s.info()["chain_slot_capacity"] // 6) + 8)
        assert b[3].info()["chain_warps_per_block"] == 8
        groups = batch.plan_groups(b)
        assert sorted(i for g in groups for i in g) == list(range(len(b)))
        assert any(g == [3] for g in groups)
        ha = batch.run_batch(a, 5)
        hb = batch.run_grouped(b, 5, groups)
        assert np.array_equal(ha.view(np.uint64), hb.view(np.uint64))
        for x, y in zip(a, b):
            assert np.array_equal(x.get(_lib.FIELD_PRIM), y.get(_lib.FIELD_PRIM))
    finally:
        for s in a + b:
            s.close()


def _call(ss, count=None, hs=None):
    n = len(ss) if count is None else count
    if hs is None:
        hs = (ctypes.c_void_p * max(n, 1))(*[ss[i % len(ss)].h.value for i in range(n)])
    t0 = np.ones(max(n, 1), dtype=np.int32)
    return _lib.lib().mfcfd_run_group(hs, n, _lib.ptr(t0), 1, None, None)


def test_group_refusals(mfcfd_lib):
    from mfcfd import cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere(6, 100, r1=1.5, seed=3)
    f64 = Solver(c, 0.4, 0.0)
    f64.initial_conditions()
    mix = Solver(c, 0.4, 0.0, precision=1)
    mix.initial_conditions()
    lev = Solver(c, 0.4, 0.0, sweep_mode=1)
    lev.initial_conditions()
    wide = []
    try:
        before = f64.get(_lib.FIELD_PRIM)
        assert _call([f64], count=0) == ARG
        assert _call([f64], count=_lib.GROUP_MAX_CLOUDS + 1) == ARG
        assert _call([f64, f64]) == ARG                       # a handle twice
        assert _call([f64, mix]) == UNSUPPORTED                # precision classes differ
        assert _call([f64, lev]) == UNSUPPORTED                # not the chain schedule
        for _ in range(3):                                     # 3 x 100 blocks do not fit
            s = Solver(c, 0.4, 0.0, chain_warps=400)
            s.initial_conditions()
            wide.append(s)
        slots = sum(s.info()["chain_slots"] for s in wide)
        assert slots > wide[0].info()["chain_slot_capacity"]
        assert _call(wide) == UNSUPPORTED
        assert "do not fit" in _lib.lib().mfcfd_last_error(wide[0].h).decode()
        # nothing ran
        assert np.array_equal(f64.get(_lib.FIELD_PRIM), before)
        assert f64.history == []
    finally:
        for s in [f64, mix, lev] + wide:
            s.close()


def test_group_wait_timeout_is_one_clouds_error(mfcfd_lib):
    """A point of one cloud publishes none of its sweep increments
    (mfcfd_set_fault_hook): that cloud's readers poll until their shortened
    bound runs out, inside the group kernel, and only that cloud reports
    MFCFD_ERR_TIMEOUT; the others finish with their own runs' bits."""
    from mfcfd import batch
    clouds = _clouds()[:3]
    want = []
    for s in _solvers(clouds, chain_warps=200):
        want.append(s.q_lskum(2))
        s.close()
    ss = _solvers(clouds, chain_warps=200)
    try:
        assert ss[1].info()["chain_terms_cross"] > 0
        _, pwa = ss[1].alias()
        ss[1].set_fault_hook(int(pwa[0]), wait_limit=1 << 12)
        st = []
        hist = batch.run_group(ss, 2, statuses=st)
        assert st == [0, TIMEOUT, 0]
        for i in (0, 2):
            assert np.array_equal(hist[i], want[i])
        # the hooked handle recovers: hook off, state set again
        ss[1].set_fault_hook(0, 0)
        ss[1].initial_conditions()
        ss[1].history.clear()
        assert np.array_equal(ss[1].q_lskum(2), want[1])
    finally:
        for s in ss:
            s.close()
