"""The device-resident set-up (gpu_setup = 1 on a handle created with its
device) against the host set-up, array by array.

Every topology array the kernels read -- the storage-order cloud, the neighbour
slots and effective lists, the least-squares geometry, the sweep terms with
their chain bits, the level schedules, the chain schedule's warp lists and
records, the residual and flux-kernel orders -- must be byte-identical to the
arrays the host set-up (build_topology, permute_topology, the chain schedule)
uploads, for clouds with and without spilled split lists, wall frames that
vary from point to point, phase-A (k_g0) points, either storage order and
every sweep schedule.  Iterations then give the same bits by construction;
that is checked too.  Configurations the device path does not cover (the
backup driver, supersonic points, power != 0) take the host path and
must still match.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ARRAYS = ["x", "y", "z", "frame", "cls", "nbhs", "conn", "eps2", "slot_nbr", "nslot", "slot_mask", "list_cnt",
          "list_ent", "geo", "swept", "consumer_shared", "fwd_lvl_ptr", "fwd_lvl_pts", "bwd_lvl_ptr",
          "bwd_lvl_pts", "fwd_off", "bwd_off", "fwd_cnt", "bwd_cnt", "fwd_ent", "bwd_ent", "fwd_need",
          "bwd_need", "fwd_old", "bwd_old", "sweep_slot_mask", "res_order", "pre_order", "g0_pts",
          "ch_ptr0", "ch_pts0", "ch_own0", "ch_items0", "ch_ptr1", "ch_pts1", "ch_own1", "ch_items1"]
FIELDS = ["PRIM", "U", "Q", "QM", "DQ", "DELT", "FLUX_RES", "DELUP", "DELUN", "DINV"]


def _clouds():
    from mfcfd import cloud, wing
    return {
        "small": lambda: cloud.small_sphere(),
        "spill": lambda: cloud.small_sphere(8, 150, seed=4),
        "ellipsoid": lambda: cloud.shell_cloud(14, 900, r1=3.0, seed=77, aspect=(1.0, 1.8, 2.6)),
        "wing": lambda: wing.swept_wing(points=20_000, nc=48, ns=16, name="wing-20k"),
    }


def _digests(s):
    return {a: s.digest(a) for a in ARRAYS}


def _pair(c, **kw):
    from mfcfd.solver import Solver
    return Solver(c, 0.8, 2.0, gpu_setup=0, **kw), Solver(c, 0.8, 2.0, gpu_setup=1, **kw)


CASES = {
    "chains": dict(),
    "chains-index-order": dict(storage_order=0),
    "chains-capacity-12": dict(split_capacity=12),
    "chains-dc": dict(precision=2),
    "chains-mixed": dict(precision=1),
    "levels": dict(sweep_mode=1),
    "dataflow": dict(sweep_mode=0),
}


@pytest.mark.parametrize("name", sorted(_clouds()))
@pytest.mark.parametrize("case", sorted(CASES))
def test_device_setup_arrays_equal_host(mfcfd_lib, name, case):
    from mfcfd._lib import MfcfdError
    c = _clouds()[name]()
    kw = CASES[case]
    try:
        host, dev = _pair(c, **kw)
    except MfcfdError as e:        # a capacity whose spills leave a list naming point 0
        assert kw.get("split_capacity"), str(e)
        from mfcfd.solver import Solver
        with pytest.raises(MfcfdError) as g:
            Solver(c, 0.8, 2.0, gpu_setup=1, **kw)
        assert str(g.value) == str(e)
        return
    try:
        a, b = _digests(host), _digests(dev)
        for k in ARRAYS:
            assert a[k] == b[k], k
        ia, ib = host.info(), dev.info()
        for k in ia:
            if k != "device_bytes":    # the device set-up keeps the query arrays resident
                assert ia[k] == ib[k], k
        for x, y in zip(host.stencils(27), dev.stencils(27)):
            assert np.array_equal(x, y)
        for x, y in zip(host.alias(), dev.alias()):
            assert np.array_equal(x, y)
        for d in (0, 1):
            assert np.array_equal(host.levels(d), dev.levels(d))
    finally:
        host.close()
        dev.close()


def test_device_setup_iterations_and_tuning(mfcfd_lib):
    """Same bits over iterations, and a chain schedule rebuilt at other warp
    counts (mfcfd_tune_chain) equal to the host's rebuild."""
    from mfcfd import _lib, cloud
    c = cloud.small_sphere()
    host, dev = _pair(c)
    try:
        out = []
        for s in (host, dev):
            s.initial_conditions()
            h = s.q_lskum(12)
            out.append((h, {f: s.get(getattr(_lib, "FIELD_" + f)) for f in FIELDS}))
        assert np.array_equal(out[0][0].view(np.uint64), out[1][0].view(np.uint64))
        for f in FIELDS:
            assert np.array_equal(out[0][1][f].view(np.uint64), out[1][1][f].view(np.uint64)), f
        for s in (host, dev):
            s.set_chain_warps(24)
        a, b = _digests(host), _digests(dev)
        for k in ARRAYS:
            assert a[k] == b[k], k
        r = [s.q_lskum(3) for s in (host, dev)]
        assert np.array_equal(r[0].view(np.uint64), r[1].view(np.uint64))
    finally:
        host.close()
        dev.close()


@pytest.mark.parametrize("kw", [dict(sweep_variant=1), dict(power=1.0)])
def test_device_setup_fallbacks_match(mfcfd_lib, kw):
    """Configurations the device path does not cover take the host set-up."""
    from mfcfd import cloud
    c = cloud.small_sphere()
    host, dev = _pair(c, **kw)
    try:
        a, b = _digests(host), _digests(dev)
        for k in ARRAYS:
            assert a[k] == b[k], k
    finally:
        host.close()
        dev.close()


def test_device_setup_supersonic_falls_back(mfcfd_lib):
    from mfcfd import cloud
    c = cloud.with_supersonic_boundary(cloud.small_sphere(7, 120, r1=1.6, seed=5))
    host, dev = _pair(c)
    try:
        a, b = _digests(host), _digests(dev)
        for k in ARRAYS:
            assert a[k] == b[k], k
    finally:
        host.close()
        dev.close()


def test_device_setup_sphere1m_equals_host(mfcfd_lib):
    """The 1,104,000-point benchmark sphere (92,000 spilled split-list
    entries): every array byte-identical to the host set-up's."""
    from mfcfd import cloud
    c = cloud.sphere_1m()
    host, dev = _pair(c)
    try:
        a, b = _digests(host), _digests(dev)
        for k in ARRAYS:
            assert a[k] == b[k], k
        assert dev.info()["split_overflows"] == host.info()["split_overflows"] > 0
    finally:
        host.close()
        dev.close()


def test_device_setup_roots_late_in_a_large_order(mfcfd_lib):
    """Points without swept lower-alias neighbours (level 0) far into a long
    sweep order: the 1.1M sphere with shell 60 made outer (not swept), so the
    points of shell 61 reached past it can be roots at about 64% of the
    order, beyond one launch-grid's worth of threads.  (A capped root launch
    once missed them on an 830k-point wing.)"""
    from mfcfd import cloud
    from mfcfd.cloud import STATUS_OUTER
    c = cloud.sphere_1m()
    st = c.status.copy()
    st[60 * 11500:61 * 11500] = STATUS_OUTER
    c.status = st
    host, dev = _pair(c)
    try:
        a, b = _digests(host), _digests(dev)
        for k in ARRAYS:
            assert a[k] == b[k], k
        assert dev.info()["n_levels_forward"] == host.info()["n_levels_forward"]
    finally:
        host.close()
        dev.close()


def _ragged_cloud(outer_all=False, seed=11):
    """A small random cloud with ragged neighbour lists (0 to 26 entries), a
    few wall points and an outer layer; with outer_all every point is outer,
    so nothing is swept."""
    from mfcfd import cloud
    from mfcfd.cloud import STATUS_INTERIOR, STATUS_OUTER, STATUS_WALL, PointCloud
    rng = np.random.default_rng(seed)
    n = 400
    pts = rng.uniform(-1.0, 1.0, size=(n, 3))
    nbhs, conn, md = cloud.knn(pts[:, 0], pts[:, 1], pts[:, 2], 26, device=-1)
    nbhs = rng.integers(0, 27, size=n).astype(np.int32)
    nbhs[0] = 26                                   # the search starts at point 1
    conn[np.arange(conn.shape[1])[None, :] >= nbhs[:, None]] = 0
    r = np.sqrt((pts * pts).sum(axis=1))
    status = np.full(n, STATUS_INTERIOR, dtype=np.int32)
    status[r > 0.95] = STATUS_OUTER
    status[:20] = STATUS_WALL
    if outer_all:
        status[:] = STATUS_OUTER
    tan1 = np.tile([1.0, 0.0, 0.0], (n, 1))
    tan2 = np.tile([0.0, 1.0, 0.0], (n, 1))
    nor = np.tile([0.0, 0.0, 1.0], (n, 1))
    return PointCloud(status=status, x=pts[:, 0].copy(), y=pts[:, 1].copy(), z=pts[:, 2].copy(), tan1=tan1,
                      tan2=tan2, nor=nor, nbhs=nbhs, conn=conn, min_dist=md, name="ragged")


@pytest.mark.parametrize("outer_all", [False, True])
@pytest.mark.parametrize("sweep_mode", [0, 2])
def test_device_setup_ragged_and_empty(mfcfd_lib, outer_all, sweep_mode):
    """Ragged neighbour counts (some points with none) and a cloud whose
    sweeps visit no point: the same arrays, or the same error, either way."""
    from mfcfd._lib import MfcfdError
    from mfcfd.solver import Solver
    c = _ragged_cloud(outer_all)
    try:
        host = Solver(c, 0.5, 1.0, gpu_setup=0, sweep_mode=sweep_mode)
    except MfcfdError as e:
        with pytest.raises(MfcfdError) as g:
            Solver(c, 0.5, 1.0, gpu_setup=1, sweep_mode=sweep_mode)
        assert str(g.value) == str(e)
        return
    dev = Solver(c, 0.5, 1.0, gpu_setup=1, sweep_mode=sweep_mode)
    try:
        a, b = _digests(host), _digests(dev)
        for k in ARRAYS:
            assert a[k] == b[k], k
        for d in (0, 1):
            assert np.array_equal(host.levels(d), dev.levels(d))
        assert host.info()["n_levels_forward"] == dev.info()["n_levels_forward"]
    finally:
        host.close()
        dev.close()
