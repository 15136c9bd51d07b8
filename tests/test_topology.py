"""Host set-up of the library (split stencils, alias order, sweep schedule)
against the oracle and the golden fixtures; needs no GPU (device = -1)."""
import numpy as np
import pytest


def _solver(cloud, **over):
    from mfcfd.solver import Solver
    return Solver(cloud, 0.4, 0.0, device=-1, **over)


def test_stencils_and_alias_match_reference(oracle_lib):
    from tests.test_oracle_golden import GOLDEN, golden_cloud
    with np.load(GOLDEN) as z:
        g = {k: z[k] for k in z.files}
    c = golden_cloud(g)
    s = _solver(c)
    counts, lists = s.stencils(27)
    assert np.array_equal(counts, g["split_counts"])
    assert np.array_equal(lists, g["split_lists"])
    a, p = s.alias()
    assert np.array_equal(a, g["case0_glibc_alias"])
    assert np.array_equal(p, g["case0_glibc_point_with_alias"])
    assert s.info()["split_overflows"] > 0


@pytest.mark.parametrize("shells,per,r1", [(8, 150, 1.7), (5, 60, 1.4)])
def test_against_oracle_small_clouds(oracle_lib, shells, per, r1):
    from mfcfd import cloud
    c = cloud.shell_cloud(shells, per, r1=r1, seed=shells * 100 + per)
    s = _solver(c)
    o = oracle_lib.Oracle(c, 0.4, 0.0)
    cs, ls = s.stencils(27)
    co, lo = o.stencils(27)
    assert np.array_equal(cs, co) and np.array_equal(ls, lo)
    assert all(np.array_equal(x, y) for x, y in zip(s.alias(), o.alias()))


def test_unlimited_capacity_has_no_overflow(small_cloud):
    s = _solver(small_cloud, split_capacity=0)
    assert s.info()["split_overflows"] == 0
    counts, lists = s.stencils(27)
    # every list is a subsequence of conn in conn order
    for i in range(0, small_cloud.n, 37):
        conn = list(small_cloud.conn[i, :small_cloud.nbhs[i]])
        for d in range(6):
            ent = list(lists[i, d, :counts[i, d]])
            it = iter(conn)
            assert all(e in it for e in ent)


def test_schedule_respects_every_dependency(small_cloud):
    """A point's level exceeds the level of every swept neighbour it reads
    (lower alias forward, higher alias backward): the level-parallel sweep
    then equals the reference's sequential one."""
    s = _solver(small_cloud)
    counts, lists = s.stencils(27)
    alias, pwa = s.alias()
    st = small_cloud.status
    swept = np.zeros(small_cloud.n, bool)
    pw = pwa[pwa > 0] - 1
    swept[pw[(st[pw] == 0) | (st[pw] == 1)]] = True
    for direction in (0, 1):
        lv = s.levels(direction)
        assert np.all((lv >= 0) == swept)
        for p in np.nonzero(swept)[0]:
            if st[p] == 1:
                nb = [k for d in range(4) for k in lists[p, d, :counts[p, d]]]
                nb += list(small_cloud.conn[p, :small_cloud.nbhs[p]])
            else:
                nb = [k for d in range(6) for k in lists[p, d, :counts[p, d]]]
            nb = np.array(nb) - 1
            dep = nb[(alias[nb] < alias[p]) if direction == 0 else (alias[nb] > alias[p])]
            dep = dep[swept[dep]]
            assert np.all(lv[dep] < lv[p])


def test_point_one_is_not_swept(small_cloud):
    """implicit_aliasing.f90:276-288: point 1's first neighbour also gets alias 1
    and takes its slot in point_with_alias, so point 1 is never swept."""
    s = _solver(small_cloud)
    alias, pwa = s.alias()
    assert alias[0] == 1
    first = small_cloud.conn[0, 0]
    assert alias[first - 1] == 1 and pwa[0] == first
    assert 1 not in set(pwa.tolist())
    assert pwa[-1] == 0
    assert s.levels(0)[0] == -1


def _nearest(c, p):
    """implicit_forward_and_reverse_sweeps.f90:39-50: first closest neighbour."""
    nb = c.conn[p, :c.nbhs[p]] - 1
    d = np.sqrt((c.x[nb] - c.x[p]) ** 2 + (c.y[nb] - c.y[p]) ** 2 + (c.z[nb] - c.z[p]) ** 2)
    return int(nb[np.argmin(d)]) if len(nb) and d.min() < 1e6 else -1


def _level_check(s, c, direction):
    """Levels are exactly the longest-path depths over swept dependencies
    (supersonic points depend on their copy source when it comes first)."""
    counts, lists = s.stencils(27)
    alias, pwa = s.alias()
    st = c.status
    swept = np.zeros(c.n, bool)
    pw = pwa[pwa > 0] - 1
    swept[pw[(st[pw] == 0) | (st[pw] == 1) | (st[pw] == 5) | (st[pw] == 6)]] = True
    ps, ks = [], []
    for d in range(6):
        for j in range(27):
            m = (counts[:, d] > j) & ((st == 0) | ((st == 1) & (d < 4)))
            ps.append(np.nonzero(m)[0])
            ks.append(lists[m, d, j] - 1)
    wall = np.nonzero(st == 1)[0]
    for j in range(27):
        m = c.nbhs[wall] > j
        ps.append(wall[m])
        ks.append(c.conn[wall[m], j] - 1)
    ss = np.nonzero((st == 5) | (st == 6))[0]
    src = np.array([_nearest(c, i) for i in ss], dtype=np.int64)
    ps.append(ss[src >= 0])
    ks.append(src[src >= 0])
    p, k = np.concatenate(ps), np.concatenate(ks)
    keep = swept[p] & swept[k] & ((alias[k] < alias[p]) if direction == 0 else (alias[k] > alias[p]))
    p, k = p[keep], k[keep]
    lv = s.levels(direction)
    assert np.array_equal(lv >= 0, swept)
    assert np.all(lv[k] < lv[p])
    deepest = np.full(c.n, -1)
    np.maximum.at(deepest, p, lv[k])
    assert np.array_equal(lv[swept], deepest[swept] + 1)


def test_large_cloud_parallel_setup(oracle_lib):
    """Above the size where the set-up runs its per-point loops on several
    host threads: stencils and alias still equal the oracle's, and the sweep
    levels are the exact longest-path depths."""
    from mfcfd import cloud
    c = cloud.shell_cloud(12, 6000, r1=3.0, seed=4242)
    assert c.n >= 8 * 4096   # every pass splits over several threads
    s = _solver(c)
    o = oracle_lib.Oracle(c, 0.4, 0.0)
    cs, ls = s.stencils(27)
    co, lo = o.stencils(27)
    assert np.array_equal(cs, co) and np.array_equal(ls, lo)
    assert all(np.array_equal(x, y) for x, y in zip(s.alias(), o.alias()))
    for direction in (0, 1):
        _level_check(s, c, direction)


def test_supersonic_points_are_swept_copies(oracle_lib):
    """Status 5/6 points join the sweep order and copy their nearest
    neighbour's increment: their level follows the copy source when it comes
    earlier in the sweep; stencils and alias still equal the oracle's."""
    from mfcfd import cloud
    c = cloud.with_supersonic_boundary(cloud.small_sphere(6, 100, r1=1.5))
    s = _solver(c)
    info = s.info()
    assert info["n_supersonic"] == int(((c.status == 5) | (c.status == 6)).sum()) > 0
    o = oracle_lib.Oracle(c, 0.4, 0.0)
    cs, ls = s.stencils(27)
    co, lo = o.stencils(27)
    assert np.array_equal(cs, co) and np.array_equal(ls, lo)
    for direction in (0, 1):
        _level_check(s, c, direction)


@pytest.mark.parametrize("capacity", [22, 20])
def test_overflowing_lists_split_on_several_threads(oracle_lib, capacity):
    """Lists longer than the storage spill into the following points' cells,
    and the reference's visiting order decides which value a cell keeps.  At
    15,000 points the split runs on several host threads (own cells first,
    then the spilled entries in that order); the effective lists still equal
    the oracle's."""
    from mfcfd import cloud
    c = cloud.shell_cloud(10, 1500, r1=2.0, seed=77)
    assert c.n >= 2 * 4096
    s = _solver(c, split_capacity=capacity)
    assert s.info()["split_overflows"] > 0
    o = oracle_lib.Oracle(c, 0.4, 0.0, split_capacity=capacity)
    cs, ls = s.stencils(27)
    co, lo = o.stencils(27)
    assert np.array_equal(cs, co) and np.array_equal(ls, lo)
    assert all(np.array_equal(x, y) for x, y in zip(s.alias(), o.alias()))
