"""Set-up of the 1,104,000-point sphere on the host, bit for bit.

The benchmark cloud (96 shells x 11,500 points, 1% jitter) has 92,000 split-
list entries written past the reference's 22-entry storage, so its stencils
exercise the spill semantics (data_structure.f90:83-88) at scale.  The
library's host-only handle (device -1) must give the oracle's split lists,
counts, alias and point_with_alias exactly (generate_connectivity.f90:12-246,
implicit_aliasing.f90:13-44).

The sweep level sets have no counterpart in the reference; they are checked
against their definition from the oracle's own stencils and alias: a swept
point's level in the forward (backward) sweep is one more than the deepest
level among the swept neighbours its L (U) routine reads, those of lower
(higher) alias (implicit_LdelU_forward_sweep_interior.f90:95-98,
implicit_UdelU_backward_sweep_interior.f90:95-98), over its split lists,
with the full conn as a wall point's z- list (implicit_LdelU_forward_sweep_
wall.f90:348-349); 0 without such neighbours.  That recursion has exactly
one solution, so checking it at every point checks every level.
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def sphere1m():
    from mfcfd import cloud
    return cloud.sphere_1m()


def _sweep_entries(c, counts, lists, lo, hi):
    """1-based entries (hi-lo, 6, 27) the sweeps read, 0 where unused."""
    from mfcfd.cloud import STATUS_WALL
    j = np.arange(lists.shape[2])
    ent = np.where(j[None, None, :] < counts[lo:hi, :, None], lists[lo:hi], 0)
    wall = c.status[lo:hi] == STATUS_WALL
    if wall.any():
        zn = np.where(j[None, :] < c.nbhs[lo:hi][wall][:, None], c.conn[lo:hi][wall], 0)
        ent[wall, 5, :] = zn[:, :lists.shape[2]]
    return ent


def test_sphere1m_setup_matches_oracle(sphere1m, oracle_lib, mfcfd_lib):
    from mfcfd.cloud import STATUS_INTERIOR, STATUS_WALL
    from mfcfd.solver import Solver
    c = sphere1m
    s = Solver(c, 0.8, 2.0, device=-1)
    counts, lists = s.stencils(27)
    alias, pwa = s.alias()
    levels = [s.levels(0), s.levels(1)]
    info = s.info()
    s.close()
    o = oracle_lib.Oracle(c, 0.8, 2.0)
    oc, ol = o.stencils(27)
    assert np.array_equal(counts, oc)
    assert np.array_equal(lists, ol)
    del ol
    oa, op = o.alias()
    o.close()
    assert np.array_equal(alias, oa)
    assert np.array_equal(pwa, op)
    assert info["split_overflows"] > 0          # the spill path is exercised

    # swept: wall and interior points the alias order visits (point 1 never is)
    n = c.n
    swept = np.zeros(n + 1, dtype=bool)         # 1-based, entry 0 false
    vis = op[op > 0]
    cls_ok = (c.status == STATUS_WALL) | (c.status == STATUS_INTERIOR)
    swept[vis] = cls_ok[vis - 1]
    a1 = np.concatenate([[0], oa])              # alias, 1-based
    for direction in (0, 1):
        lev = np.concatenate([[-1], levels[direction]])
        assert np.array_equal(lev[1:] >= 0, swept[1:]), "swept points"
        step = 131072
        for lo in range(0, n, step):
            hi = min(n, lo + step)
            ent = _sweep_entries(c, oc, lists, lo, hi)
            p_alias = a1[lo + 1:hi + 1][:, None, None]
            k_alias = a1[ent]
            dep = (ent > 0) & swept[ent] & ((k_alias < p_alias) if direction == 0 else (k_alias > p_alias))
            deepest = np.where(dep, lev[ent], -1).reshape(hi - lo, -1).max(axis=1)
            want = np.where(swept[lo + 1:hi + 1], deepest + 1, -1)
            assert np.array_equal(lev[lo + 1:hi + 1], want), (direction, lo)
    assert info["n_levels_forward"] == levels[0].max() + 1
    assert info["n_levels_backward"] == levels[1].max() + 1
