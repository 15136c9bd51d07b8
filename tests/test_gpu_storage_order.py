"""The device layout along a space-filling curve changes no result.

A handle stores its points along a Morton curve (MFCFD_ORDER_MORTON, the
default) or in the caller's index order (MFCFD_ORDER_INDEX).  The set-up runs
on the reference's indices either way and every array crossing the C ABI is
in index order, so both layouts must give the same bits for every field,
the same residual history (the reduction sums in the reference's wall-then-
interior index order in both), the same forces and the same sweep levels --
including the variants whose order the reference fixes by point index
(supersonic copies, the explicit update, the backup sweep driver).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["PRIM", "U", "Q", "QM", "DQ", "DELT", "FLUX_RES", "DELUP", "DELUN", "DINV"]


def _run(c, order, iters, **kw):
    from mfcfd import _lib
    from mfcfd.solver import Solver
    s = Solver(c, 0.8, 2.0, storage_order=order, **kw)
    s.initial_conditions()
    hist = s.q_lskum(iters)
    out = {name: s.get(getattr(_lib, "FIELD_" + name)) for name in FIELDS}
    out["hist"] = hist
    out["forces"] = s.forces()[:2]
    out["levels"] = (s.levels(0), s.levels(1))
    prim, delu, res_old = s.get_state()
    out["state"] = (prim, delu, res_old)
    s.close()
    return out


CASES = {
    "chains-fp64": dict(),
    "chains-mixed": dict(precision=1),
    "dataflow-supersonic": dict(sweep_mode=0, supersonic=True),
    "levels-explicit": dict(sweep_mode=1, update_variant=1, supersonic=True),
    "dataflow-backup": dict(sweep_mode=0, sweep_variant=1, supersonic=True),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_morton_layout_gives_the_same_bits(mfcfd_lib, case):
    from mfcfd import _lib, cloud
    kw = dict(CASES[case])
    c = cloud.small_sphere()
    if kw.pop("supersonic", False):
        c = cloud.with_supersonic_boundary(c)
    iters = 3 if kw.get("sweep_variant") == 1 else 8   # the backup driver goes NaN at outer points later on
    a = _run(c, _lib.ORDER_INDEX, iters, **kw)
    b = _run(c, _lib.ORDER_MORTON, iters, **kw)
    for name in FIELDS:
        assert np.array_equal(a[name].view(np.uint64), b[name].view(np.uint64)), name
    assert np.array_equal(a["hist"].view(np.uint64), b["hist"].view(np.uint64))
    assert a["forces"] == b["forces"]
    for x, y in zip(a["levels"], b["levels"]):
        assert np.array_equal(x, y)
    assert np.array_equal(a["state"][0], b["state"][0]) and np.array_equal(a["state"][1], b["state"][1])


def test_morton_layout_round_trips_state(mfcfd_lib):
    """set_state / get_state and set_prim cross the ABI in index order."""
    from mfcfd import _lib, cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere()
    rng = np.random.default_rng(3)
    prim = cloud.initial_state(c, 0.8, 2.0)
    prim = prim * (1.0 + 1e-3 * rng.standard_normal(prim.shape))
    delu = 1e-4 * rng.standard_normal(prim.shape)
    s = Solver(c, 0.8, 2.0, storage_order=_lib.ORDER_MORTON)
    s.set_state(prim, delu, 0.5)
    p2, d2, r2 = s.get_state()
    assert np.array_equal(p2, prim) and np.array_equal(d2, delu) and r2 == 0.5
    s.initial_conditions(prim)
    assert np.array_equal(s.get(_lib.FIELD_PRIM), prim)
    s.close()
