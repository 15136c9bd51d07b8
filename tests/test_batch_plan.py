"""Host logic of lockstep groups: batch.plan_groups and batch.plan_waves on
stand-in solvers (no device).  Groups keep one block shape, chain_spread and
precision class, at most GROUP_MAX_CLOUDS solvers and chain slots within the
device's capacity, largest clouds first; waves hold consecutive groups whose
slots fit together."""
from types import SimpleNamespace

from mfcfd import _lib, batch

CAP = 6 * (148 - 16)


def _fake(n, slots, wpb=4, precision=0, spread=0):
    info = {"chain_slots": slots, "chain_slot_capacity": CAP, "chain_warps_per_block": wpb}
    return SimpleNamespace(n=n, params=SimpleNamespace(precision=precision, chain_spread=spread),
                           info=lambda info=info: dict(info))


def _check(solvers, groups):
    assert sorted(i for g in groups for i in g) == list(range(len(solvers)))
    for g in groups:
        assert 1 <= len(g) <= _lib.GROUP_MAX_CLOUDS
        keys = {(solvers[i].info()["chain_warps_per_block"], solvers[i].params.chain_spread,
                 solvers[i].params.precision != 0) for i in g}
        assert len(keys) == 1
        assert len(g) == 1 or sum(solvers[i].info()["chain_slots"] for i in g) <= CAP
        sizes = [solvers[i].n for i in g]
        assert sizes == sorted(sizes, reverse=True)


def test_groups_split_by_shape_and_precision_class():
    s = [_fake(1000 + i, 30, wpb=4 if i % 3 else 8, precision=(0, 1, 2)[i % 3]) for i in range(30)]
    groups = batch.plan_groups(s)
    _check(s, groups)
    # MIXED and MIXED_DC share a class; FP64 is its own
    for g in groups:
        assert len({s[i].params.precision == 0 for i in g}) == 1


def test_groups_respect_capacity_and_count():
    s = [_fake(50000 - 100 * i, 60) for i in range(100)]         # 13 fit the slots
    groups = batch.plan_groups(s)
    _check(s, groups)
    assert [len(g) for g in groups[:-1]] == [CAP // 60] * (len(groups) - 1)
    s = [_fake(20000 + i, 3) for i in range(70)]                 # the count limits
    groups = batch.plan_groups(s)
    _check(s, groups)
    assert [len(g) for g in groups] == [32, 32, 6]
    # largest first: the first group holds the 32 largest clouds
    assert min(s[i].n for i in groups[0]) > max(s[i].n for g in groups[1:] for i in g)


def test_a_cloud_larger_than_the_capacity_is_its_own_group():
    s = [_fake(900000, CAP + 10), _fake(1000, 5), _fake(2000, 5)]
    groups = batch.plan_groups(s)
    _check(s, groups)
    assert [0] in groups


def test_waves_pack_consecutive_groups_within_capacity():
    s = [_fake(1000 + i, 100, precision=i % 2) for i in range(12)]
    groups = batch.plan_groups(s)
    waves = batch.plan_waves(s, groups)
    assert [gi for w in waves for gi in w] == list(range(len(groups)))
    for w in waves:
        slots = sum(s[i].info()["chain_slots"] for gi in w for i in groups[gi])
        assert len(w) == 1 or slots <= CAP
    # 6 FP64 and 6 mixed clouds of 100 slots: two groups of 6 (600 slots each), one each wave
    assert [len(g) for g in groups] == [6, 6] and len(waves) == 2
    s = [_fake(1000 + i, 40, precision=i % 2) for i in range(12)]
    groups = batch.plan_groups(s)
    assert len(batch.plan_waves(s, groups)) == 1                  # 2 x 240 slots fit together
