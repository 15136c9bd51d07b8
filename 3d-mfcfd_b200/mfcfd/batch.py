"""Concurrent iteration of several clouds on one GPU.

Each cloud keeps its own handle (state resident, own streams).  A batch call
(mfcfd_run_batch) launches every cloud's iterations in turn so that one
cloud's latency-bound LU-SGS sweeps run beside another's; clouds whose
chain-schedule sweeps would not all fit on the device together run as they
fit, each starting its next chunk as soon as there is room.  A group call
(mfcfd_run_group) runs up to 32 clouds in lockstep with each sweep
direction of all of them in one kernel launch; plan_groups packs a batch
into such groups and run_grouped runs them, side by side where their
sweeps fit the device together.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import MfcfdError, ptr


def run_batch(solvers, iters: int, t0=None, statuses=None):
    """Run `iters` iterations of every Solver; returns res_hist
    (len(solvers), iters, 2) and appends to each solver's history.  With a
    list `statuses`, a cloud's failure (a non-finite residual, say) is
    recorded there instead of raised, and the other clouds' histories are
    kept."""
    return _run("mfcfd_run_batch", solvers, iters, t0, statuses)


def run_group(solvers, iters: int, t0=None, statuses=None):
    """As run_batch, in lockstep with one chain-sweep launch per direction
    for all the solvers (mfcfd_run_group): at most GROUP_MAX_CLOUDS chain-
    schedule solvers of one block shape and precision class whose sweeps
    fit the device together (plan_groups makes such groups)."""
    return _run("mfcfd_run_group", solvers, iters, t0, statuses)


def plan_groups(solvers):
    """Pack solvers into groups that mfcfd_run_group accepts: by block shape
    and precision class, largest clouds first, each group filled while its
    chain slots fit the device and it has fewer than GROUP_MAX_CLOUDS
    solvers.  Clouds of similar size then share a group, so a lockstep
    iteration waits little for its slowest sweep.  Returns lists of indices
    into `solvers`."""
    infos = [s.info() for s in solvers]
    keys = {}
    for i, (s, inf) in enumerate(zip(solvers, infos)):
        k = (inf["chain_warps_per_block"], int(s.params.chain_spread), int(s.params.precision) != 0)
        keys.setdefault(k, []).append(i)
    groups = []
    for k in sorted(keys):
        idx = sorted(keys[k], key=lambda i: -solvers[i].n)
        cur, used = [], 0
        for i in idx:
            sl, cap = infos[i]["chain_slots"], infos[i]["chain_slot_capacity"]
            if cur and (used + sl > cap or len(cur) >= _lib.GROUP_MAX_CLOUDS):
                groups.append(cur)
                cur, used = [], 0
            cur.append(i)
            used += sl
        if cur:
            groups.append(cur)
    return groups


def plan_waves(solvers, groups):
    """Consecutive groups whose chain slots fit the device together, as
    lists of group indices: the groups of a wave may run side by side."""
    waves, cur, used = [], [], 0
    for gi, g in enumerate(groups):
        infos = [solvers[i].info() for i in g]
        sl, cap = sum(x["chain_slots"] for x in infos), infos[0]["chain_slot_capacity"]
        if cur and used + sl > cap:
            waves.append(cur)
            cur, used = [], 0
        cur.append(gi)
        used += sl
    if cur:
        waves.append(cur)
    return waves


def run_grouped(solvers, iters: int, groups=None, statuses=None):
    """run_group over plan_groups(solvers) (or the given groups); returns
    res_hist (len(solvers), iters, 2) in the solvers' order.  Groups whose
    chain sweeps fit the device together (plan_waves) run side by side, one
    host thread each (the library call releases the interpreter), so all
    their sweeps stay resident; the waves run one after another."""
    import threading
    groups = plan_groups(solvers) if groups is None else groups
    hist = np.zeros((len(solvers), iters, 2))
    st = [0] * len(solvers)
    for wave in plan_waves(solvers, groups):
        errors = []

        def one(g):
            part = [] if statuses is not None else None
            try:
                hist[g] = run_group([solvers[i] for i in g], iters, statuses=part)
            except Exception as e:          # re-raised below, after the wave
                errors.append(e)
                return
            if part is not None:
                for i, v in zip(g, part):
                    st[i] = v

        if len(wave) == 1:
            one(groups[wave[0]])
        else:
            threads = [threading.Thread(target=one, args=(groups[gi],)) for gi in wave]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
        if errors:
            raise errors[0]
    if statuses is not None:
        statuses[:] = st
    return hist


def _run(fn: str, solvers, iters: int, t0, statuses):
    n = len(solvers)
    hs = (ctypes.c_void_p * n)(*[s.h.value for s in solvers])
    if t0 is None:
        t0 = [len(s.history) + 1 for s in solvers]
    t0a = np.ascontiguousarray(t0, dtype=np.int32)
    hist = np.zeros((n, iters, 2))
    status = np.zeros(n, dtype=np.int32)
    rc = getattr(_lib.lib(), fn)(hs, n, ptr(t0a), int(iters), ptr(hist), ptr(status))
    if rc != 0 and not status.any():   # refused as a whole: nothing ran
        msg = _lib.lib().mfcfd_last_error(solvers[0].h).decode() if n else ""
        raise MfcfdError(rc, msg or "batch failed")
    if statuses is not None:
        statuses[:] = [int(v) for v in status]
    for i, s in enumerate(solvers):
        if status[i] != 0:
            if statuses is not None:
                continue
            raise MfcfdError(int(status[i]), _lib.lib().mfcfd_last_error(s.h).decode())
        for j in range(iters):
            s.history.append((int(t0a[i]) + j, float(hist[i, j, 0]), float(hist[i, j, 1])))
    return hist


def tune_all(solvers, iters: int = 3, candidates=None):
    """Autotune each Solver's chain schedule (mfcfd_tune_chain) before a
    batch; returns the chosen warp counts.  States are left unchanged."""
    return [s.tune_chain(candidates, iters)[0] for s in solvers]


def tune_batch(solvers, percents=(75, 100, 125, 150, 200), iters: int = 4):
    """Autotune a batch as a whole: for each candidate, every cloud's chain
    schedule gets that percentage of its widest sweep level in warps, and a
    round of `iters` batched iterations is timed (after an untimed round that
    captures the graphs).  Fewer warps per cloud let more clouds share the
    device at once; the fastest percentage is kept.  States and histories
    are restored; results do not depend on the choice.  Returns (percent,
    {percent: seconds per round})."""
    import time
    states = [s.get_state() for s in solvers]
    hist = [len(s.history) for s in solvers]
    widths = [s.info()["max_level_width"] for s in solvers]

    def restore():
        for s, st, h in zip(solvers, states, hist):
            s.set_state(*st)
            del s.history[h:]

    times = {}
    for pc in percents:
        for s, w in zip(solvers, widths):
            s.set_chain_warps(max(4, w * pc // 100))
        for rep in range(2 if iters % 2 == 0 else 3):
            restore()
            t = time.perf_counter()
            run_batch(solvers, iters)
            times[pc] = time.perf_counter() - t
    best = min(times, key=times.get)
    for s, w in zip(solvers, widths):
        s.set_chain_warps(max(4, w * best // 100))
    restore()
    return best, times


def solve_batch(solvers, target: float = -6.0, max_iters: int = 12000, chunk: int = 100,
                polish: float | None = -5.0, grouped: bool = False):
    """Run every Solver until its residue reaches `target` (or `max_iters`),
    in batched rounds of `chunk` iterations over the clouds still running.
    A MIXED_DC solver switches to FP64 once its residue is at or below
    `polish` (None: never), so it reaches a 1e-6 drop in about FP64's
    iteration count.  With `grouped`, each round runs as lockstep groups
    (run_grouped, planned again every round, since clouds retire and switch
    precision class); otherwise as one run_batch.  Returns, per solver, a
    dict with the iterations run, whether it converged, and the seconds
    from the call to its retirement."""
    import time
    t_start = time.perf_counter()
    live = list(range(len(solvers)))
    out = [dict(iters=0, converged=False, seconds=None, polished=False) for _ in solvers]
    while live:
        hist = (run_grouped if grouped else run_batch)([solvers[i] for i in live], chunk)
        now = time.perf_counter() - t_start
        keep = []
        for j, i in enumerate(live):
            s = solvers[i]
            out[i]["iters"] += chunk
            res = hist[j, -1, 1]
            t_last = len(s.history)
            if t_last > 2 and res <= target:
                out[i].update(converged=True, seconds=now)
                continue
            if out[i]["iters"] >= max_iters:
                out[i]["seconds"] = now
                continue
            if (polish is not None and not out[i]["polished"] and s.params.precision == _lib.PRECISION_MIXED_DC
                    and t_last > 2 and res <= polish):
                s.set_precision(_lib.PRECISION_FP64)
                out[i]["polished"] = True
            keep.append(i)
        live = keep
    return out
