"""Concurrent iteration of several clouds on one GPU (mfcfd_run_batch).

Each cloud keeps its own handle (state resident, own streams); a batch call
launches every cloud's iterations in turn so that one cloud's latency-bound
LU-SGS sweeps run beside another's.  Clouds whose chain-schedule sweeps
would not all fit on the device together are run in successive waves.
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
    n = len(solvers)
    hs = (ctypes.c_void_p * n)(*[s.h.value for s in solvers])
    if t0 is None:
        t0 = [len(s.history) + 1 for s in solvers]
    t0a = np.ascontiguousarray(t0, dtype=np.int32)
    hist = np.zeros((n, iters, 2))
    status = np.zeros(n, dtype=np.int32)
    rc = _lib.lib().mfcfd_run_batch(hs, n, ptr(t0a), int(iters), ptr(hist), ptr(status))
    if statuses is not None:
        statuses[:] = [int(v) for v in status]
    for i, s in enumerate(solvers):
        if status[i] != 0:
            if statuses is not None:
                continue
            raise MfcfdError(int(status[i]), _lib.lib().mfcfd_last_error(s.h).decode())
        for j in range(iters):
            s.history.append((int(t0a[i]) + j, float(hist[i, j, 0]), float(hist[i, j, 1])))
    if rc != 0 and (statuses is None or not any(statuses)):
        raise MfcfdError(rc, "batch failed")
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
                polish: float | None = -5.0):
    """Run every Solver until its residue reaches `target` (or `max_iters`),
    in batched rounds of `chunk` iterations over the clouds still running.
    A MIXED_DC solver switches to FP64 once its residue is at or below
    `polish` (None: never), so it reaches a 1e-6 drop in about FP64's
    iteration count.  Returns, per solver, a dict with the iterations run,
    whether it converged, and the seconds from the call to its retirement."""
    import time
    t_start = time.perf_counter()
    live = list(range(len(solvers)))
    out = [dict(iters=0, converged=False, seconds=None, polished=False) for _ in solvers]
    while live:
        hist = run_batch([solvers[i] for i in live], chunk)
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
