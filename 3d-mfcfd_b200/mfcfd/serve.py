"""Request server: steady-state solves with continuous batching on one GPU.

Python side of mfcfd_server_* (include/mfcfd.h).  Requests (a point cloud,
Mach number, angle of attack) are prepared on host threads, admitted while
their device memory fits the budget, iterate side by side in chunks of
`chunk` iterations (each started as soon as its chain sweep fits on the
device) and retire when their residue reaches the target (or at
max_iters).  Each result equals the same request solved alone.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import MfcfdError, ptr
from .cloud import PointCloud, initial_state
from .solver import params_for


def _cloud_arrays(cloud: PointCloud):
    return [np.ascontiguousarray(a) for a in (
        cloud.status.astype(np.int32), cloud.x, cloud.y, cloud.z, cloud.tan1, cloud.tan2,
        cloud.nor, cloud.nbhs.astype(np.int32), cloud.conn.astype(np.int32), cloud.min_dist)]


class Server:
    def __init__(self, device: int = 0, max_live: int = 0, setup_threads: int = 2, chunk: int = 20,
                 hbm_budget: int = 0, chain_percent: int = 100, device_setup: bool = False):
        cfg = _lib.ServerConfig(device=device, max_live=max_live, setup_threads=setup_threads,
                                chunk=chunk, hbm_budget=hbm_budget, chain_percent=chain_percent,
                                device_setup=1 if device_setup else 0)
        self.chunk = chunk
        self.h = ctypes.c_void_p()
        rc = _lib.lib().mfcfd_server_create(ctypes.byref(cfg), ctypes.byref(self.h))
        if rc != 0:
            raise MfcfdError(rc, "mfcfd_server_create failed")
        self._n = {}

    def submit(self, cloud: PointCloud, mach: float, aoa_deg: float, *, max_iters: int = 1000,
               residue_target: float = -6.0, prim: np.ndarray | None = None, forces: bool = True,
               polish_residue: float = 0.0, **params) -> int:
        """Queue one solve; returns its id.  The arrays are copied.  The
        initial state defaults to Solver.initial_conditions' (the impulsive
        start of cloud.initial_state)."""
        arrs = _cloud_arrays(cloud)
        if prim is None:
            prim = initial_state(cloud, mach, aoa_deg)
        p0 = np.ascontiguousarray(prim, dtype=np.float64)
        q = _lib.Request()
        q.params = params_for(mach, aoa_deg, **params)
        q.n = cloud.n
        for name, a in zip(("status", "x", "y", "z", "tan1", "tan2", "nor", "nbhs", "conn", "min_dist"),
                           arrs):
            setattr(q, name, a.ctypes.data)
        q.prim = p0.ctypes.data
        q.max_iters = int(max_iters)
        q.residue_target = float(residue_target)
        q.polish_residue = float(polish_residue)
        if forces:
            q.wall_area, q.ref_area = float(cloud.wall_area), float(cloud.ref_area)
        rid = ctypes.c_int64()
        rc = _lib.lib().mfcfd_server_submit(self.h, ctypes.byref(q), ctypes.byref(rid))
        if rc != 0:
            raise MfcfdError(rc, "mfcfd_server_submit failed")
        self._n[rid.value] = cloud.n
        return rid.value

    def wait(self, rid: int, timeout: float | None = None, with_prim: bool = True) -> dict:
        """The retired request's result (fields of mfcfd_result; 'prim' the
        final (N, 5) state).  Raises MfcfdError(10) if not done in time."""
        res = _lib.Result()
        prim = np.empty((self._n[rid], 5)) if with_prim else None
        rc = _lib.lib().mfcfd_server_wait(self.h, int(rid), -1.0 if timeout is None else float(timeout),
                                          ctypes.byref(res), None if prim is None else ptr(prim))
        if rc != 0:
            raise MfcfdError(rc, f"request {rid}")
        del self._n[rid]
        out = {f: getattr(res, f) for f, _ in _lib.Result._fields_}
        out["latency"] = res.t_done - res.t_submit
        if prim is not None and res.status == 0:
            out["prim"] = prim
        return out

    def stats(self) -> dict:
        st = _lib.ServerStats()
        rc = _lib.lib().mfcfd_server_get_stats(self.h, ctypes.byref(st))
        if rc != 0:
            raise MfcfdError(rc, "mfcfd_server_get_stats failed")
        return {f: getattr(st, f) for f, _ in _lib.ServerStats._fields_}

    def close(self):
        if self.h and self.h.value:
            _lib.lib().mfcfd_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_arrivals(rate: float, count: int, seed: int) -> np.ndarray:
    """Arrival times (s) of a Poisson stream of `count` requests at `rate`/s."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def latency_summary(latencies) -> dict:
    """p50 / p99 / mean / max of a list of latencies (s)."""
    a = np.asarray(latencies, dtype=np.float64)
    if a.size == 0:
        return {"p50": None, "p99": None, "mean": None, "max": None}
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
            "mean": float(a.mean()), "max": float(a.max())}


def solve_alone(cloud: PointCloud, mach: float, aoa_deg: float, chunk: int, max_iters: int,
                residue_target: float, **params) -> dict:
    """The server's convergence rule for one request on its own handle:
    rounds of `chunk` iterations from t = 1 until the residue after a round
    is <= residue_target (t > 2) or max_iters (rounded up to whole rounds)."""
    from .solver import Solver
    s = Solver(cloud, mach, aoa_deg, **params)
    s.initial_conditions()
    limit = -(-max_iters // chunk) * chunk
    t, converged = 1, False
    while t - 1 < limit:
        h = s.q_lskum(chunk, t0=t)
        t += chunk
        if t - 1 > 2 and h[-1, 1] <= residue_target:
            converged = True
            break
    cl, cd, _ = s.forces()
    out = {"iters": t - 1, "converged": converged, "res_new": float(h[-1, 0]),
           "residue": float(h[-1, 1]), "cl": cl, "cd": cd, "prim": s.get(_lib.FIELD_PRIM)}
    s.close()
    return out


def device_bytes(cloud: PointCloud, mach: float, aoa_deg: float, device: int = 0, **params) -> int:
    """Device memory a request for this cloud holds while live
    (mfcfd_prepare + mfcfd_device_bytes; nothing is allocated)."""
    L = _lib.lib()
    p = params_for(mach, aoa_deg, device=device, **params)
    arrs = _cloud_arrays(cloud)
    h = ctypes.c_void_p()
    rc = L.mfcfd_prepare(ctypes.byref(p), cloud.n, *[ptr(a) for a in arrs], ctypes.byref(h))
    try:
        if rc != 0:
            raise MfcfdError(rc, L.mfcfd_last_error(h).decode() if h.value else "")
        b = ctypes.c_int64()
        rc = L.mfcfd_device_bytes(h, ctypes.byref(b))
        if rc != 0:
            raise MfcfdError(rc, L.mfcfd_last_error(h).decode())
        return int(b.value)
    finally:
        if h.value:
            L.mfcfd_destroy(h)


def request_stream(count: int, rate: float, seed: int, n_min: int, n_max: int, pool: int = 8,
                   mach=(0.3, 0.85), alpha=(-5.0, 5.0), aspect=(1.0, 3.0), bodies: str = "mixed",
                   knn_device: int = -1):
    """A seeded stream of solve requests: Poisson arrival times at `rate`/s,
    each naming one of `pool` shell clouds (sphere or ellipsoid body with
    axis ratios U[aspect], point counts log-uniform in [n_min, n_max], shell
    count proportional to N^(1/3)) and a flow (Mach U[mach], angle of attack
    U[alpha] degrees).  bodies "mixed" alternates spheres and ellipsoids,
    "ellipsoids" makes every body one.  Returns (arrivals, clouds, [(cloud
    index, mach, alpha)])."""
    import math
    from . import cloud as cl
    rng = np.random.Generator(np.random.PCG64(seed))
    clouds = []
    for j in range(pool):
        n = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        shells = max(8, int(round(1.21 * n ** (1.0 / 3.0))))
        per = max(100, int(round(n / shells)))
        ell = bodies == "ellipsoids" or j % 2 == 1
        ax = (1.0, rng.uniform(*aspect), rng.uniform(*aspect)) if ell else (1.0, 1.0, 1.0)
        clouds.append(cl.shell_cloud(shells, per, jitter=0.02, seed=seed * 100 + j, aspect=ax,
                                     name=f"{'ellipsoid' if ell else 'sphere'}-{shells}x{per}",
                                     knn_device=knn_device))
    arrivals = poisson_arrivals(rate, count, seed + 1)
    reqs = [(int(rng.integers(pool)), float(rng.uniform(*mach)), float(rng.uniform(*alpha)))
            for _ in range(count)]
    return arrivals, clouds, reqs
