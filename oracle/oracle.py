"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by the tests, by ``__graft_entry__.smoke()`` and by the CPU-baseline
leg of ``bench.py``; never by the solver library.  See mfcfd_oracle.cpp for
what the oracle restates and how its parity is pinned.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

FIELD_PRIM, FIELD_U, FIELD_Q, FIELD_QM, FIELD_DQ, FIELD_DELT, FIELD_FLUX_RES, \
    FIELD_DELUP, FIELD_DELUN, FIELD_DINV, FIELD_DELUP_FORWARD = range(11)
FIELD_WIDTH = {FIELD_PRIM: 5, FIELD_U: 5, FIELD_Q: 5, FIELD_QM: 10, FIELD_DQ: 15,
               FIELD_DELT: 1, FIELD_FLUX_RES: 5, FIELD_DELUP: 5, FIELD_DELUN: 5,
               FIELD_DINV: 1, FIELD_DELUP_FORWARD: 5}

LIBM_GLIBC = 0
LIBM_MFMATH = 1


class _Params(ctypes.Structure):
    _fields_ = [("power", ctypes.c_double), ("vl_const", ctypes.c_double),
                ("cfl", ctypes.c_double), ("rho_inf", ctypes.c_double),
                ("u1_inf", ctypes.c_double), ("u2_inf", ctypes.c_double),
                ("u3_inf", ctypes.c_double), ("pr_inf", ctypes.c_double),
                ("inner_iterations", ctypes.c_int), ("split_capacity", ctypes.c_int),
                ("update_variant", ctypes.c_int), ("sweep_variant", ctypes.c_int)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp = ctypes.c_void_p
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [ctypes.POINTER(_Params), ctypes.c_int] + [vp] * 10
        L.oracle_set_prim.argtypes = [vp, vp]
        L.oracle_set_libm.argtypes = [ctypes.c_int]
        L.oracle_fpi_step.argtypes = [vp, ctypes.c_int, vp, vp]
        L.oracle_get.argtypes = [vp, ctypes.c_int, vp]
        L.oracle_get.restype = ctypes.c_int
        L.oracle_get_stencils.argtypes = [vp, vp, vp, ctypes.c_int]
        L.oracle_get_alias.argtypes = [vp, vp, vp]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_libm_eval.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def libm_eval(fn: str, mode: int, x) -> np.ndarray:
    """exp / log / erf over x with glibc (mode 0) or mfmath.h (mode 1)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    lib().oracle_libm_eval({"exp": 0, "log": 1, "erf": 2}[fn], int(mode), _ptr(x), _ptr(y), x.size)
    return y


class Oracle:
    """The reference's q-LSKUM iteration on the CPU, one fpi_solver call per step."""

    def __init__(self, cloud, mach, aoa_deg, cfl=5.0, vl_const=2.0, power=0.0,
                 inner_iterations=0, split_capacity=22, libm=LIBM_GLIBC, update_variant=0,
                 sweep_variant=0):
        from mfcfd.cloud import freestream   # noqa: deferred import
        L = lib()
        rho, u1, u2, u3, pr = freestream(mach, aoa_deg)
        self.params = _Params(power, vl_const, cfl, rho, u1, u2, u3, pr,
                              inner_iterations, split_capacity, update_variant, sweep_variant)
        self.n = cloud.n
        self.libm = libm
        self._keep = [np.ascontiguousarray(a) for a in (
            cloud.status.astype(np.int32), cloud.x, cloud.y, cloud.z, cloud.tan1,
            cloud.tan2, cloud.nor, cloud.nbhs.astype(np.int32),
            cloud.conn.astype(np.int32), cloud.min_dist)]
        k = self._keep
        self.h = L.oracle_create(ctypes.byref(self.params), self.n, _ptr(k[0]), _ptr(k[1]),
                                 _ptr(k[2]), _ptr(k[3]), _ptr(k[4]), _ptr(k[5]), _ptr(k[6]),
                                 _ptr(k[7]), _ptr(k[8]), _ptr(k[9]))

    def set_prim(self, prim):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        assert prim.shape == (self.n, 5)
        lib().oracle_set_prim(self.h, _ptr(prim))

    def step(self, t):
        L = lib()
        L.oracle_set_libm(self.libm)
        r = np.zeros(2)
        L.oracle_fpi_step(self.h, int(t), _ptr(r[0:1]), _ptr(r[1:2]))
        return float(r[0]), float(r[1])

    def get(self, field):
        w = FIELD_WIDTH[field]
        out = np.empty((self.n, w), dtype=np.float64)
        rc = lib().oracle_get(self.h, field, _ptr(out))
        assert rc == 0
        return out if w > 1 else out[:, 0]

    def stencils(self, width=27):
        counts = np.empty((self.n, 6), dtype=np.int32)
        lists = np.empty((self.n, 6, width), dtype=np.int32)
        lib().oracle_get_stencils(self.h, _ptr(counts), _ptr(lists), width)
        return counts, lists

    def alias(self):
        a = np.empty(self.n, dtype=np.int32)
        p = np.empty(self.n, dtype=np.int32)
        lib().oracle_get_alias(self.h, _ptr(a), _ptr(p))
        return a, p

    def close(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_FLOPS_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_flops.so")
FLOP_PHASE_NAMES = ("conserved_q", "qderiv_delt", "flux", "dinv", "sweep_fwd", "sweep_bwd", "update",
                    "other")
FLOP_KINDS = ("add", "mul", "div", "sqrt", "fma", "exp", "log", "erf", "pow")


def flop_counts(cloud, mach, aoa_deg, iters=1, libm=LIBM_MFMATH, prim0=None, skip=0):
    """FP64 operations of `iters` iterations (after `skip` uncounted ones)
    of the oracle built with counting arithmetic (oracle_flops.cpp), per
    phase of fpi_solver: {phase: {kind: count}}, fma counted once per call
    (two operations).  With libm MFMATH the transcendentals are counted
    through their own arithmetic; exp/log/erf/pow are also given as calls."""
    if not os.path.exists(_FLOPS_LIB_PATH):
        build()
    from mfcfd.cloud import freestream, initial_state   # noqa: deferred import
    L = ctypes.CDLL(_FLOPS_LIB_PATH)
    vp = ctypes.c_void_p
    L.oracle_create.restype = vp
    L.oracle_create.argtypes = [ctypes.POINTER(_Params), ctypes.c_int] + [vp] * 10
    L.oracle_set_prim.argtypes = [vp, vp]
    L.oracle_set_libm.argtypes = [ctypes.c_int]
    L.oracle_fpi_step.argtypes = [vp, ctypes.c_int, vp, vp]
    L.oracle_flops_get.argtypes = [vp]
    L.oracle_destroy.argtypes = [vp]
    rho, u1, u2, u3, pr = freestream(mach, aoa_deg)
    params = _Params(0.0, 2.0, 5.0, rho, u1, u2, u3, pr, 0, 22, 0, 0)
    keep = [np.ascontiguousarray(a) for a in (
        cloud.status.astype(np.int32), cloud.x, cloud.y, cloud.z, cloud.tan1, cloud.tan2, cloud.nor,
        cloud.nbhs.astype(np.int32), cloud.conn.astype(np.int32), cloud.min_dist)]
    h = L.oracle_create(ctypes.byref(params), cloud.n, *[_ptr(a) for a in keep])
    p0 = np.ascontiguousarray(initial_state(cloud, mach, aoa_deg) if prim0 is None else prim0,
                              dtype=np.float64)
    L.oracle_set_prim(h, _ptr(p0))
    L.oracle_set_libm(int(libm))
    r = np.zeros(2)
    for t in range(1, skip + 1):
        L.oracle_fpi_step(h, t, _ptr(r[0:1]), _ptr(r[1:2]))
    L.oracle_flops_reset()
    for t in range(skip + 1, skip + iters + 1):
        L.oracle_fpi_step(h, t, _ptr(r[0:1]), _ptr(r[1:2]))
    out = np.zeros((len(FLOP_PHASE_NAMES), len(FLOP_KINDS)), dtype=np.int64)
    L.oracle_flops_get(_ptr(out))
    L.oracle_destroy(h)
    return {ph: {k: int(out[i, j]) for j, k in enumerate(FLOP_KINDS)} for i, ph in enumerate(FLOP_PHASE_NAMES)}


def flops_of(counts: dict) -> int:
    """Operations of one phase's counts: add, mul, div, sqrt one each, fma two."""
    return counts["add"] + counts["mul"] + counts["div"] + counts["sqrt"] + 2 * counts["fma"]


def forces(cloud, prim, mach, aoa_deg, wall_area=None, ref_area=None):
    """(CL, CD, F) of a state, summed over wall points in index order (the
    project's force definition; the reference computes none):
    F = -sum (p_i - p_inf) A_i nor_i with A_i = wall_area / n_wall."""
    import math
    from mfcfd.cloud import freestream
    rho, u1, u2, u3, pr = freestream(mach, aoa_deg)
    wa = cloud.wall_area if wall_area is None else wall_area
    ra = cloud.ref_area if ref_area is None else ref_area
    wall = np.nonzero(cloud.status == 1)[0]
    each = wa / len(wall)
    F = [0.0, 0.0, 0.0]
    for i in wall:
        dp = prim[i, 4] - pr
        for r in range(3):
            F[r] = F[r] - dp * each * cloud.nor[i, r]
    v = math.sqrt(u1 * u1 + u2 * u2 + u3 * u3)
    sa, ca = u2 / v, u1 / v
    q = 0.5 * rho * v * v * ra
    return (F[0] * (-sa) + F[1] * ca) / q, (F[0] * ca + F[1] * sa) / q, np.array(F)
