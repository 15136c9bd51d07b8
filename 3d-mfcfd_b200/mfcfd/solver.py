"""Python mirror of the reference's solver interface over the C ABI.

The reference drives its solver from ``q_lskum`` (q_lskum.f90:15-36):
split stencils and aliasing once, then ``fpi_solver(t)`` per iteration,
logging ``t res_new residue``.  ``Solver`` offers the same calls on a GPU
handle: construction does ``generate_split_stencils`` + ``aliasing`` (and
the upload), ``fpi_solver(t)`` is one iteration, ``q_lskum(max_iters)`` the
loop.  Errors raise ``MfcfdError`` with the library's message.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FIELD_WIDTH, MfcfdError, ptr
from .cloud import PointCloud, initial_state


def params_for(mach: float, aoa_deg: float, **over) -> _lib.Params:
    """parameter.f90's constants for the given flow, with overrides."""
    p = _lib.Params()
    _lib.lib().mfcfd_params_init(ctypes.byref(p), float(mach), float(aoa_deg))
    for k, v in over.items():
        setattr(p, k, v)
    return p


class Solver:
    """One point cloud resident on one GPU (or a host-only handle, device=-1)."""

    def __init__(self, cloud: PointCloud, mach: float, aoa_deg: float, **params):
        self.cloud = cloud
        self.n = cloud.n
        self.mach = mach
        self.aoa = aoa_deg
        L = _lib.lib()
        self.params = params_for(mach, aoa_deg, **params)
        self._inputs = [np.ascontiguousarray(a) for a in (
            cloud.status.astype(np.int32), cloud.x, cloud.y, cloud.z, cloud.tan1, cloud.tan2,
            cloud.nor, cloud.nbhs.astype(np.int32), cloud.conn.astype(np.int32),
            cloud.min_dist)]
        h = ctypes.c_void_p()
        rc = L.mfcfd_create(ctypes.byref(self.params), self.n,
                            *[ptr(a) for a in self._inputs], ctypes.byref(h))
        self.h = h
        if rc != 0:
            msg = L.mfcfd_last_error(h).decode() if h.value else ""
            self.close()
            raise MfcfdError(rc, msg)
        self.history = []
        if cloud.wall_areas is not None and self.params.device >= 0:
            self.set_wall_areas(cloud.wall_areas)

    # -- reference entry points ------------------------------------------
    def _check(self, rc):
        if rc != 0:
            raise MfcfdError(rc, _lib.lib().mfcfd_last_error(self.h).decode())

    def initial_conditions(self, prim=None):
        """initial_conditions.f90: set prim, zero delUp/delUn."""
        if prim is None:
            prim = initial_state(self.cloud, self.mach, self.aoa)
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        assert prim.shape == (self.n, 5)
        self._check(_lib.lib().mfcfd_set_prim(self.h, ptr(prim)))

    def fpi_solver(self, t: int):
        """One iteration; returns (res_new, residue)."""
        out = np.zeros(2)
        self._check(_lib.lib().mfcfd_fpi_step(self.h, int(t), ptr(out[0:1]), ptr(out[1:2])))
        self.history.append((int(t), float(out[0]), float(out[1])))
        return float(out[0]), float(out[1])

    def q_lskum(self, max_iters: int, t0: int = 1):
        """The iteration loop on the device; returns an (iters, 2) array of
        (res_new, residue)."""
        hist = np.zeros((max_iters, 2))
        self._check(_lib.lib().mfcfd_run(self.h, int(t0), int(max_iters), ptr(hist)))
        for j in range(max_iters):
            self.history.append((t0 + j, float(hist[j, 0]), float(hist[j, 1])))
        return hist

    def print_primal_output(self, directory: str = "."):
        """post_processor.f90:13-44: primal-solution.dat, flux-residual.dat,
        qderivatives.dat and an empty normals.dat in `directory`."""
        import os
        self._check(_lib.lib().mfcfd_print_primal_output(self.h, os.fsencode(directory)))

    def forces(self, wall_area: float | None = None, ref_area: float | None = None):
        """(CL, CD, F) of the current state: F = -sum over wall points of
        (p - p_inf) A nor with A = wall_area / n_wall (defaults: the cloud's
        own areas)."""
        wa = self.cloud.wall_area if wall_area is None else wall_area
        ra = self.cloud.ref_area if ref_area is None else ref_area
        cl, cd = ctypes.c_double(), ctypes.c_double()
        f = np.zeros(3)
        self._check(_lib.lib().mfcfd_forces(self.h, float(wa), float(ra), ctypes.byref(cl),
                                            ctypes.byref(cd), ptr(f)))
        return float(cl.value), float(cd.value), f

    def set_wall_areas(self, area=None):
        """mfcfd_set_wall_areas: per-point areas (N values, index order) for
        forces(); None returns to the even split of the wall area."""
        if area is None:
            self._check(_lib.lib().mfcfd_set_wall_areas(self.h, None))
            return
        self._area = np.ascontiguousarray(area, dtype=np.float64)
        assert self._area.shape == (self.n,)
        self._check(_lib.lib().mfcfd_set_wall_areas(self.h, ptr(self._area)))

    def tune_chain(self, candidates=None, iters: int = 3):
        """mfcfd_tune_chain: time the chain schedule for each candidate warp
        count (default 1.5, 2, 3, 4 times the widest level) from the current
        state, keep the fastest; the state is left as it was.  Returns the
        kept warp count and {candidate index: ms per iteration}."""
        cand = None if candidates is None else np.ascontiguousarray(candidates, dtype=np.int32)
        count = 0 if cand is None else len(cand)
        ms = np.zeros(max(count, 4))
        chosen = ctypes.c_int32()
        self._check(_lib.lib().mfcfd_tune_chain(self.h, None if cand is None else ptr(cand), count, int(iters),
                                                ctypes.byref(chosen), ptr(ms)))
        return chosen.value, ms[:count if count else 4]

    def launch(self, t0: int, iters: int):
        """mfcfd_launch: queue iterations t0 .. t0+iters-1 and return."""
        self._check(_lib.lib().mfcfd_launch(self.h, int(t0), int(iters)))
        self._pending = (int(t0), int(iters))

    def complete(self, wait: bool = True):
        """mfcfd_complete: None while the launched iterations run (wait
        False), else their (iters, 2) (res_new, residue) history."""
        t0, iters = self._pending
        hist = np.zeros((iters, 2))
        done = ctypes.c_int32()
        self._check(_lib.lib().mfcfd_complete(self.h, 1 if wait else 0, ptr(hist), ctypes.byref(done)))
        if not done.value:
            return None
        for j in range(iters):
            self.history.append((t0 + j, float(hist[j, 0]), float(hist[j, 1])))
        return hist

    def set_chain_warps(self, warps: int) -> int:
        """mfcfd_set_chain_warps: rebuild the chain schedule for about
        `warps` warps; returns the schedule's warps."""
        actual = ctypes.c_int32()
        self._check(_lib.lib().mfcfd_set_chain_warps(self.h, int(warps), ctypes.byref(actual)))
        return actual.value

    # -- data access ---------------------------------------------------------
    def get(self, field: int) -> np.ndarray:
        w = FIELD_WIDTH[field]
        out = np.empty((self.n, w), dtype=np.float64)
        self._check(_lib.lib().mfcfd_get(self.h, int(field), ptr(out)))
        return out if w > 1 else out[:, 0]

    def get_state(self, out=None):
        """(prim, delUn, res_old); `out` = (prim, delu) arrays (N, 5) to fill,
        e.g. pinned host buffers, instead of new ones."""
        prim, delu = out if out is not None else (np.empty((self.n, 5)), np.empty((self.n, 5)))
        ro = np.zeros(1)
        self._check(_lib.lib().mfcfd_get_state(self.h, ptr(prim), ptr(delu), ptr(ro)))
        return prim, delu, float(ro[0])

    def set_state(self, prim, delu, res_old=0.0):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        delu = np.ascontiguousarray(delu, dtype=np.float64)
        self._check(_lib.lib().mfcfd_set_state(self.h, ptr(prim), ptr(delu), float(res_old)))

    def stencils(self, width: int = 27):
        counts = np.empty((self.n, 6), dtype=np.int32)
        lists = np.empty((self.n, 6, width), dtype=np.int32)
        self._check(_lib.lib().mfcfd_get_stencils(self.h, ptr(counts), ptr(lists), int(width)))
        return counts, lists

    def alias(self):
        a = np.empty(self.n, dtype=np.int32)
        p = np.empty(self.n, dtype=np.int32)
        self._check(_lib.lib().mfcfd_get_alias(self.h, ptr(a), ptr(p)))
        return a, p

    def levels(self, direction: int = 0):
        lv = np.empty(self.n, dtype=np.int32)
        self._check(_lib.lib().mfcfd_get_levels(self.h, int(direction), ptr(lv)))
        return lv

    def digest(self, name: str):
        """(FNV-1a digest, bytes) of one device topology array
        (mfcfd_debug_digest); bytes -1 when the array is not allocated."""
        dg, nb = ctypes.c_uint64(), ctypes.c_int64()
        self._check(_lib.lib().mfcfd_debug_digest(self.h, name.encode(), ctypes.byref(dg), ctypes.byref(nb)))
        return int(dg.value), int(nb.value)

    def info(self) -> dict:
        inf = _lib.Info()
        self._check(_lib.lib().mfcfd_get_info(self.h, ctypes.byref(inf)))
        return {k: getattr(inf, k) for k, _ in _lib.Info._fields_}

    def stream(self) -> int:
        sp = ctypes.c_void_p()
        self._check(_lib.lib().mfcfd_get_stream(self.h, ctypes.byref(sp)))
        return sp.value or 0

    def set_profiling(self, on: bool):
        self._check(_lib.lib().mfcfd_set_profiling(self.h, 1 if on else 0))

    def phase_times(self):
        """(dict phase -> summed ms, iterations) since profiling was enabled."""
        ms = np.zeros(_lib.NPHASE)
        it = np.zeros(1, dtype=np.int64)
        self._check(_lib.lib().mfcfd_get_phase_times(self.h, ptr(ms), ptr(it)))
        return dict(zip(_lib.PHASES, ms.tolist())), int(it[0])

    def residual_noalloc(self) -> float:
        """res_new of the last iteration, recomputed without any device
        allocation (mfcfd_residual_noalloc)."""
        out = np.zeros(1)
        self._check(_lib.lib().mfcfd_residual_noalloc(self.h, ptr(out)))
        return float(out[0])

    def set_precision(self, precision: int):
        """mfcfd_set_precision: switch between FP64 and MIXED_DC between
        iterations."""
        self._check(_lib.lib().mfcfd_set_precision(self.h, int(precision)))
        self.params.precision = int(precision)

    def set_fault_hook(self, point: int, wait_limit: int = 0):
        """Failure-detection test hook (mfcfd_set_fault_hook): point (1-based,
        0 off) publishes none of its sweep increments, and device waits give
        up after wait_limit poll rounds (0: the default)."""
        self._check(_lib.lib().mfcfd_set_fault_hook(self.h, int(point), int(wait_limit)))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            _lib.lib().mfcfd_destroy(self.h)
        self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
