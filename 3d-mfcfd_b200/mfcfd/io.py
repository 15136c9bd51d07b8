"""The reference program's files through the C ABI (csrc/mfcfd_io.cpp).

``read_input_point_data`` reads ``3d_input_data`` (point_preprocessor.f90:
25-36) into a ``PointCloud``; ``read_stored_solution`` reads
``stored-solution.dat`` (initial_conditions.f90:18-29); ``write_residue``
writes ``residue.dat`` lines (q_lskum.f90:22,31).  The output files of
``print_primal_output`` come from ``Solver.print_primal_output``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import MfcfdError, ptr
from .cloud import MAX_CONN, PointCloud


def _check(rc):
    if rc != 0:
        raise MfcfdError(rc, _lib.lib().mfcfd_last_error(None).decode())


def count_input_points(path: str) -> int:
    n = ctypes.c_int32()
    _check(_lib.lib().mfcfd_count_input_points(os.fsencode(path), ctypes.byref(n)))
    return int(n.value)


def read_input_point_data(path: str, n: int | None = None) -> PointCloud:
    """3d_input_data -> PointCloud (n records; all of them when n is None,
    where the reference takes max_points from parameter.f90)."""
    if n is None:
        n = count_input_points(path)
    status = np.zeros(n, np.int32)
    x, y, z = np.zeros(n), np.zeros(n), np.zeros(n)
    tan1, tan2, nor = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
    nbhs = np.zeros(n, np.int32)
    conn = np.zeros((n, MAX_CONN), np.int32)
    min_dist = np.zeros(n)
    _check(_lib.lib().mfcfd_read_input_point_data(
        os.fsencode(path), n, ptr(status), ptr(x), ptr(y), ptr(z), ptr(tan1), ptr(tan2), ptr(nor),
        ptr(nbhs), ptr(conn), ptr(min_dist)))
    return PointCloud(status=status, x=x, y=y, z=z, tan1=tan1, tan2=tan2, nor=nor, nbhs=nbhs,
                      conn=conn, min_dist=min_dist, name=os.path.basename(path))


def read_stored_solution(path: str, n: int) -> np.ndarray:
    """stored-solution.dat -> prim (n, 5) (x, y, z of each record dropped)."""
    prim = np.zeros((n, 5))
    _check(_lib.lib().mfcfd_read_stored_solution(os.fsencode(path), n, ptr(prim)))
    return prim


def write_residue(path: str, t0: int, res_hist: np.ndarray, append: bool = False):
    """residue.dat: `t res_new residue` per iteration of an mfcfd_run history."""
    h = np.ascontiguousarray(res_hist, dtype=np.float64).reshape(-1, 2)
    _check(_lib.lib().mfcfd_write_residue(os.fsencode(path), t0, h.shape[0], ptr(h), int(append)))
