"""ctypes binding of the C ABI in include/mfcfd.h (libmfcfd.so, built in-tree)."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmfcfd.so")

MFCFD_OK = 0
ERRORS = {1: "bad argument", 2: "CUDA error", 3: "stencil too wide",
          4: "singular least-squares system", 5: "non-finite residual",
          6: "unsupported input", 7: "out of memory", 8: "device wait timed out",
          9: "file input/output error", 10: "request not finished"}

FIELD_PRIM, FIELD_U, FIELD_Q, FIELD_QM, FIELD_DQ, FIELD_DELT, FIELD_FLUX_RES, \
    FIELD_DELUP, FIELD_DELUN, FIELD_DINV = range(10)
FIELD_WIDTH = {FIELD_PRIM: 5, FIELD_U: 5, FIELD_Q: 5, FIELD_QM: 10, FIELD_DQ: 15,
               FIELD_DELT: 1, FIELD_FLUX_RES: 5, FIELD_DELUP: 5, FIELD_DELUN: 5,
               FIELD_DINV: 1}

# Every symbol include/mfcfd.h declares.
EXPORTS = ("mfcfd_params_init", "mfcfd_create", "mfcfd_set_prim", "mfcfd_fpi_step",
           "mfcfd_run", "mfcfd_get", "mfcfd_get_state", "mfcfd_set_state",
           "mfcfd_get_stencils", "mfcfd_get_alias", "mfcfd_get_levels", "mfcfd_debug_digest", "mfcfd_knn", "mfcfd_get_info",
           "mfcfd_get_stream", "mfcfd_set_profiling", "mfcfd_get_phase_times",
           "mfcfd_residual_noalloc", "mfcfd_set_fault_hook", "mfcfd_set_precision", "mfcfd_count_input_points", "mfcfd_read_input_point_data",
           "mfcfd_read_stored_solution", "mfcfd_print_primal_output", "mfcfd_write_residue",
           "mfcfd_forces", "mfcfd_set_wall_areas", "mfcfd_run_batch", "mfcfd_run_group",
           "mfcfd_prepare", "mfcfd_device_bytes", "mfcfd_attach", "mfcfd_tune_chain",
           "mfcfd_set_chain_warps", "mfcfd_launch", "mfcfd_complete",
           "mfcfd_server_create", "mfcfd_server_submit", "mfcfd_server_wait",
           "mfcfd_server_get_stats", "mfcfd_server_destroy",
           "mfcfd_destroy", "mfcfd_last_error", "mfcfd_strerror")
NOALLOC_MAX_TERMS = 1024 * 4096
GROUP_MAX_CLOUDS = 32
NPHASE = 7
PHASES = ("qderiv", "flux", "dinv", "sweep_fwd", "sweep_bwd", "update", "residual")


class Params(ctypes.Structure):
    """mfcfd_params (include/mfcfd.h)."""
    _fields_ = [("power", ctypes.c_double), ("vl_const", ctypes.c_double),
                ("cfl", ctypes.c_double), ("rho_inf", ctypes.c_double),
                ("u1_inf", ctypes.c_double), ("u2_inf", ctypes.c_double),
                ("u3_inf", ctypes.c_double), ("pr_inf", ctypes.c_double),
                ("inner_iterations", ctypes.c_int32), ("split_capacity", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
                ("sweep_mode", ctypes.c_int32), ("update_variant", ctypes.c_int32),
                ("sweep_variant", ctypes.c_int32), ("chain_warps", ctypes.c_int32),
                ("gpu_setup", ctypes.c_int32), ("graphs", ctypes.c_int32),
                ("chain_spread", ctypes.c_int32), ("storage_order", ctypes.c_int32),
                ("flux_blocks_per_sm", ctypes.c_int32)]


ORDER_INDEX = 0
ORDER_MORTON = 1

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_MIXED_DC = 2
UPDATE_IMPLICIT = 0
UPDATE_EXPLICIT = 1
SWEEPS_ALIAS = 0
SWEEPS_BACKUP = 1
SWEEP_DATAFLOW = 0
SWEEP_LEVELS = 1
SWEEP_CHAINS = 2


class Info(ctypes.Structure):
    """mfcfd_info (include/mfcfd.h)."""
    _fields_ = [("n_points", ctypes.c_int32), ("n_wall", ctypes.c_int32),
                ("n_outer", ctypes.c_int32), ("n_interior", ctypes.c_int32),
                ("n_supersonic", ctypes.c_int32), ("n_levels_forward", ctypes.c_int32),
                ("n_levels_backward", ctypes.c_int32), ("max_level_width", ctypes.c_int32),
                ("split_overflows", ctypes.c_int32), ("shared_frame", ctypes.c_int32),
                ("device_bytes", ctypes.c_int64), ("sweep_mode", ctypes.c_int32),
                ("chain_warps", ctypes.c_int32), ("chain_terms_ring", ctypes.c_int64),
                ("chain_terms_local", ctypes.c_int64), ("chain_terms_cross", ctypes.c_int64),
                ("chain_slots", ctypes.c_int32), ("chain_slot_capacity", ctypes.c_int32),
                ("g0_points", ctypes.c_int32), ("chain_warps_per_block", ctypes.c_int32)]


class ServerConfig(ctypes.Structure):
    """mfcfd_server_config (include/mfcfd.h)."""
    _fields_ = [("device", ctypes.c_int32), ("max_live", ctypes.c_int32),
                ("setup_threads", ctypes.c_int32), ("chunk", ctypes.c_int32),
                ("hbm_budget", ctypes.c_int64), ("chain_percent", ctypes.c_int32),
                ("device_setup", ctypes.c_int32), ("reserved", ctypes.c_int32 * 6)]


class Request(ctypes.Structure):
    """mfcfd_request (include/mfcfd.h)."""
    _fields_ = [("params", Params), ("n", ctypes.c_int32)] + \
        [(f, ctypes.c_void_p) for f in ("status", "x", "y", "z", "tan1", "tan2", "nor", "nbhs",
                                        "conn", "min_dist", "prim")] + \
        [("max_iters", ctypes.c_int32), ("residue_target", ctypes.c_double),
         ("wall_area", ctypes.c_double), ("ref_area", ctypes.c_double),
         ("polish_residue", ctypes.c_double)]


class Result(ctypes.Structure):
    """mfcfd_result (include/mfcfd.h)."""
    _fields_ = [("id", ctypes.c_int64), ("status", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("iters", ctypes.c_int32), ("n", ctypes.c_int32)] + \
        [(f, ctypes.c_double) for f in ("res_new", "residue", "cl", "cd", "t_submit", "t_ready",
                                        "t_admit", "t_done")] + [("device_bytes", ctypes.c_int64),
                                                                 ("run_s", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    """mfcfd_server_stats (include/mfcfd.h)."""
    _fields_ = [(f, ctypes.c_int64) for f in (
        "submitted", "completed", "failed", "preparing", "waiting", "live", "bytes_live",
        "peak_bytes_live", "hbm_budget", "rounds", "iterations", "peak_live", "slot_capacity")] + \
        [("busy_s", ctypes.c_double), ("slot_s", ctypes.c_double)]


class MfcfdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mfcfd error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


_lib = None


def lib():
    """Load libmfcfd.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C 3d-mfcfd_b200` "
                          "or __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double
    L.mfcfd_params_init.argtypes = [ctypes.POINTER(Params), dbl, dbl]
    L.mfcfd_params_init.restype = None
    L.mfcfd_create.argtypes = [ctypes.POINTER(Params), i32] + [vp] * 10 + [ctypes.POINTER(vp)]
    L.mfcfd_set_prim.argtypes = [vp, vp]
    L.mfcfd_fpi_step.argtypes = [vp, i32, vp, vp]
    L.mfcfd_run.argtypes = [vp, i32, i32, vp]
    L.mfcfd_get.argtypes = [vp, i32, vp]
    L.mfcfd_get_state.argtypes = [vp, vp, vp, vp]
    L.mfcfd_set_state.argtypes = [vp, vp, vp, dbl]
    L.mfcfd_get_stencils.argtypes = [vp, vp, vp, i32]
    L.mfcfd_get_alias.argtypes = [vp, vp, vp]
    L.mfcfd_get_levels.argtypes = [vp, i32, vp]
    L.mfcfd_knn.argtypes = [i32, i32, vp, vp, vp, i32, vp, vp, vp]
    L.mfcfd_debug_digest.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_int64)]
    L.mfcfd_get_info.argtypes = [vp, ctypes.POINTER(Info)]
    L.mfcfd_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.mfcfd_set_profiling.argtypes = [vp, i32]
    L.mfcfd_get_phase_times.argtypes = [vp, vp, vp]
    L.mfcfd_residual_noalloc.argtypes = [vp, vp]
    L.mfcfd_set_fault_hook.argtypes = [vp, i32, i32]
    L.mfcfd_set_precision.argtypes = [vp, i32]
    cp = ctypes.c_char_p
    L.mfcfd_count_input_points.argtypes = [cp, vp]
    L.mfcfd_read_input_point_data.argtypes = [cp, i32] + [vp] * 10
    L.mfcfd_read_stored_solution.argtypes = [cp, i32, vp]
    L.mfcfd_print_primal_output.argtypes = [vp, cp]
    L.mfcfd_write_residue.argtypes = [cp, i32, i32, vp, i32]
    L.mfcfd_forces.argtypes = [vp, dbl, dbl, vp, vp, vp]
    L.mfcfd_set_wall_areas.argtypes = [vp, vp]
    L.mfcfd_run_batch.argtypes = [vp, i32, vp, i32, vp, vp]
    L.mfcfd_run_group.argtypes = [vp, i32, vp, i32, vp, vp]
    L.mfcfd_prepare.argtypes = [ctypes.POINTER(Params), i32] + [vp] * 10 + [ctypes.POINTER(vp)]
    L.mfcfd_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.mfcfd_attach.argtypes = [vp]
    L.mfcfd_tune_chain.argtypes = [vp, vp, i32, i32, ctypes.POINTER(i32), vp]
    L.mfcfd_set_chain_warps.argtypes = [vp, i32, ctypes.POINTER(i32)]
    L.mfcfd_launch.argtypes = [vp, i32, i32]
    L.mfcfd_complete.argtypes = [vp, i32, vp, ctypes.POINTER(i32)]
    L.mfcfd_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
    L.mfcfd_server_submit.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_int64)]
    L.mfcfd_server_wait.argtypes = [vp, ctypes.c_int64, dbl, ctypes.POINTER(Result), vp]
    L.mfcfd_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.mfcfd_server_destroy.argtypes = [vp]
    L.mfcfd_destroy.argtypes = [vp]
    L.mfcfd_last_error.argtypes = [vp]
    L.mfcfd_last_error.restype = ctypes.c_char_p
    L.mfcfd_strerror.argtypes = [ctypes.c_int]
    L.mfcfd_strerror.restype = ctypes.c_char_p
    for name in EXPORTS:
        if name not in ("mfcfd_params_init", "mfcfd_last_error", "mfcfd_strerror"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)
