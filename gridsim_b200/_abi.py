"""ctypes mirror of ``include/gridsim_b200.h`` and the loader of the in-tree engine library.

The structures below must match the header field for field; ``tests/test_abi.py`` checks the exported
symbol list against the header. Loading fails loudly when the shared library is missing: there is no
fallback path.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgridsim_b200.so")

c_i32, c_f64, c_u8, c_vp = ctypes.c_int32, ctypes.c_double, ctypes.c_uint8, ctypes.c_void_p

GS_OK, GS_ERR_INVALID_ARG, GS_ERR_CUDA, GS_ERR_OOM, GS_ERR_NO_DEVICE = 0, 1, 2, 3, 4
GS_ERR_TIMEOUT, GS_ERR_STATE, GS_ERR_UNSUPPORTED, GS_ERR_INTERNAL, GS_ERR_CAPACITY = 5, 6, 7, 8, 9

(PF_CONVERGED, PF_MAX_ITERATIONS, PF_NON_FINITE, PF_DIVERGED, PF_SINGULAR_PIVOT, PF_TIMEOUT, PF_NOT_RUN,
 PF_UNSOLVABLE_PART) = range(8)
PF_STATUS_NAMES = ["Converged", "MaxIterations", "NonFinite", "Diverged", "SingularPivot", "Timeout", "NotRun",
                   "UnsolvablePart"]
RATE_A, RATE_B, RATE_C = 0, 1, 2
LS_OK, LS_SINGULAR, LS_NON_FINITE_INPUT, LS_MALFORMED = 0, 1, 2, 3
OUTAGE_BRANCH, OUTAGE_GENERATOR, OUTAGE_BUS = 0, 1, 2

PREC_FP64, PREC_MIXED = 0, 1
VIOL_BRANCH_OVERLOAD, VIOL_BOUNDARY_OVERLOAD, VIOL_UNDERVOLTAGE, VIOL_OVERVOLTAGE = 0, 1, 2, 3


class CtxOpts(ctypes.Structure):
    _fields_ = [("probe_timeout_ms", c_i32), ("reserved", c_i32 * 7)]


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("n_bus", c_i32), ("n_gen", c_i32), ("n_branch", c_i32), ("reserved0", c_i32), ("base_mva", c_f64),
        ("bus_id", c_vp), ("bus_type", c_vp), ("pd", c_vp), ("qd", c_vp), ("gs", c_vp), ("bs", c_vp),
        ("vm", c_vp), ("va_deg", c_vp), ("vmin_pu", c_vp), ("vmax_pu", c_vp),
        ("gen_bus", c_vp), ("pg", c_vp), ("qg", c_vp), ("vg", c_vp), ("qmin", c_vp), ("qmax", c_vp),
        ("gen_in_service", c_vp),
        ("br_from", c_vp), ("br_to", c_vp), ("r", c_vp), ("x", c_vp), ("b", c_vp), ("tap", c_vp),
        ("shift_deg", c_vp), ("rate_a", c_vp), ("br_in_service", c_vp), ("rate_b", c_vp), ("rate_c", c_vp),
        ("n_boundary", c_i32), ("reserved1", c_i32), ("bnd_ptr", c_vp), ("bnd_branch", c_vp), ("bnd_dir", c_vp),
        ("bnd_limit_mw", c_vp),
        ("zip", c_vp),
    ]


class PfOpts(ctypes.Structure):
    _fields_ = [
        ("tolerance", c_f64), ("diverge_limit_pu", c_f64), ("max_iterations", c_i32), ("flat_start", c_i32),
        ("enforce_q_limits", c_i32), ("retry_from_dc_start", c_i32), ("per_bus_voltage_limits", c_i32),
        ("precision", c_i32), ("warm_start_from_base", c_i32), ("batch_width", c_i32), ("phase_timing", c_i32),
        ("post_fault_rating", c_i32), ("max_q_limit_passes", c_i32), ("revert_q_limits", c_i32),
        ("partial_pivoting", c_i32), ("reserved", c_i32 * 3),
    ]


class PfResult(ctypes.Structure):
    _fields_ = [
        ("status", c_i32), ("iterations", c_i32), ("max_mismatch", c_f64),
        ("vm", c_vp), ("va_deg", c_vp), ("p_inj_mw", c_vp), ("q_inj_mvar", c_vp), ("loading_pct", c_vp),
        ("sf_mva", c_vp), ("st_mva", c_vp),
    ]


class N1Result(ctypes.Structure):
    _fields_ = [
        ("status", c_vp), ("iterations", c_vp), ("max_mismatch", c_vp), ("min_vm", c_vp), ("max_vm", c_vp),
        ("max_loading_pct", c_vp), ("viol_ptr", c_vp), ("viol_capacity", c_i32), ("viol_count", c_i32),
        ("viol_kind", c_vp), ("viol_element", c_vp), ("viol_value", c_vp), ("vm", c_vp), ("va_deg", c_vp),
        ("base_status", c_i32), ("base_iterations", c_i32), ("device_ms", c_f64), ("n_singular_pivot", c_i32),
        ("n_batches", c_i32), ("kernel_launches", ctypes.c_int64), ("newton_iterations", c_i32), ("n_partial_pivot", c_i32),
        ("factor_ms", c_f64), ("solve_ms", c_f64), ("mismatch_ms", c_f64), ("other_ms", c_f64), ("factor_bytes", c_f64),
        ("level_factor_ms", c_f64), ("level_factor_bytes", c_f64), ("tail_ms", c_f64), ("islanded", c_vp),
        ("worst_boundary_pct", c_vp),
    ]


class GridInfo(ctypes.Structure):
    _fields_ = [
        ("n_bus", c_i32), ("n_branch", c_i32), ("n_pv", c_i32), ("n_pq", c_i32), ("m", c_i32), ("nnz_y", c_i32),
        ("nnz_j", c_i32), ("nnz_lu", ctypes.c_int64), ("lu_flops", ctypes.c_int64), ("n_levels", c_i32),
        ("reserved", c_i32 * 7),
    ]


class Schedule(ctypes.Structure):
    _fields_ = [("factor_cut", c_i32), ("solve_cut", c_i32), ("tail_max", c_i32), ("candidates", c_i32),
                ("default_ms", c_f64), ("tuned_ms", c_f64), ("subtree_cut", c_i32), ("reserved", c_i32 * 3)]


class MultiStats(ctypes.Structure):
    _fields_ = [("device_ms", c_f64), ("tune_ms", c_f64), ("threads_per_cta", c_i32), ("ctas", c_i32),
                ("items", c_i32), ("tuned_now", c_i32), ("system_steps", ctypes.c_int64), ("shared_top", c_i32),
                ("reserved", c_i32 * 7)]


class ServeOpts(ctypes.Structure):
    _fields_ = [("pf", PfOpts), ("slots_per_grid", c_i32), ("state_slots", c_i32), ("hbm_fraction", c_f64),
                ("scheduler_threads", c_i32), ("reserved", c_i32 * 7)]


class Request(ctypes.Structure):
    _fields_ = [("grid", c_i32), ("outage", c_i32), ("want_state", c_i32), ("reserved", c_i32), ("tag", ctypes.c_uint64)]


class Response(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("tag", ctypes.c_uint64), ("grid", c_i32), ("outage", c_i32),
                ("status", c_i32), ("iterations", c_i32), ("max_mismatch", c_f64), ("queue_ms", c_f64),
                ("latency_ms", c_f64), ("state_offset", ctypes.c_int64)]


class ServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("ticks", ctypes.c_int64),
                ("system_steps", ctypes.c_int64), ("grids", c_i32), ("slots_total", c_i32), ("in_flight", c_i32),
                ("queued", c_i32), ("slot_bytes", c_f64), ("failed", c_i32), ("reserved", c_i32 * 7)]


GS_SERVE_MAX_SLOTS = 128

# Every entry point the header declares, with its ctypes signature.
EXPORTS = {
    "gs_abi_version": (c_i32, []),
    "gs_status_str": (ctypes.c_char_p, [c_i32]),
    "gs_pf_opts_default": (None, [ctypes.POINTER(PfOpts)]),
    "gs_ctx_create": (c_i32, [c_i32, ctypes.POINTER(CtxOpts), ctypes.POINTER(c_vp)]),
    "gs_ctx_destroy": (c_i32, [c_vp]),
    "gs_last_error": (c_i32, [c_vp, ctypes.c_char_p, ctypes.c_size_t]),
    "gs_grid_create": (c_i32, [c_vp, ctypes.POINTER(GridDesc), ctypes.POINTER(c_vp)]),
    "gs_grid_destroy": (c_i32, [c_vp]),
    "gs_grid_info_get": (c_i32, [c_vp, ctypes.POINTER(GridInfo)]),
    "gs_pf_solve": (c_i32, [c_vp, ctypes.POINTER(PfOpts), ctypes.POINTER(PfResult)]),
    "gs_pf_solve_batch": (c_i32, [c_vp, c_i32, c_vp, c_vp, ctypes.POINTER(PfOpts), c_vp, c_vp, c_vp, c_vp, c_vp]),
    "gs_n1_screen": (c_i32, [c_vp, c_i32, c_vp, ctypes.POINTER(PfOpts), ctypes.POINTER(N1Result)]),
    "gs_nk_screen": (c_i32, [c_vp, c_i32, c_i32, c_vp, ctypes.POINTER(PfOpts), ctypes.POINTER(N1Result)]),
    "gs_element_screen": (c_i32, [c_vp, c_i32, c_vp, c_vp, ctypes.POINTER(PfOpts), ctypes.POINTER(N1Result)]),
    "gs_analyze_host": (c_i32, [ctypes.POINTER(GridDesc), ctypes.POINTER(GridInfo)]),
    "gs_grid_schedule_get": (c_i32, [c_vp, ctypes.POINTER(Schedule)]),
    "gs_grid_schedule_set": (c_i32, [c_vp, ctypes.POINTER(Schedule)]),
    "gs_screen_tune": (c_i32, [c_vp, c_i32, c_vp, ctypes.POINTER(PfOpts), ctypes.POINTER(Schedule)]),
    "gs_outage_topology": (c_i32, [ctypes.POINTER(GridDesc), c_f64, c_i32, c_vp, c_vp, c_vp]),
    "gs_sparse_solve_batch": (c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "gs_pf_mismatch_noalloc": (c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp]),
    "gs_pf_solve_multi": (c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(PfOpts), c_vp, c_vp, c_vp, c_vp,
                                  c_vp, ctypes.POINTER(MultiStats)]),
    "gs_serve_create": (c_i32, [c_vp, ctypes.POINTER(ServeOpts), ctypes.POINTER(c_vp)]),
    "gs_serve_add_grid": (c_i32, [c_vp, c_vp, ctypes.POINTER(c_i32)]),
    "gs_serve_start": (c_i32, [c_vp]),
    "gs_serve_submit": (c_i32, [c_vp, c_i32, c_vp, c_vp]),
    "gs_serve_poll": (c_i32, [c_vp, c_i32, c_i32, c_vp, c_vp, ctypes.c_int64, ctypes.POINTER(c_i32)]),
    "gs_serve_stats_get": (c_i32, [c_vp, ctypes.POINTER(ServeStats)]),
    "gs_serve_stop": (c_i32, [c_vp, c_i32]),
    "gs_serve_destroy": (c_i32, [c_vp]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load the engine library (once). Raises if it has not been built: there is no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"gridsim_b200 engine library not built: {path} is missing "
                           "(run __graft_entry__.build() or python -m gridsim_b200.build)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def default_opts() -> PfOpts:
    """PowerFlowOptions() defaults (``PowerFlow/PowerFlowOptions.cs``), written here so that option
    handling works without loading the engine."""
    o = PfOpts()
    o.tolerance = 1e-8
    o.diverge_limit_pu = 10.0
    o.max_iterations = 30
    o.flat_start = 0
    o.enforce_q_limits = 0
    o.retry_from_dc_start = 0
    o.per_bus_voltage_limits = 0
    o.precision = PREC_FP64
    o.warm_start_from_base = 0
    o.batch_width = 0
    return o
