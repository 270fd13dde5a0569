"""ctypes binding of the in-tree CUDA library (include/quasar_mhd.h).

The library is required: there is no CPU fallback.  If it is missing, build
it with `python -m quasar_b200.build`; if no CUDA device is present, solver
construction fails with the CUDA error.
"""
from __future__ import annotations

import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libquasar_mhd_b200.so")

QMHD_OK = 0
QMHD_INVALID_ARGUMENT = -1
QMHD_RUNTIME_ERROR = -2
QMHD_DEVICE_ERROR = -3

EXPORTS = (
    "qmhd_last_error", "qmhd_solver_create", "qmhd_solver_destroy", "qmhd_solver_grid",
    "qmhd_solver_storage_size", "qmhd_solver_seed_state", "qmhd_solver_state_component_to_host",
    "qmhd_solver_cfl_limit", "qmhd_solver_step", "qmhd_solver_step_unchecked",
    "qmhd_solver_advance", "qmhd_solver_divergence_b_max", "qmhd_solver_conserved_cell_totals",
    "qmhd_solver_last_positivity_substeps", "qmhd_solver_advance_auto",
)
EXT_EXPORTS = ("qmhd_solver_time_auto_steps", "qmhd_solver_profile_step", "qmhd_fp64_fma_peak",
               "qmhd_conserved_cell_totals_device", "qmhd_solver_set_owned_window",
               "qmhd_solver_write_halo", "qmhd_solver_gather_live", "qmhd_solver_scatter_halo")
TOTALS_DEVICE_MAX_CELLS = 67108864
BATCH_EXPORTS = ("qmhd_batch_create", "qmhd_batch_destroy", "qmhd_batch_size", "qmhd_batch_zones",
                 "qmhd_batch_instance", "qmhd_batch_advance", "qmhd_batch_time_steps",
                 "qmhd_batch_autotune", "qmhd_batch_set_tuning", "qmhd_batch_profile_step")
INDICATOR_EXPORTS = ("qmhd_indicator_create", "qmhd_indicator_destroy", "qmhd_indicator_get_params",
                     "qmhd_indicator_set_params", "qmhd_indicator_forward",
                     "qmhd_indicator_gradient", "qmhd_indicator_collect", "qmhd_indicator_rows",
                     "qmhd_indicator_labels",
                     "qmhd_indicator_clear", "qmhd_indicator_train", "qmhd_indicator_evaluate",
                     "qmhd_indicator_threshold_for_recall", "qmhd_solver_set_indicator",
                     "qmhd_solver_learned_face_counts", "qmhd_batch_set_indicator")

LAUNCH_EXPORTS = ("qmhd_launch_reconstruct", "qmhd_launch_hlld_flux", "qmhd_launch_flux_difference",
                  "qmhd_launch_ct_emf_prepare", "qmhd_launch_ct_emf_finish",
                  "qmhd_launch_emf_curl_rate", "qmhd_launch_rk_stage",
                  "qmhd_launch_admissible_fraction", "qmhd_launch_cfl_max_rate",
                  "qmhd_launch_ct_divb_linf", "qmhd_launch_ct_divb_relative_linf",
                  "qmhd_launch_fill_ghosts_fluid", "qmhd_launch_fill_ghosts_field",
                  "qmhd_launch_collocate_face_to_cell", "qmhd_launch_conserved_cell_sums",
                  "qmhd_launch_seed_initial_state")
LAUNCH_SCRATCH_BYTES = 64


class QmhdConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double),
        ("origin_x", ctypes.c_double), ("origin_y", ctypes.c_double),
        ("reconstruction_order", ctypes.c_int),
        ("gamma", ctypes.c_double), ("cfl", ctypes.c_double),
        ("boundary", ctypes.c_int * 4),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"quasar_b200 CUDA library not found at {LIB_PATH}; build it with "
            "`python -m quasar_b200.build` (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.qmhd_last_error.restype = ctypes.c_char_p
    L.qmhd_solver_create.argtypes = [ctypes.POINTER(QmhdConfig), ctypes.POINTER(vp)]
    L.qmhd_solver_destroy.argtypes = [vp]
    L.qmhd_solver_destroy.restype = None
    L.qmhd_solver_grid.argtypes = [vp, ip, ip, ip]
    L.qmhd_solver_storage_size.argtypes = [vp]
    L.qmhd_solver_storage_size.restype = ctypes.c_longlong
    L.qmhd_solver_seed_state.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_size_t]
    L.qmhd_solver_state_component_to_host.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_size_t]
    L.qmhd_solver_cfl_limit.argtypes = [vp, dp]
    L.qmhd_solver_step.argtypes = [vp, ctypes.c_double]
    L.qmhd_solver_step_unchecked.argtypes = [vp, ctypes.c_double]
    L.qmhd_solver_advance.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    L.qmhd_solver_divergence_b_max.argtypes = [vp, dp]
    L.qmhd_solver_conserved_cell_totals.argtypes = [vp, dp, dp]
    L.qmhd_solver_last_positivity_substeps.argtypes = [vp]
    L.qmhd_solver_advance_auto.argtypes = [vp, dp, ctypes.c_double, ctypes.c_int, ip]
    L.qmhd_solver_set_owned_window.argtypes = [vp] + [ctypes.c_int] * 4
    L.qmhd_solver_write_halo.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_size_t]
    L.qmhd_solver_gather_live.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_size_t, vp]
    L.qmhd_solver_scatter_halo.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_size_t, vp]
    L.qmhd_solver_time_auto_steps.argtypes = [vp, ctypes.c_int, dp, ip]
    L.qmhd_solver_profile_step.argtypes = [vp, dp, ctypes.c_int]
    L.qmhd_fp64_fma_peak.argtypes = [dp]
    L.qmhd_conserved_cell_totals_device.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int, vp, dp, dp]
    L.qmhd_batch_create.argtypes = [ctypes.POINTER(QmhdConfig), ctypes.c_int, ctypes.POINTER(vp)]
    L.qmhd_batch_destroy.argtypes = [vp]
    L.qmhd_batch_destroy.restype = None
    L.qmhd_batch_size.argtypes = [vp]
    L.qmhd_batch_zones.argtypes = [vp]
    L.qmhd_batch_zones.restype = ctypes.c_longlong
    L.qmhd_batch_instance.argtypes = [vp, ctypes.c_int]
    L.qmhd_batch_instance.restype = vp
    L.qmhd_batch_advance.argtypes = [vp, ctypes.c_int, ip]
    L.qmhd_batch_time_steps.argtypes = [vp, ctypes.c_int, dp, ctypes.POINTER(ctypes.c_longlong)]
    L.qmhd_batch_autotune.argtypes = [vp, ip, ip]
    L.qmhd_batch_set_tuning.argtypes = [vp, ip]
    L.qmhd_batch_profile_step.argtypes = [vp, dp, ctypes.c_int]
    L.qmhd_indicator_create.argtypes = [ctypes.c_ulonglong, ctypes.POINTER(vp)]
    L.qmhd_indicator_destroy.argtypes = [vp]
    L.qmhd_indicator_destroy.restype = None
    L.qmhd_indicator_get_params.argtypes = [vp, vp, ctypes.c_size_t]
    L.qmhd_indicator_set_params.argtypes = [vp, vp, ctypes.c_size_t]
    L.qmhd_indicator_forward.argtypes = [vp, vp, ctypes.c_longlong, vp]
    lp = ctypes.POINTER(ctypes.c_longlong)
    L.qmhd_indicator_gradient.argtypes = [vp, vp, vp, ctypes.c_longlong, ctypes.c_float, vp,
                                          ctypes.c_size_t, dp]
    L.qmhd_indicator_collect.argtypes = [vp, vp, ctypes.c_float]
    L.qmhd_indicator_rows.argtypes = [vp]
    L.qmhd_indicator_rows.restype = ctypes.c_longlong
    L.qmhd_indicator_labels.argtypes = [vp, vp, ctypes.c_longlong]
    L.qmhd_indicator_clear.argtypes = [vp]
    L.qmhd_indicator_train.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_int, ctypes.c_ulonglong, dp]
    L.qmhd_indicator_evaluate.argtypes = [vp, ctypes.c_float, ctypes.c_int, dp, dp, lp, lp]
    L.qmhd_indicator_threshold_for_recall.argtypes = [vp, ctypes.c_double, ctypes.c_int,
                                                      ctypes.POINTER(ctypes.c_float)]
    L.qmhd_solver_set_indicator.argtypes = [vp, vp, ctypes.c_float]
    L.qmhd_batch_set_indicator.argtypes = [vp, vp, ctypes.c_float]
    L.qmhd_solver_learned_face_counts.argtypes = [vp, lp, lp]
    from . import launch as _launch
    _launch.declare(L)
    _lib = L
    return L


def check(rc: int) -> None:
    """Map a C status to the exception the reference's binding raises."""
    if rc == QMHD_OK:
        return
    msg = lib().qmhd_last_error().decode()
    if rc == QMHD_INVALID_ARGUMENT:
        raise ValueError(msg)
    raise RuntimeError(msg)
