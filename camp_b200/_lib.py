"""ctypes bindings of libcamp_b200.so (the C ABI in include/camp_b200.h).

The library is built in-tree by ``camp_b200.build``.  There is no fallback:
if the shared library is missing or cannot be loaded, importing the solver
raises, so nothing can silently run on the CPU instead of the GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libcamp_b200.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class CellStats(C.Structure):
    _fields_ = [
        ("status", C.c_int),
        ("nst", C.c_int),
        ("nfe", C.c_int),
        ("nsetups", C.c_int),
        ("netf", C.c_int),
        ("nni", C.c_int),
        ("ncfn", C.c_int),
        ("nje", C.c_int),
        ("hu", C.c_double),
        ("hcur", C.c_double),
    ]


# every function include/camp_b200.h declares, for the export check
EXPORTED = [
    "solver_new", "solver_initialize", "solver_run", "solver_get_statistics",
    "solver_reset_timers", "solver_free", "solver_free_update_data",
    "solver_set_debug_out", "solver_set_eval_jac", "rxn_add_condensed_data",
    "rxn_update_data", "rxn_print_data", "rxn_free_update_data",
    "rxn_photolysis_create_rate_update_data", "rxn_photolysis_set_rate_update_data",
    "rxn_emission_create_rate_update_data", "rxn_emission_set_rate_update_data",
    "rxn_first_order_loss_create_rate_update_data", "rxn_first_order_loss_set_rate_update_data",
    "rxn_wet_deposition_create_rate_update_data", "rxn_wet_deposition_set_rate_update_data",
    "aero_rep_modal_binned_mass_create_gmd_update_data",
    "aero_rep_modal_binned_mass_set_gmd_update_data",
    "aero_rep_modal_binned_mass_create_gsd_update_data",
    "aero_rep_modal_binned_mass_set_gsd_update_data",
    "aero_phase_add_condensed_data", "aero_rep_add_condensed_data", "aero_rep_update_data",
    "sub_model_add_condensed_data", "sub_model_update_data", "aero_phase_print_data",
    "aero_rep_print_data", "sub_model_print_data",
    "camp_b200_last_error", "camp_b200_is_ready", "camp_b200_set_precision",
    "camp_b200_set_launch", "camp_b200_set_lu_mode", "camp_b200_set_kernel", "camp_b200_set_layout", "camp_b200_set_graph", "camp_b200_autotune", "camp_b200_get_tuning", "camp_b200_set_cost_ordering", "camp_b200_run_device",
    "camp_b200_launch_device", "camp_b200_sync_status", "camp_b200_run_device_noalloc", "camp_b200_n_photo", "camp_b200_rate_column",
    "camp_b200_set_photo_rates", "camp_b200_set_photo_rates_device", "camp_b200_get_cell_stats", "camp_b200_kernel_launches",
    "camp_b200_last_kernel_ms", "camp_b200_n_dep_var", "camp_b200_n_jac_elem",
    "camp_b200_n_lu_elem", "camp_b200_rxn_int_data_size", "camp_b200_get_solver_jac",
    "camp_b200_get_rxn_int_data", "camp_b200_get_lu_order", "camp_b200_get_block_tables",
    "camp_b200_eval_deriv",
    "camp_b200_n_mapped_values", "camp_b200_get_jac_map", "camp_b200_get_kernel",
    "camp_b200_check_precision",
    "camp_b200_eval_jac", "camp_b200_check_jac", "camp_b200_solver_from_json",
    "camp_b200_n_state_var", "camp_b200_state_name", "camp_b200_json_tolerances",
    "camp_b200_get_var_type", "camp_b200_rxn_float_data_size", "camp_b200_get_rxn_float_data",
    "camp_b200_get_aero_data",
    "camp_b200_server_new", "camp_b200_server_add_solver",
    "camp_b200_server_submit", "camp_b200_server_wait", "camp_b200_server_pending",
    "camp_b200_server_free", "camp_b200_server_open_column", "camp_b200_server_submit_column",
    "camp_b200_server_read_column", "camp_b200_server_close_column",
]

_lib = None


def load(path: str = LIB_PATH):
    """Loads the library (raising if it is absent) and declares signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m camp_b200.build` "
            "(the solver has no CPU fallback)"
        )
    lib = C.CDLL(path)
    vp, ip, dp = C.c_void_p, C.c_int, C.c_double
    lib.solver_new.restype = vp
    lib.solver_new.argtypes = [ip, ip, _i32p] + [ip] * 15
    lib.solver_initialize.argtypes = [vp, _f64p, dp, ip, ip]
    lib.solver_run.restype = ip
    lib.solver_run.argtypes = [vp, _f64p, _f64p, dp, dp]
    lib.solver_get_statistics.argtypes = [vp] + [C.POINTER(C.c_int)] * 9 + [C.POINTER(C.c_double)] * 2 + [C.POINTER(C.c_int)] * 3 + [C.POINTER(C.c_double)] * 3
    lib.solver_free.argtypes = [vp]
    lib.solver_free_update_data.argtypes = [vp]
    lib.rxn_add_condensed_data.argtypes = [ip, ip, ip, ip, _i32p, _f64p, vp]
    lib.rxn_update_data.argtypes = [ip, C.POINTER(C.c_int), ip, vp, vp]
    lib.aero_phase_add_condensed_data.argtypes = [ip, ip, _i32p, _f64p, vp]
    lib.aero_rep_add_condensed_data.argtypes = [ip, ip, ip, ip, _i32p, _f64p, vp]
    lib.sub_model_add_condensed_data.argtypes = [ip, ip, ip, ip, _i32p, _f64p, vp]
    lib.aero_rep_update_data.argtypes = [ip, C.POINTER(C.c_int), ip, vp, vp]
    for kind in ("photolysis", "emission", "first_order_loss", "wet_deposition"):
        getattr(lib, f"rxn_{kind}_create_rate_update_data").restype = vp
        getattr(lib, f"rxn_{kind}_set_rate_update_data").argtypes = [vp, ip, dp]
    for what in ("gmd", "gsd"):
        getattr(lib, f"aero_rep_modal_binned_mass_create_{what}_update_data").restype = vp
        getattr(lib, f"aero_rep_modal_binned_mass_set_{what}_update_data").argtypes = [
            vp, ip, ip, dp]
    lib.camp_b200_last_error.restype = C.c_char_p
    lib.camp_b200_is_ready.restype = ip
    lib.camp_b200_is_ready.argtypes = [vp]
    lib.camp_b200_set_precision.argtypes = [vp, ip]
    lib.camp_b200_set_launch.argtypes = [vp, ip, ip]
    lib.camp_b200_set_cost_ordering.argtypes = [vp, ip]
    lib.camp_b200_set_lu_mode.restype = ip
    lib.camp_b200_set_lu_mode.argtypes = [vp, ip]
    lib.camp_b200_autotune.restype = ip
    lib.camp_b200_autotune.argtypes = [vp, _f64p, _f64p, ip, dp, dp]
    lib.camp_b200_check_precision.restype = ip
    lib.camp_b200_check_precision.argtypes = [vp, _f64p, _f64p, ip, dp, _f64p]
    lib.camp_b200_get_kernel.restype = ip
    lib.camp_b200_get_kernel.argtypes = [vp]
    lib.camp_b200_get_tuning.restype = ip
    lib.camp_b200_get_tuning.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.camp_b200_set_graph.restype = ip
    lib.camp_b200_set_graph.argtypes = [vp, ip]
    lib.camp_b200_set_layout.restype = ip
    lib.camp_b200_set_layout.argtypes = [vp, ip]
    lib.camp_b200_set_kernel.restype = ip
    lib.camp_b200_set_kernel.argtypes = [vp, ip, ip]
    lib.camp_b200_run_device.restype = ip
    lib.camp_b200_run_device.argtypes = [vp, vp, vp, ip, dp, dp, vp]
    lib.camp_b200_launch_device.restype = ip
    lib.camp_b200_launch_device.argtypes = [vp, vp, vp, ip, dp, dp, vp]
    lib.camp_b200_run_device_noalloc.restype = ip
    lib.camp_b200_run_device_noalloc.argtypes = [vp, vp, vp, vp, vp, ip, dp, dp, vp]
    lib.camp_b200_sync_status.restype = ip
    lib.camp_b200_sync_status.argtypes = [vp, vp]
    lib.camp_b200_n_photo.restype = ip
    lib.camp_b200_n_photo.argtypes = [vp]
    lib.camp_b200_rate_column.restype = ip
    lib.camp_b200_rate_column.argtypes = [vp, ip] + [C.POINTER(C.c_int)] * 3
    lib.camp_b200_set_photo_rates.argtypes = [vp, _f64p, ip]
    lib.camp_b200_set_photo_rates_device.restype = ip
    lib.camp_b200_set_photo_rates_device.argtypes = [vp, vp, ip]
    lib.camp_b200_get_cell_stats.restype = ip
    lib.camp_b200_get_cell_stats.argtypes = [vp, C.POINTER(CellStats), ip]
    lib.camp_b200_kernel_launches.restype = C.c_long
    lib.camp_b200_kernel_launches.argtypes = [vp]
    lib.camp_b200_last_kernel_ms.restype = dp
    lib.camp_b200_last_kernel_ms.argtypes = [vp]
    for name in ("camp_b200_n_dep_var", "camp_b200_n_jac_elem", "camp_b200_n_lu_elem",
                 "camp_b200_rxn_int_data_size", "camp_b200_n_mapped_values"):
        getattr(lib, name).restype = ip
        getattr(lib, name).argtypes = [vp]
    lib.camp_b200_get_solver_jac.argtypes = [vp, _i32p, _i32p]
    lib.camp_b200_get_rxn_int_data.argtypes = [vp, _i32p]
    lib.camp_b200_get_lu_order.argtypes = [vp, _i32p]
    lib.camp_b200_get_block_tables.restype = C.c_long
    lib.camp_b200_get_block_tables.argtypes = [vp, vp, C.c_long]
    lib.camp_b200_get_jac_map.restype = ip
    lib.camp_b200_get_jac_map.argtypes = [vp, _i32p]
    lib.camp_b200_eval_deriv.restype = ip
    lib.camp_b200_eval_deriv.argtypes = [vp, _f64p, _f64p, ip, dp, _f64p, _f64p, _f64p]
    lib.camp_b200_eval_jac.restype = ip
    lib.camp_b200_eval_jac.argtypes = [vp, _f64p, _f64p, ip, dp, _f64p, _f64p]
    lib.camp_b200_solver_from_json.restype = vp
    lib.camp_b200_solver_from_json.argtypes = [C.POINTER(C.c_char_p), ip, ip]
    for name in ("camp_b200_n_state_var", "camp_b200_rxn_float_data_size"):
        getattr(lib, name).restype = ip
        getattr(lib, name).argtypes = [vp]
    lib.camp_b200_state_name.restype = ip
    lib.camp_b200_state_name.argtypes = [vp, ip, C.c_char_p, ip]
    lib.camp_b200_json_tolerances.restype = ip
    lib.camp_b200_json_tolerances.argtypes = [vp, _f64p, C.POINTER(C.c_double)]
    lib.camp_b200_get_var_type.restype = ip
    lib.camp_b200_get_var_type.argtypes = [vp, _i32p]
    lib.camp_b200_get_rxn_float_data.restype = ip
    lib.camp_b200_get_rxn_float_data.argtypes = [vp, _f64p]
    lib.camp_b200_get_aero_data.restype = ip
    lib.camp_b200_get_aero_data.argtypes = [vp, ip, ip, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                            vp, vp]
    lib.camp_b200_check_jac.restype = ip
    lib.camp_b200_check_jac.argtypes = [vp, _f64p, _f64p, ip, dp, dp, dp, _f64p, _i32p]
    lib.camp_b200_server_new.restype = vp
    lib.camp_b200_server_new.argtypes = [ip, dp, dp]
    lib.camp_b200_server_add_solver.restype = ip
    lib.camp_b200_server_add_solver.argtypes = [vp, vp]
    lib.camp_b200_server_submit.restype = C.c_long
    lib.camp_b200_server_submit.argtypes = [vp, ip, vp, vp, vp, ip, dp, dp]
    lib.camp_b200_server_wait.restype = ip
    lib.camp_b200_server_wait.argtypes = [vp, C.c_long, C.POINTER(C.c_double), vp, ip]
    lib.camp_b200_server_pending.restype = ip
    lib.camp_b200_server_pending.argtypes = [vp]
    lib.camp_b200_server_free.argtypes = [vp]
    lib.camp_b200_server_open_column.restype = C.c_long
    lib.camp_b200_server_open_column.argtypes = [vp, ip, vp, ip]
    lib.camp_b200_server_submit_column.restype = C.c_long
    lib.camp_b200_server_submit_column.argtypes = [vp, C.c_long, vp, vp, dp, dp]
    lib.camp_b200_server_read_column.restype = ip
    lib.camp_b200_server_read_column.argtypes = [vp, C.c_long, vp]
    lib.camp_b200_server_close_column.restype = ip
    lib.camp_b200_server_close_column.argtypes = [vp, C.c_long]
    _lib = lib
    return lib


def last_error() -> str:
    return load().camp_b200_last_error().decode()
