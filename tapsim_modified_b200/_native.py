"""ctypes binding of libtapsim_b200.so (include/tapsim_gpu.h).

The library is built in-tree by tapsim_modified_b200.build.  Loading fails
loudly when it is missing: there is no CPU fallback for the device path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libtapsim_b200.so"

TG_OK = 0
ERRORS = {
    1: "TG_ERR_ARGUMENT", 2: "TG_ERR_CUDA", 3: "TG_ERR_NAN", 4: "TG_ERR_SINGULAR", 5: "TG_ERR_NOT_SURFACE",
    6: "TG_ERR_RELAX_FAULT", 7: "TG_ERR_ITERATION_CAP", 8: "TG_ERR_OUTSIDE", 9: "TG_ERR_WALK_LIMIT",
    10: "TG_ERR_NO_SURFACE", 11: "TG_ERR_HOST", 12: "TG_ERR_UNKNOWN_TYPE",
}
TG_ERR_ARGUMENT = 1
TG_ERR_RELAX_FAULT = 6
TG_ERR_ITERATION_CAP = 7
TG_ERR_NO_SURFACE = 10
TG_ERR_HOST = 11


class tg_type(C.Structure):
    _fields_ = [("id", C.c_int32), ("charge_density", C.c_float), ("epsilon", C.c_float), ("removable", C.c_int32),
                ("neumann", C.c_int32), ("dirichlet", C.c_int32), ("phi", C.c_float), ("mass", C.c_float),
                ("evap_charge", C.c_int32), ("evap_field", C.c_float), ("evap_energy", C.c_float)]


class tg_mesh_desc(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("xyz", C.c_void_p), ("type_id", C.c_void_p), ("hull", C.c_void_p),
                ("phi", C.c_void_p), ("row_ptr", C.c_void_p), ("col", C.c_void_p), ("coupling", C.c_void_p),
                ("geom", C.c_void_p), ("area_pos", C.c_void_p), ("volume", C.c_void_p), ("num_tets", C.c_int32),
                ("tet_v", C.c_void_p), ("tet_n", C.c_void_p), ("node_tet", C.c_void_p), ("num_types", C.c_int32),
                ("types", C.POINTER(tg_type))]


class tg_solve_opts(C.Structure):
    _fields_ = [("rel_tol", C.c_double), ("max_outer", C.c_int32), ("max_inner", C.c_int32),
                ("inner_rtol", C.c_double), ("warm_start", C.c_int32), ("preconditioner", C.c_int32),
                ("inner_precision", C.c_int32)]


class tg_solve_info(C.Structure):
    _fields_ = [("outer", C.c_int32), ("inner", C.c_int32), ("rel_residual", C.c_double),
                ("initial_rel_residual", C.c_double), ("inner_neumann", C.c_int32), ("residual_cells", C.c_int32),
                ("setup_seconds", C.c_double)]


class tg_select_info(C.Structure):
    _fields_ = [("num_surface", C.c_int32), ("candidate", C.c_int32), ("best_ratio", C.c_float),
                ("second_ratio", C.c_float), ("ratio_sum", C.c_double), ("probability", C.c_float),
                ("apex", C.c_int32), ("prob_mode", C.c_int32), ("best_probability", C.c_float),
                ("second_probability", C.c_float), ("score_sum", C.c_double)]


class tg_trace_opts(C.Structure):
    _fields_ = [("time_step", C.c_double), ("min_time_step", C.c_double), ("error_threshold", C.c_double),
                ("max_steps", C.c_int32), ("stepper_limit", C.c_int32), ("walk_limit", C.c_int32), ("integrator", C.c_int32), ("stepper", C.c_int32),
                ("precision", C.c_int32), ("fp64_radius", C.c_double)]


class tg_impact(C.Structure):
    _fields_ = [("stop", C.c_float * 3), ("stop_time", C.c_float), ("last_pos", C.c_float * 3),
                ("last_tet", C.c_int32), ("last_phi", C.c_float), ("steps", C.c_int32), ("status", C.c_int32),
                ("trials", C.c_int32)]


class tg_path_point(C.Structure):
    _fields_ = [("time", C.c_float), ("position", C.c_float * 3), ("velocity", C.c_float * 3), ("tet", C.c_int32)]


class tg_result_row(C.Structure):
    _fields_ = [("index", C.c_uint32), ("id", C.c_int32), ("number", C.c_uint32), ("voltage", C.c_float),
                ("start", C.c_float * 3), ("stop", C.c_float * 3), ("tof", C.c_float), ("probability", C.c_float),
                ("potential_before", C.c_float), ("field_before", C.c_float * 3), ("potential_after", C.c_float),
                ("field_after", C.c_float * 3), ("normal", C.c_float * 3), ("apex", C.c_float * 3)]


class tg_trajectory_item(C.Structure):
    _fields_ = [("index", C.c_uint32), ("number", C.c_uint32), ("time_scale", C.c_float), ("status", C.c_int32),
                ("charge", C.c_float), ("mass", C.c_float), ("num_points", C.c_int32), ("points", C.c_void_p),
                ("error", C.c_float * 6)]


# tg_path_point as a numpy record (the same 32 bytes)
PATH_POINT = np.dtype([("time", "<f4"), ("position", "<f4", 3), ("velocity", "<f4", 3), ("tet", "<i4")])


class tg_event_opts(C.Structure):
    _fields_ = [("vacuum_id", C.c_int32), ("relax_mode", C.c_int32), ("local_threshold", C.c_double),
                ("local_shell", C.c_int32), ("local_cycle", C.c_int32), ("local_queue", C.c_int32),
                ("global_steps", C.c_int32), ("refresh_interval", C.c_int32), ("refresh_threshold", C.c_double),
                ("refresh_cycle", C.c_int32), ("refresh_queue", C.c_int32), ("refresh_max_sweeps", C.c_int64),
                ("solve", tg_solve_opts), ("trace", tg_trace_opts), ("trace_enabled", C.c_int32),
                ("normal_enabled", C.c_int32), ("prob_mode", C.c_int32), ("choice_mode", C.c_int32),
                ("temperature", C.c_float), ("rng_seed", C.c_uint32), ("initial_velocity", C.c_int32),
                ("path_cap", C.c_int32), ("path_points", C.c_void_p), ("path_errors", C.c_void_p),
                ("force_nodes", C.c_void_p), ("force_count", C.c_int32)]


class tg_event_record(C.Structure):
    _fields_ = [("node", C.c_int32), ("type_id", C.c_int32), ("probability", C.c_float), ("best_ratio", C.c_float),
                ("second_ratio", C.c_float), ("scaling_reference", C.c_float), ("phi_before", C.c_float),
                ("field_before", C.c_float * 3), ("phi_after", C.c_float), ("field_after", C.c_float * 3),
                ("apex", C.c_float * 3), ("normal", C.c_float * 3), ("impact", tg_impact), ("detached", C.c_int32),
                ("relax_iterations", C.c_int32), ("rel_residual", C.c_double), ("relax_status", C.c_int32), ("best_probability", C.c_float),
                ("second_probability", C.c_float)]


class tg_tip_params(C.Structure):
    _fields_ = [("lattice_a", C.c_double), ("cap_radius", C.c_double), ("shank_length", C.c_double),
                ("half_angle_deg", C.c_double), ("box_half_width", C.c_double), ("box_height", C.c_double),
                ("fine_shell", C.c_double), ("layers_per_level", C.c_int32), ("coarsen", C.c_double),
                ("max_spacing", C.c_double), ("solute_fraction", C.c_double), ("precip_density", C.c_double),
                ("precip_rmin", C.c_double), ("precip_rmax", C.c_double), ("precip_mu", C.c_double),
                ("precip_sigma", C.c_double), ("seed", C.c_uint64)]


class tg_sample_params(C.Structure):
    _fields_ = [("box_half_width", C.c_double), ("box_height", C.c_double), ("fine_shell", C.c_double),
                ("exclusion", C.c_double), ("layers_per_level", C.c_int32), ("coarsen", C.c_double),
                ("max_spacing", C.c_double), ("vacuum_id", C.c_int32), ("top_id", C.c_int32),
                ("bottom_id", C.c_int32), ("sides_id", C.c_int32), ("seed", C.c_uint64)]


# every symbol include/tapsim_gpu.h declares, with its ctypes signature
_P = C.c_void_p
_I = C.c_int32
SIGNATURES = {
    "tg_create": (C.c_int, [C.POINTER(tg_mesh_desc), C.POINTER(_P)]),
    "tg_destroy": (None, [_P]),
    "tg_last_error": (C.c_char_p, [_P]),
    "tg_num_nodes": (C.c_int, [_P]),
    "tg_relax_cycles": (C.c_int, [_P, _I, C.POINTER(C.c_double)]),
    "tg_relax_threshold": (C.c_int, [_P, C.c_double, _I, _I, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    "tg_local_relax": (C.c_int, [_P, _I, _I, C.c_double, _I, _I, C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    "tg_solve": (C.c_int, [_P, C.POINTER(tg_solve_opts), C.POINTER(tg_solve_info)]),
    "tg_residual": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "tg_get_phi": (C.c_int, [_P, _P]),
    "tg_set_phi": (C.c_int, [_P, _P]),
    "tg_field_o1": (C.c_int, [_P, _I, _P, _P]),
    "tg_field_o1_noalloc": (C.c_int, [_P, _I, _P, _P]),
    "tg_get_couplings": (C.c_int, [_P, _P]),
    "tg_get_types": (C.c_int, [_P, _P]),
    "tg_surface_init": (C.c_int, [_P, _I, C.POINTER(_I)]),
    "tg_surface_select": (C.c_int, [_P, C.POINTER(tg_select_info)]),
    "tg_surface_select_mode": (C.c_int, [_P, _I, C.c_float, C.POINTER(tg_select_info)]),
    "tg_surface_pick": (C.c_int, [_P, C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "tg_get_surface": (C.c_int, [_P, _I, _P, _P, C.POINTER(_I)]),
    "tg_surface_normal": (C.c_int, [_P, _I, _P]),
    "tg_take_away": (C.c_int, [_P, _I, _I, _P, C.POINTER(_I)]),
    "tg_update_coordination": (C.c_int, [_P]),
    "tg_trace": (C.c_int, [_P, _I, _P, _P, _P, _P, C.POINTER(tg_trace_opts), _P]),
    "tg_trace_path": (C.c_int, [_P, _I, _P, _P, _P, _P, C.POINTER(tg_trace_opts), _I, _P, _P, _P]),
    "tg_cell_values": (C.c_int, [_P, _I, _P, _P, _P, _P]),
    "tg_surface_normals": (C.c_int, [_P, _I, _P, _P]),
    "tg_surface_cells": (C.c_int, [_P, _I, C.c_float, _I, C.POINTER(_I), _P, _P]),
    "tg_log_grid": (C.c_int, [_P, C.c_char_p, _I, _I, _P]),
    "tg_log_surface": (C.c_int, [_P, C.c_char_p, _I, _I, _I, _I, C.c_float, _P]),
    "tg_mesh_numbers": (C.c_int, [_P, _P]),
    "tg_grid_log_write": (C.c_int, [C.c_char_p, _I, _I, _P, _P, _P, _P, _P]),
    "tg_results_write": (C.c_int, [C.c_char_p, _I, C.c_char_p, _I, _P, _I]),
    "tg_trajectory_write": (C.c_int, [C.c_char_p, _I, _I, _P, _I]),
    "tg_surface_log_write": (C.c_int, [C.c_char_p, _I, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P]),
    "tg_potential_at": (C.c_int, [_P, _I, _P, _P, _P]),
    "tg_run_event": (C.c_int, [_P, C.POINTER(tg_event_opts), _I, C.POINTER(tg_event_record)]),
    "tg_run_events": (C.c_int, [_P, C.POINTER(tg_event_opts), _I, _I, _P, C.POINTER(C.c_int32)]),
    "tg_run_tips": (C.c_int, [_P, _I, _P, _I, _P, _P, _P, _I]),
    "tg_amg_schedule": (C.c_int, [_P, _I, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "tg_timer_start": (C.c_int, [_P]),
    "tg_timer_stop": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "tg_launch_count": (C.c_int64, [_P]),
    "tg_set_launch_mode": (C.c_int, [_P, _I]),
    "tg_bench_kernel": (C.c_int, [_P, _I, _I, C.POINTER(C.c_float), C.POINTER(C.c_double)]),
    "tg_gemm_bf16": (C.c_int, [_P, _P, _P, _I, _I, _I]),
    "tg_amg_host_build": (C.c_int, [_I, _P, _P, _P, C.POINTER(C.c_void_p)]),
    "tg_amg_host_levels": (C.c_int32, [_P]),
    "tg_amg_host_matrix": (C.c_int, [_P, _I, _I, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                     _P, _P, _P]),
    "tg_amg_host_destroy": (None, [_P]),
    "tg_amg_host_inject_worker_failure": (None, [_I]),
    "tg_learner_create": (C.c_int, [_I, _I, _I, C.c_uint64, C.POINTER(C.c_void_p)]),
    "tg_learner_destroy": (None, [_P]),
    "tg_learner_last_error": (C.c_char_p, [_P]),
    "tg_learner_num_params": (C.c_int32, []),
    "tg_learner_set_gain": (C.c_int, [_P, C.c_float]),
    "tg_learner_set_refine": (C.c_int, [_P, _I]),
    "tg_learner_attach": (C.c_int, [_P, _P, _I]),
    "tg_learner_samples": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "tg_learner_get_params": (C.c_int, [_P, _P]),
    "tg_learner_set_params": (C.c_int, [_P, _P]),
    "tg_learner_get_sample": (C.c_int, [_P, _I, C.POINTER(C.c_int32), _P, _P, _P, _P]),
    "tg_learner_gradients": (C.c_int, [_P, _I, _I, C.POINTER(C.c_float), _P, _P]),
    "tg_learner_train": (C.c_int, [_P, _I, _I, C.c_float, C.c_uint64, _I, _I, C.POINTER(C.c_float)]),
    "tg_tip_params_default": (None, [C.POINTER(tg_tip_params)]),
    "tg_mesh_from_tip": (C.c_int, [C.POINTER(tg_tip_params), _I, C.POINTER(_P)]),
    "tg_mesh_from_files": (C.c_int, [C.c_char_p, C.c_char_p, _I, C.POINTER(_P)]),
    "tg_sample_params_default": (None, [C.POINTER(tg_sample_params)]),
    "tg_mesh_from_sample": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(tg_sample_params), _I, C.POINTER(_P)]),
    "tg_mesh_from_dump": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_P)]),
    "tg_mesh_destroy": (None, [_P]),
    "tg_mesh_temperature": (C.c_float, [_P]),
    "tg_mesh_type_id": (C.c_int32, [_P, C.c_char_p]),
    "tg_mesh_describe": (C.c_int, [_P, C.POINTER(tg_mesh_desc), C.POINTER(_I)]),
    "tg_mesh_write_node_file": (C.c_int, [_P, C.c_char_p, _I]),
    "tg_mesh_write_grid_nodes": (C.c_int, [_P, C.c_char_p, _I, _P]),
    "tg_mesh_dump_index": (C.c_uint32, [_P]),
    "tg_mesh_write_config": (C.c_int, [_P, C.c_char_p]),
    "tg_mesh_write_dump": (C.c_int, [_P, C.c_char_p, _P]),
}

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m tapsim_modified_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class TapsimError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def check(code: int, handle=None) -> int:
    if code != TG_OK:
        msg = lib().tg_last_error(handle)
        raise TapsimError(code, msg.decode() if msg else "")
    return code


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
