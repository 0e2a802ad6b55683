"""ctypes bindings of libcufil.so (declarations in include/cufil.h).

The library is loaded from this package directory.  There is no fallback: if
the CUDA library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libcufil.so"

CF_OK = 0
CF_EINVAL = 1
CF_ENOMEM = 2
CF_ECUDA = 3
CF_NOT_CONVERGED = 4
CF_NONFINITE = 5
CF_TIMEOUT = 6
CF_ENOTSUP = 7

CF_BEAT_FULFORD_BLAKE = 1
CF_BEAT_FULFORD_BLAKE_ORIGINAL = 4

CF_PRECOND_NONE = 0
CF_PRECOND_BLOCK_DIAG = 1
CF_PRECOND_LEARNED = 2
CF_PRECOND_LINE = 3
CF_PRECOND_LEARNED_LINE = 4

_STATUS_NAMES = {0: "CF_OK", 1: "CF_EINVAL", 2: "CF_ENOMEM", 3: "CF_ECUDA", 4: "CF_NOT_CONVERGED",
                 5: "CF_NONFINITE", 6: "CF_TIMEOUT", 7: "CF_ENOTSUP"}


class CufilError(RuntimeError):
    def __init__(self, code: int, fn: str, msg: str):
        super().__init__(f"{fn} -> {_STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class MobilityConfig(ctypes.Structure):
    _fields_ = [("n_seg", ctypes.c_int), ("n_blob", ctypes.c_int), ("wall", ctypes.c_int),
                ("seg_dof", ctypes.c_int), ("seg_radius", ctypes.c_double), ("blob_radius", ctypes.c_double),
                ("mu", ctypes.c_double), ("device", ctypes.c_int)]


_dp = ctypes.POINTER(ctypes.c_double)


class SimConfig(ctypes.Structure):
    _fields_ = [("n_fil", ctypes.c_int), ("n_seg", ctypes.c_int), ("seg_sep", ctypes.c_double),
                ("beat", ctypes.c_int), ("dynamic_phase", ctypes.c_int), ("dynamic_angle", ctypes.c_int),
                ("dt", ctypes.c_double), ("spring_factor", ctypes.c_double), ("gmres_tol", ctypes.c_double),
                ("gmres_max_iter", ctypes.c_int), ("precond", ctypes.c_int),
                ("base_pos", ctypes.c_void_p), ("omega0", ctypes.c_void_p),
                ("phase0", ctypes.c_void_p), ("angle0", ctypes.c_void_p),
                ("gen_phase_force_refs", ctypes.c_void_p), ("n_gen_phase_refs", ctypes.c_int),
                ("gen_angle_force_refs", ctypes.c_void_p), ("n_gen_angle_refs", ctypes.c_int),
                ("s_values_ref", ctypes.c_void_p), ("s_ref_rows", ctypes.c_int), ("s_ref_cols", ctypes.c_int),
                ("s_tol_factor", ctypes.c_double), ("device", ctypes.c_int),
                ("line_patch", ctypes.c_int), ("precond_refresh", ctypes.c_int)]


class SwimConfig(ctypes.Structure):
    _fields_ = [("n_fil", ctypes.c_int), ("n_seg", ctypes.c_int), ("n_blob", ctypes.c_int),
                ("seg_sep", ctypes.c_double), ("beat", ctypes.c_int), ("dt", ctypes.c_double),
                ("spring_factor", ctypes.c_double), ("gmres_tol", ctypes.c_double), ("gmres_max_iter", ctypes.c_int),
                ("fil_refs", ctypes.c_void_p), ("fil_dirs", ctypes.c_void_p), ("blob_refs", ctypes.c_void_p),
                ("body_x0", ctypes.c_void_p), ("body_q0", ctypes.c_void_p), ("omega0", ctypes.c_void_p),
                ("phase0", ctypes.c_void_p), ("angle0", ctypes.c_void_p),
                ("gen_phase_force_refs", ctypes.c_void_p), ("n_gen_phase_refs", ctypes.c_int),
                ("gen_angle_force_refs", ctypes.c_void_p), ("n_gen_angle_refs", ctypes.c_int),
                ("s_values_ref", ctypes.c_void_p), ("s_ref_rows", ctypes.c_int), ("s_ref_cols", ctypes.c_int),
                ("s_tol_factor", ctypes.c_double), ("device", ctypes.c_int)]


class ElasticConfig(ctypes.Structure):
    _fields_ = [("n_fil", ctypes.c_int), ("n_seg", ctypes.c_int), ("seg_sep", ctypes.c_double),
                ("base_pos", ctypes.c_void_p), ("dt", ctypes.c_double), ("dimensionless_force", ctypes.c_double),
                ("kb", ctypes.c_double), ("kt", ctypes.c_double), ("repulsion_factor", ctypes.c_double),
                ("broyden_tol", ctypes.c_double), ("max_broyden_iter", ctypes.c_int),
                ("jacobian_confidence", ctypes.c_double), ("ic_type", ctypes.c_int), ("perturbations", ctypes.c_void_p),
                ("device", ctypes.c_int)]


class FcmConfig(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("rh", ctypes.c_double), ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
                ("eta", ctypes.c_double), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("boxsize", ctypes.c_double), ("device", ctypes.c_int)]


class FlowConfig(ctypes.Structure):
    _fields_ = [("max_flow", ctypes.c_int), ("max_seg", ctypes.c_int), ("max_blob", ctypes.c_int),
                ("max_bodies", ctypes.c_int), ("mu", ctypes.c_double), ("remove_net_force", ctypes.c_int),
                ("device", ctypes.c_int)]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "cf_last_error": [],
    "cf_version": [],
    "cf_mobility_create": [ctypes.POINTER(MobilityConfig), ctypes.POINTER(_vp)],
    "cf_mobility_destroy": [_vp],
    "cf_copy_segment_positions_to_device": [_vp, _vp],
    "cf_copy_segment_forces_to_device": [_vp, _vp],
    "cf_copy_blob_positions_to_device": [_vp, _vp],
    "cf_copy_blob_forces_to_device": [_vp, _vp],
    "cf_copy_segment_velocities_to_host": [_vp, _vp],
    "cf_copy_blob_velocities_to_host": [_vp, _vp],
    "cf_wait_for_device": [_vp],
    "cf_evaluate_segment_segment_mobility": [_vp],
    "cf_evaluate_segment_blob_mobility": [_vp],
    "cf_evaluate_blob_blob_mobility": [_vp],
    "cf_evaluate_blob_segment_mobility": [_vp],
    "cf_evaluate_full_mobility": [_vp],
    "cf_apply_mobility": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "cf_apply_mobility_device": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "cf_rpy_wall_segments_noalloc": [_vp, _vp, _vp, _i, _vp],
    "cf_set_wait_limit": [ctypes.c_uint],
    "cf_fcm_create": [ctypes.POINTER(FcmConfig), ctypes.POINTER(_vp)],
    "cf_fcm_destroy": [_vp],
    "cf_fcm_apply": [_vp, _vp, _vp, _vp],
    "cf_fcm_apply_device": [_vp, _vp, _vp, _vp, _vp],
    "cf_fcm_apply_segments_blobs": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp],
    "cf_fcm_info": [_vp, _vp],
    "cf_fcm_set_timing": [_vp, _i],
    "cf_fcm_stage_times": [_vp, _vp],
    "cf_flow_create": [ctypes.POINTER(FlowConfig), ctypes.POINTER(_vp)],
    "cf_flow_destroy": [_vp],
    "cf_flow_velocities": [_vp, _vp, _i, _vp, _vp, _i, _i, _vp, _vp, _i, _i, _vp, _vp],
    "cf_flow_velocities_device": [_vp, _vp, _i, _vp, _vp, _i, _i, _vp, _vp, _i, _i, _vp, _vp, _vp],
    "cf_sim_create": [ctypes.POINTER(SimConfig), ctypes.POINTER(_vp)],
    "cf_sim_destroy": [_vp],
    "cf_sim_step": [_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(_d)],
    "cf_sim_step_async": [_vp, _i],
    "cf_sim_last_solve": [_vp, ctypes.POINTER(_i), ctypes.POINTER(_d)],
    "cf_sim_get_state": [_vp, _vp, _vp, _vp, _vp],
    "cf_sim_get_segments": [_vp, _vp, _vp],
    "cf_sim_get_directions": [_vp, _vp, _vp],
    "cf_sim_step_io": [_vp, _i] + [_vp] * 12,
    "cf_sim_get_arclengths": [_vp, _vp],
    "cf_sim_system_size": [_vp],
    "cf_sim_stream": [_vp, ctypes.POINTER(_vp)],
    "cf_sim_set_state": [_vp, _vp, _vp, _vp, _vp],
    "cf_sim_get_solution": [_vp, _vp],
    "cf_sim_set_solution": [_vp, _vp],
    "cf_sim_iteration_log": [_vp, _vp, _i],
    "cf_sim_launches_per_step": [_vp, _i],
    "cf_sim_initial_guess": [_vp, _i],
    "cf_sim_assemble_rhs": [_vp, _i, _vp],
    "cf_sim_apply_preconditioner": [_vp, _vp, _vp],
    "cf_sim_system_matvec": [_vp, _vp, _vp],
    "cf_sim_write_data": [_vp, _i, _d, ctypes.c_char_p],
    "cf_sim_write_config": [_vp, ctypes.c_char_p, _i],
    "cf_read_ic": [ctypes.c_char_p, _i, _vp, _vp, _vp],
    "cf_sim_solve": [_vp, _vp, _vp, _d, _i, ctypes.POINTER(_i), ctypes.POINTER(_d)],
    "cf_sim_autotune": [_vp, _i, _vp],
    "cf_sim_refresh_preconditioner": [_vp],
    "cf_sim_learned_dims": [_vp, _vp, _vp],
    "cf_sim_set_network": [_vp, _vp],
    "cf_sim_set_network_weight": [_vp, ctypes.c_double],
    "cf_sim_collect_pairs": [_vp, _i, _i, _vp, _vp, _vp],
    "cf_sim_features": [_vp, _vp, _vp],
    "cf_sim_precond_info": [_vp, _vp, _vp, _vp, _vp],
    "cf_sim_set_tuning": [_vp, _vp],
    "cf_sim_get_tuning": [_vp, _vp],
    "cf_mlp_create": [_i, _i, _i, _i, ctypes.c_ulonglong, _i, ctypes.POINTER(_vp)],
    "cf_mlp_destroy": [_vp],
    "cf_mlp_num_params": [_vp],
    "cf_mlp_forward": [_vp, _vp, _i, _vp, _vp],
    "cf_mlp_gradients": [_vp, _vp, _vp, _i, _vp, _vp],
    "cf_mlp_train_step": [_vp, _vp, _vp, _i, ctypes.c_float, _vp],
    "cf_mlp_get_params": [_vp, _vp],
    "cf_mlp_set_params": [_vp, _vp],
    "cf_mlp_stream": [_vp, ctypes.POINTER(_vp)],
    "cf_precond_save": [_vp, _d, ctypes.c_char_p],
    "cf_precond_load": [ctypes.c_char_p, _i, _i, ctypes.POINTER(_vp), ctypes.POINTER(_d)],
    "cf_batch_create": [_vp, _i, ctypes.POINTER(_vp)],
    "cf_batch_destroy": [_vp],
    "cf_batch_shape": [_vp, _vp, _vp, _vp, _vp],
    "cf_batch_step": [_vp, _i, _vp, _vp],
    "cf_batch_step_async": [_vp, _i],
    "cf_batch_last_solve": [_vp, _vp, _vp, _vp],
    "cf_batch_get_state": [_vp, _vp, _vp, _vp, _vp],
    "cf_batch_set_state": [_vp, _vp, _vp, _vp, _vp],
    "cf_batch_get_segments": [_vp, _vp],
    "cf_batch_get_solution": [_vp, _i, _vp],
    "cf_batch_iteration_log": [_vp, _i, _vp, _i],
    "cf_batch_stream": [_vp, ctypes.POINTER(_vp)],
    "cf_batch_launches_per_step": [_vp, _i],
    "cf_batch_autotune": [_vp, _i, _vp],
    "cf_batch_set_tuning": [_vp, _vp],
    "cf_batch_get_tuning": [_vp, _vp],
    "cf_swim_create": [ctypes.POINTER(SwimConfig), ctypes.POINTER(_vp)],
    "cf_swim_destroy": [_vp],
    "cf_swim_step": [_vp, _i, _vp, _vp],
    "cf_swim_get_state": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "cf_swim_get_particles": [_vp, _vp, _vp, _vp, _vp],
    "cf_swim_get_directions": [_vp, _vp, _vp],
    "cf_swim_system_matvec": [_vp, _vp, _vp],
    "cf_swim_apply_preconditioner": [_vp, _vp, _vp],
    "cf_swim_system_size": [_vp],
    "cf_elastic_create": [ctypes.POINTER(ElasticConfig), ctypes.POINTER(_vp)],
    "cf_elastic_destroy": [_vp],
    "cf_elastic_step": [_vp, _i, _vp],
    "cf_elastic_get_segments": [_vp, _vp, _vp, _vp],
    "cf_elastic_get_jacobian_inverse": [_vp, _i, _vp],
    "cf_elastic_first_evaluation": [_vp, _i, _vp],
    "cf_elastic_stats": [_vp, _vp, _vp, _vp, _vp],
    "cf_elastic_system_size": [_vp],
    "cf_tc_tile_product": [_vp, _vp, _vp, ctypes.c_uint],
}
_RESTYPES = {"cf_last_error": ctypes.c_char_p, "cf_mlp_num_params": ctypes.c_longlong}

_lib = None


def load():
    """Loads libcufil.so once; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m cufcm_fil_b200.build` "
                               "(the engine has no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, argtypes in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = L
    return _lib


def last_error() -> str:
    msg = load().cf_last_error()
    return msg.decode() if msg else ""


def call(name: str, *args, ok=(CF_OK,)) -> int:
    rc = getattr(load(), name)(*args)
    if rc not in ok:
        raise CufilError(rc, name, last_error())
    return rc
