"""ctypes binding of the C ABI in include/femorax_b200.h (the library built in this folder).

Loading fails loudly when the library is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfemorax_b200.so")

FX_OK = 0
FX_E_INVALID = 1
FX_E_UNSUPPORTED = 2
FX_E_NOMEM = 3
FX_E_NOT_SPD = 4
FX_E_DIVERGED = 5
FX_E_TIMEOUT = 6
FX_E_CUDA = 7
FX_E_UNSTABLE = 8

FX_ELEM_STDBRICK = 0
FX_ELEM_SSPBRICK = 1
FX_MAT_ELASTIC = 0
FX_MAT_J2 = 1
FX_RENUMBER_OFF = 0
FX_RENUMBER_RCM = 1
FX_PATH_AUTO = 0
FX_PATH_GENERAL = 1
FX_PATH_BOX = 2
FX_SOLVER_CG = 0
FX_SOLVER_GMRES = 1
FX_SOLVER_KRYLOV = 2
FX_SOLVER_IR = 3
FX_ENGINE_INNER_FP32 = 0
FX_ENGINE_INNER_FP64 = 1
FX_MATH_EXP, FX_MATH_LOG, FX_MATH_POW, FX_MATH_COS = 0, 1, 2, 3

p_i32 = C.POINTER(C.c_int32)
p_i64 = C.POINTER(C.c_int64)
p_f64 = C.POINTER(C.c_double)
p_i8 = C.POINTER(C.c_int8)
vp = C.c_void_p


class fx_material(C.Structure):
    _fields_ = [("kind", C.c_int32), ("element", C.c_int32), ("E", C.c_double), ("nu", C.c_double),
                ("rho", C.c_double), ("sigma_y", C.c_double), ("H", C.c_double), ("hk", C.c_double)]


class fx_param_set(C.Structure):
    _fields_ = [("kind", C.c_int32), ("mass_type", C.c_int32), ("E", C.c_double), ("nu", C.c_double),
                ("rho", C.c_double), ("b", C.c_double * 3), ("alphaM", C.c_double), ("betaK", C.c_double),
                ("betaKinit", C.c_double), ("betaKcomm", C.c_double), ("sigma_y", C.c_double), ("H", C.c_double),
                ("hk", C.c_double), ("element", C.c_int32), ("pad_", C.c_int32)]


class fx_mesh(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_equations", C.c_int32), ("coords", p_f64), ("count", C.c_int32),
                ("padded", C.c_int32), ("node", p_i32), ("eq", p_i32), ("param", p_i32), ("num_params", C.c_int32),
                ("pad_", C.c_int32), ("params", C.POINTER(fx_param_set)), ("lumped_mass", p_f64),
                ("nodal_mass", p_f64), ("nodal_alpha_mass", p_f64), ("eq_dof", p_i8)]


class fx_coeffs(C.Structure):
    _fields_ = [("stiffness", C.c_double), ("damping", C.c_double), ("mass", C.c_double), ("initial", C.c_int32),
                ("pad_", C.c_int32)]


class fx_solve_opts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("max_iterations", C.c_int32), ("lanes", C.c_int32),
                ("restart", C.c_int32), ("pad_", C.c_int32)]


class fx_solve_result(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32), ("rhs_norm", C.c_double),
                ("initial_residual", C.c_double), ("final_residual", C.c_double), ("indefinite", C.c_int32),
                ("status", C.c_int32), ("refinements", C.c_int32), ("pad_", C.c_int32)]


FX_TEST_NORM_UNBALANCE = 0
FX_TEST_NORM_DISP_INCR = 1

# name: (restype, argtypes)
PROTOTYPES = {
    "fx_last_error": (C.c_char_p, []),
    "fx_version": (C.c_char_p, []),
    "fx_model_create": (C.c_int, [C.c_int32, p_i32, p_f64, C.POINTER(vp)]),
    "fx_model_destroy": (None, [vp]),
    "fx_model_add_group": (C.c_int, [vp, C.POINTER(fx_material), p_f64, C.c_int32, C.c_int32, p_i32, p_i32]),
    "fx_model_add_fix": (C.c_int, [vp, C.c_int32, p_i32, p_i32]),
    "fx_model_add_equal_dof": (C.c_int, [vp, C.c_int32, p_i32, p_i32, p_i32]),
    "fx_model_add_rayleigh": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32, p_i32]),
    "fx_model_add_mass": (C.c_int, [vp, C.c_int32, p_i32, p_i32, p_f64]),
    "fx_compile": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, C.POINTER(vp)]),
    "fx_compiled_destroy": (None, [vp]),
    "fx_compiled_sizes": (C.c_int, [vp, p_i64]),
    "fx_compiled_array_i32": (C.c_int64, [vp, C.c_char_p, p_i32]),
    "fx_compiled_array_f64": (C.c_int64, [vp, C.c_char_p, p_f64]),
    "fx_compiled_mesh": (C.c_int, [vp, C.POINTER(fx_param_set), C.POINTER(fx_mesh)]),
    "fx_force_create": (C.c_int, [C.POINTER(fx_mesh), C.c_int32, C.POINTER(vp)]),
    "fx_force_destroy": (None, [vp]),
    "fx_force_set_path": (C.c_int, [vp, C.c_int32]),
    "fx_force_info": (C.c_int, [vp, p_i64]),
    "fx_force_set_launch": (C.c_int, [vp, C.c_int32, C.c_int32]),
    "fx_force_get_launch": (C.c_int, [vp, p_i32]),
    "fx_force_tune": (C.c_int, [vp, vp]),
    "fx_apply_operator": (C.c_int, [vp, fx_coeffs, vp, vp, vp]),
    "fx_apply_operator_f32": (C.c_int, [vp, fx_coeffs, vp, vp, vp]),
    "fx_device_memory": (C.c_int, [C.c_int32, p_i64, p_i64]),
    "fx_ssp_element_constants": (C.c_int, [p_f64, C.c_double, C.c_double, p_f64, p_f64]),
    "fx_force_set_general_mode": (C.c_int, [vp, C.c_int32]),
    "fx_force_set_soil_corrector": (C.c_int, [vp, C.c_int32]),
    "fx_apply_operator_host": (C.c_int, [vp, fx_coeffs, vp, vp, vp]),
    "fx_operator_diagonal_host": (C.c_int, [vp, fx_coeffs, vp, vp]),
    "fx_operator_diagonal": (C.c_int, [vp, fx_coeffs, vp, vp]),
    "fx_force_compute": (C.c_int, [vp, vp, vp, vp, vp]),
    "fx_force_compute_f32": (C.c_int, [vp, vp, vp, vp, vp]),
    "fx_mass_times_ground": (C.c_int, [vp, C.c_int32, vp, vp]),
    "fx_min_critical_dt": (C.c_int, [vp, C.c_int32, p_f64]),
    "fx_element_critical_dts": (C.c_int, [vp, C.c_int32, vp, vp]),
    "fx_stability_may_change": (C.c_int, [vp, p_i32]),
    "fx_stability_prepare": (C.c_int, [vp, vp]),
    "fx_min_critical_dt_bound": (C.c_int, [vp, C.c_int32, p_f64, vp]),
    "fx_explicit_checks": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32]),
    "fx_force_commit": (C.c_int, [vp, vp]),
    "fx_force_plastic_points": (C.c_int, [vp, p_i64]),
    "fx_vops_create": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, C.POINTER(vp)]),
    "fx_vops_destroy": (None, [vp]),
    "fx_vops_dot": (C.c_int, [vp, vp, vp, C.c_int64, vp, p_f64, vp]),
    "fx_dot_noalloc": (C.c_int, [vp, vp, C.c_int64, C.c_int32, vp, p_f64, vp]),
    "fx_pimy_create": (C.c_int, [p_f64, p_f64, C.POINTER(vp)]),
    "fx_pimy_destroy": (None, [vp]),
    "fx_pimy_info": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "fx_pimy_setup_values": (C.c_int, [vp, p_f64]),
    "fx_pimy_init": (C.c_int, [vp, C.c_int64, vp, vp]),
    "fx_pimy_update": (C.c_int, [vp, C.c_int32, C.c_int64, vp, vp, vp, vp, vp, vp, vp]),
    "fx_pimy_init_host": (C.c_int, [vp, C.c_int64, p_f64]),
    "fx_force_set_pimy": (C.c_int, [vp, C.c_int32, vp]),
    "fx_force_set_pdmy": (C.c_int, [vp, C.c_int32, vp]),
    "fx_pdmy_create": (C.c_int, [p_f64, p_f64, C.POINTER(vp)]),
    "fx_pdmy_destroy": (None, [vp]),
    "fx_pdmy_info": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "fx_pdmy_setup_values": (C.c_int, [vp, p_f64]),
    "fx_pdmy_init": (C.c_int, [vp, C.c_int64, vp, vp]),
    "fx_pdmy_update": (C.c_int, [vp, C.c_int32, C.c_int64, vp, vp, vp, vp, vp, vp, vp]),
    "fx_pdmy_init_host": (C.c_int, [vp, C.c_int64, p_f64]),
    "fx_pdmy_update_host": (C.c_int, [vp, C.c_int32, C.c_int64, p_f64, p_f64, p_f64, p_f64, p_f64,
                                      C.POINTER(C.c_int32)]),
    "fx_force_set_material_stage": (C.c_int, [vp, C.c_int32, C.c_int32]),
    "fx_force_pimy_failed": (C.c_int, [vp, C.POINTER(C.c_int64)]),
    "fx_pimy_update_host": (C.c_int, [vp, C.c_int32, C.c_int64, p_f64, p_f64, p_f64, p_f64, p_f64,
                                      C.POINTER(C.c_int32)]),
    "fx_axpy": (C.c_int, [C.c_double, vp, vp, C.c_int64, vp]),
    "fx_xpay": (C.c_int, [vp, C.c_double, vp, C.c_int64, vp]),
    "fx_multiply": (C.c_int, [vp, vp, vp, C.c_int64, vp]),
    "fx_solver_create": (C.c_int, [vp, C.c_int32, fx_solve_opts, C.POINTER(vp)]),
    "fx_solver_destroy": (None, [vp]),
    "fx_solver_setup": (C.c_int, [vp, fx_coeffs, vp]),
    "fx_solver_set_inner_tolerance": (C.c_int, [vp, C.c_double]),
    "fx_solver_solve": (C.c_int, [vp, vp, vp, C.POINTER(fx_solve_result), vp]),
    "fx_solver_newmark": (C.c_int, [vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_double,
                                    C.c_int32, C.POINTER(C.c_int32), C.POINTER(fx_solve_result), vp]),
    "fx_solver_newmark_recover": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, C.c_int32,
                                            C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_int32, p_i32,
                                            C.POINTER(fx_solve_result), vp]),
    "fx_solver_newton_recover": (C.c_int, [vp, vp, vp, C.c_int32, C.c_double, C.c_int32, C.c_int32, p_i32,
                                           C.POINTER(fx_solve_result), vp]),
    "fx_solver_newton": (C.c_int, [vp, vp, vp, C.c_int32, C.c_double, C.c_int32, C.POINTER(C.c_int32),
                                   C.POINTER(fx_solve_result), vp]),
    "fx_explicit_run": (C.c_int, [vp, vp, C.c_int32, p_f64, C.c_int32, C.c_double, vp, vp, vp, vp, vp]),
    "fx_explicit_run_f32": (C.c_int, [vp, vp, C.c_int32, p_f64, C.c_int32, C.c_double, vp, vp, vp, vp, vp]),
    "fx_explicit_record": (C.c_int, [vp, C.c_int32, vp, C.c_int32]),
    "fx_force_get_launches": (C.c_int, [vp, C.POINTER(C.c_int32)]),
    "fx_nbatch_set_inner": (C.c_int, [vp, C.c_int32, C.c_double]),
    "fx_motions_create": (C.c_int, [C.POINTER(vp)]),
    "fx_motions_destroy": (C.c_int, [vp]),
    "fx_motions_add": (C.c_int, [vp, C.c_int32, C.c_double, p_f64, p_f64, C.c_int32, C.c_double, C.c_double,
                                 C.c_int32, C.c_int32]),
    "fx_motions_evaluate": (C.c_int, [vp, C.c_double, p_f64]),
    "fx_explicit_stage": (C.c_int, [vp, C.c_int32, vp, vp, vp, C.c_int32, C.c_double, p_f64, vp, vp, vp, C.c_int32,
                                    vp]),
    "fx_newmark_predict": (C.c_int, [C.c_int64, vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_double,
                                     C.c_double, vp]),
    "fx_newmark_update": (C.c_int, [C.c_int64, vp, vp, vp, vp, C.c_double, C.c_double, vp]),
    "fx_force_state": (C.c_int, [vp, C.c_int32, p_f64, C.c_int64]),
    "fx_force_set_state": (C.c_int, [vp, C.c_int32, p_f64, C.c_int64]),
    "fx_nbatch_create": (C.c_int, [C.POINTER(fx_mesh), C.c_int32, C.c_int32, fx_solve_opts, C.POINTER(vp)]),
    "fx_nbatch_destroy": (None, [vp]),
    "fx_nbatch_layout": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "fx_nbatch_force": (vp, [vp]),
    "fx_nbatch_step": (C.c_int, [vp, vp, vp, C.c_double, C.c_int32, C.POINTER(C.c_int32), C.POINTER(fx_solve_result),
                                 vp]),
    "fx_engine_create": (C.c_int, [C.c_int32, C.c_int64, C.c_int32, fx_coeffs, fx_solve_opts, C.c_double,
                                   C.POINTER(vp)]),
    "fx_engine_destroy": (None, [vp]),
    "fx_engine_set_precision": (C.c_int, [vp, C.c_int32]),
    "fx_engine_set_persistent": (C.c_int, [vp, C.c_int32]),
    "fx_math_eval": (C.c_int, [C.c_int32, vp, vp, vp, C.c_int64, vp]),
    "fx_server_create": (C.c_int, [vp, C.c_int32, C.c_int64, C.c_int32, C.c_int32, C.POINTER(vp)]),
    "fx_server_destroy": (None, [vp]),
    "fx_server_add_static": (C.c_int, [vp, C.c_int64, vp, p_f64, C.c_double]),
    "fx_server_add_j2": (C.c_int, [vp, C.c_int64, C.POINTER(fx_mesh), p_f64, C.c_int64, C.c_int32, C.c_int32,
                                   C.c_double, C.c_int32, C.c_double, C.c_int32, C.c_double]),
    "fx_server_run": (C.c_int, [vp, C.c_int32, C.POINTER(C.c_double)]),
    "fx_server_result": (C.c_int, [vp, C.c_int64, p_f64, C.POINTER(fx_solve_result), p_f64, p_f64, p_i32]),
    "fx_math_eval_host": (C.c_int, [C.c_int32, p_f64, p_f64, p_f64, C.c_int64]),
    "fx_engine_admit": (C.c_int, [vp, vp, p_f64, C.POINTER(C.c_int32)]),
    "fx_engine_round": (C.c_int, [vp, C.POINTER(C.c_int32)]),
    "fx_engine_finished": (C.c_int, [vp, C.c_int32, C.POINTER(C.c_int32)]),
    "fx_engine_retire": (C.c_int, [vp, C.c_int32, p_f64, C.POINTER(fx_solve_result)]),
    "fx_engine_info": (C.c_int, [vp, C.POINTER(C.c_int64)]),
}

_lib = None


class FxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib() -> C.CDLL:
    """The loaded library (raises if it is not built: there is no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"femorax_b200: {LIB_PATH} is not built (run `python -m femorax_b200.build`); "
                               "there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != FX_OK:
        raise FxError(code, lib().fx_last_error().decode())
