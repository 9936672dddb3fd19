"""ctypes binding of ``libfhs_b200.so`` (the C ABI declared in include/fhs_b200.h).

The library is loaded from this package directory only; if it is missing the
import fails loudly (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfhs_b200.so")

FHS_OK = 0
STATUS_NAMES = {
    0: "FHS_OK", 1: "FHS_ERR_INVALID_ARG", 2: "FHS_ERR_CUDA", 3: "FHS_ERR_OUT_OF_MEMORY",
    4: "FHS_ERR_STATE", 5: "FHS_ERR_NUMERIC", 6: "FHS_ERR_UNSUPPORTED", 7: "FHS_ERR_NO_DEVICE",
}

ALGO_SARA, ALGO_HS, ALGO_FHS = 0, 1, 2
WINDOW_NONE, WINDOW_TRIANGULAR = 0, 1


class FhsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class SolverConfig(C.Structure):
    _fields_ = [("algo", C.c_int), ("nlevel", C.c_int), ("n_groups", C.c_int), ("Qy", C.c_int),
                ("Qx", C.c_int), ("splits_y", C.POINTER(C.c_int)), ("splits_x", C.POINTER(C.c_int)),
                ("overlap_y", C.c_int), ("overlap_x", C.c_int), ("window", C.c_int)]


class SolverParams(C.Structure):
    _fields_ = [("nu0", C.c_double), ("nu1", C.c_double), ("nu2", C.POINTER(C.c_double)),
                ("gamma", C.POINTER(C.c_double)), ("gamma0", C.POINTER(C.c_double)),
                ("reweighting_sig", C.POINTER(C.c_double)),
                ("reweighting_sig_bar", C.POINTER(C.c_double)),
                ("reweighting_alpha", C.c_double), ("reweighting_flag", C.c_int),
                ("reweighting_min_iter", C.c_int), ("reweighting_max_iter", C.c_int),
                ("reweighting_rel_var", C.c_double), ("pdfb_min_iter", C.c_int),
                ("pdfb_max_iter", C.c_int), ("pdfb_rel_var", C.c_double),
                ("pdfb_fidelity_tolerance", C.c_double), ("pdfb_rel_var_low", C.c_double),
                ("elipse_proj_max_iter", C.c_int), ("elipse_proj_min_iter", C.c_int),
                ("elipse_proj_eps", C.c_double), ("adjust_flag_noise", C.c_int),
                ("adjust_noise_min_iter", C.c_int), ("adjust_noise_rel_var", C.c_double),
                ("adjust_noise_start_iter", C.c_int), ("adjust_noise_change_percentage", C.c_double),
                ("alph", C.c_double), ("alph_bar", C.c_double)]


class IterInfo(C.Structure):
    _fields_ = [("rel_val", C.c_double), ("residual", C.c_double), ("epsilon", C.c_double),
                ("nuclear", C.c_double)]


class RunInfo(C.Structure):
    _fields_ = [("n_iter", C.c_int), ("n_reweights", C.c_int), ("converged", C.c_int),
                ("rel_val", C.c_double), ("residual", C.c_double), ("epsilon", C.c_double),
                ("seconds", C.c_double), ("n_noise_adjustments", C.c_int)]


class Tuning(C.Structure):
    _fields_ = [("tuned", C.c_int), ("fft_chunk", C.c_int), ("grid_slice", C.c_int), ("n_fft", C.c_int),
                ("n_grid", C.c_int), ("fft_candidates", C.c_int * 8), ("fft_ms", C.c_double * 8),
                ("grid_candidates", C.c_int * 8), ("grid_ms", C.c_double * 8)]

    def as_dict(self):
        return {"tuned": bool(self.tuned), "fft_chunk": self.fft_chunk, "grid_slice": self.grid_slice,
                "fft_ms": {int(self.fft_candidates[i]): round(float(self.fft_ms[i]), 4) for i in range(self.n_fft)},
                "grid_ms": {int(self.grid_candidates[i]): round(float(self.grid_ms[i]), 4)
                            for i in range(self.n_grid)}}


class WarmInfo(C.Structure):
    _fields_ = [("used", C.c_int), ("objective_warm", C.c_double), ("objective_cold", C.c_double),
                ("seconds", C.c_double)]


_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_vp = C.c_void_p
_i64p = C.POINTER(C.c_int64)

# name -> (restype, argtypes); the list is every symbol of include/fhs_b200.h
SIGNATURES = {
    "fhs_abi_version": (C.c_int, []),
    "fhs_last_error": (C.c_char_p, []),
    "fhs_kernel_launch_count": (C.c_ulonglong, []),
    "fhs_measop_create": (C.c_int, [C.c_int] * 8 + [C.POINTER(_vp)]),
    "fhs_measop_destroy": (C.c_int, [_vp]),
    "fhs_measop_set_channel": (C.c_int, [_vp, C.c_int, C.c_int64, _dp, _dp, _dp, C.c_int, _i64p]),
    "fhs_measop_commit": (C.c_int, [_vp]),
    "fhs_measop_n_vis": (C.c_int64, [_vp, C.c_int]),
    "fhs_measop_create_dr": (C.c_int, [_vp, C.POINTER(_vp)]),
    "fhs_measop_is_dr": (C.c_int, [_vp]),
    "fhs_measop_dr_cells": (C.c_int, [_vp, C.c_int, _i64p]),
    "fhs_measop_dr_lambda": (C.c_int, [_vp, C.c_int, _dp]),
    "fhs_measop_autotune": (C.c_int, [_vp, C.POINTER(Tuning)]),
    "fhs_measop_set_tuning": (C.c_int, [_vp, C.c_int, C.c_int]),
    "fhs_measop_tuning": (C.c_int, [_vp, C.POINTER(Tuning)]),
    "fhs_measop_grid_size": (C.c_int64, [_vp]),
    "fhs_measop_n_blocks": (C.c_int, [_vp, C.c_int]),
    "fhs_measop_image_size": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fhs_scaled_fft": (C.c_int, [_vp, _dp, _dp]),
    "fhs_scaled_fft_adjoint": (C.c_int, [_vp, _dp, _dp]),
    "fhs_apply_direct_operator": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "fhs_apply_adjoint_operator": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "fhs_forward_operator": (C.c_int, [_vp, _dp, _dp]),
    "fhs_adjoint_operator": (C.c_int, [_vp, _dp, _dp]),
    "fhs_operator_norm": (C.c_int, [_vp, C.c_int, C.c_double, _dp]),
    "fhs_compute_residual_images": (C.c_int, [_vp, _dp, _dp, _dp]),
    "fhs_update_dual_data_fidelity": (C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "fhs_gen_preconditioning_matrix": (C.c_int, [C.c_int64, _dp, _dp, C.c_int, C.c_int, C.c_int, _dp]),
    "fhs_measop_set_preconditioner": (C.c_int, [_vp, C.c_int, _dp]),
    "fhs_forward_operator_precond": (C.c_int, [_vp, _dp, _dp]),
    "fhs_adjoint_operator_precond": (C.c_int, [_vp, _dp, _dp]),
    "fhs_operator_norm_precond": (C.c_int, [_vp, C.c_int, C.c_double, _dp]),
    "fhs_update_dual_data_fidelity_precond": (C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int,
                                                        C.c_double, _dp, _dp, _dp, _dp, _dp,
                                                        C.POINTER(C.c_int)]),
    "fhs_proj_l2ball": (C.c_int, [C.c_int, C.c_int64, _dp, C.c_double, _dp, _dp]),
    "fhs_proj_l2ball_noalloc": (C.c_int, [C.c_int, C.c_int64, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
    "fhs_nuclear_norm": (C.c_int, [C.c_int, C.c_int64, C.c_int, _dp, _dp]),
    "fhs_sara_n_coefs": (C.c_int64, [C.c_int, C.c_int, C.c_int]),
    "fhs_sara_analysis": (C.c_int, [C.c_int] * 5 + [_dp, _dp]),
    "fhs_sara_synthesis": (C.c_int, [C.c_int] * 5 + [_dp, _dp]),
    "fhs_compute_sara_prior": (C.c_int, [C.c_int] * 5 + [_dp, _dp]),
    "fhs_solver_create": (C.c_int, [_vp, C.POINTER(SolverConfig), C.POINTER(_vp)]),
    "fhs_solver_destroy": (C.c_int, [_vp]),
    "fhs_solver_set_data": (C.c_int, [_vp, _dp, _dp]),
    "fhs_solver_set_params": (C.c_int, [_vp, C.POINTER(SolverParams)]),
    "fhs_solver_init": (C.c_int, [_vp, _dp]),
    "fhs_solver_iterate": (C.c_int, [_vp, C.c_int, C.POINTER(IterInfo)]),
    "fhs_solver_run": (C.c_int, [_vp, C.c_int, C.POINTER(RunInfo)]),
    "fhs_solver_get_x": (C.c_int, [_vp, _dp]),
    "fhs_unet_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(_vp)]),
    "fhs_unet_destroy": (C.c_int, [_vp]),
    "fhs_unet_n_params": (C.c_int64, [_vp]),
    "fhs_unet_set_params": (C.c_int, [_vp, _fp]),
    "fhs_unet_get_params": (C.c_int, [_vp, _fp]),
    "fhs_unet_forward": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _fp, _fp]),
    "fhs_unet_gradient": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _fp, _fp, _fp, _dp]),
    "fhs_unet_train_step": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _fp, _fp, C.c_float, _dp]),
    "fhs_solver_init_warm": (C.c_int, [_vp, _vp, C.c_int, C.POINTER(WarmInfo)]),
    "fhs_solver_group_stats": (C.c_int, [_vp, _dp]),
    "fhs_solver_update_weights": (C.c_int, [_vp]),
    "fhs_solver_ellipse_iterations": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "fhs_solver_epsilon": (C.c_int, [_vp, _dp]),
    "fhs_solver_set_epsilon": (C.c_int, [_vp, _dp]),
    "fhs_solver_regularization": (C.c_int, [_vp, _dp, _dp]),
    "fhs_solver_field_size": (C.c_int64, [_vp, C.c_int]),
    "fhs_solver_get_field": (C.c_int, [_vp, C.c_int, _dp]),
    "fhs_solver_set_field": (C.c_int, [_vp, C.c_int, _dp]),
    "fhs_solver_stage_count": (C.c_int, []),
    "fhs_solver_stage_name": (C.c_char_p, [C.c_int]),
    "fhs_solver_time_iterations": (C.c_int, [_vp, C.c_int, _dp]),
    "fhs_solver_profile_stages": (C.c_int, [_vp, C.c_int, _dp]),
}

# fhs_field (include/fhs_b200.h)
FIELDS = {"xsol": 0, "g": 1, "v0": 2, "v1": 3, "v2": 4, "proj": 5, "weights0": 6, "weights1": 7}

_lib = None


def lib():
    """Load the library once (raises if the CUDA build is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built: run faceted-hypersara_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            try:
                fn = getattr(L, name)
            except AttributeError:  # reported by the symbol test, not at import
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int):
    if status != FHS_OK:
        raise FhsError(status, lib().fhs_last_error().decode())


def dptr(a):
    """double* of a contiguous float64 numpy array (None -> NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(_dp)
