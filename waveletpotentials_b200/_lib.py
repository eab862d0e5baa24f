"""ctypes binding of the in-tree CUDA library ``libwp_b200.so`` (declared in include/wp_api.h).

There is no CPU fallback: if the library is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwp_b200.so")
HEADER = os.path.join(HERE, "..", "include", "wp_api.h")

WP_OK = 0
STATUS = {0: "WP_OK", 1: "WP_ERR_INVALID_ARG", 2: "WP_ERR_UNSUPPORTED", 3: "WP_ERR_CUDA", 4: "WP_ERR_WORKSPACE",
          5: "WP_ERR_NOT_CONVERGED", 6: "WP_ERR_NONFINITE", 7: "WP_ERR_DEVICE_WAIT"}
WP_ERR_NOT_CONVERGED, WP_ERR_NONFINITE, WP_ERR_DEVICE_WAIT = 5, 6, 7
WAIT_SITE_GRID_BARRIER, WAIT_SITE_CONV_PIPELINE, WAIT_SITE_BATCH_PUBLISH = 1, 2, 3
BATCH_GRAPH, BATCH_PERSISTENT, BATCH_AUTO = 0, 1, 2
CDF3_5, CDF2_6, CDF4_4, CDF4_6, CDF2_8, CDF3_7 = 2, 5, 6, 7, 10, 11
CDF2_0, CDF1_1, CDF1_7 = 16, 17, 18
PREC_FP32, PREC_MIXED, PREC_FP64 = 0, 1, 2
PROLONG_CONSTANT, PROLONG_TRILINEAR = 0, 1
START_ZERO, START_FMG = 0, 1


class WPError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)}: {msg}")


class MgParams(ctypes.Structure):
    _fields_ = [("max_cycles", ctypes.c_int), ("nu1", ctypes.c_int), ("nu2", ctypes.c_int),
                ("omega", ctypes.c_double), ("rel_tol", ctypes.c_double), ("precision", ctypes.c_int),
                ("prolongation", ctypes.c_int), ("start", ctypes.c_int), ("host_loop", ctypes.c_int),
                ("inner_cycles", ctypes.c_int)]


class MgReport(ctypes.Structure):
    _fields_ = [("cycles", ctypes.c_int), ("rel_residual", ctypes.c_double), ("history", ctypes.c_double * 64),
                ("steps", ctypes.c_int)]


_lib = None
P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double
C = ctypes.c_char
S = ctypes.c_size_t
PP = ctypes.POINTER(ctypes.c_void_p)

SIGNATURES = {
    "wp_last_error": (ctypes.c_char_p, []),
    "wp_version": (I, []),
    "wp_debug_withhold_wait": (I, [I, I, ctypes.c_double]),
    "wp_profile_enable": (None, [I]),
    "wp_profile_reset": (None, []),
    "wp_launch_count": (ctypes.c_longlong, []),
    "wp_profile_collect": (I, []),
    "wp_profile_entry": (I, [I, ctypes.c_char_p, I, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(D),
                             ctypes.POINTER(D)]),
    "wp_dwt1d": (I, [P, P, I, I, I, I, C, C, I, I, P]),
    "wp_dwt1d_f64": (I, [P, P, I, I, I, I, C, C, I, I, P]),
    "wp_ip_diag": (I, [P, I, I, C]),
    "wp_recover3d_create": (I, [PP, I, I, I, D, D, D, C, I, I]),
    "wp_recover3d_run": (I, [P, P, P, P, P, P, P, P]),
    "wp_recover3d_project": (I, [P, P, P, P, P, P, P, P]),
    "wp_recover3d_cut": (I, [P, P, P, P, P, P, P, I, P]),
    "wp_recover3d_destroy": (I, [P]),
    "wp_recover2d_create": (I, [PP, I, I, D, D, C, I, I]),
    "wp_recover2d_run": (I, [P, P, P, P, P]),
    "wp_recover2d_project": (I, [P, P, P, P, P]),
    "wp_recover2d_destroy": (I, [P]),
    "wp_mgfrac3d_create": (I, [PP, P, P, P, I, I, I, D, D, D, C, P]),
    "wp_mgfrac3d_solve": (I, [P, P, P, P, I, I, I, D, P]),
    "wp_mgfrac3d_solve_index": (I, [P, P, P, P, I, I, I, D, P]),
    "wp_mgfrac3d_solve_index64": (I, [P, P, P, P, I, I, I, D, P]),
    "wp_mgfrac3d_index_sizes": (I, [P, P, P, I, P, P]),
    "wp_mgfrac3d_solve_tol": (I, [P, P, P, P, ctypes.POINTER(MgParams), ctypes.POINTER(MgReport), P]),
    "wp_mgfrac3d_residual": (I, [P, P, P, ctypes.POINTER(D), P]),
    "wp_mgfrac3d_iterate64": (I, [P, P, P]),
    "wp_mgfrac3d_iterate64_view": (I, [P, P]),
    "wp_mgfrac3d_destroy": (I, [P]),
    "wp_mgfrac2d_create": (I, [PP, P, P, I, I, D, D, C, P]),
    "wp_mgfrac2d_solve": (I, [P, P, P, P, I, I, I, D, P]),
    "wp_mgfrac2d_solve_tol": (I, [P, P, P, P, ctypes.POINTER(MgParams), ctypes.POINTER(MgReport), P]),
    "wp_mgfrac2d_residual": (I, [P, P, P, ctypes.POINTER(D), P]),
    "wp_mgfrac2d_destroy": (I, [P]),
    "wp_divergence_frac3d": (I, [P, P, P, P, P, P, P, I, I, I, D, D, D, P]),
    "wp_divergence_frac2d": (I, [P, P, P, P, P, I, I, D, D, P]),
    "wp_grad_subtract_frac3d": (I, [P, P, P, P, P, P, P, I, I, I, D, D, D, I, P]),
    "wp_grad_subtract_frac3d_p64": (I, [P, P, P, P, P, P, P, I, I, I, D, D, D, I, P]),
    "wp_grad_subtract_frac2d": (I, [P, P, P, P, P, I, I, D, D, I, P]),
    "wp_max_abs": (I, [P, S, ctypes.POINTER(D), P]),
    "wp_sdf_spheres3d": (I, [P, I, I, I, D, P, P, I, P]),
    "wp_fractions3d": (I, [P, P, P, P, I, I, I, D, P]),
    "wp_fractions3d_subsampled": (I, [P, P, P, P, I, I, I, D, P]),
    "wp_fast_sweep_solve": (I, [P, I, I, I, D, I, P]),
    "wp_fast_sweep_reinit": (I, [P, I, I, I, D, I, P]),
    "wp_particles_to_ls": (I, [P, P, I, I, I, I, D, D, D, I, P]),
    "wp_particles_to_ls_narrow": (I, [P, P, I, I, I, I, D, D, D, I, P]),
    "wp_sdf_boxes3d": (I, [P, I, I, I, D, P, P, I, P]),
    "wp_sdf_circles2d": (I, [P, I, I, D, P, P, I, P]),
    "wp_fractions2d": (I, [P, P, P, I, I, D, P]),
    "wp_dst3d_create": (I, [PP, I, I, I, D, D, D]),
    "wp_dst3d_solve": (I, [P, P, P, P]),
    "wp_dst3d_destroy": (I, [P]),
    "wp_dst3d_solve_noalloc": (I, [P, P, I, I, I, D, D, D, P]),
    "wp_sweep3d_create": (I, [PP, I, I, I, D, D, D, C]),
    "wp_sweep3d_solve": (I, [P, P, P, P, P, P, P, P]),
    "wp_sweep3d_solve_from_mid": (I, [P, P, P, P, P, P, P, I, I, I, P]),
    "wp_sweep3d_project": (I, [P, P, P, P, P]),
    "wp_sweep3d_destroy": (I, [P]),
    "wp_sweep2d_solve": (I, [P, P, P, I, I, D, D, C, P]),
    "wp_mgfrac3d_autotune": (I, [P, P]),
    "wp_mgfrac3d_tiles": (I, [P, P, P, P, I, P]),
    "wp_mgfrac3d_uniform_rows": (I, [P, I, P, P]),
    "wp_mgfrac3d_set_tile": (I, [P, I, I, I, I]),
    "wp_conv3_forward": (I, [P, P, I, P, P, I, P, P, I, I, I, I, I, P, P, P]),
    "wp_conv3_wgrad": (I, [P, P, I, P, I, I, I, I, P]),
    "wp_random_field3d": (I, [P, I, I, I, D, D, I, ctypes.c_ulonglong, P]),
    "wp_velocity3d": (I, [P, P, P, I, I, I, ctypes.c_ulonglong, D, D, D, D, I, P]),
    "wp_unet_create": (I, [PP, I, I, I, ctypes.c_ulonglong]),
    "wp_unet_predict": (I, [P, P, P, P, D, P]),
    "wp_unet_train_step": (I, [P, P, P, P, D, D, P, P]),
    "wp_unet_params": (I, [P, I, P, S, P]),
    "wp_unet_set_params": (I, [P, P, S]),
    "wp_unet_destroy": (I, [P]),
    "wp_batch_create": (I, [PP, I, P, P, P, P, P, P, P, I]),
    "wp_batch_plan": (I, [P, P, P, P, P, P]),
    "wp_batch_run": (I, [P, P, P, P, P, P, P, P]),
    "wp_batch_results": (I, [P, P, P, P, P]),
    "wp_batch_set_mode": (I, [P, I, ctypes.c_longlong]),
    "wp_batch_profile": (I, [P, I, P, I, P]),
    "wp_batch_get_mode": (I, [P, P, P, P]),
    "wp_batch_destroy": (I, [P]),
}


def header_symbols() -> list[str]:
    """Every function declared with CUWHHD_API in include/wp_api.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"CUWHHD_API\s+[\w\s\*]+?\b(wp_\w+)\s*\(", txt)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m waveletpotentials_b200.build` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    m = lib().wp_last_error()
    return m.decode() if m else ""


def check(status: int, where: str) -> None:
    if status != WP_OK:
        raise WPError(status, where, last_error())
