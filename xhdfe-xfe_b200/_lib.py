"""ctypes binding of libb200fe.so (the C ABI declared in include/b200fe.h).

The library is built in-tree by ``build.py`` next to this file.  Loading fails
loudly when it is missing: there is no CPU fallback behind this package.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libb200fe.so"

OK, NOT_CONVERGED, UNAVAILABLE, CUDA_ERROR, INVALID_ARG = 0, 1, 2, 3, 4
PREC_FP64, PREC_MIXED = 0, 1
MAX_DIMS = 8
PROF_CATEGORIES = 8
PROF_NAMES = ("pass", "gather", "finalize", "vector", "rhs", "final", "setup", "couple")

STATUS_NAMES = {
    OK: "ok",
    NOT_CONVERGED: "not converged",
    UNAVAILABLE: "CUDA device unavailable",
    CUDA_ERROR: "CUDA error",
    INVALID_ARG: "invalid argument",
}

# Every symbol include/b200fe.h declares.
EXPORTED_SYMBOLS = (
    "b200fe_version",
    "b200fe_device_available",
    "b200fe_default_options",
    "b200fe_context_create",
    "b200fe_context_destroy",
    "b200fe_last_error",
    "b200fe_context_stream",
    "b200fe_absorb",
    "b200fe_absorb_device",
    "b200fe_absorb_fe",
    "b200fe_absorb_slopes",
    "b200fe_absorb_slopes_device",
    "b200fe_absorb_group_individual",
    "b200fe_demean_raw",
    "b200fe_fe_recovery_max_delta",
    "b200fe_demean_sorted_noalloc",
    "b200fe_dense_ids_device",
    "b200fe_drop_singletons_device",
    "b200fe_first_pair_components_device",
    "b200fe_ols_device",
    "b200fe_ols",
    "b200fe_kss_create",
    "b200fe_kss_destroy",
    "b200fe_kss_last_error",
    "b200fe_kss_max_lanes",
    "b200fe_kss_pack_buffer",
    "b200fe_kss_solve_multi",
    "b200fe_kss_solve",
    "b200fe_kss_jla",
    "b200fe_stable_sort_u64",
    "b200fe_mlp_num_params",
    "b200fe_mlp_forward",
    "b200fe_mlp_grad",
    "b200fe_mlp_adam",
    "b200fe_warmstart_set",
    "b200fe_warmstart_samples",
)


class GroupIndividual(ctypes.Structure):
    _fields_ = [
        ("num_individuals", ctypes.c_int32),
        ("num_edges", ctypes.c_int64),
        ("group_ptr", ctypes.c_void_p),
        ("group_individual", ctypes.c_void_p),
        ("individual_ptr", ctypes.c_void_p),
        ("individual_group", ctypes.c_void_p),
        ("group_scale", ctypes.c_void_p),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("tol", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("certify", ctypes.c_int),
        ("check_interval", ctypes.c_int),
        ("reuse_structure", ctypes.c_int),
        ("inner_tol", ctypes.c_double),
        ("tolerance_mode", ctypes.c_int),
        ("max_outer", ctypes.c_int),
        ("profile", ctypes.c_int),
        ("pass_kernel", ctypes.c_int),
        ("fe_linf_tol", ctypes.c_double),
    ]


OLS_MAX_P = 32


class OlsResult(ctypes.Structure):
    """b200fe_ols_result (include/b200fe.h)."""
    _fields_ = [
        ("p", ctypes.c_int), ("num_clusters", ctypes.c_int),
        ("rss", ctypes.c_double), ("sigma2", ctypes.c_double), ("df_resid", ctypes.c_double),
        ("cov_scale", ctypes.c_double), ("cluster_u2", ctypes.c_double),
        ("coef", ctypes.c_double * OLS_MAX_P), ("se", ctypes.c_double * OLS_MAX_P),
        ("cov", ctypes.c_double * (OLS_MAX_P * OLS_MAX_P)),
        ("xtx_inv", ctypes.c_double * (OLS_MAX_P * OLS_MAX_P)),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("outer_iterations", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("precision_certified", ctypes.c_int),
        ("primary_dim", ctypes.c_int),
        ("num_levels_present", ctypes.c_int * MAX_DIMS),
        ("abs_residual", ctypes.c_double),
        ("abs_residual_rel", ctypes.c_double),
        ("rel_residual", ctypes.c_double),
        ("setup_ms", ctypes.c_double),
        ("solve_ms", ctypes.c_double),
        ("h2d_ms", ctypes.c_double),
        ("d2h_ms", ctypes.c_double),
        ("kernel_launches", ctypes.c_longlong),
        ("library_calls", ctypes.c_longlong),
        ("prof_ms", ctypes.c_double * PROF_CATEGORIES),
        ("prof_bytes", ctypes.c_double * PROF_CATEGORIES),
        ("prof_launches", ctypes.c_longlong * PROF_CATEGORIES),
        ("warm_columns", ctypes.c_int),
    ]


_LIB = None


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load libb200fe.so and declare argument types.  Raises when missing."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with build.build() (nvcc, sm_100a); "
            "this package has no CPU fallback")
    lib = ctypes.CDLL(str(p))
    vp, i64, c_int = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    pp = ctypes.POINTER(ctypes.c_void_p)
    lib.b200fe_version.restype = c_int
    lib.b200fe_device_available.restype = c_int
    lib.b200fe_default_options.argtypes = [ctypes.POINTER(Options)]
    lib.b200fe_default_options.restype = None
    lib.b200fe_context_create.argtypes = [c_int, ctypes.POINTER(vp)]
    lib.b200fe_context_create.restype = c_int
    lib.b200fe_context_destroy.argtypes = [vp]
    lib.b200fe_context_destroy.restype = None
    lib.b200fe_last_error.argtypes = [vp]
    lib.b200fe_last_error.restype = ctypes.c_char_p
    lib.b200fe_context_stream.argtypes = [vp]
    lib.b200fe_context_stream.restype = vp
    lib.b200fe_absorb.argtypes = [vp, vp, vp, i64, c_int, c_int, pp, vp, vp,
                                  ctypes.POINTER(Options), vp, vp, ctypes.POINTER(Result)]
    lib.b200fe_absorb.restype = c_int
    lib.b200fe_absorb_device.argtypes = [vp, vp, i64, c_int, c_int, pp, vp, vp,
                                         ctypes.POINTER(Options), vp, ctypes.POINTER(Result), vp]
    lib.b200fe_absorb_device.restype = c_int
    lib.b200fe_demean_raw.argtypes = [vp, vp, i64, c_int, c_int, pp, vp, ctypes.c_double,
                                      c_int, ctypes.POINTER(c_int)]
    lib.b200fe_demean_raw.restype = c_int
    lib.b200fe_fe_recovery_max_delta.argtypes = [vp, vp, i64, c_int, pp, vp, vp, vp,
                                                 ctypes.POINTER(ctypes.c_double)]
    lib.b200fe_fe_recovery_max_delta.restype = c_int
    lib.b200fe_demean_sorted_noalloc.argtypes = [vp, i64, c_int, vp, ctypes.c_int32, vp, vp, vp]
    lib.b200fe_demean_sorted_noalloc.restype = c_int
    lib.b200fe_absorb_fe.argtypes = [vp, vp, vp, i64, c_int, c_int, pp, vp, vp,
                                     ctypes.POINTER(Options), vp, vp, pp, ctypes.POINTER(Result)]
    lib.b200fe_absorb_fe.restype = c_int
    lib.b200fe_absorb_slopes.argtypes = [vp, vp, vp, i64, c_int, c_int, pp, vp, pp, vp, vp,
                                         ctypes.POINTER(Options), vp, vp, ctypes.POINTER(Result)]
    lib.b200fe_absorb_slopes.restype = c_int
    lib.b200fe_absorb_slopes_device.argtypes = [vp, vp, i64, c_int, c_int, pp, vp, pp, vp, vp,
                                                ctypes.POINTER(Options), vp,
                                                ctypes.POINTER(Result), vp]
    lib.b200fe_absorb_slopes_device.restype = c_int
    lib.b200fe_absorb_group_individual.argtypes = [
        vp, vp, vp, i64, c_int, c_int, pp, vp, ctypes.POINTER(GroupIndividual), vp,
        ctypes.POINTER(Options), vp, vp, ctypes.POINTER(Result)]
    lib.b200fe_absorb_group_individual.restype = c_int
    lib.b200fe_dense_ids_device.argtypes = [vp, vp, i64, vp, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_int32)]
    lib.b200fe_dense_ids_device.restype = c_int
    lib.b200fe_drop_singletons_device.argtypes = [vp, c_int, pp, vp, i64, vp, c_int,
                                                  ctypes.POINTER(ctypes.c_int64),
                                                  ctypes.POINTER(c_int)]
    lib.b200fe_drop_singletons_device.restype = c_int
    lib.b200fe_first_pair_components_device.argtypes = [
        vp, vp, vp, i64, vp, ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_int64),
        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.b200fe_first_pair_components_device.restype = c_int
    lib.b200fe_ols_device.argtypes = [vp, vp, vp, i64, c_int, vp, vp, ctypes.c_int32, c_int,
                                      ctypes.c_double, c_int, ctypes.POINTER(OlsResult)]
    lib.b200fe_ols_device.restype = c_int
    lib.b200fe_ols.argtypes = [vp, vp, vp, i64, c_int, vp, vp, ctypes.c_int32, c_int,
                               ctypes.c_double, c_int, ctypes.POINTER(OlsResult)]
    lib.b200fe_ols.restype = c_int
    lib.b200fe_kss_create.argtypes = [c_int, c_int, vp, vp, vp, i64, vp, vp, vp, vp, vp, vp,
                                      ctypes.POINTER(vp)]
    lib.b200fe_kss_create.restype = c_int
    lib.b200fe_kss_destroy.argtypes = [vp]
    lib.b200fe_kss_destroy.restype = None
    lib.b200fe_kss_last_error.argtypes = [vp]
    lib.b200fe_kss_last_error.restype = ctypes.c_char_p
    lib.b200fe_kss_max_lanes.argtypes = []
    lib.b200fe_kss_max_lanes.restype = c_int
    lib.b200fe_kss_pack_buffer.argtypes = [vp, c_int]
    lib.b200fe_kss_pack_buffer.restype = vp
    lib.b200fe_kss_solve_multi.argtypes = [vp, vp, vp, c_int, ctypes.c_double, c_int, vp]
    lib.b200fe_kss_solve_multi.restype = c_int
    lib.b200fe_kss_solve.argtypes = [vp, vp, vp, ctypes.c_double, c_int, ctypes.POINTER(c_int)]
    lib.b200fe_kss_solve.restype = c_int
    lib.b200fe_kss_jla.argtypes = [vp, ctypes.c_int64, vp, vp, vp, vp, ctypes.c_double, ctypes.c_uint64, c_int,
                                   c_int, ctypes.c_double, c_int, vp, vp, vp, vp, vp, vp,
                                   ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_longlong)]
    lib.b200fe_kss_jla.restype = c_int
    lib.b200fe_stable_sort_u64.argtypes = [vp, vp, i64]
    lib.b200fe_stable_sort_u64.restype = c_int
    lib.b200fe_mlp_num_params.argtypes = []
    lib.b200fe_mlp_num_params.restype = c_int
    lib.b200fe_mlp_forward.argtypes = [vp, vp, vp, i64, vp]
    lib.b200fe_mlp_forward.restype = c_int
    lib.b200fe_mlp_grad.argtypes = [vp, vp, vp, vp, i64, vp]
    lib.b200fe_mlp_grad.restype = c_int
    lib.b200fe_mlp_adam.argtypes = [vp, vp, vp, vp, vp, c_int, ctypes.c_double]
    lib.b200fe_mlp_adam.restype = c_int
    lib.b200fe_warmstart_set.argtypes = [vp, vp, c_int]
    lib.b200fe_warmstart_set.restype = c_int
    lib.b200fe_warmstart_samples.argtypes = [vp, vp, i64, c_int, c_int, pp, vp, vp,
                                             ctypes.POINTER(Options), vp, vp, vp, i64,
                                             ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(Result)]
    lib.b200fe_warmstart_samples.restype = c_int
    if path is None:
        _LIB = lib
    return lib


def default_options(lib=None) -> Options:
    o = Options()
    (lib or load()).b200fe_default_options(ctypes.byref(o))
    return o
