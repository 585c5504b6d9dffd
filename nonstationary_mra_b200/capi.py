"""ctypes binding of include/mra_b200.h (the C ABI of libmra_b200.so).

The product path always goes through the compiled CUDA library; when the
library is missing or the device is not an sm_100 GPU the calls raise -- there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmra_b200.so")

MRA_OK, MRA_ERR_ARG, MRA_ERR_CUDA, MRA_ERR_OOM, MRA_ERR_NOT_SPD, MRA_ERR_TIMEOUT, MRA_ERR_STATE, MRA_ERR_NO_DEVICE = range(8)
STATUS_NAMES = ["OK", "ARG", "CUDA", "OOM", "NOT_SPD", "TIMEOUT", "STATE", "NO_DEVICE"]

DIST_CHORDAL, DIST_GREAT_CIRCLE, DIST_EUCLID2D = 0, 1, 2
BASIS_WENDLAND, BASIS_GAUSSIAN = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1

_p_u64 = C.POINTER(C.c_uint64)
_p_f64 = C.POINTER(C.c_double)


class mra_structure(C.Structure):
    _fields_ = [("J", C.c_int32), ("M", C.c_int32), ("r", C.c_int32), ("reserved", C.c_int32),
                ("n_interior", C.c_uint64), ("n_finest", C.c_uint64), ("finest_parent", _p_u64),
                ("knots", _p_f64), ("obs_offset", _p_u64), ("obs", _p_f64), ("obs_value", _p_f64),
                ("pred_offset", _p_u64), ("pred", _p_f64)]


class mra_field(C.Structure):
    _fields_ = [("n_basis", C.c_uint64), ("centers", _p_f64), ("weights", _p_f64), ("intercept", C.c_double)]


class mra_model(C.Structure):
    _fields_ = [("nonstationary", C.c_int32), ("distance", C.c_int32), ("nu_x2", C.c_int32), ("basis", C.c_int32),
                ("prefactor_exp", C.c_double), ("dist_scale", C.c_double), ("basis_len", C.c_double),
                ("field", mra_field * 3)]


class mra_theta(C.Structure):
    _fields_ = [("sill", C.c_double), ("range", C.c_double), ("nugget", C.c_double),
                ("sill_scale", C.c_double), ("range_scale", C.c_double), ("nugget_scale", C.c_double),
                ("weights", _p_f64 * 3), ("intercepts", _p_f64)]


class mra_stats(C.Structure):
    _fields_ = [("d", C.c_double), ("loglik", C.c_double), ("ms_total", C.c_double), ("ms_fields", C.c_double),
                ("ms_prior", C.c_double), ("ms_finest", C.c_double), ("ms_posterior", C.c_double),
                ("ms_predict", C.c_double), ("flop_last", C.c_double), ("flop_reference", C.c_double),
                ("bytes_device", C.c_uint64),
                ("bad_region", C.c_int64), ("kernel_launches", C.c_int32), ("graph_replays", C.c_int32),
                ("n_timed", C.c_int32), ("timed_kind", C.c_int32 * 40), ("timed_level", C.c_int32 * 40),
                ("timed_ms", C.c_double * 40), ("timed_flop", C.c_double * 40),
                ("timed_ms_cov", C.c_double * 40)]

class mra_opt_config(C.Structure):
    _fields_ = [("rho_begin", C.c_double), ("rho_end", C.c_double), ("npt", C.c_int32), ("max_evals", C.c_int32)]


class mra_opt_result(C.Structure):
    _fields_ = [("f_best", C.c_double), ("evals", C.c_int32), ("status", C.c_int32), ("rho_final", C.c_double)]


# double (*)(const double* x, void* user, int32_t* stop)
OBJECTIVE_FN = C.CFUNCTYPE(C.c_double, _p_f64, C.c_void_p, C.POINTER(C.c_int32))
_p_f32 = C.POINTER(C.c_float)

KERNEL_NAMES = {0: "fields", 1: "prior_level", 2: "finest_group", 3: "posterior_level", 4: "reduce", 5: "predict",
                6: "convert"}


# (name, restype, argtypes) of every exported entry point of include/mra_b200.h and include/mra_surrogate.h
SIGNATURES = [
    ("mra_create", C.c_int, [C.POINTER(mra_structure), C.POINTER(mra_model), C.c_int32, C.POINTER(C.c_void_p)]),
    ("mra_destroy", C.c_int, [C.c_void_p]),
    ("mra_set_theta", C.c_int, [C.c_void_p, C.POINTER(mra_theta)]),
    ("mra_set_obs_values", C.c_int, [C.c_void_p, _p_f64]),
    ("mra_loglik", C.c_int, [C.c_void_p, _p_f64, _p_f64]),
    ("mra_predict", C.c_int, [C.c_void_p, _p_f64, _p_f64]),
    ("mra_capture_graph", C.c_int, [C.c_void_p]),
    ("mra_get_stats", C.c_int, [C.c_void_p, C.POINTER(mra_stats)]),
    ("mra_get_terms", C.c_int, [C.c_void_p, _p_f64, C.c_int32]),
    ("mra_shard_set", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_uint8)]),
    ("mra_shard_loglik_subtrees", C.c_int, [C.c_void_p]),
    ("mra_shard_record_size", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("mra_shard_export", C.c_int, [C.c_void_p, C.c_uint64, _p_f64, C.c_uint64]),
    ("mra_shard_import", C.c_int, [C.c_void_p, C.c_uint64, _p_f64, C.c_uint64]),
    ("mra_shard_loglik_top", C.c_int, [C.c_void_p, _p_f64, _p_f64]),
    ("mra_sample_prior", C.c_int, [C.c_void_p, _p_f64, _p_f64, _p_f64]),
    ("mra_eval_covariance", C.c_int, [C.POINTER(mra_model), C.POINTER(mra_theta), _p_f64, C.c_uint64, _p_f64,
                                      C.c_uint64, C.c_int32, _p_f64]),
    ("mra_eval_fields", C.c_int, [C.POINTER(mra_model), C.POINTER(mra_theta), _p_f64, C.c_uint64, _p_f64]),
    ("mra_eval_covariance_static", C.c_int, [C.POINTER(mra_model), C.POINTER(mra_theta), C.c_void_p, C.c_uint64,
                                             C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p]),
    ("mra_autotune", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), _p_f64]),
    ("mra_set_device", C.c_int, [C.c_int32]),
    ("mra_timer_start", C.c_int, [C.c_void_p]),
    ("mra_timer_stop", C.c_int, [C.c_void_p, _p_f64]),
    ("mra_last_error", C.c_char_p, []),
    # include/mra_surrogate.h
    ("mra_opt_minimize", C.c_int, [C.c_int32, _p_f64, _p_f64, _p_f64, C.POINTER(mra_opt_config), OBJECTIVE_FN,
                                   C.c_void_p, C.POINTER(mra_opt_result)]),
    ("mra_mlp_create", C.c_int, [C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("mra_mlp_destroy", C.c_int, [C.c_void_p]),
    ("mra_mlp_num_params", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("mra_mlp_get_params", C.c_int, [C.c_void_p, _p_f32]),
    ("mra_mlp_set_params", C.c_int, [C.c_void_p, _p_f32]),
    ("mra_mlp_set_data", C.c_int, [C.c_void_p, _p_f32, _p_f32, C.c_int64]),
    ("mra_mlp_grad", C.c_int, [C.c_void_p, _p_f32, _p_f32]),
    ("mra_mlp_train", C.c_int, [C.c_void_p, C.c_int32, C.c_float, _p_f32]),
    ("mra_mlp_predict", C.c_int, [C.c_void_p, _p_f32, C.c_int64, _p_f32, _p_f32]),
]

_lib: Optional[C.CDLL] = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads libmra_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m nonstationary_mra_b200.build`")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MRAError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else status}: {msg}")


def check(status: int, where: str) -> None:
    if status != MRA_OK:
        msg = load().mra_last_error()
        raise MRAError(status, where, msg.decode() if msg else "")


def f64p(a: np.ndarray):
    return a.ctypes.data_as(_p_f64)


def u64p(a: np.ndarray):
    return a.ctypes.data_as(_p_u64)


def f32p(a: np.ndarray):
    return a.ctypes.data_as(_p_f32)
