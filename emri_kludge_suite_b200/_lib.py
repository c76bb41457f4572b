"""ctypes binding of libaak_b200.so (the C ABI declared in include/aak.h).

The library is built in-tree by ``emri_kludge_suite_b200.build``.  Loading
fails loudly when it is missing: there is no Python or CPU fallback for the
waveform kernels.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libaak_b200.so")

AAK_OK = 0
STATUS_NAMES = {
    0: "AAK_OK",
    1: "AAK_ERR_INVALID_PARAM",
    2: "AAK_ERR_UNSTABLE_START",
    3: "AAK_ERR_FIT_TOO_CLOSE_TO_PLUNGE",
    4: "AAK_ERR_SOLVER_NO_CONVERGE",
    5: "AAK_ERR_CUDA",
    6: "AAK_ERR_NO_MEMORY",
    7: "AAK_ERR_TOO_FEW_STEPS",
    8: "AAK_ERR_CAPACITY",
    9: "AAK_ERR_DEVICE_TIMEOUT",
}

PARAM_FIELDS = "length dt p T f T_fit mu M s e iota gamma psi theta_S phi_S theta_K phi_K alpha D".split()


class AAKParams(ctypes.Structure):
    """struct aak_params (include/aak.h); the reference SetPar fields."""

    _fields_ = [("length", ctypes.c_int64)] + [(n, ctypes.c_double) for n in PARAM_FIELDS[1:]] + [
        ("backint", ctypes.c_int32),
        ("LISA", ctypes.c_int32),
    ]


class AAKMapped(ctypes.Structure):
    """struct aak_mapped (include/aak.h)."""

    _fields_ = [
        ("steps", ctypes.c_int32),
        ("inspiral_flag", ctypes.c_int32),
        ("newton_iterations", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("Phi0", ctypes.c_double),
        ("e_traj", ctypes.c_double * 100),
        ("v_map", ctypes.c_double * 100),
        ("M_map", ctypes.c_double * 100),
        ("s_map", ctypes.c_double * 100),
        ("dt_map", ctypes.c_double * 100),
    ]


class AAKError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        msg = f"{what}: {name}" if what else name
        try:
            msg += f" ({lib().aak_status_string(status).decode()})"
            detail = lib().aak_last_error_detail().decode()
            if status in (5, 6) and detail:
                msg += f" [{detail}]"
        except Exception:
            pass
        super().__init__(msg)


class AAKValueError(AAKError, ValueError):
    """Parameter-level failures (the reference would exit the process)."""


_VALUE_STATUSES = {1, 2, 3, 4, 7, 8}


def check(status: int, what: str = "") -> None:
    if status != AAK_OK:
        if status in _VALUE_STATUSES:
            raise AAKValueError(status, what)
        raise AAKError(status, what)


_lib = None

_d = ctypes.c_double
_dp = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.c_int32
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64 = ctypes.c_int64
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p


def lib():
    """Load libaak_b200.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first (python -m emri_kludge_suite_b200.build)"
        )
    L = ctypes.CDLL(LIB_PATH)
    L.aak_status_string.restype = ctypes.c_char_p
    L.aak_status_string.argtypes = [ctypes.c_int]
    L.aak_version.restype = ctypes.c_int
    L.aak_last_error_detail.restype = ctypes.c_char_p
    L.aak_last_error_detail.argtypes = []
    L.aak_front_end.argtypes = [ctypes.POINTER(AAKParams), _dp, ctypes.POINTER(AAKMapped)]
    L.aak_coarse_kerr.argtypes = [ctypes.POINTER(AAKParams), _i32p, _dp, _dp, _dp, _dp, _dp]
    L.aak_parmap.argtypes = [_dp, _d, _d, _d, _d, _d, _dp, _dp, _i32p]
    L.aak_wave.argtypes = [ctypes.POINTER(AAKParams), _dp, _dp, _dp, _dp]
    L.aak_phase.argtypes = [ctypes.POINTER(AAKParams)] + [_dp] * 9
    L.aak_tdi.argtypes = [ctypes.POINTER(AAKParams)] + [_dp] * 8
    L.aak_tdi_batch_host.argtypes = [_vp, ctypes.POINTER(AAKParams), _i32, _i32, _dp, _i64p, _i32p]
    L.aak_batch_run_phase.argtypes = [_vp, _vp, _i64, _vp]
    L.aak_phase_batch_host.argtypes = [_vp, ctypes.POINTER(AAKParams), _i32, _i32, _dp, _i64p, _i32p]
    L.aak_genwave.argtypes = [_dp, _dp, _dp, _d, _i32, _dp, _dp, _d, _dp, _d, _d, _dp, _d, _d, _d, _d, _d, _d, _d,
                              _d, _d, _dp, _i32, _i32, _i32, _i32]
    L.aak_ctx_create.argtypes = [_i32, ctypes.POINTER(_vp)]
    L.aak_ctx_destroy.argtypes = [_vp]
    L.aak_ctx_destroy.restype = None
    L.aak_batch_plan.argtypes = [_vp, ctypes.POINTER(AAKParams), _i32, _i32p, _i32]
    L.aak_batch_plan_mapped.argtypes = [_vp, ctypes.POINTER(AAKParams), ctypes.POINTER(AAKMapped), _i32, _i32p, _i32]
    L.aak_batch_info.argtypes = [_vp, _i64p, _i64p, _i32p, _i32p, _i32p]
    L.aak_batch_upload.argtypes = [_vp, _vp]
    L.aak_batch_plan_bytes.argtypes = [_vp, _i64p]
    L.aak_batch_run.argtypes = [_vp, _vp, _vp, _vp, _vp, _i64, _i32, _vp]
    L.aak_batch_run_noalloc.argtypes = [_vp, _vp, _i64, _i64p, _vp, _vp, _vp]
    L.aak_batch_run_plain.argtypes = [_vp, _vp, _vp, _vp, _i64, _vp]
    L.aak_batch_last_launches.argtypes = [_vp]
    L.aak_batch_device_status.argtypes = [_vp]
    L.aak_selftest_lookback_timeout.argtypes = [_i64]
    L.aak_batch_set_profiling.argtypes = [_vp, _i32]
    L.aak_batch_kernel_ms.argtypes = [_vp, ctypes.POINTER(ctypes.c_float)]
    L.aak_probe_fp64_tflops.argtypes = [_i32, _dp]
    L.aak_probe_fp32_tflops.argtypes = [_i32, _dp]
    L.aak_batch_run_graph.argtypes = [_vp, _vp, _vp, _i32, _vp]
    L.aak_ctx_set_precision.argtypes = [_vp, _i32]
    L.aak_ctx_set_lookback_bound.argtypes = [_vp, _i64]
    L.aak_ctx_autotune.argtypes = [_vp, _vp, _vp, _i32, ctypes.c_char_p, _i32p, ctypes.POINTER(ctypes.c_float)]
    L.aak_ctx_set_variant.argtypes = [_vp, _i32, _i32]
    L.aak_wave_batch_host.argtypes = [_vp, ctypes.POINTER(AAKParams), _i32, _i32p, _i32, _dp, _dp, _i64p, _i32p]
    # learned ParMap warm start
    _fp = ctypes.POINTER(ctypes.c_float)
    L.aak_mlp_num_params.argtypes = []
    L.aak_mlp_max_train_rows.argtypes = []
    L.aak_mlp_create.argtypes = [_i32, ctypes.POINTER(_vp)]
    L.aak_mlp_destroy.argtypes = [_vp]
    L.aak_mlp_destroy.restype = None
    L.aak_mlp_set_params.argtypes = [_vp, _fp]
    L.aak_mlp_get_params.argtypes = [_vp, _fp]
    L.aak_mlp_set_norm.argtypes = [_vp, _fp, _fp, _fp, _fp]
    L.aak_mlp_set_adam.argtypes = [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float]
    L.aak_mlp_forward.argtypes = [_vp, _vp, _vp, _i64, _vp]
    L.aak_mlp_gradients.argtypes = [_vp, _vp, _vp, _vp, _i64, _vp, _fp, _vp]
    L.aak_mlp_train_step.argtypes = [_vp, _vp, _vp, _vp, _i64, ctypes.c_float, _fp, _vp]
    L.aak_mlp_status.argtypes = [_vp]
    L.aak_mlp_predict_host.argtypes = [_vp, _dp, _dp, _i64]
    L.aak_parmap_separatrix.argtypes = [_d, _d, _d, _dp]
    L.aak_parmap_dataset.argtypes = [_i64, ctypes.c_uint64, ctypes.c_uint64, _i32, _dp, _dp, _dp, _i32p]
    L.aak_parmap_solve_batch.argtypes = [_i64, _dp, _dp, _dp, _i32, _dp, _i32p, _i32p, _dp, _dp, _i32p]
    L.aak_ctx_set_parmap_model.argtypes = [_vp, _vp]
    L.aak_batch_newton_stats.argtypes = [_vp, _i64p, _i64p, _i64p]
    L.aak_gpu_set_parmap_model.argtypes = [_vp, _vp]
    L.aak_ctx_set_parmap_device.argtypes = [_vp, _i32]
    L.aak_ctx_set_evolve_device.argtypes = [_vp, _i32]
    L.aak_batch_plan_ms.argtypes = [_vp, _dp]
    L.aak_lpt_partition.argtypes = [_dp, _i64, _i32, _i32p, _dp]
    L.aak_gpu_set_parmap_device.argtypes = [_vp, _i32]
    _lib = L
    return L


def ptr(a: np.ndarray):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    if a.dtype == np.float32:
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    if a.dtype == np.int32:
        return a.ctypes.data_as(_i32p)
    if a.dtype == np.int64:
        return a.ctypes.data_as(_i64p)
    raise TypeError(a.dtype)


def make_params(pars: dict) -> AAKParams:
    """AAKwrapper-style pars dict -> struct aak_params."""
    kw = {k: float(pars[k]) for k in PARAM_FIELDS[1:]}
    return AAKParams(length=int(pars["length"]), **kw, backint=int(bool(pars["backint"])), LISA=int(bool(pars["LISA"])))


def params_array(plist) -> ctypes.Array:
    arr = (AAKParams * len(plist))()
    for i, p in enumerate(plist):
        arr[i] = p if isinstance(p, AAKParams) else make_params(p)
    return arr
