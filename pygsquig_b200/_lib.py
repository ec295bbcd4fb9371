"""ctypes binding of libsqg.so (include/sqg.h).

The library is built in-tree (``python -m pygsquig_b200.build``).  Loading
fails loudly when it is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

from .exceptions import ConfigurationError, NumericalError, SimulationError

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsqg.so")

SQG_MAX_SCALARS = 4
SQG_OK, SQG_ERR_INVALID, SQG_ERR_CUDA, SQG_ERR_NONFINITE, SQG_ERR_WORKSPACE, SQG_ERR_STATE = range(6)
SQG_F64, SQG_F32 = 0, 1
SQG_EXPLICIT_RK4, SQG_IF_RK4 = 0, 1
SQG_BUF_STAGE, SQG_BUF_UV, SQG_BUF_RING_FORCE, SQG_BUF_STATUS = range(4)
SQG_DIAG_COUNT = 6


class SqgDesc(C.Structure):
    _fields_ = [
        ("N", C.c_int32),
        ("precision", C.c_int32),
        ("scheme", C.c_int32),
        ("p", C.c_int32),
        ("L", C.c_double),
        ("alpha", C.c_double),
        ("nu_p", C.c_double),
        ("has_damping", C.c_int32),
        ("p_damp", C.c_int32),
        ("mu", C.c_double),
        ("kf_damp", C.c_double),
        ("nu_damp", C.c_double),
        ("has_ring", C.c_int32),
        ("reserved0", C.c_int32),
        ("ring_kf", C.c_double),
        ("ring_dk", C.c_double),
        ("ring_epsilon", C.c_double),
        ("ring_tau_f", C.c_double),
        ("ring_amplitude", C.c_double),
        ("n_scalars", C.c_int32),
        ("reserved1", C.c_int32),
        ("kappa", C.c_double * SQG_MAX_SCALARS),
        ("mean_gradient", C.c_int32 * SQG_MAX_SCALARS),
        ("grad_x", C.c_double * SQG_MAX_SCALARS),
        ("grad_y", C.c_double * SQG_MAX_SCALARS),
    ]


class SqgMember(C.Structure):
    _fields_ = [
        ("theta", C.c_void_p),
        ("alpha", C.c_double),
        ("n_scalars", C.c_int32),
        ("reserved", C.c_int32),
        ("scalars", C.c_void_p * SQG_MAX_SCALARS),
        ("kappa", C.c_double * SQG_MAX_SCALARS),
    ]


# Every symbol include/sqg.h declares, with its argument types.
_vp, _i32, _dbl, _sz = C.c_void_p, C.c_int32, C.c_double, C.c_size_t
SIGNATURES = {
    "sqg_plan_create": [C.POINTER(SqgDesc), C.POINTER(C.c_void_p)],
    "sqg_plan_destroy": [_vp],
    "sqg_plan_workspace_bytes": [_vp, C.POINTER(_sz)],
    "sqg_plan_set_workspace": [_vp, _vp, _sz, _vp],
    "sqg_plan_buffer": [_vp, _i32, C.POINTER(_sz), C.POINTER(_sz)],
    "sqg_ring_mode_count": [_vp, C.POINTER(_i32)],
    "sqg_ring_modes": [_vp, C.POINTER(_i32), C.POINTER(_i32)],
    "sqg_rhs": [_vp, _vp, _vp, _vp],
    "sqg_rhs_noalloc": [C.POINTER(SqgDesc), _vp, _vp, _vp],
    "sqg_step": [_vp, _vp, _vp, _dbl, _vp, _vp],
    "sqg_multistep": [_vp, _vp, _i32, _dbl, _vp, _i32, _vp],
    "sqg_stage_begin": [_vp, _vp, _vp],
    "sqg_stage": [_vp, _i32, _vp, _vp, _dbl, _vp, _vp, _vp],
    "sqg_stage_physical": [_vp, _i32, _vp, _vp, _dbl, _vp, _vp, _vp],
    "sqg_plan_shape": [_vp, _vp, _vp, _vp, _vp],
    "sqg_plan_set_shape": [_vp, _i32, _i32],
    "sqg_plan_autotune": [_vp, _i32, _vp],
    "sqg_ring_substeps": [_vp, _vp, _i32, _dbl, _vp, _vp],
    "sqg_max_speed": [_vp, _vp, _vp, _vp, _vp],
    "sqg_spectrum_absmax": [_vp, _vp, _vp, _vp],
    "sqg_velocity": [_vp, _vp, _vp, _vp, _vp],
    "sqg_to_physical": [_vp, _vp, _vp, _vp],
    "sqg_to_spectral": [_vp, _vp, _vp, _vp],
    "sqg_damping": [_vp, _vp, _vp, _vp],
    "sqg_hyperviscosity": [_vp, _vp, _vp, _vp],
    "sqg_ring_forcing": [_vp, _vp, _vp, _dbl, _vp, _vp],
    "sqg_inner": [_vp, _vp, _vp, _vp, _vp],
    "sqg_diagnostics": [_vp, _vp, _vp, _vp],
    "sqg_energy_spectrum": [_vp, _vp, _vp, _vp],
    "sqg_scalar_variance": [_vp, _vp, _vp, _vp],
    "sqg_scalars_step": [_vp, _vp, _vp, _vp, _dbl, _vp],
    "sqg_check_status": [_vp, C.POINTER(C.c_uint32), _vp],
    "sqg_last_launch_count": [_vp, C.POINTER(C.c_int64)],
    "sqg_plan_host_tables": [_vp, _vp, _vp, _vp],
    "sqg_set_timing": [_vp, _i32],
    "sqg_timing_read": [_vp, _vp, _vp, _i32],
    "sqg_batch_create": [C.POINTER(SqgDesc), _i32, C.POINTER(SqgMember), C.POINTER(C.c_void_p)],
    "sqg_batch_workspace_bytes": [_vp, C.POINTER(_sz)],
    "sqg_batch_set_workspace": [_vp, _vp, _sz, _vp],
    "sqg_batch_multistep": [_vp, _i32, _dbl, _i32, _vp],
    "sqg_batch_last_launch_count": [_vp, C.POINTER(C.c_int64)],
    "sqg_batch_destroy": [_vp],
    "sqg_ensemble_create": [C.POINTER(C.c_void_p), _i32, C.POINTER(C.c_void_p)],
    "sqg_ensemble_multistep": [_vp, _i32, _dbl, _i32, _vp],
    "sqg_ensemble_last_launch_count": [_vp, C.POINTER(C.c_int64)],
    "sqg_ensemble_destroy": [_vp],
    "closure_conv64": [_i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp],
    "closure_wgrad64": [_i32, _i32, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _vp],
    "closure_conv_in": [_i32, _i32, _i32, C.c_float, _vp, _vp, _vp, _vp, _vp, _vp],
    "closure_conv_out": [_i32, _i32, _i32, C.c_float, _vp, _vp, _vp, _vp, _vp],
    "closure_conv_out_dgrad": [_i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp],
    "closure_small_grad": [_i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "closure_mse": [C.c_int64, _vp, _vp, _vp, _vp, _vp],
    "closure_adam": [C.c_int64, _vp, _vp, _vp, _vp, C.c_float, C.c_float, C.c_float, C.c_float, _i32, _vp],
    "closure_weights_bf16": [_vp, _vp, _vp, _vp],
    "closure_ops_last_error_string": [],
    "closure_last_error_string": [],
    "sqg_last_error_string": [],
    "sqg_version": [],
}

_lib = None
_lock = threading.Lock()


def load():
    """Load libsqg.so (raises RuntimeError when it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libsqg.so not found at {LIB_PATH}; build it with "
                "`python -m pygsquig_b200.build` (nvcc, sm_100a). There is no CPU fallback."
            )
        lib = C.CDLL(LIB_PATH)
        for name, argt in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argt
            fn.restype = C.c_char_p if name.endswith("_last_error_string") else C.c_int
        _lib = lib
        return lib


def check(rc: int) -> None:
    """Map an sqg_status to the reference's exception types."""
    if rc == SQG_OK:
        return
    msg = load().sqg_last_error_string().decode(errors="replace")
    if rc == SQG_ERR_INVALID:
        raise ValueError(msg)
    if rc == SQG_ERR_NONFINITE:
        raise NumericalError(msg)
    if rc == SQG_ERR_WORKSPACE or rc == SQG_ERR_STATE:
        raise ConfigurationError(msg)
    raise SimulationError(f"CUDA error in libsqg: {msg}")
