"""ctypes binding of libpsdm_rtm.so (the C ABI declared in include/psdm_rtm.h).

The library is the product: there is no CPU fallback.  Loading fails loudly
if the shared library has not been built (python -m psdm_b200.build).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libpsdm_rtm.so")

PSDM_OK, PSDM_ERR_ARG, PSDM_ERR_CUDA, PSDM_ERR_NOMEM, PSDM_ERR_STATE = 0, -1, -2, -3, -4
PREC_FP32, PREC_FP16, PREC_BF16 = 0, 1, 2

# Every symbol include/psdm_rtm.h declares (checked by tests/test_abi.py).
EXPORTS = [
    "psdm_last_error", "psdm_engine_create", "psdm_engine_destroy", "psdm_engine_device_bytes",
    "psdm_engine_trim", "psdm_engine_set_stream", "psdm_engine_set_profiling", "psdm_engine_stats",
    "psdm_engine_reset_stats", "psdm_dynamic_window_solver_forward_ram", "psdm_dynamic_window_solver_backward_ram",
    "psdm_rtm_shot", "psdm_rtm_shot_device", "psdm_model_shot", "psdm_fd_coef", "psdm_pml_coeffs", "psdm_ricker_mcs",
    "psdm_dynamic_window", "psdm_taper_pad_trace", "psdm_optimization_dt", "psdm_normalize_psdm",
    "psdm_model_shot_noalloc", "psdm_plan_memory", "psdm_engine_autotune", "psdm_rtm_shot_fp64", "psdm_rtm_batch", "psdm_rtm_batch_device", "psdm_engine_batch_slots",
    "psdm_engine_check_wait_timeout", "psdm_engine_dt_quotients", "psdm_trace_windows", "psdm_condition_traces", "psdm_condition_traces_device",
    "psdm_su_write_image", "psdm_su_read_shot", "psdm_su_read_header_i32", "psdm_engine_set_checkpointing", "psdm_engine_set_pass_launch", "psdm_engine_set_steps_per_launch", "psdm_engine_set_reconstruction",
    "psdm_freq_filter", "psdm_freq_filter_device", "psdm_butterworth_response",
    "psdm_nav_read", "psdm_channel_positions", "psdm_geometry_mcs", "psdm_linear_2d", "psdm_batmodel_from_velocity",
    "psdm_nav_read_was", "psdm_nav_read_obs", "psdm_geometry_was", "psdm_bathymetry_nav", "psdm_relocate_obs",
]


class Params(C.Structure):
    _fields_ = [("dPML", C.c_int32), ("fs", C.c_int32), ("strategy", C.c_int32), ("precision", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("launches", C.c_int64), ("fwd_steps", C.c_int64), ("bwd_steps", C.c_int64), ("shots", C.c_int64),
                ("fwd_ms", C.c_double), ("bwd_ms", C.c_double)]


class Plan(C.Structure):
    """psdm_plan (include/psdm_rtm.h)."""
    _fields_ = [("steps_per_launch", C.c_int32), ("slots", C.c_int32), ("checkpoint_interval", C.c_int32),
                ("fits", C.c_int32), ("bytes_per_slot", C.c_int64), ("budget_bytes", C.c_int64),
                ("probe_us", C.c_float * 2)]


class Shot(C.Structure):
    """struct psdm_shot (one shot of a batched call)."""
    _fields_ = [("NumRec", C.c_int32), ("nxSou", C.c_int32), ("nySou", C.c_int32), ("nxRec", C.c_void_p),
                ("nyRec", C.c_void_p), ("nx_w", C.c_int32), ("nt_prop2", C.c_int32), ("nt_taper", C.c_int32),
                ("Vp_w", C.c_void_p), ("Data_target", C.c_void_p), ("PSDM_w", C.c_void_p)]


class Conditioning(C.Structure):
    """struct psdm_conditioning."""
    _fields_ = [("cut_multiple", C.c_int32), ("cut_sf", C.c_int32), ("taper_option", C.c_int32),
                ("T_taper", C.c_float), ("T_zeros", C.c_float)]


class PsdmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"psdm error {code}: {msg}")
        self.code = code


_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I, _F, _P = C.c_int32, C.c_float, C.c_void_p


def lib():
    """Load libpsdm_rtm.so (raises if it is missing: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m psdm_b200.build` "
                          "(the RTM engine has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.psdm_last_error.restype = C.c_char_p
    L.psdm_engine_create.argtypes = [_I, C.POINTER(_P)]
    L.psdm_engine_destroy.argtypes = [_P]
    L.psdm_engine_device_bytes.argtypes = [_P]
    L.psdm_engine_device_bytes.restype = C.c_int64
    L.psdm_engine_trim.argtypes = [_P]
    L.psdm_engine_set_stream.argtypes = [_P, _P]
    L.psdm_engine_set_profiling.argtypes = [_P, _I]
    L.psdm_engine_stats.argtypes = [_P, C.POINTER(Stats)]
    L.psdm_engine_reset_stats.argtypes = [_P]
    PP = C.POINTER(Params)
    L.psdm_dynamic_window_solver_forward_ram.argtypes = [
        _P, PP, _I, _i32p, _i32p, _i32p, _i32p, _f32p, _F, _F, _I, _I, _I, _f32p, _F, _I, _I, _I, _P, _P]
    L.psdm_dynamic_window_solver_backward_ram.argtypes = [
        _P, PP, _I, _i32p, _i32p, _i32p, _i32p, _f32p, _F, _F, _I, _I, _I, _f32p, _F, _I, _I, _I, _P, _f32p]
    L.psdm_rtm_shot.argtypes = [
        _P, PP, _I, _I, _I, _i32p, _i32p, _f32p, _f32p, _F, _F, _I, _I, _I, _f32p, _F, _I, _I, _I, _I, _I, _I, _I,
        _f32p]
    L.psdm_rtm_shot_device.argtypes = [
        _P, PP, _I, _I, _I, _i32p, _i32p, _P, _P, _F, _F, _I, _I, _I, _P, _F, _I, _I, _I, _I, _I, _I, _I, _P]
    L.psdm_model_shot.argtypes = [_P, PP, _I, _I, _I, _i32p, _i32p, _f32p, _F, _F, _I, _I, _I, _f32p, _F, _I, _f32p]
    L.psdm_rtm_shot_fp64.argtypes = [_I, PP, _I, _I, _I, _i32p, _i32p, _f32p, _f32p, _F, _F, _I, _I, _I, _f32p, _F,
                                     _I, _I, _I, _I, _I, _I, _f64p, _P]
    L.psdm_plan_memory.argtypes = [PP, _I, _I, _I, _I, _I, _I, C.c_int64, _I, C.POINTER(Plan)]
    L.psdm_engine_autotune.argtypes = [_P, PP, _I, _I, _I, _I, _I, _I, C.c_int64, _I, _I, C.POINTER(Plan)]
    L.psdm_model_shot_noalloc.argtypes = [PP, _I, _I, _I, _i32p, _i32p, _P, _F, _F, _I, _I, _I, _P, _F, _I, _P, _P]
    L.psdm_rtm_batch.argtypes = [_P, PP, _I, C.POINTER(Shot), _f32p, _F, _F, _I, _I, _F, _I, _I, _I, _I, _I]
    L.psdm_rtm_batch_device.argtypes = [_P, PP, _I, C.POINTER(Shot), _P, _F, _F, _I, _I, _F, _I, _I, _I, _I, _I]
    L.psdm_engine_batch_slots.argtypes = [_P]
    L.psdm_engine_batch_slots.restype = _I
    L.psdm_engine_check_wait_timeout.argtypes = [_P]
    L.psdm_engine_dt_quotients.argtypes = [_P, _F, _f32p, _I, _f32p]
    L.psdm_engine_set_checkpointing.argtypes = [_P, _I]
    L.psdm_engine_set_pass_launch.argtypes = [_P, _I]
    L.psdm_engine_set_steps_per_launch.argtypes = [_P, _I]
    L.psdm_engine_set_reconstruction.argtypes = [_P, _I]
    L.psdm_freq_filter.argtypes = [_P, _f32p, _I, _F, _I, _I, _F, _F]
    L.psdm_freq_filter_device.argtypes = [_P, _P, _I, _F, _I, _I, _F, _F]
    L.psdm_su_write_image.argtypes = [C.c_char_p, _I, _I, _F, _F, _I, _f32p, _I]
    L.psdm_su_read_shot.argtypes = [C.c_char_p, _I, _I, _I, _I, _I, _f32p, _P]
    L.psdm_su_read_header_i32.argtypes = [C.c_char_p, _I, _I, _I, _I, _i32p]
    L.psdm_butterworth_response.argtypes = [_I, _F, _I, _F, _F, _f32p]
    L.psdm_nav_read.argtypes = [C.c_char_p, _I, _I, _F, _I, _I, _I, _P, _P, _P, _i32p]
    L.psdm_channel_positions.argtypes = [_F, _I, _I, _I, _F, _P, _F, _F, _f32p]
    L.psdm_geometry_mcs.argtypes = [_F, _I, _f32p, _F, _F, _F, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _i32p,
                                    _i32p]
    L.psdm_linear_2d.argtypes = [_I, _I, _F, _f32p, _I, _I, _F, _f32p]
    L.psdm_batmodel_from_velocity.argtypes = [_I, _I, _F, _F, _f32p, _f32p]
    L.psdm_nav_read_was.argtypes = [C.c_char_p, _I, _I, _F, _F, _F, _I, _I, _i32p, _f32p, _f32p, _i32p, _f32p]
    L.psdm_nav_read_obs.argtypes = [C.c_char_p, _I, _F, _i32p, _f32p, _f32p, _i32p, _i32p]
    L.psdm_geometry_was.argtypes = [_I, _I, _I, _f32p, _F, _F, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _i32p,
                                    _i32p]
    L.psdm_bathymetry_nav.argtypes = [_I, _f32p, _f32p, _F, _I, _F, _f32p]
    L.psdm_relocate_obs.argtypes = [_I, _i32p, _f32p, _I, _F, _f32p, _i32p]
    CP = C.POINTER(Conditioning)
    L.psdm_trace_windows.argtypes = [CP, _I, _I, _I, _i32p, _i32p, _f32p, _F, _F, _I, _i32p, _i32p, _i32p]
    L.psdm_trace_windows.restype = None
    L.psdm_condition_traces.argtypes = [_P, CP, _I, _f32p, _I, _F, _F, _i32p, _i32p, _i32p, _f32p]
    L.psdm_condition_traces_device.argtypes = [_P, CP, _I, _P, _I, _F, _F, _i32p, _i32p, _i32p, _P]
    L.psdm_fd_coef.argtypes = [_I, _I, _f32p]
    L.psdm_fd_coef.restype = None
    L.psdm_pml_coeffs.argtypes = [_I, _I, _F, _F, _I, _f32p, _f32p, _P]
    L.psdm_pml_coeffs.restype = None
    L.psdm_ricker_mcs.argtypes = [_I, _F, _F, _F, _f32p]
    L.psdm_ricker_mcs.restype = None
    L.psdm_dynamic_window.argtypes = [_I, _I, _i32p, _F, _I, _F, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]
    L.psdm_dynamic_window.restype = None
    L.psdm_taper_pad_trace.argtypes = [_f32p, _I, _I, _I, _I]
    L.psdm_taper_pad_trace.restype = None
    L.psdm_optimization_dt.argtypes = [_F, _F, _F, _I, C.POINTER(_F), C.POINTER(_I), C.POINTER(_I)]
    L.psdm_optimization_dt.restype = None
    L.psdm_normalize_psdm.argtypes = [_I, _I, _f32p, _f32p, _f32p]
    L.psdm_normalize_psdm.restype = None
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != PSDM_OK:
        raise PsdmError(rc, lib().psdm_last_error().decode(errors="replace"))
