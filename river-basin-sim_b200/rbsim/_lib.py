"""ctypes binding of librbsim.so (the C ABI declared in include/rbsim.h).

The library is the only compute path: if it is missing, or no CUDA device is
present when a kernel is needed, calls raise -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librbsim.so")

RB_OK = 0
RB_ERR_ARG = -1
RB_ERR_CUDA = -2
RB_ERR_DEVICE = -3
RB_ERR_TIMEOUT = -4
RB_ERR_STEP = -5

RB_DEVERR_NONFINITE = 1
RB_DEVERR_CLOCK = 2
RB_DEVERR_STEPS = 4
RB_DEVERR_TIMEOUT = 8
RB_ARITH_EXACT = 0
RB_ARITH_FAST = 1

EDGES = ("north", "south", "east", "west")  # the ABI's per-edge order
BC_CODE = {"closed": 0, "open": 1, "fixed_stage": 2}

_P = ctypes.c_void_p


class LiFields(ctypes.Structure):
    _fields_ = [
        ("ny", ctypes.c_int32), ("nx", ctypes.c_int32), ("dx", ctypes.c_double),
        ("h", _P * 2), ("qx", _P * 2), ("qy", _P * 2), ("z", _P), ("n", _P),
        ("h_comp", _P), ("rain_field", _P), ("infil", _P), ("bc", ctypes.c_int32 * 4),
        ("d50", _P), ("qs_int_x", _P), ("qs_comp_x", _P), ("qs_int_y", _P), ("qs_comp_y", _P),
        ("chan_w", _P), ("chan_d", _P), ("chan_n", _P),
        ("qx_ch", _P * 2), ("qx_fp", _P * 2), ("qy_ch", _P * 2), ("qy_fp", _P * 2),
    ]  # fmt: skip


class HllcFields(ctypes.Structure):
    _fields_ = [
        ("ny", ctypes.c_int32), ("nx", ctypes.c_int32), ("dx", ctypes.c_double),
        ("h", _P * 2), ("hu", _P * 2), ("hv", _P * 2), ("z", _P), ("n", _P),
        ("h_comp", _P), ("rain_field", _P), ("infil", _P), ("bc", ctypes.c_int32 * 4),
    ]  # fmt: skip


class StepArgs(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double), ("rain", ctypes.c_double), ("rain_scale", ctypes.c_double),
        ("limit", ctypes.c_int32), ("reserved", ctypes.c_int32), ("stage", ctypes.c_double * 4),
    ]  # fmt: skip


class ClockConfig(ctypes.Structure):
    _fields_ = [
        ("alpha", ctypes.c_double), ("dt_max", ctypes.c_double), ("t0", ctypes.c_double), ("sync", _P),
        ("nsync", ctypes.c_int32), ("rain_is_field", ctypes.c_int32), ("rain_rate", ctypes.c_double),
        ("rain_until", ctypes.c_double), ("rain_field_sum", ctypes.c_double), ("limit", ctypes.c_int32),
        ("nsrc", ctypes.c_int32), ("src_cell", _P), ("knot_off", _P), ("knot_t", _P), ("knot_q", _P),
        ("src_comp", _P), ("stage_off", ctypes.c_int32 * 5), ("reserved", ctypes.c_int32), ("stage_t", _P),
        ("stage_v", _P),
    ]  # fmt: skip


class ClockState(ctypes.Structure):
    _fields_ = [
        ("t", ctypes.c_double), ("dt", ctypes.c_double), ("rain_volume", ctypes.c_double),
        ("inflow_volume", ctypes.c_double),
        ("cur", ctypes.c_int32), ("steps", ctypes.c_int32), ("err", ctypes.c_uint32), ("reserved", ctypes.c_int32),
    ]  # fmt: skip


class EnsembleLayout(ctypes.Structure):
    _fields_ = [
        ("ndom", ctypes.c_int32), ("n_li", ctypes.c_int32), ("n_hllc", ctypes.c_int32),
        ("li_variant", ctypes.c_int32), ("hllc_variant", ctypes.c_int32), ("li_grid", ctypes.c_int32),
        ("hllc_grid", ctypes.c_int32), ("reserved", ctypes.c_int32), ("li_tiles", ctypes.c_int64),
        ("hllc_tiles", ctypes.c_int64), ("off_clocks", ctypes.c_int64), ("off_li", ctypes.c_int64),
        ("off_hllc", ctypes.c_int64), ("off_map_li", ctypes.c_int64), ("off_map_hllc", ctypes.c_int64),
        ("off_targets", ctypes.c_int64), ("bytes", ctypes.c_int64),
    ]  # fmt: skip


# name -> (restype, argtypes) for every exported entry point of include/rbsim.h
SIGNATURES = {
    "rb_li_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    "rb_hllc_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    "rb_workspace_init": (ctypes.c_int, [_P, ctypes.c_size_t, _P]),
    "rb_li_step": (ctypes.c_int, [ctypes.POINTER(LiFields), ctypes.c_int32, ctypes.POINTER(StepArgs), _P, _P]),
    "rb_li_compute_dt": (ctypes.c_int, [ctypes.POINTER(LiFields), ctypes.c_int32, ctypes.c_double,
                                        ctypes.c_double, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "rb_hllc_step": (ctypes.c_int, [ctypes.POINTER(HllcFields), ctypes.c_int32, ctypes.POINTER(StepArgs), _P, _P]),
    "rb_hllc_stage": (ctypes.c_int, [ctypes.POINTER(HllcFields), ctypes.c_int32, ctypes.POINTER(StepArgs), _P, _P,
                                     ctypes.c_int32]),
    "rb_hllc_compute_dt": (ctypes.c_int, [ctypes.POINTER(HllcFields), ctypes.c_int32, ctypes.c_double,
                                          ctypes.c_double, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "rb_inject_points": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P, _P]),
    "rb_exner_apply": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _P, _P, _P, _P,
                                      ctypes.c_float, _P, _P, _P, _P, _P]),
    "rb_ledger_loss": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _P, ctypes.POINTER(ctypes.c_double)]),
    "rb_sum_f64": (ctypes.c_int, [_P, ctypes.c_int64, _P, ctypes.c_size_t, _P, ctypes.POINTER(ctypes.c_double)]),
    "rb_read_device_error": (ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_uint32)]),
    "rb_li_clock_start": (ctypes.c_int, [ctypes.POINTER(LiFields), ctypes.c_int32, ctypes.POINTER(ClockConfig),
                                         _P, _P]),
    "rb_hllc_clock_start": (ctypes.c_int, [ctypes.POINTER(HllcFields), ctypes.c_int32,
                                           ctypes.POINTER(ClockConfig), _P, _P]),
    "rb_clock_set_target": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int32, _P]),
    "rb_clock_plan": (ctypes.c_int, [_P, _P]),
    "rb_li_step_clocked": (ctypes.c_int, [ctypes.POINTER(LiFields), _P, _P]),
    "rb_hllc_stage_clocked": (ctypes.c_int, [ctypes.POINTER(HllcFields), ctypes.c_int32, _P, _P]),
    "rb_clock_inflow": (ctypes.c_int, [_P, _P, _P, _P]),
    "rb_li_enqueue_steps": (ctypes.c_int, [ctypes.POINTER(LiFields), ctypes.c_int32, ctypes.c_int32, _P, _P]),
    "rb_hllc_enqueue_steps": (ctypes.c_int, [ctypes.POINTER(HllcFields), ctypes.c_int32, ctypes.c_int32, _P, _P]),
    "rb_clock_read": (ctypes.c_int, [_P, _P, ctypes.POINTER(ClockState)]),
    "rb_ensemble_layout_make": (ctypes.c_int, [ctypes.c_int32, _P, _P, _P, ctypes.c_int32, ctypes.c_int32,
                                               ctypes.POINTER(EnsembleLayout)]),
    "rb_ensemble_init": (ctypes.c_int, [ctypes.POINTER(EnsembleLayout), _P, _P, _P, _P, _P, _P, _P, _P]),
    "rb_ensemble_set_targets": (ctypes.c_int, [ctypes.POINTER(EnsembleLayout), _P, _P, _P, _P]),
    "rb_ensemble_enqueue": (ctypes.c_int, [ctypes.POINTER(EnsembleLayout), _P, ctypes.c_int32, _P]),
    "rb_ensemble_read": (ctypes.c_int, [ctypes.POINTER(EnsembleLayout), _P, _P, _P]),
    "rb_li_set_kernel_variant": (ctypes.c_int, [ctypes.c_int32]),
    "rb_li_kernel_variants": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    "rb_launch_config": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)] * 3),
    "rb_set_arith_mode": (ctypes.c_int, [ctypes.c_int32]),
    "rb_arith_mode": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    "rb_hllc_set_kernel_variant": (ctypes.c_int, [ctypes.c_int32]),
    "rb_hllc_kernel_variants": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    "rb_li_clock_reseed": (ctypes.c_int, [ctypes.POINTER(LiFields), ctypes.c_int32, _P, _P]),
    "rb_hllc_clock_reseed": (ctypes.c_int, [ctypes.POINTER(HllcFields), ctypes.c_int32, _P, _P]),
    "rb_reservoir_withdraw": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_float, _P, _P]),
    "rb_reservoir_deliver": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _P, _P]),
    "rb_hllc_step_noalloc": (ctypes.c_int, [ctypes.POINTER(HllcFields), ctypes.c_int32, ctypes.POINTER(StepArgs),
                                            _P, _P]),
    "rb_hllc_noalloc_read_error": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint32), _P]),
    "rb_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "rb_version": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)] * 3),
}  # fmt: skip

_LIB: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """Load librbsim.so once; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python river-basin-sim_b200/build.py` "
                "(there is no CPU fallback for the solver path)"
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


class DeviceError(RuntimeError):
    """A kernel raised a device-side error bit (e.g. a non-finite depth)."""


def launch_config() -> tuple[int, int, int]:
    """(LI kernel variant, HLLC kernel variant, arithmetic mode) the library launches with now."""
    li, hl, mode = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
    check(lib().rb_launch_config(ctypes.byref(li), ctypes.byref(hl), ctypes.byref(mode)))
    return li.value, hl.value, mode.value


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    lib().rb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    """Map a non-zero status to the exception class the reference raises."""
    if rc == RB_OK:
        return
    msg = last_error()
    if rc == RB_ERR_ARG:
        raise ValueError(msg)
    if rc == RB_ERR_STEP:
        raise RuntimeError(msg)
    if rc == RB_ERR_DEVICE:
        raise DeviceError(msg)
    raise RuntimeError(f"librbsim error {rc}: {msg}")
