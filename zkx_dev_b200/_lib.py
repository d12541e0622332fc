"""ctypes binding of libzkx_rd.so (include/zkx_rd.h).

The library is the only compute path: if it is missing, importing an operator raises
immediately instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzkx_rd.so")

SUCCESS = 0
INVALID_ARGUMENT = 1001
INVALID_SHAPE = 1002
UNSUPPORTED_OPERATION = 1004
OUT_OF_MEMORY = 2003
RESOURCE_FAILED = 3002

WINDOW_NONE, WINDOW_HANN, WINDOW_HAMMING, WINDOW_EXPLICIT_FP32, WINDOW_EXPLICIT_FP64 = range(5)
CFAR_ACCURATE, CFAR_COMPAT = 0, 1
PRECISION_FP32, PRECISION_TC_F16, PRECISION_TC_BF16 = 0, 1, 2
PAD_ODD, PAD_EVEN, PAD_CONSTANT, PAD_NONE = range(4)
FIR_AUTO, FIR_DIRECT, FIR_FFT = range(3)
PAD_ROUND_F32, PAD_ROUND_F16, PAD_ROUND_I8, PAD_ROUND_I16, PAD_ROUND_I32 = range(5)

# Every symbol the header declares, with its ctypes signature.
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double


class ResampleLayout(ctypes.Structure):
    _fields_ = [("up", _I), ("down", _I), ("identity", _I), ("output_samples", _I),
                ("coefficient_count", _I), ("half_length", _I), ("prefix_zeros", _I),
                ("output_start", _I)]


class WorkItem(ctypes.Structure):
    """zkx_rd_work_item"""
    _fields_ = [("plan", ctypes.c_void_p), ("x", ctypes.c_void_p), ("power", ctypes.c_void_p),
                ("threshold", ctypes.c_void_p), ("detections", ctypes.c_void_p)]


class RdDesc(ctypes.Structure):
    _fields_ = [("num_pulses", _I), ("samples_per_pulse", _I), ("range_nfft", _I),
                ("doppler_nfft", _I), ("replica_length", _I), ("normalize", _I),
                ("range_window", _I), ("doppler_window", _I), ("guard_cells", _I * 2),
                ("reference_cells", _I * 2), ("pfa", _D), ("cfar_mode", _I), ("precision", _I)]


class RdTuning(ctypes.Structure):
    _fields_ = [("compression_variant", _I), ("doppler_columns", _I), ("cfar_tile", _I),
                ("compression_radix", _I), ("compression_ctas_per_sm", _I), ("cfar_ctas_per_sm", _I)]


class ServerDesc(ctypes.Structure):
    _fields_ = [("normalize", _I), ("range_window", _I), ("doppler_window", _I),
                ("guard_cells", _I * 2), ("reference_cells", _I * 2), ("pfa", _D),
                ("cfar_mode", _I), ("streams", _I), ("max_inflight", _I), ("max_batch", _I),
                ("hbm_fraction", _D), ("budget_bytes", ctypes.c_size_t), ("max_pending", _I)]


class Request(ctypes.Structure):
    _fields_ = [("num_pulses", _I), ("samples_per_pulse", _I), ("waveform_id", ctypes.c_uint64),
                ("replica", _P), ("replica_length", _I), ("x", _P), ("detections", _P),
                ("threshold", _P), ("power", _P), ("rd", _P)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("mean_batch", _D),
                ("p50_us", _D), ("p99_us", _D), ("max_us", _D), ("mean_us", _D),
                ("cpis_per_s", _D), ("budget_bytes", ctypes.c_size_t),
                ("peak_bytes", ctypes.c_size_t), ("plan_bytes", ctypes.c_size_t), ("plans", _I),
                ("refused", ctypes.c_uint64)]


class SynthTarget(ctypes.Structure):
    _fields_ = [("delay", _I), ("doppler_bin", _I), ("amplitude", _D), ("phase", _D)]


SIGNATURES = {
    "zkx_last_error": (ctypes.c_char_p, []),
    "zkx_version": (ctypes.c_char_p, []),
    "zkx_kernel_status": (_I, [_I, ctypes.POINTER(_I)]),
    "zkx_selftest_wait_timeout": (_I, [ctypes.c_longlong, _P]),
    "zkx_pulse_compression_c64": (_I, [_P, _I, _I, _P, _I, _I, _I, _I, _P, _P, _P]),
    "zkx_pulse_compression_c64_noalloc": (_I, [_P, _I, _I, _P, _I, _I, _I, _I, _P, _P, _P]),
    "zkx_replica_spectrum_c64": (_I, [_P, _I, _I, _I, _I, _P, _P, _P]),
    "zkx_pulse_compression_spectrum_c64": (_I, [_P, _I, _I, _I, _P, _P, _P]),
    "zkx_pulse_compression_spectrum_ex_c64": (_I, [_P, _I, _I, _I, _P, _I, _P, _P]),
    "zkx_pulse_doppler_c64": (_I, [_P, _I, _I, _I, _I, _P, _P, _P, _P]),
    "zkx_fft_c2c_c64": (_I, [_P, _I, _I, _I, _P, _P]),
    "zkx_cfar_alpha": (_I, [_D, _I, ctypes.POINTER(_D)]),
    "zkx_ambgfun_c64": (_I, [_P, _I, _I, _P, _I, _I, _I, _D, _D, _P, _P]),
    "zkx_lfm_waveform_c64": (_I, [_I, _D, _D, _P, _P]),
    "zkx_task1_echo_c64": (_I, [_P, _I, _I, _I, _I, _D, ctypes.c_uint32, _D, _D, _D, _D, _P, _P, _P, _P]),
    "zkx_synth_cpi_c64": (_I, [_I, _I, _I, _D, ctypes.POINTER(SynthTarget), _I, ctypes.c_uint64, _D, _P, _P]),
    "zkx_ambgfun_shape": (_I, [_I, _I, _I, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_I),
                               ctypes.POINTER(_I)]),
    "zkx_cfar_reference_count": (_I, [_I, _I, _I, _I, _I]),
    "zkx_ca_cfar_f32": (_I, [_P, _I, _I, _I, _I, _I, _I, _I, _D, _I, _P, _P, _P]),
    "zkx_fir_f32": (_I, [_P, _I, _P, _I, _I, _P, _P, _P, _P]),
    "zkx_fir_ex_f32": (_I, [_P, _I, _P, _I, _I, _P, _P, _P, _I, _P]),
    "zkx_firfilter2_f32": (_I, [_P, _I, _P, _I, _I, _I, _I, _I, _I, _P, _P]),
    "zkx_firfilter2_ex_f32": (_I, [_P, _I, _P, _I, _I, _I, _I, _I, _I, _P, _I, _P]),
    "zkx_hilbert_f32": (_I, [_P, _I, _I, _I, _P, _P]),
    "zkx_upfirdn_length": (ctypes.c_longlong, [_I, _I, _I, _I]),
    "zkx_upfirdn_f32": (_I, [_P, _I, _P, _I, _I, _I, _I, _P, _P]),
    "zkx_resample_poly_layout": (_I, [_I, _I, _I, _I, _I, ctypes.POINTER(ResampleLayout)]),
    "zkx_resample_poly_design": (_I, [ctypes.POINTER(ResampleLayout), _D, _P]),
    "zkx_resample_poly_f32": (_I, [_P, _I, _I, ctypes.POINTER(ResampleLayout), _P, _P, _P]),
    "zkx_convert_to_f32": (_I, [_P, _I, ctypes.c_longlong, _P, _P]),
    "zkx_widen_f32_to_f64": (_I, [_P, ctypes.c_longlong, _P, _P]),
    "zkx_cfar_detect_int": (_I, [_P, _I, _P, ctypes.c_longlong, _P, _P]),
    "zkx_transpose_f32": (_I, [_P, _I, _I, _P, _P]),
    "zkx_transpose_c64": (_I, [_P, _I, _I, _P, _P]),
    "zkx_resample_poly_design_window": (_I, [ctypes.POINTER(ResampleLayout), _P, _P]),
    "zkx_rd_plan_create": (_I, [ctypes.POINTER(RdDesc), _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "zkx_rd_plan_destroy": (_I, [_P]),
    "zkx_rd_plan_shape": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "zkx_rd_execute": (_I, [_P, _P, _P, _P, _P, _P, _P, _P]),
    "zkx_rd_execute_batch": (_I, [_P, _P, _I, _P, _P, _P, _P, _P, _P]),
    "zkx_rd_graph_create": (_I, [_P, _P, _I, _P, _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "zkx_rd_graph_launch": (_I, [_P, _P]),
    "zkx_rd_graph_destroy": (_I, [_P]),
    "zkx_rd_worklist_create": (_I, [ctypes.POINTER(WorkItem), _I, ctypes.POINTER(_P)]),
    "zkx_rd_worklist_launch": (_I, [_P, _P]),
    "zkx_rd_worklist_info": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_longlong)]),
    "zkx_rd_worklist_destroy": (_I, [_P]),
    "zkx_rd_plan_autotune": (_I, [_P, _P, _I, _P, ctypes.POINTER(RdTuning)]),
    "zkx_rd_plan_get_tuning": (_I, [_P, ctypes.POINTER(RdTuning)]),
    "zkx_rd_plan_set_tuning": (_I, [_P, ctypes.POINTER(RdTuning)]),
    "zkx_rd_server_create": (_I, [ctypes.POINTER(ServerDesc), ctypes.POINTER(_P)]),
    "zkx_rd_server_destroy": (_I, [_P]),
    "zkx_rd_submit": (_I, [_P, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]),
    "zkx_rd_poll": (_I, [_P, ctypes.c_uint64, _I, ctypes.POINTER(_I)]),
    "zkx_rd_server_stats_get": (_I, [_P, ctypes.POINTER(ServerStats)]),
    "zkx_rd_server_stats_reset": (_I, [_P]),
}

_lib: Optional[ctypes.CDLL] = None


class ZkxError(RuntimeError):
    """A failing libzkx_rd call; `code` is the reference's ErrorCode number."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class ZkxValueError(ZkxError, ValueError):
    """Invalid shape or argument (the reference throws std::invalid_argument)."""


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m zkx_dev_b200.build`")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(rc: int) -> None:
    if rc != SUCCESS:
        msg = lib().zkx_last_error().decode(errors="replace")
        if rc in (INVALID_ARGUMENT, INVALID_SHAPE):
            raise ZkxValueError(rc, msg)
        raise ZkxError(rc, msg)


def stream_handle(stream=None) -> Optional[int]:
    """Raw cudaStream_t of a torch stream (default: torch's current stream)."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


def kernel_status(clear: bool = True) -> int:
    """Synchronise the device and return (and by default clear) the kernel error word."""
    code = ctypes.c_int()
    check(lib().zkx_kernel_status(int(clear), ctypes.byref(code)))
    return code.value
