"""ctypes binding of ``libftdx.so`` (the C ABI declared in ``include/ftdx.h``).

The library is loaded from the package directory.  There is no fallback: if
the shared library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libftdx.so")

FTDX_OK = 0
STATUS_NAMES = {
    0: "FTDX_OK", 1: "FTDX_ERR_INVALID_ARG", 2: "FTDX_ERR_UNSUPPORTED", 3: "FTDX_ERR_CUDA",
    4: "FTDX_ERR_NO_DEVICE", 5: "FTDX_ERR_ALLOC", 6: "FTDX_ERR_CAPACITY", 7: "FTDX_ERR_TIMEOUT",
    8: "FTDX_ERR_CACHE",
}

# enum values (include/ftdx.h)
IN_FP16, IN_INT4, IN_FP32 = 0, 1, 2
COMPUTE_FP8, COMPUTE_FP6, COMPUTE_FP4, COMPUTE_FP8_SPLIT, COMPUTE_FP4_SPLIT = 0, 1, 2, 3, 4
OUT_FP16, OUT_FP32 = 0, 1
FORMAT_PACKED_TRIANGLE = 0
LAYOUT_TIME_ANT_CHAN_POL, LAYOUT_CHAN_POL_ANT_TIME = 0, 1


class FtdxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class ChannelDesc(ctypes.Structure):
    _fields_ = [("A", ctypes.c_void_p), ("C", ctypes.c_void_p), ("n_inputs", ctypes.c_int),
                ("K", ctypes.c_int), ("lda", ctypes.c_int64), ("active", ctypes.c_void_p)]


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("verbosity", ctypes.c_int),
                ("tune_cache", ctypes.c_char_p), ("reserved", ctypes.c_int * 8)]


class FtdDesc(ctypes.Structure):
    _fields_ = [("n_ant", ctypes.c_int), ("n_chan", ctypes.c_int), ("n_pol", ctypes.c_int),
                ("n_time", ctypes.c_int), ("n_time_inner", ctypes.c_int), ("layout", ctypes.c_int),
                ("pol_sum", ctypes.c_int), ("reserved", ctypes.c_int * 4)]


class ImagingConfig(ctypes.Structure):
    _fields_ = [("n_ant", ctypes.c_int), ("n_chan", ctypes.c_int), ("n_pol", ctypes.c_int),
                ("n_grid", ctypes.c_int), ("n_beam", ctypes.c_int), ("chan_tile", ctypes.c_int),
                ("cell_size_rad", ctypes.c_float), ("baseline_uv_m", ctypes.c_void_p),
                ("freq_hz", ctypes.c_void_p), ("taper", ctypes.c_void_p),
                ("beam_pixels", ctypes.c_void_p), ("output_stage", ctypes.c_int),
                ("reserved", ctypes.c_int * 7)]


class PipelineConfig(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("K", ctypes.c_int), ("batch", ctypes.c_int),
                ("output", ctypes.c_int), ("ftd", ctypes.POINTER(FtdDesc)),
                ("host_threads", ctypes.c_int), ("reserved", ctypes.c_int * 7)]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float

# name -> (restype, argtypes); every function include/ftdx.h declares.
PROTOTYPES = {
    "ftdx_version": (_i, []),
    "ftdx_status_string": (ctypes.c_char_p, [_i]),
    "ftdx_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(Config)]),
    "ftdx_destroy": (_i, [_vp]),
    "ftdx_last_error": (ctypes.c_char_p, [_vp]),
    "ftdx_herk": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _f, _f, _vp, _i]),
    "ftdx_init_herk": (_i, [_vp, _i, _i, _i, _vp]),
    "ftdx_herk_adjoint": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _vp]),
    "ftdx_gain_gradient": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp]),
    "ftdx_herk_kahan": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp]),
    "ftdx_herk_batched_v": (_i, [_vp, ctypes.c_void_p, _i, _i, _f, _f, _vp, _i]),
    "ftdx_herk_ftd": (_i, [_vp, _vp, _vp, ctypes.POINTER(FtdDesc), _i, _f, _f, _vp]),
    "ftdx_strided_batch_gemm": (ctypes.c_longlong, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _i,
                                                    _i, _vp]),
    "ftdx_set_strided_mode": (_i, [_vp, _i]),
    "ftdx_peak_probe": (_i, [_vp, _i, _i, _i, ctypes.POINTER(ctypes.c_double)]),
    "ftdx_wait_selftest": (_i, [_vp, _i, _vp]),
    "ftdx_xengine": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _vp]),
    "ftdx_image_beams": (_i, [_vp, ctypes.POINTER(ImagingConfig), _vp, _vp, _vp, _vp]),
    "ftdx_pipeline_create": (_i, [_vp, ctypes.POINTER(PipelineConfig), ctypes.POINTER(_vp)]),
    "ftdx_pipeline_correlate": (_i, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _i]),
    "ftdx_pipeline_destroy": (_i, [_vp]),
    "ftdx_pipeline_sizes": (_i, [_vp, ctypes.POINTER(ctypes.c_size_t),
                                 ctypes.POINTER(ctypes.c_size_t)]),
    "ftdx_end_herk": (_i, [_vp]),
    "ftdx_device_status": (_i, [_vp, _vp, ctypes.POINTER(ctypes.c_uint32)]),
    "ftdx_set_profiling": (_i, [_vp, _i]),
    "ftdx_set_tune_cache": (_i, [_vp, ctypes.c_char_p]),
    "ftdx_tune": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, ctypes.POINTER(_i),
                       ctypes.POINTER(_i), ctypes.POINTER(_f)]),
    "ftdx_lookup_tuned": (_i, [_vp, _i, _i, _i, _i, _i, ctypes.POINTER(_i), ctypes.POINTER(_i),
                               ctypes.POINTER(_f)]),
    "ftdx_lookup_tuned_compute": (_i, [_vp, _i, _i, _i, _i, _i, _i, ctypes.POINTER(_i),
                                       ctypes.POINTER(_i), ctypes.POINTER(_f)]),
    "ftdx_set_graph_mode": (_i, [_vp, _i]),
    "ftdx_graph_count": (_i, [_vp]),
    "ftdx_set_strategy": (_i, [_vp, _i, _i]),
    "ftdx_set_split_k": (_i, [_vp, _i]),
    "ftdx_tuned_split_k": (_i, [_vp, _i, _i, _i, _i, _i]),
    "ftdx_herk_static": (_i, [_vp, _vp, _i, _i, _i, _vp, ctypes.POINTER(ctypes.c_uint32),
                              ctypes.POINTER(ctypes.c_size_t)]),
    "ftdx_profile_read": (_i, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i)]),
}

_lib = None


def load():
    """Load libftdx.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FtdxError(4, f"{LIB_PATH} is missing; build it with `python -m ftd_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(h, status: int, what: str):
    if status != FTDX_OK:
        msg = load().ftdx_last_error(h) if h else b""
        raise FtdxError(status, f"{what}: {(msg or b'').decode(errors='replace')}")
