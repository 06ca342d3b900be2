"""ctypes binding of ``libpstm_cuda.so`` (the C ABI in ``include/pstm_cuda.h``).

The structures below mirror the header field for field.  Loading fails loudly
when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpstm_cuda.so")

ABI_VERSION = 5

# pstm_status
OK, ERR_INVALID_ARGUMENT, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_NOT_INITIALIZED, \
    ERR_UNSUPPORTED, ERR_TIMEOUT, ERR_INJECTED = range(8)
STATUS_NAMES = {
    OK: "PSTM_OK", ERR_INVALID_ARGUMENT: "PSTM_ERR_INVALID_ARGUMENT", ERR_CUDA: "PSTM_ERR_CUDA",
    ERR_OUT_OF_MEMORY: "PSTM_ERR_OUT_OF_MEMORY", ERR_NOT_INITIALIZED: "PSTM_ERR_NOT_INITIALIZED",
    ERR_UNSUPPORTED: "PSTM_ERR_UNSUPPORTED", ERR_TIMEOUT: "PSTM_ERR_TIMEOUT",
    ERR_INJECTED: "PSTM_ERR_INJECTED",
}

AMP_F32, AMP_BF16, AMP_F16 = 0, 1, 2
IMAGE_F64, IMAGE_F32 = 0, 1
TT_STRAIGHT, TT_CURVED, TT_VTI, TT_CURVED_VTI = 0, 1, 2, 3
PREC_EXACT, PREC_FAST, PREC_FP32 = 0, 1, 2
# pstm_interp, named as KernelConfig.interpolation_method (aliases of interpolation.py:42-51)
INTERP_BY_NAME = {"linear": 0, "nearest": 1, "cubic": 2, "sinc4": 3, "sinc8": 4, "sinc16": 5,
                  "lanczos3": 6, "lanczos5": 7}
INTERP_ALIASES = {"sinc": "sinc8", "spline": "cubic", "lanczos": "lanczos3"}


def interp_code(name) -> int:
    """pstm_interp code of an interpolation method name or enum (None: linear)."""
    if name is None:
        return 0
    key = str(getattr(name, "value", name)).lower().strip()
    key = INTERP_ALIASES.get(key, key)
    if key not in INTERP_BY_NAME:
        raise ValueError(f"unknown interpolation method {name!r}")
    return INTERP_BY_NAME[key]
STREAM_LEGACY = 1   # cudaStreamLegacy

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


class TracesDesc(ctypes.Structure):
    _fields_ = [
        ("amplitudes", _vp), ("amp_dtype", ctypes.c_int32), ("n_samples", ctypes.c_int32),
        ("n_traces", ctypes.c_int64), ("amp_row_stride", ctypes.c_int64),
        ("source_x", _vp), ("source_y", _vp), ("receiver_x", _vp), ("receiver_y", _vp),
        ("midpoint_x", _vp), ("midpoint_y", _vp), ("weights", _vp),
        ("sample_rate_ms", ctypes.c_double), ("start_time_ms", ctypes.c_double),
    ]


class OutputDesc(ctypes.Structure):
    _fields_ = [
        ("image", _vp), ("image_dtype", ctypes.c_int32), ("fold_is_3d", ctypes.c_int32),
        ("fold", _vp), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nt", ctypes.c_int32),
        ("x_axis", _vp), ("y_axis", _vp), ("x_grid", _vp), ("y_grid", _vp), ("t_axis_ms", _vp),
    ]


class VelocityDesc(ctypes.Structure):
    _fields_ = [("vrms", _vp), ("is_3d", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Params(ctypes.Structure):
    _fields_ = [
        ("max_aperture_m", ctypes.c_double), ("min_aperture_m", ctypes.c_double),
        ("max_dip_degrees", ctypes.c_double), ("taper_fraction", ctypes.c_double),
        ("apply_spreading", ctypes.c_int32), ("apply_obliquity", ctypes.c_int32),
        ("aa_enabled", ctypes.c_int32), ("traveltime", ctypes.c_int32),
        ("aa_dominant_freq", ctypes.c_double), ("grid_dx", ctypes.c_double),
        ("grid_dy", ctypes.c_double), ("curved_v0", ctypes.c_double), ("curved_k", ctypes.c_double),
        ("eta", _vp), ("eta_is_3d", ctypes.c_int32), ("compensated", ctypes.c_int32),
        ("eta_constant", ctypes.c_double), ("precision", ctypes.c_int32), ("interpolation", ctypes.c_int32),
    ]


class BinDesc(ctypes.Structure):
    _fields_ = [("trace_begin", ctypes.c_int64), ("n_traces", ctypes.c_int64), ("image", _vp), ("fold", _vp)]


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("pillars_per_cta", ctypes.c_int32), ("times_per_lane", ctypes.c_int32),
        ("traces_per_chunk", ctypes.c_int32), ("n_candidates", ctypes.c_int32),
        ("best_ms", ctypes.c_float), ("default_ms", ctypes.c_float),
    ]


class SurrogateDomain(ctypes.Structure):
    _fields_ = [
        ("traveltime", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("curved_v0", ctypes.c_double), ("curved_k", ctypes.c_double),
        ("t0_max_s", ctypes.c_double), ("h_max_m", ctypes.c_double),
        ("v_a", ctypes.c_double), ("v_b", ctypes.c_double), ("v_rel", ctypes.c_double),
        ("eta_slope", ctypes.c_double), ("eta_jitter", ctypes.c_double), ("eta_max", ctypes.c_double),
    ]


class Surrogate(ctypes.Structure):
    _fields_ = [
        ("shift", ctypes.c_float * 8), ("scale", ctypes.c_float * 8), ("out_scale", ctypes.c_float),
        ("traveltime", ctypes.c_int32), ("params", _vp),
    ]


class LearnedReport(ctypes.Structure):
    _fields_ = [
        ("probe_max_ms", ctypes.c_float), ("probe_rms_ms", ctypes.c_float),
        ("n_probe_used", ctypes.c_int32), ("used_surrogate", ctypes.c_int32),
    ]


# name -> (restype, argtypes); the exported surface of include/pstm_cuda.h
SIGNATURES = {
    "pstm_cuda_abi_version": (ctypes.c_int32, []),
    "pstm_cuda_create": (ctypes.c_int32, [ctypes.c_int32, ctypes.POINTER(_vp)]),
    "pstm_cuda_destroy": (None, [_vp]),
    "pstm_cuda_migrate_tile_dev": (ctypes.c_int32, [_vp, ctypes.POINTER(TracesDesc), ctypes.POINTER(OutputDesc),
                                                    ctypes.POINTER(VelocityDesc), ctypes.POINTER(Params), _vp]),
    "pstm_cuda_migrate_tile_runs_dev": (ctypes.c_int32, [_vp, ctypes.POINTER(TracesDesc), ctypes.POINTER(ctypes.c_int64),
                                                         ctypes.c_int32, ctypes.POINTER(OutputDesc),
                                                         ctypes.POINTER(VelocityDesc), ctypes.POINTER(Params), _vp]),
    "pstm_cuda_migrate_scatter_dev": (ctypes.c_int32, [_vp, ctypes.POINTER(TracesDesc), ctypes.c_int64,
                                                       ctypes.POINTER(OutputDesc), ctypes.POINTER(VelocityDesc),
                                                       ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_int64), _vp]),
    "pstm_cuda_migrate_tile_host": (ctypes.c_int32, [_vp, ctypes.POINTER(TracesDesc), ctypes.POINTER(OutputDesc),
                                                     ctypes.POINTER(VelocityDesc), ctypes.POINTER(Params)]),
    "pstm_cuda_migrate_tile_noalloc": (ctypes.c_int32, [ctypes.POINTER(TracesDesc), ctypes.POINTER(OutputDesc),
                                                        ctypes.POINTER(VelocityDesc), ctypes.POINTER(Params), _vp]),
    "pstm_cuda_noalloc_status": (ctypes.c_int32, [_vp]),
    "pstm_cuda_migrate_bins_dev": (ctypes.c_int32, [_vp, ctypes.POINTER(TracesDesc), ctypes.POINTER(OutputDesc),
                                                    ctypes.POINTER(VelocityDesc), ctypes.POINTER(Params),
                                                    ctypes.POINTER(BinDesc), ctypes.c_int32, _vp]),
    "pstm_cuda_autotune_bins": (ctypes.c_int32, [_vp, ctypes.POINTER(TracesDesc), ctypes.POINTER(OutputDesc),
                                                 ctypes.POINTER(VelocityDesc), ctypes.POINTER(Params),
                                                 ctypes.POINTER(BinDesc), ctypes.c_int32, ctypes.c_int64,
                                                 ctypes.POINTER(TuneResult)]),
    "pstm_cuda_surrogate_param_count": (ctypes.c_int32, []),
    "pstm_cuda_surrogate_samples": (ctypes.c_int32, [_vp, ctypes.POINTER(SurrogateDomain), ctypes.c_uint64,
                                                     ctypes.c_int64, ctypes.c_int32, _vp, _vp, _vp, _vp]),
    "pstm_cuda_surrogate_gradients": (ctypes.c_int32, [_vp, ctypes.POINTER(Surrogate), _vp, _vp, ctypes.c_int32,
                                                       _vp, _vp, _vp]),
    "pstm_cuda_surrogate_adam": (ctypes.c_int32, [_vp, _vp, _vp, _vp, _vp, ctypes.c_int32, ctypes.c_float, _vp]),
    "pstm_cuda_surrogate_eval": (ctypes.c_int32, [_vp, ctypes.POINTER(Surrogate), _vp, ctypes.c_int32, _vp, _vp]),
    "pstm_cuda_migrate_tile_learned_dev": (ctypes.c_int32, [_vp, ctypes.POINTER(TracesDesc),
                                                            ctypes.POINTER(OutputDesc), ctypes.POINTER(VelocityDesc),
                                                            ctypes.POINTER(Params), ctypes.POINTER(Surrogate),
                                                            ctypes.c_float, ctypes.c_int32,
                                                            ctypes.POINTER(LearnedReport), _vp]),
    "pstm_cuda_interp_rows": (ctypes.c_int32, [_vp, ctypes.c_int32, _vp, ctypes.c_int64, ctypes.c_int32, _vp,
                                               ctypes.c_int32, _vp, _vp, _vp]),
    "pstm_cuda_traces_to_f16": (ctypes.c_int32, [_vp, _vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int64, _vp,
                                                 ctypes.c_int64, _vp, _vp, _vp]),
    "pstm_cuda_measure_sfu_peak": (ctypes.c_int32, [ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    "pstm_cuda_synchronize": (ctypes.c_int32, [_vp]),
    "pstm_cuda_last_error": (ctypes.c_char_p, [_vp]),
}

_lib = None


class PstmCudaError(RuntimeError):
    """A nonzero pstm_status, carrying the code and the library's message."""

    def __init__(self, code: int, message: str):
        self.code = code
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")


def load(path: str | None = None):
    """Load the library (once) and bind every declared entry point."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build it with `python -m pstm_b200.build` (there is no CPU fallback)")
    L = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.pstm_cuda_abi_version() != ABI_VERSION:
        raise RuntimeError("libpstm_cuda.so ABI version mismatch; rebuild")
    if path is None:
        _lib = L
    return L


def check(rc: int, ctx=None, lib=None) -> None:
    if rc != OK:
        L = lib or load()
        msg = L.pstm_cuda_last_error(ctx)
        msg = msg.decode() if msg else ""
        if rc == ERR_INVALID_ARGUMENT:
            raise ValueError(f"PSTM_ERR_INVALID_ARGUMENT: {msg}")
        raise PstmCudaError(rc, msg)
