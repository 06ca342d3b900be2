"""ctypes wrapper of the FP64 CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs, always as the checker or the timed CPU baseline, never as
the product path.  The restated algorithm and its reference citations are in
``oracle/pstm_oracle.c``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libpstm_oracle.so")
_lib = None

TT_STRAIGHT, TT_CURVED, TT_VTI, TT_CURVED_VTI = 0, 1, 2, 3
KIND_BY_NAME = {
    "straight_ray": TT_STRAIGHT, "curved_ray": TT_CURVED,
    "anisotropic_vti": TT_VTI, "curved_vti": TT_CURVED_VTI,
}

_dp = ctypes.POINTER(ctypes.c_double)


class _Args(ctypes.Structure):
    _fields_ = [
        ("n_traces", ctypes.c_int64), ("n_samples", ctypes.c_int32),
        ("amp_is_f64", ctypes.c_int32), ("amplitudes", ctypes.c_void_p),
        ("source_x", _dp), ("source_y", _dp), ("receiver_x", _dp), ("receiver_y", _dp),
        ("midpoint_x", _dp), ("midpoint_y", _dp), ("weights", _dp),
        ("sample_rate_ms", ctypes.c_double), ("start_time_ms", ctypes.c_double),
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nt", ctypes.c_int32),
        ("x_axis", _dp), ("y_axis", _dp), ("x_grid", _dp), ("y_grid", _dp),
        ("t_axis_ms", _dp), ("image", _dp), ("fold", ctypes.POINTER(ctypes.c_int32)),
        ("fold_is_3d", ctypes.c_int32),
        ("vrms", _dp), ("vel_is_3d", ctypes.c_int32),
        ("max_aperture_m", ctypes.c_double), ("min_aperture_m", ctypes.c_double),
        ("max_dip_degrees", ctypes.c_double), ("taper_fraction", ctypes.c_double),
        ("apply_spreading", ctypes.c_int32), ("apply_obliquity", ctypes.c_int32),
        ("aa_enabled", ctypes.c_int32), ("aa_dominant_freq", ctypes.c_double),
        ("grid_dx", ctypes.c_double), ("grid_dy", ctypes.c_double),
        ("traveltime_kind", ctypes.c_int32), ("curved_v0", ctypes.c_double),
        ("curved_k", ctypes.c_double), ("eta", _dp), ("eta_is_3d", ctypes.c_int32),
        ("eta_constant", ctypes.c_double),
        ("pillar_begin", ctypes.c_int64), ("pillar_end", ctypes.c_int64),
        ("n_threads", ctypes.c_int32), ("interp_method", ctypes.c_int32),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (plain gcc) if it is missing or stale."""
    src = os.path.join(_HERE, "pstm_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.pstm_oracle_migrate.argtypes = [ctypes.POINTER(_Args)]
        L.pstm_oracle_migrate.restype = ctypes.c_int
        L.pstm_oracle_traveltime.argtypes = [ctypes.c_int32, ctypes.c_int64, _dp,
                                             ctypes.c_double, ctypes.c_double, _dp]
        L.pstm_oracle_traveltime.restype = None
        L.pstm_oracle_linear_interp.argtypes = [_dp, ctypes.c_int32, ctypes.c_double]
        L.pstm_oracle_linear_interp.restype = ctypes.c_double
        L.pstm_oracle_interp.argtypes = [_dp, ctypes.c_int32, ctypes.c_double, ctypes.c_int32]
        L.pstm_oracle_interp.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def migrate(traces, output, velocity, config, kind=None, pillars=None, n_threads=0,
            image=None, fold=None):
    """Run the FP64 oracle on reference-shaped carriers.

    ``kind`` defaults to ``config.kernel_type``.  ``pillars=(begin, end)``
    restricts the work to a flattened (ix*ny+iy) pillar range.  ``image`` and
    ``fold`` default to ``output.image``/``output.fold`` and are accumulated
    in place (``+=``) like the reference.
    """
    L = lib()
    amps = np.asarray(traces.amplitudes)
    if amps.dtype == np.float64:
        amps = np.ascontiguousarray(amps)
        amp_is_f64 = 1
    else:
        amps = np.ascontiguousarray(amps, dtype=np.float32)
        amp_is_f64 = 0
    keep = []

    def k(a):
        keep.append(a)
        return a

    sx, sy = k(_f64(traces.source_x)), k(_f64(traces.source_y))
    rx, ry = k(_f64(traces.receiver_x)), k(_f64(traces.receiver_y))
    mx, my = k(_f64(traces.midpoint_x)), k(_f64(traces.midpoint_y))
    w = k(_f64(traces.weights)) if getattr(traces, "weights", None) is not None else None
    img = output.image if image is None else image
    fld = output.fold if fold is None else fold
    assert img.dtype == np.float64 and img.flags["C_CONTIGUOUS"]
    nx, ny, nt = len(output.x_axis), len(output.y_axis), len(output.t_axis_ms)
    xg = getattr(output, "x_grid", None)
    yg = getattr(output, "y_grid", None)
    xg = k(_f64(np.reshape(xg, -1))) if xg is not None else None
    yg = k(_f64(np.reshape(yg, -1))) if yg is not None else None
    v = k(_f64(velocity.vrms))
    vel3d = 0 if velocity.is_1d else 1
    if vel3d:
        assert v.shape == (nx, ny, nt), v.shape
    else:
        assert v.shape == (nt,), v.shape
    eta = getattr(config, "vti_eta_array", None)
    eta_is_3d = 0
    if eta is not None:
        eta = k(_f64(eta))
        eta_is_3d = 0 if eta.ndim == 1 else 1
    if kind is None:
        kind = KIND_BY_NAME.get(getattr(config, "kernel_type", "straight_ray"), TT_STRAIGHT)
    elif isinstance(kind, str):
        kind = KIND_BY_NAME[kind]
    fold_ptr = None
    fold_is_3d = 0
    if fld is not None:
        assert fld.dtype == np.int32 and fld.flags["C_CONTIGUOUS"]
        fold_is_3d = 1 if fld.ndim == 3 else 0
        fold_ptr = fld.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    xa, ya, ta = k(_f64(output.x_axis)), k(_f64(output.y_axis)), k(_f64(output.t_axis_ms))
    a = _Args(
        n_traces=amps.shape[0], n_samples=amps.shape[1], amp_is_f64=amp_is_f64,
        amplitudes=amps.ctypes.data,
        source_x=_p(sx), source_y=_p(sy), receiver_x=_p(rx), receiver_y=_p(ry),
        midpoint_x=_p(mx), midpoint_y=_p(my), weights=_p(w),
        sample_rate_ms=float(traces.sample_rate_ms), start_time_ms=float(traces.start_time_ms),
        nx=nx, ny=ny, nt=nt, x_axis=_p(xa), y_axis=_p(ya), x_grid=_p(xg), y_grid=_p(yg),
        t_axis_ms=_p(ta), image=_p(img), fold=fold_ptr, fold_is_3d=fold_is_3d,
        vrms=_p(v), vel_is_3d=vel3d,
        max_aperture_m=float(config.max_aperture_m), min_aperture_m=float(config.min_aperture_m),
        max_dip_degrees=float(config.max_dip_degrees), taper_fraction=float(config.taper_fraction),
        apply_spreading=int(bool(config.apply_spreading)),
        apply_obliquity=int(bool(config.apply_obliquity)),
        aa_enabled=int(bool(config.aa_enabled)),
        aa_dominant_freq=float(getattr(config, "aa_dominant_freq", 30.0)),
        grid_dx=float(config.grid_dx), grid_dy=float(config.grid_dy),
        traveltime_kind=int(kind), curved_v0=float(config.curved_ray_v0),
        curved_k=float(config.curved_ray_k), eta=_p(eta), eta_is_3d=eta_is_3d,
        eta_constant=float(getattr(config, "vti_eta_constant", 0.0)),
        pillar_begin=0 if pillars is None else int(pillars[0]),
        pillar_end=0 if pillars is None else int(pillars[1]),
        n_threads=int(n_threads), interp_method=interp_code(getattr(config, "interpolation_method", None)),
    )
    rc = L.pstm_oracle_migrate(ctypes.byref(a))
    if rc != 0:
        raise ValueError(f"oracle rejected its arguments (code {rc})")
    return img, fld


def traveltime(kind, feat7, v0=1500.0, k=0.5):
    """Exact FP64 traveltime for rows (t0, dx_s, dy_s, dx_r, dy_r, v, eta)."""
    if isinstance(kind, str):
        kind = KIND_BY_NAME[kind]
    f = np.ascontiguousarray(feat7, dtype=np.float64).reshape(-1, 7)
    out = np.empty(f.shape[0], np.float64)
    lib().pstm_oracle_traveltime(int(kind), f.shape[0], _p(f), float(v0), float(k), _p(out))
    return out


# trace interpolators (names and aliases of pstm/kernels/interpolation.py:26-51)
INTERP_BY_NAME = {"linear": 0, "nearest": 1, "cubic": 2, "sinc4": 3, "sinc8": 4, "sinc16": 5,
                  "lanczos3": 6, "lanczos5": 7}
INTERP_ALIASES = {"sinc": "sinc8", "spline": "cubic", "lanczos": "lanczos3"}


def interp_code(name) -> int:
    if name is None:
        return 0
    name = str(getattr(name, "value", name)).lower().strip()
    return INTERP_BY_NAME[INTERP_ALIASES.get(name, name)]


def interp(trace, t_sample, method):
    """One interpolated sample by the restated reference interpolator."""
    tr = np.ascontiguousarray(trace, dtype=np.float64)
    return lib().pstm_oracle_interp(_p(tr), len(tr), float(t_sample), interp_code(method))


def linear_interp(trace, t_sample):
    tr = np.ascontiguousarray(trace, dtype=np.float64)
    return lib().pstm_oracle_linear_interp(_p(tr), len(tr), float(t_sample))
