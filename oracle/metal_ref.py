"""The reference's Metal compute shaders compiled as C++ on the CPU.

Test infrastructure only: it checks the oracle, it is never measured or
shipped.  ``oracle/Makefile``'s ``ref`` target compiles ``metal_ref.cpp`` --
which includes ``pstm/metal/shaders/pstm_migration.metal``,
``pstm_curved_ray.metal`` and ``pstm_anisotropic_vti.metal`` from the reference
tree, unchanged, with the Metal standard-library subset of
``metal_compat/metal_stdlib`` -- into ``oracle/_ref/libpstm_metal_ref.so``.
The library exists only where the reference tree does;
``tests/golden/make_metal_golden.py`` runs it and commits its outputs as
fixtures, which the tests compare with the oracle everywhere.

A migration runs a shader kernel once per (ix, iy, it), as a Metal dispatch
of nx x ny x nt threads would, on FP32 inputs laid out as the kernels take
them: per-time tables t0 (s), (t0/2)^2, 1/v^2 (or 1/v^2 per sample with 3-D
velocity), aperture, eta.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libpstm_metal_ref.so")

_f = ctypes.c_float
_pf = ctypes.POINTER(ctypes.c_float)
_pi = ctypes.POINTER(ctypes.c_int32)


class Call(ctypes.Structure):
    """Mirror of pstm_ref_call (metal_ref.cpp)."""
    _fields_ = [(n, _pf) for n in ("amps", "sx", "sy", "rx", "ry", "mx", "my", "x_coords", "y_coords", "t0_s",
                                   "t0_half_sq", "apertures", "eta", "inv_v_sq", "image")] + \
               [("fold", _pi)] + \
               [(n, ctypes.c_int32) for n in ("n_traces", "n_samples", "nx", "ny", "nt", "spreading", "obliquity",
                                              "aa", "use_3d_velocity", "eta_is_1d")] + \
               [(n, _f) for n in ("dx", "dy", "dt_ms", "t_start_ms", "max_aperture", "min_aperture",
                                  "taper_fraction", "max_dip_deg", "aa_dominant_freq", "v0", "k", "eta_constant")]


class Window(ctypes.Structure):
    """Mirror of the shader's TimeWindow (pstm_migration.metal:495-502)."""
    _fields_ = [("t_start_ms", _f), ("t_end_ms", _f), ("dt_effective_ms", _f), ("downsample_factor", ctypes.c_int32),
                ("sample_offset", ctypes.c_int32), ("n_samples", ctypes.c_int32)]


_REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
def build(reference_root: str | None = None) -> str | None:
    """Build the library from the reference tree; None when the tree is absent."""
    ref = reference_root or os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref, "pstm", "metal", "shaders")):
        return None
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)
    return LIB_PATH


def available() -> bool:
    return os.path.exists(LIB_PATH)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB_PATH} is not built (needs the reference tree; see oracle/Makefile)")
        L = ctypes.CDLL(LIB_PATH)
        for name in ("pstm_ref_aa_weight",):
            getattr(L, name).argtypes = [_f] * 9
        L.pstm_ref_dsr.argtypes = [_f] * 4
        L.pstm_ref_time_to_depth.argtypes = [_f] * 3
        L.pstm_ref_curved_dsr.argtypes = [_f] * 5
        L.pstm_ref_vti_dsr.argtypes = [_f] * 5
        for name in ("pstm_ref_aa_weight", "pstm_ref_dsr", "pstm_ref_time_to_depth", "pstm_ref_curved_dsr",
                     "pstm_ref_vti_dsr"):
            getattr(L, name).restype = _f
        for name in ("pstm_ref_migrate_straight", "pstm_ref_migrate_curved", "pstm_ref_migrate_vti"):
            getattr(L, name).argtypes = [ctypes.POINTER(Call), ctypes.c_int32]
            getattr(L, name).restype = None
        L.pstm_ref_migrate_time_variant.argtypes = [ctypes.POINTER(Call), _pf, ctypes.c_int32,
                                                    ctypes.POINTER(Window), ctypes.c_int32]
        L.pstm_ref_migrate_time_variant.restype = None
        _lib = L
    return _lib


def _rows(fn, *cols):
    """fn applied row by row to FP32 columns; FP32 result."""
    cols = [np.asarray(c, np.float32).ravel() for c in cols]
    return np.array([fn(*(float(c[i]) for c in cols)) for i in range(len(cols[0]))], np.float32)


def aa_weight(ox, oy, mx, my, v, t, dx, dy, fdom):
    """compute_aa_weight of pstm_migration.metal:95-132."""
    return _rows(lib().pstm_ref_aa_weight, ox, oy, mx, my, v, t, dx, dy, fdom)


def curved_dsr(h_s, h_r, z, v0, k):
    """curved_ray_dsr_traveltime of pstm_curved_ray.metal:86-96."""
    return _rows(lib().pstm_ref_curved_dsr, h_s, h_r, z, v0, k)


def time_to_depth(t_s, v0, k):
    """time_to_depth of pstm_curved_ray.metal:50-56."""
    return _rows(lib().pstm_ref_time_to_depth, t_s, v0, k)


def vti_dsr(t0_s, h_s, h_r, v, eta):
    """vti_dsr_traveltime of pstm_anisotropic_vti.metal:135-148."""
    return _rows(lib().pstm_ref_vti_dsr, t0_s, h_s, h_r, v, eta)


def migrate(kind: str, amps, sx, sy, rx, ry, x_coords, y_coords, t_axis_ms, vrms, *, aperture_m: float,
            taper: float, dx: float, dy: float, dt_ms: float, t_start_ms: float = 0.0, spreading=True,
            obliquity=True, aa=True, aa_dominant_freq=30.0, v0=1500.0, k=0.5, eta=None, eta_constant=0.0,
            max_dip_deg=45.0, simd=False):
    """Image (nx, ny, nt) FP32 and fold of one shader kernel (``simd``: its
    ``_simd`` variant, the Metal backend's default).

    ``kind`` is "straight" (pstm_migrate_3d; ``vrms`` (nt) or (nx, ny, nt)),
    "curved" (pstm_migrate_curved_ray; ``vrms`` unused) or "vti"
    (pstm_migrate_vti; ``vrms`` (nt), ``eta`` (nt) or None for
    ``eta_constant``).  Midpoints are (s + r) / 2 formed in FP64 and rounded
    to FP32, as the reference's host path does (``create_trace_block``,
    base.py:339-340, then the FP32 buffers of the Metal call); the aperture
    table is ``aperture_m`` at every time.
    """
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    amps = f32(amps)
    n_traces, ns = amps.shape
    mx = f32((np.asarray(sx, np.float64) + np.asarray(rx, np.float64)) / 2.0)
    my = f32((np.asarray(sy, np.float64) + np.asarray(ry, np.float64)) / 2.0)
    sx, sy, rx, ry = f32(sx), f32(sy), f32(rx), f32(ry)
    xc, yc = f32(x_coords).ravel(), f32(y_coords).ravel()
    nx, ny = np.shape(x_coords)
    t_ms = np.asarray(t_axis_ms, np.float64)
    nt = len(t_ms)
    t0 = t_ms / 1000.0
    v = np.asarray(vrms, np.float64)
    use3d = v.ndim == 3
    tabs = {"t0_s": f32(t0), "t0_half_sq": f32((t0 / 2.0) ** 2), "apertures": f32(np.full(nt, aperture_m)),
            "eta": f32(eta if eta is not None else np.zeros(nt)), "inv_v_sq": f32(1.0 / v ** 2).ravel()}
    image = np.zeros((nx, ny, nt), np.float32)
    fold = np.zeros((nx, ny, nt) if kind == "straight" else (nx, ny), np.int32)
    c = Call()
    keep = [amps, sx, sy, rx, ry, mx, my, xc, yc, image, fold] + list(tabs.values())
    ptr = lambda a: a.ctypes.data_as(_pf)
    c.amps, c.sx, c.sy, c.rx, c.ry, c.mx, c.my = map(ptr, (amps, sx, sy, rx, ry, mx, my))
    c.x_coords, c.y_coords, c.image = ptr(xc), ptr(yc), ptr(image)
    for name, a in tabs.items():
        setattr(c, name, ptr(a))
    c.fold = fold.ctypes.data_as(_pi)
    c.n_traces, c.n_samples, c.nx, c.ny, c.nt = n_traces, ns, nx, ny, nt
    c.spreading, c.obliquity, c.aa = int(spreading), int(obliquity), int(aa)
    c.use_3d_velocity, c.eta_is_1d = int(use3d), int(eta is not None)
    c.dx, c.dy, c.dt_ms, c.t_start_ms = dx, dy, dt_ms, t_start_ms
    c.max_aperture = c.min_aperture = aperture_m
    c.taper_fraction, c.max_dip_deg, c.aa_dominant_freq = taper, max_dip_deg, aa_dominant_freq
    c.v0, c.k, c.eta_constant = v0, k, eta_constant
    fn = {"straight": lib().pstm_ref_migrate_straight, "curved": lib().pstm_ref_migrate_curved,
          "vti": lib().pstm_ref_migrate_vti}[kind]
    fn(ctypes.byref(c), int(bool(simd)))
    del keep
    return image, fold


def migrate_time_variant(amps, sx, sy, rx, ry, x_coords, y_coords, vrms_base, windows, *, aperture_m: float,
                         taper: float, dx: float, dy: float, dt_ms: float, t_start_ms: float = 0.0, spreading=True,
                         obliquity=True, aa=True, aa_dominant_freq=30.0, max_dip_deg=45.0):
    """Image (nx, ny, n_windowed) FP32 and per-sample fold of
    pstm_migrate_time_variant (pstm_migration.metal:544-701).

    ``windows`` are ``pstm_b200.time_variant.TimeWindow`` records;
    ``vrms_base`` is v_rms at the trace sampling ``dt_ms`` ((nt_base) or
    (nx, ny, nt_base)).  The shader's aperture is min(max, min + v t / 2);
    ``aperture_m`` sets both ends, so it is that value at every time.
    """
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    amps = f32(amps)
    n_traces, ns = amps.shape
    mx = f32((np.asarray(sx, np.float64) + np.asarray(rx, np.float64)) / 2.0)
    my = f32((np.asarray(sy, np.float64) + np.asarray(ry, np.float64)) / 2.0)
    sx, sy, rx, ry = f32(sx), f32(sy), f32(rx), f32(ry)
    xc, yc = f32(x_coords).ravel(), f32(y_coords).ravel()
    nx, ny = np.shape(x_coords)
    v = f32(vrms_base)
    use3d = v.ndim == 3
    nt_base = v.shape[-1]
    win = (Window * max(1, len(windows)))()
    for i, w in enumerate(windows):
        win[i] = Window(w.t_start_ms, w.t_end_ms, w.dt_effective_ms, w.downsample_factor, w.sample_start,
                        w.n_samples)
    total = int(sum(w.n_samples for w in windows))
    image = np.zeros((nx, ny, total), np.float32)
    fold = np.zeros((nx, ny, total), np.int32)
    c = Call()
    ptr = lambda a: a.ctypes.data_as(_pf)
    c.amps, c.sx, c.sy, c.rx, c.ry, c.mx, c.my = map(ptr, (amps, sx, sy, rx, ry, mx, my))
    c.x_coords, c.y_coords, c.image = ptr(xc), ptr(yc), ptr(image)
    c.fold = fold.ctypes.data_as(_pi)
    c.n_traces, c.n_samples, c.nx, c.ny, c.nt = n_traces, ns, nx, ny, total
    c.spreading, c.obliquity, c.aa, c.use_3d_velocity = int(spreading), int(obliquity), int(aa), int(use3d)
    c.dx, c.dy, c.dt_ms, c.t_start_ms = dx, dy, dt_ms, t_start_ms
    c.max_aperture = c.min_aperture = aperture_m
    c.taper_fraction, c.max_dip_deg, c.aa_dominant_freq = taper, max_dip_deg, aa_dominant_freq
    lib().pstm_ref_migrate_time_variant(ctypes.byref(c), ptr(v), nt_base, win, len(windows))
    return image, fold
