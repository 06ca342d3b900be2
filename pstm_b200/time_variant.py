"""Time-variant output sampling (the reference's second speed-up path).

Deep output times carry less bandwidth, so the reference migrates each time
window at a coarser rate and interpolates the result back to the uniform
axis (``pstm/algorithm/time_variant.py``, used by the executor at
``pstm/pipeline/executor.py:1697-1727`` through the backend method
``migrate_tile_time_variant``).  This module keeps the reference's interface
(``FrequencyTimeTable``, ``TimeWindow``, ``compute_time_windows``,
``compute_downsample_factor``, ``nearest_power_of_2``, ``interpolate_fmax``,
``estimate_speedup``, ``resample_to_uniform``) so that windows computed by
either side are the same; the migration at the window times runs on the
ordinary CUDA kernel (its time axis may be non-uniform) and the resampling
of device images runs on a CUDA interpolation kernel.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat


@dataclass
class FrequencyTimeTable:
    """Maximum signal frequency (Hz) against output time (ms); times strictly
    increasing, frequencies positive (time_variant.py:19-83)."""

    times_ms: list = field(default_factory=list)
    frequencies_hz: list = field(default_factory=list)

    def __post_init__(self):
        if len(self.times_ms) != len(self.frequencies_hz):
            raise ValueError("times and frequencies must have same length")
        if len(self.times_ms) < 2:
            raise ValueError("Table must have at least 2 entries")
        if any(b <= a for a, b in zip(self.times_ms, self.times_ms[1:])):
            raise ValueError(f"Times must be monotonically increasing: {self.times_ms}")
        if any(f <= 0 for f in self.frequencies_hz):
            raise ValueError(f"Frequencies must be positive: {self.frequencies_hz}")

    @classmethod
    def from_list(cls, pairs) -> "FrequencyTimeTable":
        if not pairs:
            raise ValueError("pairs list cannot be empty")
        pairs = sorted(pairs, key=lambda p: p[0])
        return cls(times_ms=[p[0] for p in pairs], frequencies_hz=[p[1] for p in pairs])

    def to_list(self):
        return list(zip(self.times_ms, self.frequencies_hz))

    @classmethod
    def default(cls) -> "FrequencyTimeTable":
        """The reference's default table (80 Hz at 0 s down to 15 Hz at 5 s)."""
        return cls(times_ms=[0, 500, 1500, 3000, 5000], frequencies_hz=[80, 60, 40, 25, 15])

    @property
    def t_min(self) -> float:
        return self.times_ms[0]

    @property
    def t_max(self) -> float:
        return self.times_ms[-1]

    @property
    def n_entries(self) -> int:
        return len(self.times_ms)


@dataclass
class TimeWindow:
    """A run of output samples at one effective rate (time_variant.py:86-121)."""

    t_start_ms: float
    t_end_ms: float
    dt_effective_ms: float
    downsample_factor: int
    sample_start: int
    sample_end: int
    f_max_hz: float

    @property
    def n_samples(self) -> int:
        return self.sample_end - self.sample_start

    @property
    def duration_ms(self) -> float:
        return self.t_end_ms - self.t_start_ms


def interpolate_fmax(t_ms: float, table: FrequencyTimeTable) -> float:
    """Shape-preserving piecewise-cubic (PCHIP, Fritsch-Carlson) interpolation
    of the table, constant beyond its ends."""
    if t_ms <= table.t_min:
        return float(table.frequencies_hz[0])
    if t_ms >= table.t_max:
        return float(table.frequencies_hz[-1])
    from scipy.interpolate import PchipInterpolator
    return float(PchipInterpolator(table.times_ms, table.frequencies_hz)(t_ms))


def nearest_power_of_2(n: int) -> int:
    """The power of two nearest to n (the lower one on a tie), at least 1."""
    if n <= 1:
        return 1
    lo = 1 << (int(n).bit_length() - 1)
    return 2 * lo if n - lo > 2 * lo - n else lo


def compute_downsample_factor(f_max_hz: float, base_dt_ms: float, min_factor: int = 1, max_factor: int = 8) -> int:
    """Power-of-two decimation that keeps f_max below Nyquist: the number of
    base samples in 1000 / (2 f_max) ms, rounded to a power of two, clamped."""
    k = nearest_power_of_2(int((1000.0 / (2.0 * f_max_hz)) / base_dt_ms))
    return max(min_factor, min(max_factor, k))


def compute_time_windows(t_min_ms: float, t_max_ms: float, base_dt_ms: float, freq_table: FrequencyTimeTable,
                         min_factor: int = 1, max_factor: int = 8) -> list:
    """Cover [t_min, t_max] with windows of constant decimation.

    A window starts at t with the factor of f_max(t); it grows in steps of its
    effective rate while the factor at the next step is unchanged, keeps at
    least one sample, and ends on a whole number of samples (clipped to
    t_max).  Window times are accumulated in the same order as the reference
    (time_variant.py:201-286), so both give identical windows.
    """
    factor_at = lambda t: compute_downsample_factor(interpolate_fmax(t, freq_table), base_dt_ms, min_factor,
                                                    max_factor)
    out, t, first = [], t_min_ms, 0
    while t < t_max_ms:
        f = interpolate_fmax(t, freq_table)
        k = compute_downsample_factor(f, base_dt_ms, min_factor, max_factor)
        step = base_dt_ms * k
        end = t
        while end < t_max_ms and factor_at(end + step) == k:
            end += step
        if end <= t:
            end = min(t + step, t_max_ms)
        end = min(end, t_max_ms)
        n = max(1, int((end - t) / step))
        end = t + n * step
        if end > t_max_ms:
            end = t_max_ms
            n = max(1, int((end - t) / step))
        out.append(TimeWindow(t, end, step, k, first, first + n, f))
        first += n
        t = end
    return out


def estimate_speedup(t_min_ms: float, t_max_ms: float, base_dt_ms: float, freq_table: FrequencyTimeTable) -> float:
    uniform = int((t_max_ms - t_min_ms) / base_dt_ms)
    tv = sum(w.n_samples for w in compute_time_windows(t_min_ms, t_max_ms, base_dt_ms, freq_table))
    return 1.0 if tv == 0 else uniform / tv


def window_times(windows) -> np.ndarray:
    """Output times (ms) of the samples the windows compute, in order."""
    if not windows:
        return np.zeros(0)
    return np.concatenate([w.t_start_ms + np.arange(w.n_samples) * w.dt_effective_ms for w in windows])


def interp_rows(src, src_times, dst_times, ctx=None):
    """Linear interpolation of every row of src (.., n_src) from src_times onto
    dst_times with np.interp's end rule (the edge value outside).  CUDA
    tensors run the CUDA kernel, NumPy arrays run np.interp."""
    if hasattr(src, "is_cuda") and src.is_cuda:
        import torch
        L = nat.load()
        own = None
        if ctx is None:
            h = ctypes.c_void_p()
            nat.check(L.pstm_cuda_create(src.device.index or 0, ctypes.byref(h)), None, L)
            ctx = own = h
        try:
            s = src.contiguous()
            if s.dtype not in (torch.float64, torch.float32):
                raise ValueError("interp_rows takes float64 or float32 tensors")
            xs = torch.as_tensor(np.ascontiguousarray(src_times, np.float64), device=s.device)
            xd = torch.as_tensor(np.ascontiguousarray(dst_times, np.float64), device=s.device)
            n_src, n_dst = s.shape[-1], int(xd.numel())
            if xs.numel() != n_src:
                raise ValueError("src_times does not match the last axis of src")
            out = torch.empty(tuple(s.shape[:-1]) + (n_dst,), dtype=s.dtype, device=s.device)
            rows = s.numel() // max(1, n_src)
            stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY
            nat.check(L.pstm_cuda_interp_rows(ctx, nat.IMAGE_F32 if s.dtype == torch.float32 else nat.IMAGE_F64,
                                              s.data_ptr(), rows, n_src, xs.data_ptr(), n_dst, xd.data_ptr(),
                                              out.data_ptr(), ctypes.c_void_p(stream)), ctx, L)
            torch.cuda.synchronize()
            return out
        finally:
            if own is not None:
                L.pstm_cuda_destroy(own)
    a = np.asarray(src)
    flat = a.reshape(-1, a.shape[-1])
    res = np.stack([np.interp(dst_times, src_times, r) for r in flat]) if flat.size else np.zeros((0, len(dst_times)))
    return res.reshape(a.shape[:-1] + (len(dst_times),))


def resample_to_uniform(tv_image, windows, base_dt_ms: float, output_nt: int, ctx=None):
    """The time-variant image (nx, ny, n_tv) linearly interpolated onto the
    uniform axis arange(output_nt) * base_dt_ms (time_variant.py:354-397)."""
    times = window_times(windows)
    if len(times) <= 1:   # nothing to interpolate between: zeros, as the reference
        if hasattr(tv_image, "is_cuda"):
            return tv_image.new_zeros(tuple(tv_image.shape[:-1]) + (output_nt,))
        return np.zeros(np.shape(tv_image)[:-1] + (output_nt,))
    return interp_rows(tv_image, times, np.arange(output_nt) * base_dt_ms, ctx)
