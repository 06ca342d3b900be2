"""Data carriers of the kernel-backend boundary.

These mirror the reference's ``pstm/kernels/base.py`` (``TraceBlock`` :27-116,
``OutputTile`` :119-177, ``VelocitySlice`` :180-194, ``KernelConfig``
:197-265, ``KernelMetrics`` :268-287, ``MigrationKernel`` :290-318,
``create_trace_block`` :321-357, ``create_output_tile`` :360-384) field for
field, so that objects built by the reference executor can be handed to the
CUDA backend unchanged and the other way round.  The backend only duck-types
its arguments; these classes exist so this package runs without the
reference installed.

Defaults that the reference pulls from ``pstm.settings`` (``settings.py:90-133``)
are fixed here to the same values.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from enum import Enum
from typing import Protocol, runtime_checkable

import numpy as np

# Reference settings defaults (pstm/settings.py:94-133; grid dt from GridSettings).
DEFAULT_MAX_APERTURE_M = 5000.0
DEFAULT_MIN_APERTURE_M = 500.0
DEFAULT_MAX_DIP_DEG = 45.0
DEFAULT_TAPER_FRACTION = 0.1
DEFAULT_AA_ENABLED = True
DEFAULT_APPLY_SPREADING = True
DEFAULT_INTERPOLATION = "linear"
DEFAULT_OUTPUT_DT_MS = 2.0
# The Metal host reads ``config.aa_dominant_freq`` through ``hasattr`` and
# falls back to 30 Hz (pstm/kernels/metal_compiled.py:706).
DEFAULT_AA_DOMINANT_FREQ = 30.0


class KernelCapability(Enum):
    """Same members as the reference enum (base.py:17-24)."""

    FP16 = "fp16"
    FP64 = "fp64"
    COMPLEX = "complex"
    ASYNC = "async"
    BATCH = "batch"


@dataclass
class TraceBlock:
    """Trace panel and geometry: amplitudes (n_traces, n_samples), FP64 coords."""

    amplitudes: np.ndarray
    source_x: np.ndarray
    source_y: np.ndarray
    receiver_x: np.ndarray
    receiver_y: np.ndarray
    offset: np.ndarray
    midpoint_x: np.ndarray
    midpoint_y: np.ndarray
    weights: np.ndarray | None = None
    sample_rate_ms: float = 2.0
    start_time_ms: float = 0.0

    @property
    def n_traces(self) -> int:
        return int(self.amplitudes.shape[0])

    @property
    def n_samples(self) -> int:
        return int(self.amplitudes.shape[1])

    @property
    def time_axis_ms(self) -> np.ndarray:
        return self.start_time_ms + self.sample_rate_ms * np.arange(self.n_samples)

    def validate(self) -> list[str]:
        n = self.n_traces
        errs = []
        for name in ("source_x", "source_y", "receiver_x", "receiver_y",
                     "offset", "midpoint_x", "midpoint_y"):
            arr = getattr(self, name)
            if len(arr) != n:
                errs.append(f"{name} length mismatch: {len(arr)} != {n}")
        if not self.amplitudes.flags["C_CONTIGUOUS"]:
            errs.append("amplitudes must be C-contiguous")
        if not np.all(np.isfinite(self.amplitudes)):
            errs.append("amplitudes contains NaN or Inf values")
        return errs

    def ensure_contiguous(self) -> "TraceBlock":
        c = np.ascontiguousarray
        return TraceBlock(
            amplitudes=c(self.amplitudes), source_x=c(self.source_x),
            source_y=c(self.source_y), receiver_x=c(self.receiver_x),
            receiver_y=c(self.receiver_y), offset=c(self.offset),
            midpoint_x=c(self.midpoint_x), midpoint_y=c(self.midpoint_y),
            weights=None if self.weights is None else c(self.weights),
            sample_rate_ms=self.sample_rate_ms, start_time_ms=self.start_time_ms,
        )


@dataclass
class OutputTile:
    """Output accumulator: image (nx, ny, nt) f64, fold (nx, ny, nt) int32."""

    image: np.ndarray
    fold: np.ndarray
    x_axis: np.ndarray
    y_axis: np.ndarray
    t_axis_ms: np.ndarray
    x_grid: np.ndarray | None = None
    y_grid: np.ndarray | None = None

    @property
    def nx(self) -> int:
        return len(self.x_axis)

    @property
    def ny(self) -> int:
        return len(self.y_axis)

    @property
    def nt(self) -> int:
        return len(self.t_axis_ms)

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.nx, self.ny, self.nt)

    @property
    def x_range(self) -> tuple[float, float]:
        return (float(self.x_axis[0]), float(self.x_axis[-1]))

    @property
    def y_range(self) -> tuple[float, float]:
        return (float(self.y_axis[0]), float(self.y_axis[-1]))

    @property
    def dt_ms(self) -> float:
        if len(self.t_axis_ms) < 2:
            return 1.0
        return float(self.t_axis_ms[1] - self.t_axis_ms[0])

    @property
    def x_coords(self) -> np.ndarray:
        return self.x_axis

    @property
    def y_coords(self) -> np.ndarray:
        return self.y_axis

    @property
    def t_coords_ms(self) -> np.ndarray:
        return self.t_axis_ms

    def reset(self) -> None:
        self.image[...] = 0.0
        self.fold[...] = 0


@dataclass
class VelocitySlice:
    """RMS velocity: (nt,) when ``is_1d`` else (nx, ny, nt)."""

    vrms: np.ndarray
    is_1d: bool = True
    x_axis: np.ndarray | None = None
    y_axis: np.ndarray | None = None
    t_axis_ms: np.ndarray | None = None

    def get_velocity_at(self, ix: int, iy: int, it: int) -> float:
        return float(self.vrms[it] if self.is_1d else self.vrms[ix, iy, it])


@dataclass
class KernelConfig:
    """Kernel parameters; ``None`` fields take the reference settings defaults."""

    max_aperture_m: float | None = None
    min_aperture_m: float | None = None
    max_dip_degrees: float | None = None
    taper_fraction: float | None = None
    aa_enabled: bool | None = None
    aa_filter_indices: np.ndarray | None = None
    aa_filter_bank: np.ndarray | None = None
    apply_spreading: bool | None = None
    apply_obliquity: bool = True
    interpolation_method: str | None = None
    output_dt_ms: float | None = None
    accumulate_fold: bool = True
    time_variant_enabled: bool = False
    time_variant_windows: list | None = None
    kernel_type: str = "straight_ray"
    curved_ray_enabled: bool = False
    curved_ray_v0: float = 1500.0
    curved_ray_k: float = 0.5
    vti_enabled: bool = False
    vti_eta_constant: float = 0.0
    vti_eta_array: np.ndarray | None = None
    vti_eta_is_1d: bool = True
    grid_dx: float = 25.0
    grid_dy: float = 12.5
    aa_dominant_freq: float = DEFAULT_AA_DOMINANT_FREQ

    def __post_init__(self) -> None:
        if self.max_aperture_m is None:
            self.max_aperture_m = DEFAULT_MAX_APERTURE_M
        if self.min_aperture_m is None:
            self.min_aperture_m = DEFAULT_MIN_APERTURE_M
        if self.max_dip_degrees is None:
            self.max_dip_degrees = DEFAULT_MAX_DIP_DEG
        if self.taper_fraction is None:
            self.taper_fraction = DEFAULT_TAPER_FRACTION
        if self.aa_enabled is None:
            self.aa_enabled = DEFAULT_AA_ENABLED
        if self.apply_spreading is None:
            self.apply_spreading = DEFAULT_APPLY_SPREADING
        if self.interpolation_method is None:
            self.interpolation_method = DEFAULT_INTERPOLATION
        if self.output_dt_ms is None:
            self.output_dt_ms = DEFAULT_OUTPUT_DT_MS

    def get_aperture_at_time(self, t_ms: float, velocity: float) -> float:
        ap = velocity * (t_ms / 1000.0) * np.tan(np.radians(self.max_dip_degrees))
        return float(np.clip(ap, self.min_aperture_m, self.max_aperture_m))


@dataclass
class KernelMetrics:
    n_traces_processed: int = 0
    n_samples_output: int = 0
    compute_time_s: float = 0.0
    memory_peak_mb: float = 0.0

    @property
    def traces_per_second(self) -> float:
        return self.n_traces_processed / self.compute_time_s if self.compute_time_s > 0 else 0.0

    @property
    def samples_per_second(self) -> float:
        return self.n_samples_output / self.compute_time_s if self.compute_time_s > 0 else 0.0


@runtime_checkable
class MigrationKernel(Protocol):
    @property
    def name(self) -> str: ...

    @property
    def capabilities(self) -> set: ...

    def initialize(self, config) -> None: ...

    def migrate_tile(self, traces, output, velocity, config=None): ...

    def synchronize(self) -> None: ...

    def cleanup(self) -> None: ...


def create_trace_block(amplitudes, source_x, source_y, receiver_x, receiver_y,
                       sample_rate_ms, start_time_ms=0.0, weights=None) -> TraceBlock:
    """FP64 offsets/midpoints from FP64 coordinates, as base.py:321-357."""
    sx = np.asarray(source_x, dtype=np.float64)
    sy = np.asarray(source_y, dtype=np.float64)
    rx = np.asarray(receiver_x, dtype=np.float64)
    ry = np.asarray(receiver_y, dtype=np.float64)
    amps = np.asarray(amplitudes)
    if amps.dtype not in (np.float32, np.float16) and amps.dtype.name != "bfloat16":
        amps = amps.astype(np.float32)
    amps = np.ascontiguousarray(amps)
    return TraceBlock(
        amplitudes=amps, source_x=sx, source_y=sy, receiver_x=rx, receiver_y=ry,
        offset=np.sqrt((rx - sx) ** 2 + (ry - sy) ** 2),
        midpoint_x=(sx + rx) / 2.0, midpoint_y=(sy + ry) / 2.0,
        weights=None if weights is None else np.asarray(weights, dtype=np.float64),
        sample_rate_ms=float(sample_rate_ms), start_time_ms=float(start_time_ms),
    )


def create_output_tile(x_min, x_max, dx, y_min, y_max, dy, t_min_ms, t_max_ms, dt_ms) -> OutputTile:
    """Axes by arange with a half-step end guard, as base.py:360-384."""
    x = np.arange(x_min, x_max + dx / 2, dx, dtype=np.float64)
    y = np.arange(y_min, y_max + dy / 2, dy, dtype=np.float64)
    t = np.arange(t_min_ms, t_max_ms + dt_ms / 2, dt_ms, dtype=np.float64)
    shape = (len(x), len(y), len(t))
    return OutputTile(image=np.zeros(shape, np.float64), fold=np.zeros(shape, np.int32),
                      x_axis=x, y_axis=y, t_axis_ms=t)
