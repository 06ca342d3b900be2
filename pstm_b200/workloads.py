"""Seeded synthetic workloads with the shapes of the five benchmark cases.

No public dataset is used: every trace panel here is a sum of 25 Hz Ricker
diffraction responses plus Gaussian noise, generated from a fixed seed.

* ``config1``  plain straight-ray tile: 64x64 bins at 25 m, 500 samples at
  4 ms, 16,384 FP32 traces of 500 samples, s/r uniform in a 1.6 km square
  (offset <= 2 km), diffractors (800,800,0.6 s), (500,1100,1.0 s),
  (1200,400,1.4 s) in v = 2000 m/s, SNR 10; aperture 1000 m, dip 60 deg,
  weights on, AA off.
* ``binned_survey``  the batched case: traces sorted into common-offset bins
  of equal width (40 bins over 0-4 km), the trace count of each bin drawn
  lognormal between 5k and 200k (about 2M in all), midpoints uniform over the
  patch, azimuths uniform; each bin is a contiguous range of the panel.
* ``survey``   the larger cases (2-5): bins of 12.5 m, laterally varying
  v_rms(t,x,y) = (1500 + 2500 t/3 s)(1 + 0.05 G(x,y)), G a unit-variance
  Gaussian-smoothed field with a 300 m correlation length, eta(t0) rising
  linearly to 0.15 at 3 s, triangle AA on.

Diffraction traveltimes use the kernel's own straight-ray DSR convention,
t = sqrt((t0/2)^2 + ds^2/v^2) + sqrt((t0/2)^2 + dr^2/v^2).  SNR is the ratio
of the panel's RMS signal to the RMS of the added noise.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .base import KernelConfig, OutputTile, TraceBlock, VelocitySlice, create_trace_block

RICKER_HZ = 25.0
SNR = 10.0
C1_DIFFRACTORS = ((800.0, 800.0, 0.6), (500.0, 1100.0, 1.0), (1200.0, 400.0, 1.4))


def ricker(t: np.ndarray, f: float = RICKER_HZ) -> np.ndarray:
    a = (np.pi * f * t) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def draw_geometry(rng, n, lo, hi, max_offset):
    """Uniform source/receiver pairs in [lo, hi]^2 with |r - s| <= max_offset."""
    s = rng.uniform(lo, hi, (n, 2))
    r = rng.uniform(lo, hi, (n, 2))
    bad = np.hypot(*(r - s).T) > max_offset
    while bad.any():
        k = int(bad.sum())
        s[bad] = rng.uniform(lo, hi, (k, 2))
        r[bad] = rng.uniform(lo, hi, (k, 2))
        bad = np.hypot(*(r - s).T) > max_offset
    return s, r


def diffraction_panel(s, r, diffractors, v_of_t0, ns, dt_s, rng, snr=SNR, dtype=np.float32,
                      block=65536):
    """(n, ns) panel: Ricker responses of point diffractors + Gaussian noise."""
    n = s.shape[0]
    t = np.arange(ns) * dt_s
    panel = np.zeros((n, ns), dtype=np.float32)
    for b0 in range(0, n, block):
        sl = slice(b0, min(n, b0 + block))
        acc = np.zeros((sl.stop - sl.start, ns), dtype=np.float64)
        for (xd, yd, t0d) in diffractors:
            v = float(v_of_t0(t0d))
            ds2 = (s[sl, 0] - xd) ** 2 + (s[sl, 1] - yd) ** 2
            dr2 = (r[sl, 0] - xd) ** 2 + (r[sl, 1] - yd) ** 2
            T = np.sqrt((t0d / 2) ** 2 + ds2 / v ** 2) + np.sqrt((t0d / 2) ** 2 + dr2 / v ** 2)
            acc += ricker(t[None, :] - T[:, None])
        panel[sl] = acc
    rms = float(np.sqrt(np.mean(panel.astype(np.float64) ** 2)))
    panel += (rng.standard_normal(panel.shape, dtype=np.float32) * (rms / snr)).astype(np.float32)
    return panel.astype(dtype)


@dataclass
class Case:
    traces: TraceBlock
    output: OutputTile
    velocity: VelocitySlice
    config: KernelConfig
    kernel_type: str = "straight_ray"

    @property
    def pairs(self) -> int:
        return self.output.nx * self.output.ny * self.output.nt * self.traces.n_traces


def config1(seed: int = 1234, n_traces: int = 16384, nx: int = 64, ny: int = 64, nt: int = 500) -> Case:
    rng = np.random.default_rng(seed)
    s, r = draw_geometry(rng, n_traces, 0.0, 1600.0, 2000.0)
    ns, dt_ms = 500, 4.0
    amps = diffraction_panel(s, r, C1_DIFFRACTORS, lambda t0: 2000.0, ns, dt_ms / 1000.0, rng)
    tb = create_trace_block(amps, s[:, 0], s[:, 1], r[:, 0], r[:, 1], sample_rate_ms=dt_ms)
    x = np.arange(nx) * 25.0
    y = np.arange(ny) * 25.0
    t = np.arange(nt) * 4.0
    out = OutputTile(image=np.zeros((nx, ny, nt)), fold=np.zeros((nx, ny, nt), np.int32),
                     x_axis=x, y_axis=y, t_axis_ms=t)
    vel = VelocitySlice(vrms=np.full(nt, 2000.0), is_1d=True)
    cfg = KernelConfig(max_aperture_m=1000.0, min_aperture_m=500.0, max_dip_degrees=60.0,
                       taper_fraction=0.1, apply_spreading=True, apply_obliquity=True,
                       aa_enabled=False, interpolation_method="linear", grid_dx=25.0, grid_dy=25.0)
    return Case(tb, out, vel, cfg)


# ----------------------------------------------------------------- larger surveys
def lateral_field(nx, ny, dx, corr_m, seed):
    """Unit-variance white noise smoothed by a Gaussian of std corr_m metres."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    g = gaussian_filter(rng.standard_normal((nx, ny)), sigma=corr_m / dx, mode="wrap")
    g -= g.mean()
    return g / g.std()


def survey_velocity(t_ms: np.ndarray, G: np.ndarray) -> np.ndarray:
    """v_rms(t, x, y) = (1500 + 2500 t/3 s) (1 + 0.05 G(x, y)), shape (nx, ny, nt)."""
    vt = 1500.0 + 2500.0 * (t_ms / 1000.0) / 3.0
    return vt[None, None, :] * (1.0 + 0.05 * G[:, :, None])


def survey_eta(t_ms: np.ndarray) -> np.ndarray:
    """eta(t0) rising linearly from 0 to 0.15 at 3 s (smooth, 1-D)."""
    return np.clip(0.15 * (t_ms / 1000.0) / 3.0, 0.0, 0.15)


@dataclass
class Survey:
    """A survey patch: trace panel + geometry + the full output grid."""

    s: np.ndarray
    r: np.ndarray
    amps: np.ndarray
    dt_ms: float
    x_axis: np.ndarray
    y_axis: np.ndarray
    t_axis_ms: np.ndarray
    G: np.ndarray
    dx: float

    def velocity(self, ix0=0, ix1=None, iy0=0, iy1=None) -> np.ndarray:
        ix1 = len(self.x_axis) if ix1 is None else ix1
        iy1 = len(self.y_axis) if iy1 is None else iy1
        return survey_velocity(self.t_axis_ms, self.G[ix0:ix1, iy0:iy1])

    def trace_block(self) -> TraceBlock:
        return create_trace_block(self.amps, self.s[:, 0], self.s[:, 1], self.r[:, 0], self.r[:, 1],
                                  sample_rate_ms=self.dt_ms)

    def tile(self, ix0, ix1, iy0, iy1, image_dtype=np.float64) -> tuple[OutputTile, VelocitySlice]:
        nx, ny, nt = ix1 - ix0, iy1 - iy0, len(self.t_axis_ms)
        out = OutputTile(image=np.zeros((nx, ny, nt), image_dtype), fold=np.zeros((nx, ny, nt), np.int32),
                         x_axis=self.x_axis[ix0:ix1].copy(), y_axis=self.y_axis[iy0:iy1].copy(),
                         t_axis_ms=self.t_axis_ms.copy())
        vel = VelocitySlice(vrms=np.ascontiguousarray(self.velocity(ix0, ix1, iy0, iy1)), is_1d=False)
        return out, vel


def survey(n_traces: int, nx: int, ny: int, nt: int, dt_ms: float, ns: int, dx: float = 12.5,
           max_offset: float = 1e9, n_diffractors: int = 6, seed: int = 7,
           amp_dtype=np.float32, with_amplitudes: bool = True) -> Survey:
    rng = np.random.default_rng(seed)
    extent = nx * dx
    s, r = draw_geometry(rng, n_traces, 0.0, extent, max_offset)
    G = lateral_field(nx, ny, dx, 300.0, seed + 1)
    t_axis = np.arange(nt) * dt_ms
    tmax = (nt - 1) * dt_ms / 1000.0
    diffr = [(rng.uniform(0.2, 0.8) * extent, rng.uniform(0.2, 0.8) * ny * dx,
              rng.uniform(0.25, 0.7) * tmax) for _ in range(n_diffractors)]
    amps = None
    if with_amplitudes:
        amps = diffraction_panel(s, r, diffr, lambda t0: 1500.0 + 2500.0 * t0 / 3.0, ns, dt_ms / 1000.0,
                                 rng, dtype=amp_dtype)
    return Survey(s=s, r=r, amps=amps, dt_ms=dt_ms, x_axis=np.arange(nx) * dx,
                  y_axis=np.arange(ny) * dx, t_axis_ms=t_axis, G=G, dx=dx)


def estimate_gradient_from_vrms(vrms, t_ms, window_ms: float = 500.0) -> tuple[float, float]:
    """(v0, k) of a linear V(z) = v0 + k z from a v_rms(t) function, as the
    reference suggests them (``pstm/algorithm/curved_ray.py:145-201``):
    a least-squares line v_rms ~ v0 + slope t over t <= window_ms (the first
    len // 2 samples when fewer than two fall inside; v_rms[0] and k = 0 when
    fewer than two remain), k = 2 slope / v0,
    then v0 clamped to [1000, 6000] m/s and k to [0, 2] 1/s."""
    v = np.asarray(vrms, np.float64)
    t = np.asarray(t_ms, np.float64)
    if len(v) < 2:
        return (float(v[0]) if len(v) else 1500.0), 0.0
    mask = t <= window_ms
    if mask.sum() < 2:
        mask = np.zeros(len(t), bool)
        mask[:len(t) // 2] = True
    if mask.sum() < 2:
        return float(v[0]), 0.0
    ts, vs = t[mask] / 1000.0, v[mask]
    tm, vm = ts.mean(), vs.mean()
    slope = float(((ts - tm) * (vs - vm)).sum() / ((ts - tm) ** 2).sum())
    v0 = float(vm - slope * tm)
    k = 2.0 * slope / v0 if v0 > 0 else 0.0
    return max(1000.0, min(v0, 6000.0)), max(0.0, min(k, 2.0))


def survey_config(kernel_type: str = "straight_ray", aa: bool = True, dx: float = 12.5,
                  eta: np.ndarray | None = None, v0: float = 1500.0, k: float = 0.5) -> KernelConfig:
    """Reference defaults (5 km aperture, 45 deg dip) with AA on, as cases 2-5."""
    return KernelConfig(aa_enabled=aa, grid_dx=dx, grid_dy=dx, kernel_type=kernel_type,
                        curved_ray_v0=v0, curved_ray_k=k, vti_eta_array=eta,
                        vti_enabled=eta is not None, curved_ray_enabled=kernel_type.startswith("curved"))


def config2_small(n_traces=4096, nx=16, ny=16, nt=300, ns=300, seed=7) -> Case:
    """A reduced case-2 style tile (3-D velocity, AA on) for parity tests."""
    sv = survey(n_traces, nx, ny, nt, 2.0, ns, seed=seed)
    out, vel = sv.tile(0, nx, 0, ny)
    return Case(sv.trace_block(), out, vel, survey_config(aa=True))


def diffraction_panel_torch(s, r, diffractors, v_of_t0, ns, dt_s, seed, device="cuda",
                            dtype=None, snr=SNR, block=32768):
    """Device-side version of ``diffraction_panel`` for the large cases.

    Same model (Ricker responses + Gaussian noise at the given SNR), generated
    with a seeded ``torch.Generator`` on ``device``; returns a torch tensor.
    """
    import torch
    dtype = dtype or torch.float32
    n = s.shape[0]
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    t = torch.arange(ns, device=device, dtype=torch.float32) * dt_s
    S = torch.as_tensor(s, device=device, dtype=torch.float64)
    Rr = torch.as_tensor(r, device=device, dtype=torch.float64)
    panel = torch.empty((n, ns), device=device, dtype=dtype)
    sumsq = 0.0
    for b0 in range(0, n, block):
        b1 = min(n, b0 + block)
        acc = torch.zeros((b1 - b0, ns), device=device, dtype=torch.float32)
        for (xd, yd, t0d) in diffractors:
            v = float(v_of_t0(t0d))
            ds2 = (S[b0:b1, 0] - xd) ** 2 + (S[b0:b1, 1] - yd) ** 2
            dr2 = (Rr[b0:b1, 0] - xd) ** 2 + (Rr[b0:b1, 1] - yd) ** 2
            T = (torch.sqrt((t0d / 2) ** 2 + ds2 / v ** 2) + torch.sqrt((t0d / 2) ** 2 + dr2 / v ** 2)).float()
            a = (torch.pi * RICKER_HZ * (t[None, :] - T[:, None])) ** 2
            acc += (1.0 - 2.0 * a) * torch.exp(-a)
        sumsq += float((acc.double() ** 2).sum())
        panel[b0:b1] = acc.to(dtype)
    rms = (sumsq / (n * ns)) ** 0.5
    for b0 in range(0, n, block):
        b1 = min(n, b0 + block)
        noise = torch.randn((b1 - b0, ns), generator=g, device=device, dtype=torch.float32) * (rms / snr)
        panel[b0:b1] = (panel[b0:b1].float() + noise).to(dtype)
    return panel


def survey_device(n_traces: int, nx: int, ny: int, nt: int, dt_ms: float, ns: int, dx: float = 12.5,
                  max_offset: float = 1e9, n_diffractors: int = 6, seed: int = 7, device="cuda",
                  dtype=None):
    """``survey`` with the trace panel generated on the device (torch tensor)."""
    sv = survey(n_traces, nx, ny, nt, dt_ms, ns, dx=dx, max_offset=max_offset,
                n_diffractors=n_diffractors, seed=seed, with_amplitudes=False)
    rng = np.random.default_rng(seed + 100)
    extent = nx * dx
    tmax = (nt - 1) * dt_ms / 1000.0
    diffr = [(rng.uniform(0.2, 0.8) * extent, rng.uniform(0.2, 0.8) * ny * dx,
              rng.uniform(0.25, 0.7) * tmax) for _ in range(n_diffractors)]
    amps = diffraction_panel_torch(sv.s, sv.r, diffr, lambda t0: 1500.0 + 2500.0 * t0 / 3.0, ns,
                                   dt_ms / 1000.0, seed + 200, device=device, dtype=dtype)
    return sv, amps


# ----------------------------------------------------------------- offset bins
def offset_bin_counts(n_bins: int, lo: int, hi: int, total: int, seed: int) -> np.ndarray:
    """Trace counts per bin: lognormal between lo and hi, scaled to about `total`."""
    rng = np.random.default_rng(seed)
    mu = 0.5 * (np.log(lo) + np.log(hi))
    sigma = (np.log(hi) - np.log(lo)) / 4.0
    c = np.clip(np.exp(rng.normal(mu, sigma, n_bins)), lo, hi)
    c = np.clip(c * (total / c.sum()), lo, hi)
    return np.rint(c).astype(np.int64)


@dataclass
class BinnedSurvey:
    survey: Survey
    starts: np.ndarray      # first trace of each bin
    counts: np.ndarray      # traces of each bin
    bin_width_m: float
    amps_device: object = None   # torch tensor when generated on the device


def binned_survey(counts, nx: int, ny: int, nt: int, dt_ms: float, ns: int, dx: float = 12.5,
                  bin_width_m: float = 100.0, n_diffractors: int = 6, seed: int = 11,
                  device=None, dtype=None) -> BinnedSurvey:
    """Traces of common-offset bins [b w, (b+1) w), bin after bin, over an
    nx*dx x ny*dx patch with the ``survey`` velocity.  With ``device`` the
    amplitudes are generated there (``amps_device``), else on the host."""
    counts = np.asarray(counts, dtype=np.int64)
    rng = np.random.default_rng(seed)
    n = int(counts.sum())
    h = np.concatenate([rng.uniform(b * bin_width_m, (b + 1) * bin_width_m, int(c))
                        for b, c in enumerate(counts)]) if n else np.zeros(0)
    az = rng.uniform(0.0, 2.0 * np.pi, n)
    m = np.stack([rng.uniform(0.0, nx * dx, n), rng.uniform(0.0, ny * dx, n)], axis=1)
    d = 0.5 * h[:, None] * np.stack([np.cos(az), np.sin(az)], axis=1)
    s, r = m - d, m + d
    G = lateral_field(nx, ny, dx, 300.0, seed + 1)
    tmax = (nt - 1) * dt_ms / 1000.0
    diffr = [(rng.uniform(0.2, 0.8) * nx * dx, rng.uniform(0.2, 0.8) * ny * dx,
              rng.uniform(0.25, 0.7) * tmax) for _ in range(n_diffractors)]
    v_of_t0 = lambda t0: 1500.0 + 2500.0 * t0 / 3.0
    amps, amps_dev = None, None
    if device is not None:
        amps_dev = diffraction_panel_torch(s, r, diffr, v_of_t0, ns, dt_ms / 1000.0, seed + 200,
                                           device=device, dtype=dtype)
    else:
        amps = diffraction_panel(s, r, diffr, v_of_t0, ns, dt_ms / 1000.0, rng, dtype=dtype or np.float32)
    sv = Survey(s=s, r=r, amps=amps, dt_ms=dt_ms, x_axis=np.arange(nx) * dx, y_axis=np.arange(ny) * dx,
                t_axis_ms=np.arange(nt) * dt_ms, G=G, dx=dx)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    return BinnedSurvey(sv, starts, counts, bin_width_m, amps_dev)

