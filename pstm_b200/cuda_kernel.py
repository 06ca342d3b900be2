"""CUDA backend implementing the reference ``MigrationKernel`` protocol.

Drop-in for the reference's kernel backends (``pstm/kernels/base.py:290-318``):
``name``, ``capabilities``, ``initialize``, ``migrate_tile``, ``synchronize``,
``cleanup``, plus the optional methods the reference executor discovers with
``hasattr`` (``pstm/pipeline/executor.py:1710-1745``):
``migrate_tile_curved_ray``, ``migrate_tile_vti`` and ``migrate_tile_time_variant``
(:1712-1717).  ``migrate_tile_curved_vti``, ``migrate_tile_learned``,
``migrate_bins`` and ``autotune_bins`` are extensions with no reference
counterpart.

Arguments are duck-typed, so the reference's own ``TraceBlock``/``OutputTile``/
``VelocitySlice``/``KernelConfig`` objects work as well as this package's
mirrors.  NumPy arrays go through the host-pointer C entry point (copies in,
kernel, copies out); CUDA ``torch`` tensors go through the device-pointer entry
point without copies.

Semantics follow the reference Numba backend
(``pstm/kernels/numba_cpu_optimized.py:545-626``): the image and fold are
accumulated in place (``+=``), a 1-D velocity shorter or longer than the
output time axis is interpolated onto it with ``np.interp`` (:569-578), and
calling ``migrate_tile`` before ``initialize`` raises
``RuntimeError("Kernel not initialized")`` (:555-556).
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

from . import _native as nat
from .base import KernelCapability, KernelMetrics

_TT_BY_TYPE = {
    "straight_ray": nat.TT_STRAIGHT,
    "curved_ray": nat.TT_CURVED,
    "anisotropic_vti": nat.TT_VTI,
    "curved_vti": nat.TT_CURVED_VTI,
}


def _is_torch_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and hasattr(x, "data_ptr") and bool(x.is_cuda)


def lateral_velocity_choice(v3):
    """The Metal host's choice between a 3-D velocity cube and its centre
    pillar (``metal_compiled.py:631-664``): with max |v - v_centre| /
    mean(v_centre) > 5 % the cube is used, else the centre pillar
    v[nx // 2, ny // 2, :] stands for every pillar.  ``v3`` is (nx, ny, nt),
    NumPy or torch; returns (velocity, is_3d)."""
    nx, ny = v3.shape[0], v3.shape[1]
    centre = v3[nx // 2, ny // 2, :]
    rel = float((v3 - centre[None, None, :]).abs().max() / centre.mean()) if hasattr(v3, "abs") \
        else float(np.abs(v3 - centre[None, None, :]).max() / centre.mean())
    return (v3, True) if rel > 0.05 else (centre.contiguous() if hasattr(centre, "contiguous") else centre, False)


def float32_to_bf16_bits(a: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even FP32 -> BF16, returned as uint16 bit patterns."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    rounding = ((u >> 16) & 1) + 0x7FFF
    return ((u + rounding) >> 16).astype(np.uint16)


def scaled_f16(amps: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """FP32 traces -> (FP16 traces, per-trace 2^-e): the precision form's
    format, the rule of ``pstm_cuda_traces_to_f16`` -- each trace times 2^e
    with its largest |amplitude| in [2^13, 2^14), rounded to nearest even."""
    a = np.asarray(amps, dtype=np.float32)
    m = np.abs(a).max(axis=1) if a.shape[1] else np.zeros(a.shape[0], np.float32)
    ok = (m > 0) & np.isfinite(m)
    ex = np.frexp(np.where(ok, m, 1.0))[1]
    e = np.where(ok, 14 - ex, 0).astype(np.int32)
    out = (a * np.ldexp(np.float32(1.0), e)[:, None].astype(np.float32)).astype(np.float16)
    return out, np.ldexp(1.0, -e)


def bf16_bits_to_float32(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


class CudaKernel:
    """Kirchhoff PSTM on one CUDA device (sm_100a) through ``libpstm_cuda.so``.

    Parameters
    ----------
    device:
        CUDA device index (default: ``PSTM_CUDA_DEVICE`` or 0).
    trace_dtype:
        ``"auto"`` keeps float32/float16 amplitudes as given and treats uint16
        arrays as BF16 bit patterns; ``"bf16"``/``"f16"``/``"f32"`` convert
        host arrays first.  ``"f16"`` is the precision form: FP16 with one
        power-of-two scale per trace carried by the trace weight
        (:meth:`to_f16_panel`, which also converts device panels).
    compensated:
        TwoSum-compensated FP32 partial sums between the flushes into the
        image (``True``/``False``); ``"auto"`` compensates for 16-bit traces
        (the precision form) and not for FP32 traces.
    velocity_mode:
        ``"exact"`` uses a 3-D velocity slice per pillar; ``"auto"`` follows the
        Metal host rule (``metal_compiled.py:631-664``): the centre pillar is
        used for every pillar unless the lateral variation exceeds 5 %.
    precision:
        ``"exact"`` forms the sample index in FP64 (the reference Numba path's
        interpolation position and trace-end test); ``"fast"`` uses FP32
        traveltime and re-takes in FP64 the trace-end tests within 0.01
        samples of a trace end; ``"fp32"`` is FP32 throughout (traveltime,
        sample index, trace-end tests), FP64 staying in the coordinate
        differences and the fold test: the precision form's arithmetic.
    """

    def __init__(self, device: int | None = None, trace_dtype: str = "auto",
                 compensated="auto", velocity_mode: str = "exact", precision: str = "exact"):
        self._device = int(os.environ.get("PSTM_CUDA_DEVICE", "0")) if device is None else int(device)
        self._trace_dtype = trace_dtype
        if compensated not in ("auto", True, False):
            raise ValueError("compensated must be 'auto', True or False")
        self._compensated = compensated
        self._velocity_mode = velocity_mode
        modes = {"exact": nat.PREC_EXACT, "fast": nat.PREC_FAST, "fp32": nat.PREC_FP32}
        if precision not in modes:
            raise ValueError("precision must be 'exact', 'fast' or 'fp32'")
        self._precision = modes[precision]
        self._config = None
        self._ctx = None
        self._lib = None

    # ------------------------------------------------------------- protocol
    @property
    def name(self) -> str:
        return "cuda_b200"

    @property
    def capabilities(self) -> set:
        try:  # report the reference's own enum members when it is importable
            from pstm.kernels.base import KernelCapability as RefCap  # type: ignore
            return {RefCap.FP16, RefCap.ASYNC, RefCap.BATCH}
        except Exception:
            return {KernelCapability.FP16, KernelCapability.ASYNC, KernelCapability.BATCH}

    def initialize(self, config) -> None:
        self._lib = nat.load()
        if self._ctx is None:
            h = ctypes.c_void_p()
            rc = self._lib.pstm_cuda_create(self._device, ctypes.byref(h))
            nat.check(rc, None, self._lib)
            self._ctx = h
        self._config = config

    def migrate_tile(self, traces, output, velocity, config=None) -> KernelMetrics:
        return self._migrate(traces, output, velocity, config, nat.TT_STRAIGHT)

    def migrate_tile_curved_ray(self, traces, output, velocity, config=None) -> KernelMetrics:
        return self._migrate(traces, output, velocity, config, nat.TT_CURVED)

    def migrate_tile_vti(self, traces, output, velocity, config=None) -> KernelMetrics:
        return self._migrate(traces, output, velocity, config, nat.TT_VTI)

    def migrate_tile_curved_vti(self, traces, output, velocity, config=None) -> KernelMetrics:
        return self._migrate(traces, output, velocity, config, nat.TT_CURVED_VTI)

    def migrate_tile_time_variant(self, traces, output, velocity, config, windows) -> KernelMetrics:
        """Migrate at the sample times of the time-variant ``windows`` (straight
        rays; the reference's ``migrate_tile_time_variant``,
        ``metal_compiled.py:940-1275``).  As the reference, ``output.image`` is
        replaced by the (nx, ny, n_windowed_samples) image, which the caller
        brings back to the uniform axis with ``time_variant.resample_to_uniform``;
        the fold (per pillar, the same at every time) is added into
        ``output.fold``.  Host arrays or CUDA tensors, like ``migrate_tile``."""
        from . import time_variant as tvm
        from .base import OutputTile, VelocitySlice
        if self._ctx is None or self._config is None:
            raise RuntimeError("Kernel not initialized")
        cfg = config if config is not None else self._config
        t_start = time.perf_counter()
        tv = tvm.window_times(windows)
        if len(tv) == 0:
            raise ValueError("no time windows")
        nx, ny = len(output.x_axis), len(output.y_axis)
        on_dev = _is_torch_cuda(output.image)
        t_out = output.t_axis_ms.cpu().numpy() if _is_torch_cuda(output.t_axis_ms) else np.asarray(output.t_axis_ms)
        v = velocity.vrms
        vt = getattr(velocity, "t_axis_ms", None)
        vt = t_out if vt is None else (vt.cpu().numpy() if _is_torch_cuda(vt) else np.asarray(vt, np.float64))
        is_1d = bool(getattr(velocity, "is_1d", True))
        if is_1d:
            v_np = v.cpu().numpy() if _is_torch_cuda(v) else np.asarray(v, np.float64)
            v_tv = np.interp(tv, vt[:len(v_np)], v_np)
            if on_dev:
                import torch
                v_tv = torch.as_tensor(v_tv, device=output.image.device)
        else:
            v_tv = tvm.interp_rows(v, vt[:v.shape[-1]], tv, ctx=self._ctx if _is_torch_cuda(v) else None)
        if on_dev:
            import torch
            dev = output.image.device
            img = torch.zeros((nx, ny, len(tv)), dtype=output.image.dtype, device=dev)
            fold = torch.zeros((nx, ny), dtype=torch.int32, device=dev)
            t_axis = torch.as_tensor(tv, device=dev)
        else:
            img = np.zeros((nx, ny, len(tv)), dtype=np.asarray(output.image).dtype)
            fold = np.zeros((nx, ny), np.int32)
            t_axis = tv
        tv_out = OutputTile(image=img, fold=fold, x_axis=output.x_axis, y_axis=output.y_axis, t_axis_ms=t_axis,
                            x_grid=getattr(output, "x_grid", None), y_grid=getattr(output, "y_grid", None))
        self._migrate(traces, tv_out, VelocitySlice(vrms=v_tv, is_1d=is_1d), cfg, nat.TT_STRAIGHT)
        output.image = img
        if output.fold is not None:
            if len(output.fold.shape) == 3:
                output.fold += fold[..., None]
            else:
                output.fold += fold
        return KernelMetrics(n_traces_processed=int(traces.amplitudes.shape[0]), n_samples_output=nx * ny * len(tv),
                             compute_time_s=time.perf_counter() - t_start)

    def migrate_tile_learned(self, traces, output, velocity, surrogate, config=None,
                             kernel_type: str = "anisotropic_vti", max_residual_ms: float = 0.1,
                             n_probe: int = 4096):
        """The learned form: probe ``surrogate`` (a ``pstm_b200.surrogate.Net``)
        against the exact traveltime on ``n_probe`` random in-aperture pairs of
        this tile and migrate with it when the largest residual is at most
        ``max_residual_ms`` (negative: always), else with the exact kernel.
        Device tensors only.  Returns (KernelMetrics, report dict)."""
        if self._ctx is None or self._config is None:
            raise RuntimeError("Kernel not initialized")
        if kernel_type not in ("anisotropic_vti", "curved_vti"):
            raise ValueError("the learned form covers anisotropic_vti and curved_vti")
        cfg = config if config is not None else self._config
        t_start = time.perf_counter()
        keep: list = []
        devs: list = []
        td = self._trace_desc(traces, keep, devs)
        od = nat.OutputDesc()
        img = output.image
        if not _is_torch_cuda(img):
            raise ValueError("the learned form takes CUDA tensors")
        import torch
        if img.dtype not in (torch.float64, torch.float32) or not img.is_contiguous():
            raise ValueError("device image must be a contiguous float64/float32 tensor")
        od.image = img.data_ptr()
        od.image_dtype = nat.IMAGE_F64 if img.dtype == torch.float64 else nat.IMAGE_F32
        if output.fold is not None:
            od.fold = output.fold.data_ptr()
            od.fold_is_3d = 1 if len(output.fold.shape) == 3 else 0
            devs.append(_is_torch_cuda(output.fold))
        self._output_axes(output, od, keep, devs)
        vd = nat.VelocityDesc()
        vd.vrms, vd.is_3d, dv = self._velocity(velocity, output, od.nx, od.ny, od.nt, keep)
        devs.append(dv)
        prm = self._params(cfg, _TT_BY_TYPE[kernel_type], keep, devs=devs)
        self._auto_compensation(prm, td)
        if not all(devs):
            raise ValueError("the learned form takes CUDA tensors only")
        net = surrogate.to_struct()
        rep = nat.LearnedReport()
        stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY
        rc = self._lib.pstm_cuda_migrate_tile_learned_dev(self._ctx, ctypes.byref(td), ctypes.byref(od),
                                                          ctypes.byref(vd), ctypes.byref(prm), ctypes.byref(net),
                                                          float(max_residual_ms), int(n_probe), ctypes.byref(rep),
                                                          ctypes.c_void_p(stream))
        nat.check(rc, self._ctx, self._lib)
        report = {"probe_max_ms": rep.probe_max_ms, "probe_rms_ms": rep.probe_rms_ms,
                  "n_probe_used": rep.n_probe_used, "used_surrogate": bool(rep.used_surrogate)}
        return KernelMetrics(n_traces_processed=td.n_traces, n_samples_output=od.nx * od.ny * od.nt,
                             compute_time_s=time.perf_counter() - t_start), report

    def migrate_bins(self, traces, bins, geometry, velocity, config=None,
                     kernel_type: str = "straight_ray") -> KernelMetrics:
        """The batched form; see :func:`migrate_bins`."""
        return migrate_bins(self, traces, bins, geometry, velocity, config, kernel_type)

    def autotune_bins(self, traces, bins, geometry, velocity, config=None, kernel_type: str = "straight_ray",
                      pairs_per_candidate: int = 0) -> dict:
        """The autotuner of the batched form; see :func:`autotune_bins`."""
        return autotune_bins(self, traces, bins, geometry, velocity, config, kernel_type, pairs_per_candidate)

    def synchronize(self) -> None:
        """Wait for this backend's work, then report device-side failures
        (a bounded wait that gave up raises ``PstmCudaError`` with
        ``ERR_TIMEOUT``).  Device-tensor calls run on torch's current stream,
        so that device is synchronised first."""
        if self._ctx is not None:
            import sys
            torch = sys.modules.get("torch")
            if torch is not None and torch.cuda.is_initialized():
                torch.cuda.synchronize(self._device)
            nat.check(self._lib.pstm_cuda_synchronize(self._ctx), self._ctx, self._lib)

    def cleanup(self) -> None:
        if self._ctx is not None:
            self._lib.pstm_cuda_destroy(self._ctx)
        self._ctx = None
        self._config = None

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass

    # ------------------------------------------------------------- internals
    @property
    def context(self):
        return self._ctx

    def _params(self, cfg, tt: int, keep: list, eta_override=None, devs: list | None = None) -> nat.Params:
        p = nat.Params()
        p.max_aperture_m = float(cfg.max_aperture_m)
        p.min_aperture_m = float(cfg.min_aperture_m)
        p.max_dip_degrees = float(cfg.max_dip_degrees)
        p.taper_fraction = float(cfg.taper_fraction)
        p.apply_spreading = int(bool(cfg.apply_spreading))
        p.apply_obliquity = int(bool(cfg.apply_obliquity))
        p.aa_enabled = int(bool(cfg.aa_enabled))
        p.traveltime = int(tt)
        p.aa_dominant_freq = float(getattr(cfg, "aa_dominant_freq", 30.0))
        p.grid_dx = float(getattr(cfg, "grid_dx", 25.0))
        p.grid_dy = float(getattr(cfg, "grid_dy", 12.5))
        p.curved_v0 = float(getattr(cfg, "curved_ray_v0", 1500.0))
        p.curved_k = float(getattr(cfg, "curved_ray_k", 0.5))
        p.eta_constant = float(getattr(cfg, "vti_eta_constant", 0.0))
        p.compensated = 0 if self._compensated == "auto" else int(bool(self._compensated))
        p.precision = self._precision
        p.interpolation = nat.interp_code(getattr(cfg, "interpolation_method", None))
        eta = eta_override if eta_override is not None else getattr(cfg, "vti_eta_array", None)
        if eta is not None and tt in (nat.TT_VTI, nat.TT_CURVED_VTI):
            ptr, on_dev = self._arr(eta, np.float64, keep)
            if devs is not None:
                devs.append(on_dev)
            p.eta = ptr
            p.eta_is_3d = 0 if len(eta.shape) == 1 else 1
        return p

    def _auto_compensation(self, prm, td) -> None:
        """compensated="auto": TwoSum-compensated partial sums for 16-bit traces
        (the precision form), plain FP32 partials for FP32 traces."""
        if self._compensated == "auto":
            prm.compensated = int(td.amp_dtype != nat.AMP_F32)

    def _arr(self, a, dtype, keep: list):
        """(pointer, on_device) for a numpy array or a CUDA torch tensor."""
        if a is None:
            return None, False
        if _is_torch_cuda(a):
            if not a.is_contiguous():
                a = a.contiguous()
                keep.append(a)
            return a.data_ptr(), True
        arr = np.ascontiguousarray(a, dtype=dtype)
        keep.append(arr)
        return arr.ctypes.data, False

    def _amplitudes(self, amps, keep: list):
        if _is_torch_cuda(amps):
            import torch
            code = {torch.float32: nat.AMP_F32, torch.float16: nat.AMP_F16,
                    torch.bfloat16: nat.AMP_BF16}.get(amps.dtype)
            if code is None:
                raise ValueError(f"unsupported amplitude dtype {amps.dtype}")
            if amps.dim() != 2 or amps.stride(1) != 1:
                raise ValueError("amplitudes must be (n_traces, n_samples) with unit sample stride")
            return amps.data_ptr(), code, int(amps.stride(0)), True
        a = np.asarray(amps)
        want = self._trace_dtype
        if want == "bf16" and a.dtype != np.uint16:
            a = float32_to_bf16_bits(a)
        elif want == "f16" and a.dtype != np.float16:
            a = a.astype(np.float16)
        elif want == "f32" and a.dtype != np.float32:
            a = a.astype(np.float32)
        if a.dtype == np.float32:
            code = nat.AMP_F32
        elif a.dtype == np.float16:
            code = nat.AMP_F16
        elif a.dtype == np.uint16:
            code = nat.AMP_BF16
        else:
            a = a.astype(np.float32)
            code = nat.AMP_F32
        if a.ndim != 2 or a.strides[1] != a.itemsize:
            a = np.ascontiguousarray(a)
        keep.append(a)
        stride = a.strides[0] // a.itemsize if a.shape[0] > 1 else a.shape[1]
        return a.ctypes.data, code, max(stride, a.shape[1]), False

    def _velocity(self, velocity, output, nx, ny, nt, keep: list):
        v = velocity.vrms
        is_1d = bool(getattr(velocity, "is_1d", True))
        if _is_torch_cuda(v):
            if (is_1d and tuple(v.shape) != (nt,)) or (not is_1d and tuple(v.shape) != (nx, ny, nt)):
                raise ValueError("device velocity must match the output tile shape")
            if not is_1d and self._velocity_mode == "auto":
                v, use3d = lateral_velocity_choice(v)
                is_1d = not use3d
            return self._arr(v, np.float64, keep)[0], (0 if is_1d else 1), True
        v = np.asarray(v, dtype=np.float64)
        t_out = np.asarray(output.t_axis_ms, dtype=np.float64)
        if is_1d:
            if len(v) != nt:   # numba_cpu_optimized.py:574-578
                vt = getattr(velocity, "t_axis_ms", None)
                vt = t_out if vt is None else np.asarray(vt, dtype=np.float64)
                v = np.interp(t_out, vt, v)
            is3d = 0
        else:
            if v.shape != (nx, ny, nt):
                raise ValueError(f"3-D velocity shape {v.shape} != tile {(nx, ny, nt)}")
            is3d = 1
            if self._velocity_mode == "auto":
                v, use3d = lateral_velocity_choice(v)
                is3d = int(use3d)
        if not np.all(v > 0):
            raise ValueError("velocity must be > 0")
        v = np.ascontiguousarray(v)
        keep.append(v)
        return v.ctypes.data, is3d, False

    def to_f16_panel(self, traces):
        """The precision form of a trace panel: a TraceBlock whose amplitudes
        are FP16 with one power-of-two scale per trace and whose weights carry
        the inverse scales (``pstm_cuda_traces_to_f16``; host arrays follow the
        same rule in NumPy).  Geometry is shared with ``traces``."""
        import dataclasses
        amps = traces.amplitudes
        w = getattr(traces, "weights", None)
        if _is_torch_cuda(amps):
            import torch
            if amps.dtype != torch.float32 or amps.dim() != 2 or amps.stride(1) != 1:
                raise ValueError("to_f16_panel takes (n_traces, n_samples) float32 CUDA amplitudes")
            if self._ctx is None:
                raise RuntimeError("Kernel not initialized")
            n, ns = amps.shape
            out = torch.empty((n, ns), dtype=torch.float16, device=amps.device)
            wout = torch.empty((n,), dtype=torch.float64, device=amps.device)
            win = None
            if w is not None:
                win = torch.as_tensor(w, dtype=torch.float64, device=amps.device).contiguous()
            stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY
            rc = self._lib.pstm_cuda_traces_to_f16(self._ctx, amps.data_ptr(), n, ns, amps.stride(0),
                                                   out.data_ptr(), ns, win.data_ptr() if win is not None else None,
                                                   wout.data_ptr(), ctypes.c_void_p(stream))
            nat.check(rc, self._ctx, self._lib)
            return dataclasses.replace(traces, amplitudes=out, weights=wout)
        a16, inv = scaled_f16(np.asarray(amps, np.float32))
        w = inv if w is None else np.asarray(w, np.float64) * inv
        return dataclasses.replace(traces, amplitudes=a16, weights=w)

    def _trace_desc(self, traces, keep: list, devs: list) -> nat.TracesDesc:
        if self._trace_dtype == "f16" and not _is_torch_cuda(traces.amplitudes) \
                and np.asarray(traces.amplitudes).dtype != np.float16:
            traces = self.to_f16_panel(traces)   # the precision form: per-trace scaled FP16
        amp_ptr, amp_code, amp_stride, amp_dev = self._amplitudes(traces.amplitudes, keep)
        td = nat.TracesDesc()
        td.amplitudes = amp_ptr
        td.amp_dtype = amp_code
        td.n_samples = int(traces.amplitudes.shape[1])
        td.n_traces = int(traces.amplitudes.shape[0])
        td.amp_row_stride = amp_stride
        devs.append(amp_dev)
        for name in ("source_x", "source_y", "receiver_x", "receiver_y", "midpoint_x", "midpoint_y"):
            ptr, d = self._arr(getattr(traces, name), np.float64, keep)
            setattr(td, name, ptr)
            devs.append(d)
        w = getattr(traces, "weights", None)
        if w is not None:
            ptr, d = self._arr(w, np.float64, keep)
            td.weights = ptr
            devs.append(d)
        td.sample_rate_ms = float(traces.sample_rate_ms)
        td.start_time_ms = float(traces.start_time_ms)
        return td

    def _output_axes(self, output, od: nat.OutputDesc, keep: list, devs: list) -> None:
        od.nx, od.ny, od.nt = len(output.x_axis), len(output.y_axis), len(output.t_axis_ms)
        od.x_axis, d1 = self._arr(output.x_axis, np.float64, keep)
        od.y_axis, d2 = self._arr(output.y_axis, np.float64, keep)
        od.t_axis_ms, d3 = self._arr(output.t_axis_ms, np.float64, keep)
        devs += [d1, d2, d3]
        xg, yg = getattr(output, "x_grid", None), getattr(output, "y_grid", None)
        if xg is not None and yg is not None:
            od.x_grid, d4 = self._arr(xg, np.float64, keep)
            od.y_grid, d5 = self._arr(yg, np.float64, keep)
            devs += [d4, d5]

    def migrate_tile_runs(self, traces, runs, output, velocity, config=None,
                          kernel_type: str = "straight_ray") -> KernelMetrics:
        """Migrate one tile against row ranges of a resident panel.

        ``runs`` is an (n, 2) array of [begin, end) row ranges of ``traces``
        (CUDA tensors), ascending and disjoint; the tile receives what
        ``migrate_tile`` would add for the concatenation of the ranges (up to
        the order of floating-point additions), without copying them together.
        A panel in midpoint order (``pstm_b200.spatial``) gives a tile's
        traces as such ranges.  ``kernel_type`` picks the traveltime as the
        executor's dispatch does (``executor.py:1691-1745``).
        """
        if kernel_type not in _TT_BY_TYPE:
            raise ValueError(f"unknown kernel_type {kernel_type!r}")
        r = np.ascontiguousarray(np.asarray(runs, dtype=np.int64).reshape(-1, 2))
        return self._migrate(traces, output, velocity, config, _TT_BY_TYPE[kernel_type], runs=r)

    def migrate_scatter(self, traces, output, velocity, config=None, kernel_type: str = "straight_ray",
                        segment_traces: int = 0, count_items: bool = False) -> KernelMetrics:
        """Migrate an output grid with the trace-centric (scatter) schedule:
        every trace is read once for the whole grid, as in the reference's
        trace-centric kernel (``pstm_trace_centric.metal:112-236``), with the
        gather kernel's partial sums and one atomic add per output sample per
        (segment, pillar block, time block) item.  ``traces`` are CUDA tensors,
        best in midpoint order (``pstm_b200.spatial.sort_panel``); the output
        has a regular grid (ascending ``x_axis``, ``y_axis``).  The result is
        ``migrate_tile``'s up to the order of floating-point additions.  With
        ``count_items`` the call synchronises and the metrics carry the number
        of items in ``n_items``."""
        if kernel_type not in _TT_BY_TYPE:
            raise ValueError(f"unknown kernel_type {kernel_type!r}")
        return self._migrate(traces, output, velocity, config, _TT_BY_TYPE[kernel_type],
                             scatter=(int(segment_traces), bool(count_items)))

    def _migrate(self, traces, output, velocity, config, tt: int, runs=None, scatter=None) -> KernelMetrics:
        if self._ctx is None or self._config is None:
            raise RuntimeError("Kernel not initialized")
        cfg = config if config is not None else self._config
        t_start = time.perf_counter()
        keep: list = []
        nx, ny, nt = len(output.x_axis), len(output.y_axis), len(output.t_axis_ms)
        ntr = int(traces.amplitudes.shape[0])

        devs: list = []
        td = self._trace_desc(traces, keep, devs)

        od = nat.OutputDesc()
        img = output.image
        if _is_torch_cuda(img):
            import torch
            if img.dtype not in (torch.float64, torch.float32) or not img.is_contiguous():
                raise ValueError("device image must be a contiguous float64/float32 tensor")
            od.image = img.data_ptr()
            od.image_dtype = nat.IMAGE_F64 if img.dtype == torch.float64 else nat.IMAGE_F32
            devs.append(True)
        else:
            if not isinstance(img, np.ndarray) or img.dtype not in (np.float64, np.float32) \
                    or not img.flags["C_CONTIGUOUS"]:
                raise ValueError("image must be a C-contiguous float64/float32 array")
            od.image = img.ctypes.data
            od.image_dtype = nat.IMAGE_F64 if img.dtype == np.float64 else nat.IMAGE_F32
            devs.append(False)
        if tuple(img.shape) != (nx, ny, nt):
            raise ValueError(f"image shape {tuple(img.shape)} != {(nx, ny, nt)}")
        fold = output.fold
        if fold is not None:
            if _is_torch_cuda(fold):
                od.fold = fold.data_ptr()
                devs.append(True)
            else:
                if not isinstance(fold, np.ndarray) or fold.dtype != np.int32 or not fold.flags["C_CONTIGUOUS"]:
                    raise ValueError("fold must be a C-contiguous int32 array")
                od.fold = fold.ctypes.data
                devs.append(False)
            od.fold_is_3d = 1 if len(fold.shape) == 3 else 0
        self._output_axes(output, od, keep, devs)

        vd = nat.VelocityDesc()
        vd.vrms, vd.is_3d, dv = self._velocity(velocity, output, nx, ny, nt, keep)
        devs.append(dv)
        prm = self._params(cfg, tt, keep, devs=devs)
        self._auto_compensation(prm, td)

        on_dev = all(devs)
        if any(devs) and not on_dev:
            raise ValueError("mixing device tensors and host arrays in one call is not supported")
        if runs is not None:
            if not on_dev:
                raise ValueError("migrate_tile_runs takes CUDA tensors only")
            import torch
            stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY
            rc = self._lib.pstm_cuda_migrate_tile_runs_dev(
                self._ctx, ctypes.byref(td), runs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(runs),
                ctypes.byref(od), ctypes.byref(vd), ctypes.byref(prm), ctypes.c_void_p(stream))
            nat.check(rc, self._ctx, self._lib)
            return KernelMetrics(n_traces_processed=int((runs[:, 1] - runs[:, 0]).sum()) if len(runs) else 0,
                                 n_samples_output=nx * ny * nt, compute_time_s=time.perf_counter() - t_start)
        if scatter is not None:
            if not on_dev:
                raise ValueError("migrate_scatter takes CUDA tensors only")
            import torch
            stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY
            n_items = ctypes.c_int64(0)
            rc = self._lib.pstm_cuda_migrate_scatter_dev(
                self._ctx, ctypes.byref(td), scatter[0], ctypes.byref(od), ctypes.byref(vd), ctypes.byref(prm),
                ctypes.byref(n_items) if scatter[1] else None, ctypes.c_void_p(stream))
            nat.check(rc, self._ctx, self._lib)
            m = KernelMetrics(n_traces_processed=ntr, n_samples_output=nx * ny * nt,
                              compute_time_s=time.perf_counter() - t_start)
            if scatter[1]:
                m.n_items = int(n_items.value)
            return m
        if on_dev:
            import torch   # order the launch after the producers of the caller's tensors
            stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY
            rc = self._lib.pstm_cuda_migrate_tile_dev(self._ctx, ctypes.byref(td), ctypes.byref(od),
                                                      ctypes.byref(vd), ctypes.byref(prm),
                                                      ctypes.c_void_p(stream))
        else:
            rc = self._lib.pstm_cuda_migrate_tile_host(self._ctx, ctypes.byref(td), ctypes.byref(od),
                                                       ctypes.byref(vd), ctypes.byref(prm))
        nat.check(rc, self._ctx, self._lib)
        return KernelMetrics(n_traces_processed=ntr, n_samples_output=nx * ny * nt,
                             compute_time_s=time.perf_counter() - t_start)


class Bin:
    """One output of the batched form: traces [trace_begin, trace_begin +
    n_traces) of the batch's trace block, migrated into its own image (and
    fold).  Reference: one gather bin of ``executor.py:960-975``."""

    def __init__(self, trace_begin: int, n_traces: int, image, fold=None):
        self.trace_begin = int(trace_begin)
        self.n_traces = int(n_traces)
        self.image = image
        self.fold = fold


def _batch_descs(kernel: "CudaKernel", traces, bins, geometry, velocity, config, kernel_type: str):
    """Descriptors of a batched call (device tensors only)."""
    if kernel._ctx is None or kernel._config is None:
        raise RuntimeError("Kernel not initialized")
    if kernel_type not in _TT_BY_TYPE:
        raise ValueError(f"unknown kernel_type {kernel_type!r}")
    import torch
    cfg = config if config is not None else kernel._config
    keep: list = []
    devs: list = []
    td = kernel._trace_desc(traces, keep, devs)
    od = nat.OutputDesc()
    kernel._output_axes(geometry, od, keep, devs)
    nx, ny, nt = od.nx, od.ny, od.nt
    vd = nat.VelocityDesc()
    vd.vrms, vd.is_3d, dv = kernel._velocity(velocity, geometry, nx, ny, nt, keep)
    devs.append(dv)
    prm = kernel._params(cfg, _TT_BY_TYPE[kernel_type], keep, devs=devs)
    kernel._auto_compensation(prm, td)
    if not all(devs):
        raise ValueError("the batched form takes CUDA tensors only (traces, axes, velocity and eta)")
    arr = (nat.BinDesc * max(1, len(bins)))()
    img_dtype = None
    fold3 = None
    for i, b in enumerate(bins):
        img = b.image
        if not _is_torch_cuda(img) or not img.is_contiguous() or img.dtype not in (torch.float64, torch.float32):
            raise ValueError(f"bin {i}: image must be a contiguous float64/float32 CUDA tensor")
        if tuple(img.shape) != (nx, ny, nt):
            raise ValueError(f"bin {i}: image shape {tuple(img.shape)} != {(nx, ny, nt)}")
        if img_dtype is None:
            img_dtype = img.dtype
        elif img.dtype != img_dtype:
            raise ValueError("all bins' images must have one dtype")
        arr[i].trace_begin, arr[i].n_traces, arr[i].image = b.trace_begin, b.n_traces, img.data_ptr()
        if b.fold is not None:
            f = b.fold
            if not _is_torch_cuda(f) or f.dtype != torch.int32 or not f.is_contiguous():
                raise ValueError(f"bin {i}: fold must be a contiguous int32 CUDA tensor")
            shape = (nx, ny, nt) if len(f.shape) == 3 else (nx, ny)
            if tuple(f.shape) != shape or (fold3 is not None and fold3 != (len(shape) == 3)):
                raise ValueError(f"bin {i}: fold must be (nx, ny, nt) or (nx, ny), the same for every bin")
            fold3 = len(shape) == 3
            arr[i].fold = f.data_ptr()
    od.fold_is_3d = 1 if fold3 else 0
    od.image_dtype = nat.IMAGE_F32 if img_dtype == torch.float32 else nat.IMAGE_F64
    keep.append(arr)
    return td, od, vd, prm, arr, keep


def migrate_bins(kernel: "CudaKernel", traces, bins, geometry, velocity, config=None,
                 kernel_type: str = "straight_ray") -> KernelMetrics:
    """Migrate many bins sharing one tile geometry in ONE persistent launch
    (replayed from a CUDA graph while the arguments repeat).

    ``traces`` holds every bin's traces (CUDA tensors), ``bins`` is a list of
    :class:`Bin`, ``geometry`` gives the tile axes (an ``OutputTile``; its own
    image is not used).  Replaces the executor's per-bin loop of
    ``migrate_tile`` calls (``executor.py:960-975``).  Asynchronous on the
    current torch stream; ``kernel.synchronize()`` reports kernel-side errors.
    """
    import torch
    t0 = time.perf_counter()
    td, od, vd, prm, arr, keep = _batch_descs(kernel, traces, bins, geometry, velocity, config, kernel_type)
    stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY
    rc = kernel._lib.pstm_cuda_migrate_bins_dev(kernel._ctx, ctypes.byref(td), ctypes.byref(od), ctypes.byref(vd),
                                                ctypes.byref(prm), arr, len(bins), ctypes.c_void_p(stream))
    nat.check(rc, kernel._ctx, kernel._lib)
    return KernelMetrics(n_traces_processed=sum(b.n_traces for b in bins),
                         n_samples_output=od.nx * od.ny * od.nt * len(bins),
                         compute_time_s=time.perf_counter() - t0)


def autotune_bins(kernel: "CudaKernel", traces, bins, geometry, velocity, config=None,
                  kernel_type: str = "straight_ray", pairs_per_candidate: int = 0) -> dict:
    """Time the candidate launch shapes of the batched form on a sample of
    this batch and keep the fastest in the kernel's context (later
    :func:`migrate_bins` calls of the same workload class use it)."""
    import torch
    torch.cuda.synchronize()
    td, od, vd, prm, arr, keep = _batch_descs(kernel, traces, bins, geometry, velocity, config, kernel_type)
    res = nat.TuneResult()
    rc = kernel._lib.pstm_cuda_autotune_bins(kernel._ctx, ctypes.byref(td), ctypes.byref(od), ctypes.byref(vd),
                                             ctypes.byref(prm), arr, len(bins), int(pairs_per_candidate),
                                             ctypes.byref(res))
    nat.check(rc, kernel._ctx, kernel._lib)
    return {"pillars_per_cta": res.pillars_per_cta, "times_per_lane": res.times_per_lane,
            "traces_per_chunk": res.traces_per_chunk, "n_candidates": res.n_candidates,
            "best_ms": res.best_ms, "default_ms": res.default_ms}


def create_cuda_kernel(**kw) -> CudaKernel:
    """Factory in the style of ``create_optimized_numba_kernel``."""
    return CudaKernel(**kw)
