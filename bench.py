#!/usr/bin/env python
"""Throughput of the CUDA Kirchhoff PSTM backend, in migrated sample-trace pairs/s.

Workload (default ``c2tile``): the production-tile case -- 1,048,576 traces of
1500 samples at 2 ms with random source/receiver positions in a 3.2 x 3.2 km
patch, output bins of 12.5 m with 1500 samples at 2 ms, laterally varying
v_rms(t,x,y), triangle AA on, reference default 5 km aperture (every trace is
inside it).  One step is one ``migrate_tile`` call: a 64 x 64-pillar tile of the
256 x 256 output grid against the whole trace panel (6.44e12 sample-trace
pairs), the unit of work the reference executor hands a backend.  Successive
steps walk the 16 tiles of the grid; with N GPUs rank r takes tiles r, r+N, ...
(disjoint outputs, no collective on the data path: weak scaling).

``value``      device-resident inputs, timed with CUDA events on the launch stream.
``e2e``        through the public backend (``CudaKernel.migrate_tile``) with
               pinned host arrays: every step copies the panel, geometry,
               velocity and image/fold in and the image/fold out.
``cpu_baseline`` the FP64 CPU oracle (a port of the reference algorithm) on a
               bounded sample of the same workload, on this host's cores.
``--impl reference`` times that CPU port alone, as the reference arm.

Inputs are larger than L2 (the FP32 panel is 6.3 GB), so no L2 flush is needed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "migrated sample-trace pairs/s"
UNIT = "pairs/s"

# algorithmic work per sample-trace pair of the straight-ray kernel with AA on
# (16 FP32 FLOP + 3 MUFU for DSR, interpolation and weights; AA adds 4 + 1)
FLOP_PER_PAIR = 20
MUFU_PER_PAIR = 4

# DRAM traffic of one 64 x 64 x 1500 tile launch per trace of the panel, from an
# ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of one launch over
# 262,144 traces (a 1.6 GB panel, 24 MiB trace segments): 16.23 + 5.02 GB.  The
# segment-major schedule reads each segment and re-adds the tile once per
# segment, so the traffic grows with the trace count; scaled per trace.
DRAM_BYTES_PER_TRACE_TILE64 = 21.25e9 / 262144


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--dtype", choices=["f32", "bf16", "f16"], default="f32")
    ap.add_argument("--precision", choices=["exact", "fast", "fp32"], default="exact")
    ap.add_argument("--traces", type=int, default=1 << 20)
    ap.add_argument("--tile", type=int, default=64)
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="tiles timed end to end (0: the first min(steps, 4) tiles of the timed device steps)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the precision-form measurement")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-form measurement")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-form measurement")
    ap.add_argument("--learned-steps", type=int, default=60000, help="Adam steps of the surrogate training")
    ap.add_argument("--case5", action="store_true",
                    help="run the large-survey case (512x512x2000, FP16 traces, curved+VTI) instead")
    ap.add_argument("--case5-tiles", type=int, default=2, help="64x64 tiles of the case-5 grid to migrate")
    ap.add_argument("--no-case5", action="store_true", help="skip the case-5 line of the default run")
    ap.add_argument("--no-streaming", action="store_true", help="skip the streaming-executor part of case 5")
    ap.add_argument("--no-scatter", action="store_true", help="skip the scatter-vs-gather line")
    ap.add_argument("--case5-aperture", type=float, default=1000.0, help="max aperture (m) of the case-5 run")
    ap.add_argument("--no-numba", action="store_true", help="skip the reference's Numba CPU leg")
    ap.add_argument("--numba-leg", default=None, help=argparse.SUPPRESS)   # internal: the child process
    ap.add_argument("--batch-scale", type=int, default=1,
                    help="the batched form migrates 1/this of every bin's traces (1: the full ~2M traces)")
    return ap.parse_args()


# ------------------------------------------------------------------ workload
GRID, NT, NS, DT_MS, DX = 256, 1500, 1500, 2.0, 12.5


def tiles_of(tile):
    from pstm_b200 import replicas
    return replicas.grid_tiles(GRID, GRID, tile)


def config():
    from pstm_b200 import workloads
    return workloads.survey_config(kernel_type="straight_ray", aa=True, dx=DX)


def measured_sfu_peak(device: int) -> float:
    """MUFU operations/s of this GPU from the library's throughput kernel (0 on failure)."""
    import ctypes
    from pstm_b200 import _native as nat
    L = nat.load()
    v = ctypes.c_double(0.0)
    if L.pstm_cuda_measure_sfu_peak(device, ctypes.byref(v)) != nat.OK:
        return 0.0
    return float(v.value)


# ------------------------------------------------------------------ the reference's Numba path
REF_PKG = os.path.join(ROOT, "baseline", "_ref")
C2_SAMPLE = dict(n_traces=1 << 16, pillars=16)   # labelled case-2 sample of the Numba leg


def c2_numba_sample():
    """The case-2 sample the reference's Numba kernel can run: the first 65,536
    traces of the seeded case-2 survey (1500 samples at 2 ms), the 16 x 16
    pillars at the centre of the grid x 1500 output samples, the centre
    pillar's v_rms as a 1-D velocity (Numba takes no 3-D velocity), AA off
    (Numba has none), reference defaults otherwise (5 km aperture, 45 deg dip).
    Returns (traces, x_axis, y_axis, t_axis, vrms, config) as plain arrays."""
    from pstm_b200 import workloads
    n, pb = C2_SAMPLE["n_traces"], C2_SAMPLE["pillars"]
    sv = workloads.survey(n, GRID, GRID, NT, DT_MS, NS, dx=DX, seed=7)
    c0 = GRID // 2 - pb // 2
    xa, ya = sv.x_axis[c0:c0 + pb].copy(), sv.y_axis[c0:c0 + pb].copy()
    v = np.ascontiguousarray(sv.velocity(GRID // 2, GRID // 2 + 1, GRID // 2, GRID // 2 + 1)[0, 0])
    cfg = workloads.survey_config(kernel_type="straight_ray", aa=False, dx=DX)
    return sv, xa, ya, sv.t_axis_ms.copy(), v, cfg


def _to_reference(rb, amps, sx, sy, rx, ry, dt_ms, xa, ya, ta, vrms, cfg):
    import dataclasses
    tb = rb.create_trace_block(np.ascontiguousarray(amps, np.float32), sx, sy, rx, ry, sample_rate_ms=dt_ms,
                               start_time_ms=0.0)
    out = rb.OutputTile(image=np.zeros((len(xa), len(ya), len(ta))), fold=np.zeros((len(xa), len(ya), len(ta)),
                                                                                      np.int32),
                        x_axis=xa, y_axis=ya, t_axis_ms=ta)
    vel = rb.VelocitySlice(vrms=np.ascontiguousarray(vrms, np.float64), is_1d=True)
    names = {f.name for f in dataclasses.fields(rb.KernelConfig)}
    kw = {f.name: getattr(cfg, f.name) for f in dataclasses.fields(cfg) if f.name in names}
    return tb, out, vel, rb.KernelConfig(**kw)


def numba_leg_child(outdir):
    """Child process of :func:`numba_reference`: times the reference's own
    registered CPU backend, OptimizedNumbaKernel.migrate_tile
    (pstm/kernels/numba_cpu_optimized.py:545-626), from the installed reference
    in baseline/_ref, on every host core, after a JIT warm-up call with the
    same array ranks; saves its images for the parity check."""
    sys.path.insert(0, REF_PKG)
    import numba
    from pstm.kernels import base as rb
    from pstm.kernels.numba_cpu_optimized import OptimizedNumbaKernel
    from pstm_b200 import workloads
    numba.set_num_threads(os.cpu_count())
    res = {"threads": numba.get_num_threads(), "cores": os.cpu_count(), "numba": numba.__version__,
           "cpu_model": _cpu_model()}
    case = workloads.config1()
    tbc = case.traces
    args1 = (tbc.amplitudes, tbc.source_x, tbc.source_y, tbc.receiver_x, tbc.receiver_y, tbc.sample_rate_ms,
             case.output.x_axis, case.output.y_axis, case.output.t_axis_ms, case.velocity.vrms, case.config)
    k = OptimizedNumbaKernel()
    # warm-up: the same array ranks (3-D fold) on 2 x 2 pillars and 64 traces
    w = _to_reference(rb, tbc.amplitudes[:64], tbc.source_x[:64], tbc.source_y[:64], tbc.receiver_x[:64],
                      tbc.receiver_y[:64], tbc.sample_rate_ms, case.output.x_axis[:2], case.output.y_axis[:2],
                      case.output.t_axis_ms, case.velocity.vrms, case.config)
    t0 = time.perf_counter()
    k.initialize(w[3])
    k.migrate_tile(*w)
    res["jit_warmup_s"] = time.perf_counter() - t0
    tb, out, vel, cfg = _to_reference(rb, *args1)
    k.initialize(cfg)
    t0 = time.perf_counter()
    k.migrate_tile(tb, out, vel, cfg)
    dt = time.perf_counter() - t0
    res["case1"] = {"value": case.pairs / dt, "unit": UNIT, "seconds": dt, "pairs": case.pairs,
                    "workload": "case 1 in full: 64x64x500 @4 ms, 16,384 FP32 traces x 500, straight rays, "
                                "1000 m aperture, 60 deg dip, weights on, AA off"}
    np.savez(os.path.join(outdir, "numba_case1.npz"), image=out.image, fold=out.fold)
    sv, xa, ya, ta, v, c2cfg = c2_numba_sample()
    tb, out, vel, cfg = _to_reference(rb, sv.amps, sv.s[:, 0], sv.s[:, 1], sv.r[:, 0], sv.r[:, 1], DT_MS, xa, ya,
                                      ta, v, c2cfg)
    k.initialize(cfg)
    t0 = time.perf_counter()
    k.migrate_tile(tb, out, vel, cfg)
    dt = time.perf_counter() - t0
    pairs = len(xa) * len(ya) * len(ta) * sv.amps.shape[0]
    res["case2_sample"] = {"value": pairs / dt, "unit": UNIT, "seconds": dt, "pairs": pairs,
                           "workload": f"case-2 sample: {len(xa)}x{len(ya)} centre pillars x {len(ta)} @2 ms, "
                                       f"{sv.amps.shape[0]} traces x {NS}; centre-pillar 1-D v_rms, AA off "
                                       "(Numba supports neither 3-D velocity nor AA), 5 km aperture"}
    np.savez(os.path.join(outdir, "numba_case2_sample.npz"), image=out.image, fold=out.fold)
    k.cleanup()
    print("NUMBA_LEG " + json.dumps(res), flush=True)


def numba_comparison(outdir):
    """The reference's Numba path beside the CUDA kernel on the same inputs:
    its timings (child process, all host cores) and, on the GPU, the CUDA
    backend on the identical case-1 tile and case-2 sample -- rate (CUDA
    events, device-resident inputs), fold equality and image relative L2
    against the Numba images."""
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.cuda_kernel import CudaKernel
    res = numba_reference(outdir)
    if "unavailable" in res:
        return res
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")

    def cuda_run(amps, sx, sy, rx, ry, dt_ms, xa, ya, ta, vrms, cfg, reps):
        mx, my = (sx + rx) / 2.0, (sy + ry) / 2.0
        tb = TraceBlock(amplitudes=dev(np.asarray(amps, np.float32)), source_x=dev(sx), source_y=dev(sy),
                        receiver_x=dev(rx), receiver_y=dev(ry), offset=dev(np.hypot(rx - sx, ry - sy)),
                        midpoint_x=dev(mx), midpoint_y=dev(my), sample_rate_ms=dt_ms, start_time_ms=0.0)
        shape = (len(xa), len(ya), len(ta))
        mk = lambda: OutputTile(image=torch.zeros(shape, dtype=torch.float64, device="cuda"),
                                fold=torch.zeros(shape, dtype=torch.int32, device="cuda"), x_axis=dev(xa),
                                y_axis=dev(ya), t_axis_ms=dev(ta))
        vel = VelocitySlice(vrms=dev(vrms), is_1d=True)
        k = CudaKernel()
        k.initialize(cfg)
        o = mk()
        k.migrate_tile(tb, o, vel)   # the compared result (one call)
        k.synchronize()
        img, fold = o.image.cpu().numpy(), o.fold.cpu().numpy()
        scratch = mk()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            k.migrate_tile(tb, scratch, vel)
        e1.record()
        torch.cuda.synchronize()
        k.cleanup()
        return img, fold, e0.elapsed_time(e1) / reps

    def compare(name, img, fold):
        z = np.load(os.path.join(outdir, name))
        ref = z["image"]
        return {"fold_equal": bool(np.array_equal(fold, z["fold"])),
                "image_rel_l2": float(np.linalg.norm(img - ref) / np.linalg.norm(ref))}

    case = workloads.config1()
    tb = case.traces
    img, fold, ms = cuda_run(tb.amplitudes, tb.source_x, tb.source_y, tb.receiver_x, tb.receiver_y,
                             tb.sample_rate_ms, case.output.x_axis, case.output.y_axis, case.output.t_axis_ms,
                             case.velocity.vrms, case.config, 10)
    res["case1"]["cuda"] = {"value": case.pairs / (ms / 1e3), "ms": ms, **compare("numba_case1.npz", img, fold)}
    res["case1"]["cuda_over_numba"] = res["case1"]["cuda"]["value"] / res["case1"]["value"]
    sv, xa, ya, ta, v, cfg = c2_numba_sample()
    img, fold, ms = cuda_run(sv.amps, sv.s[:, 0], sv.s[:, 1], sv.r[:, 0], sv.r[:, 1], DT_MS, xa, ya, ta, v, cfg, 5)
    c2 = res["case2_sample"]
    c2["cuda"] = {"value": c2["pairs"] / (ms / 1e3), "ms": ms, **compare("numba_case2_sample.npz", img, fold)}
    c2["cuda_over_numba"] = c2["cuda"]["value"] / c2["value"]
    return res


def _cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def numba_reference(outdir, timeout_s=900):
    """Run :func:`numba_leg_child` in a fresh process (Numba's thread pool and
    torch's stay apart); None when the reference is not installed."""
    if not os.path.isdir(os.path.join(REF_PKG, "pstm")):
        return {"unavailable": "the reference is not installed in baseline/_ref"}
    env = dict(os.environ, NUMBA_NUM_THREADS=str(os.cpu_count()), PYTHONDONTWRITEBYTECODE="1",
               NUMBA_CACHE_DIR=os.path.join(outdir, "numba_cache"))
    try:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--numba-leg", outdir], env=env,
                           capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"the Numba leg exceeded {timeout_s} s"}
    for line in r.stdout.splitlines():
        if line.startswith("NUMBA_LEG "):
            return json.loads(line[len("NUMBA_LEG "):])
    return {"unavailable": f"the Numba leg failed (rc {r.returncode}): {r.stderr.strip()[-300:]}"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU legs
def cpu_sample(sv, cfg, tile, n_traces, pillars_x, pillars_y, amps_host):
    """Time the FP64 oracle on pillars [0:px, 0:py] of the first tile x n_traces."""
    from oracle import oracle
    from pstm_b200.base import create_trace_block
    ix0, _, iy0, _ = tile
    out, vel = sv.tile(ix0, ix0 + pillars_x, iy0, iy0 + pillars_y)
    tb = create_trace_block(amps_host[:n_traces], sv.s[:n_traces, 0], sv.s[:n_traces, 1],
                            sv.r[:n_traces, 0], sv.r[:n_traces, 1], sample_rate_ms=DT_MS)
    t0 = time.perf_counter()
    oracle.migrate(tb, out, vel, cfg)
    dt = time.perf_counter() - t0
    pairs = pillars_x * pillars_y * NT * n_traces
    return pairs / dt, pairs, dt


def reference_arm(args):
    """The reference algorithm on the host cores (the CPU port), rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    from pstm_b200 import workloads
    oracle.build()
    n_tr = 1 << 18
    sv = workloads.survey(n_tr, GRID, GRID, NT, DT_MS, NS, dx=DX, seed=7)
    cfg = config()
    tile = tiles_of(args.tile)[0]
    cores = os.cpu_count()
    px, py = 4, 4
    for _ in range(args.warmup):
        cpu_sample(sv, cfg, tile, n_tr, px, py, sv.amps)
    rates, secs = [], 0.0
    for _ in range(args.steps):
        r, pairs, dt = cpu_sample(sv, cfg, tile, n_tr, px, py, sv.amps)
        rates.append(r)
        secs += dt
    value = args.steps * pairs / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "case-2 production tile (256x256x1500 @12.5 m/2 ms, 1,048,576 traces x 1500, "
                               "3-D v_rms, AA on), CPU sample per step", "parallelism": "openmp"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{px}x{py} pillars x {NT} samples x {n_tr} traces per step (FP64 C port "
                                   "of the reference Numba/Metal semantics, OpenMP, all host threads)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ forms
def accuracy_vs_fp64(kernel_factory, sv, cfg, n_tr, amps_host, pillars=2):
    """Relative L2 of a form against the FP64 oracle on a pillars x pillars x nt
    sample of the first tile against the first n_tr traces (host arrays)."""
    from oracle import oracle
    from pstm_b200.base import create_trace_block
    out, vel = sv.tile(20, 20 + pillars, 20, 20 + pillars)
    tb = create_trace_block(amps_host[:n_tr], sv.s[:n_tr, 0], sv.s[:n_tr, 1], sv.r[:n_tr, 0], sv.r[:n_tr, 1],
                            sample_rate_ms=DT_MS)
    ref_out, _ = sv.tile(20, 20 + pillars, 20, 20 + pillars)
    oracle.migrate(tb, ref_out, vel, cfg)
    k = kernel_factory()
    k.initialize(cfg)
    k.migrate_tile(tb, out, vel)
    k.cleanup()
    return float(np.linalg.norm(out.image - ref_out.image) / np.linalg.norm(ref_out.image))


def measure_forms(args, k_plain, tb, amps, tile_args, my_tiles, pairs_per_step, world, dist, sv, cfg):
    """Plain form (exact sample index, FP32 traces) and the precision form (FP16
    traces with a power-of-two scale per trace carried by the trace weight,
    FP32 traveltime, sample index and trace-end tests, compensated FP32
    accumulation; the FP32-arithmetic kernel on FP32 traces, FP16 with the
    FP64 sample index or with FP64 trace-end re-decisions, and BF16 beside
    it): pairs/s on the timed tiles of the full case-2 panel and rel-L2 vs
    the FP64 oracle on the FP32 traces."""
    import dataclasses
    import torch
    from oracle import oracle
    from pstm_b200 import replicas
    from pstm_b200.cuda_kernel import CudaKernel
    oracle.build()
    n_acc = 1 << 17
    amps_host = amps[:n_acc].float().cpu().numpy()
    res = {}
    specs = [("plain_exact_f32", "f32", "exact"), ("precision_f16_fp32", "f16", "fp32"),
             ("fp32_arithmetic_f32", "f32", "fp32"), ("precision_f16_exact", "f16", "exact"),
             ("precision_f16_fast", "f16", "fast"), ("precision_bf16_fast", "bf16", "fast")]
    f32_tb = tb if amps.dtype == torch.float32 else dataclasses.replace(tb, amplitudes=amps.float())
    f16_tb = None
    for name, dt, prec in specs:
        tdt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[dt]
        kf = CudaKernel(precision=prec)
        kf.initialize(cfg)
        if dt == "f16":   # the precision form's format, converted once on the device
            if f16_tb is None:
                f16_tb = kf.to_f16_panel(f32_tb)
            tbf = f16_tb
        else:
            tbf = tb if tdt == amps.dtype else dataclasses.replace(tb, amplitudes=amps.to(tdt))
        kf.migrate_tile(tbf, *tile_args[my_tiles[0]])
        torch.cuda.synchronize()
        steps = min(2, args.steps)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for j in range(args.warmup, args.warmup + steps):
            kf.migrate_tile(tbf, *tile_args[my_tiles[j]])
        e1.record()
        torch.cuda.synchronize()
        ms = replicas.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda")
        kf.cleanup()
        # the FP64 oracle is fed the FP32 traces; the CUDA form converts them itself
        err = accuracy_vs_fp64(lambda: CudaKernel(precision=prec, trace_dtype=dt), sv, cfg, n_acc, amps_host)
        res[name] = {"value": world * steps * pairs_per_step / (ms / 1e3), "unit": UNIT,
                     "trace_dtype": dt + ("_scaled_per_trace" if dt == "f16" else ""), "traveltime": prec,
                     "steps": steps, "rel_l2_vs_fp64": err, "meets_1e-3": bool(err <= 1e-3),
                     "rel_l2_sample": f"2x2 pillars x {NT} samples x {n_acc} traces, FP64 oracle on FP32 traces"}
    plain = res["plain_exact_f32"]["value"]
    for name in res:
        res[name]["vs_plain_exact_f32"] = res[name]["value"] / plain
    return res


def measure_case1_interp(method: str = "sinc8", precision: str = "exact"):
    """The case-1 tile with a higher-order trace interpolator instead of
    linear: pairs/s on device inputs.  precision "exact" runs the FP64
    interpolation kernel, "fast" its FP64-index / FP32-tap variant."""
    import dataclasses
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.cuda_kernel import CudaKernel
    case = workloads.config1()
    tb, out = case.traces, case.output
    cfg = dataclasses.replace(case.config, interpolation_method=method)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    o = OutputTile(image=torch.zeros(out.image.shape, dtype=torch.float64, device="cuda"),
                   fold=torch.zeros(out.fold.shape, dtype=torch.int32, device="cuda"),
                   x_axis=dev(out.x_axis), y_axis=dev(out.y_axis), t_axis_ms=dev(out.t_axis_ms))
    vel = VelocitySlice(vrms=dev(case.velocity.vrms), is_1d=True)
    k = CudaKernel(precision=precision)
    k.initialize(cfg)
    k.migrate_tile(dtb, o, vel, cfg)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    k.migrate_tile(dtb, o, vel, cfg)
    e1.record()
    torch.cuda.synchronize()
    k.cleanup()
    ms = e0.elapsed_time(e1)
    return {"value": case.pairs / (ms / 1e3), "unit": UNIT, "ms_per_tile": ms, "interpolation": method,
            "precision": precision,
            "workload": "case 1 tile with the higher-order interpolation kernel "
                        + ("(FP64 throughout)" if precision == "exact" else "(FP64 index, FP32 taps and weights)")}


def measure_case1():
    """The CPU-runnable case: 64 x 64 bins at 25 m x 500 samples at 4 ms against
    16,384 FP32 traces of 500 samples (3.36e10 pairs), straight rays, aperture
    1000 m, weights on, AA off; device-resident inputs, CUDA events."""
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.cuda_kernel import CudaKernel
    case = workloads.config1()
    tb, out = case.traces, case.output
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    o = OutputTile(image=torch.zeros(out.image.shape, dtype=torch.float64, device="cuda"),
                   fold=torch.zeros(out.fold.shape, dtype=torch.int32, device="cuda"),
                   x_axis=dev(out.x_axis), y_axis=dev(out.y_axis), t_axis_ms=dev(out.t_axis_ms))
    vel = VelocitySlice(vrms=dev(case.velocity.vrms), is_1d=True)
    k = CudaKernel()
    k.initialize(case.config)
    for _ in range(3):
        k.migrate_tile(dtb, o, vel)
    torch.cuda.synchronize()
    reps = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        k.migrate_tile(dtb, o, vel)
    e1.record()
    torch.cuda.synchronize()
    k.cleanup()
    ms = e0.elapsed_time(e1) / reps
    return {"value": case.pairs / (ms / 1e3), "unit": UNIT, "ms_per_tile": ms, "pairs": case.pairs,
            "workload": "case 1: 64x64x500 tile, 16,384 FP32 traces x 500 @4 ms, straight exact, AA off",
            "l2": "inputs (33 MB) fit in L2; consecutive calls on the same tile"}


def measure_batched(args, world, dist, scale: int = 1, per_bin_compare: bool = True):
    """The batched form on the common-offset case: 40 offset bins over 0-4 km,
    lognormal trace counts between 5k and 200k (about 2M), 1000 BF16 samples at
    4 ms, each bin into its own 128 x 128 x 1000 FP32 image, VTI traveltime with
    the case-2 velocity and eta(t0).  All bins in one persistent, graph-replayed
    launch with the autotuned shape, against the same bins as one per-tile call
    each (the reference's bin loop).  Every bin keeps 1/scale of its traces
    (the first ones); at scale 1 the full case (~2M traces, one ~100 s launch)
    is timed once and the per-bin comparison is left to a reduced run."""
    import torch
    from oracle import oracle
    from pstm_b200 import replicas, workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice, create_trace_block
    from pstm_b200.cuda_kernel import Bin, CudaKernel
    rank = int(os.environ.get("RANK", "0"))
    nx = ny = 128
    nt, ns, dt_ms = 1000, 1000, 4.0
    full = workloads.offset_bin_counts(40, 5000, 200000, 2_000_000, seed=4)
    counts = np.maximum(1, full // max(1, scale))
    bs = workloads.binned_survey(counts, nx, ny, nt, dt_ms, ns, dx=DX, bin_width_m=100.0, seed=40 + rank,
                                 device="cuda", dtype=torch.bfloat16)
    sv = bs.survey
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    mx, my = (sv.s[:, 0] + sv.r[:, 0]) / 2.0, (sv.s[:, 1] + sv.r[:, 1]) / 2.0
    tb = TraceBlock(amplitudes=bs.amps_device, source_x=dev(sv.s[:, 0]), source_y=dev(sv.s[:, 1]),
                    receiver_x=dev(sv.r[:, 0]), receiver_y=dev(sv.r[:, 1]),
                    offset=dev(np.hypot(sv.r[:, 0] - sv.s[:, 0], sv.r[:, 1] - sv.s[:, 1])),
                    midpoint_x=dev(mx), midpoint_y=dev(my), sample_rate_ms=dt_ms, start_time_ms=0.0)
    geom = OutputTile(image=None, fold=None, x_axis=dev(sv.x_axis), y_axis=dev(sv.y_axis), t_axis_ms=dev(sv.t_axis_ms))
    vel = VelocitySlice(vrms=dev(sv.velocity()), is_1d=False)
    eta = workloads.survey_eta(sv.t_axis_ms)
    cfg = workloads.survey_config(kernel_type="anisotropic_vti", aa=True, dx=DX, eta=eta)
    cfg.vti_eta_array = dev(eta)
    imgs = [torch.zeros((nx, ny, nt), dtype=torch.float32, device="cuda") for _ in counts]
    folds = [torch.zeros((nx, ny), dtype=torch.int32, device="cuda") for _ in counts]
    bins = [Bin(b0, n, imgs[i], folds[i]) for i, (b0, n) in enumerate(zip(bs.starts, bs.counts))]
    pairs = int(counts.sum()) * nx * ny * nt
    k = CudaKernel(precision="fp32")   # the forms' FP32 arithmetic (1e-3 bar)
    k.initialize(cfg)
    t0 = time.perf_counter()
    tune = k.autotune_bins(tb, bins, geom, vel, cfg, kernel_type="anisotropic_vti")
    tune["seconds"] = time.perf_counter() - t0

    def timed(fn, reps):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return replicas.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda") / reps

    batched = lambda: k.migrate_bins(tb, bins, geom, vel, cfg, kernel_type="anisotropic_vti")
    if scale == 1:   # the full case: time the first call (graph capture is host-side, ~ms of ~100 s)
        reps = 1
        ms_batched = timed(batched, 1)
        k.synchronize()
    else:
        batched()   # capture the graph
        torch.cuda.synchronize()
        k.synchronize()
        reps = max(1, min(2, args.steps))
        ms_batched = timed(batched, reps)

    kp = CudaKernel(precision="fp32")   # a second context: untuned default shape, per-tile launches
    kp.initialize(cfg)

    def per_bin():
        for b in bins:
            sl = slice(b.trace_begin, b.trace_begin + b.n_traces)
            sub = TraceBlock(amplitudes=tb.amplitudes[sl], source_x=tb.source_x[sl], source_y=tb.source_y[sl],
                             receiver_x=tb.receiver_x[sl], receiver_y=tb.receiver_y[sl], offset=tb.offset[sl],
                             midpoint_x=tb.midpoint_x[sl], midpoint_y=tb.midpoint_y[sl],
                             sample_rate_ms=dt_ms, start_time_ms=0.0)
            kp.migrate_tile_vti(sub, OutputTile(image=b.image, fold=b.fold, x_axis=geom.x_axis, y_axis=geom.y_axis,
                                               t_axis_ms=geom.t_axis_ms), vel, cfg)
    ms_per_bin = None
    if per_bin_compare:
        per_bin()
        ms_per_bin = timed(per_bin, 1)
    kp.cleanup()

    # accuracy: the smallest bin, 2 x 2 pillars, against the FP64 oracle fed the
    # same (BF16-valued) traces; a fresh image so the bin is migrated once
    i = int(np.argmin(counts))
    b = bins[i]
    sl = slice(b.trace_begin, b.trace_begin + b.n_traces)
    one = torch.zeros((nx, ny, nt), dtype=torch.float32, device="cuda")
    k.migrate_bins(tb, [Bin(b.trace_begin, b.n_traces, one)], geom, vel, cfg, kernel_type="anisotropic_vti")
    torch.cuda.synchronize()
    htb = create_trace_block(bs.amps_device[sl].float().cpu().numpy(), sv.s[sl, 0], sv.s[sl, 1], sv.r[sl, 0],
                             sv.r[sl, 1], sample_rate_ms=dt_ms)
    px = 60
    ref_out, ref_vel = sv.tile(px, px + 2, px, px + 2)
    ocfg = workloads.survey_config(kernel_type="anisotropic_vti", aa=True, dx=DX, eta=eta)
    oracle.build()
    oracle.migrate(htb, ref_out, ref_vel, ocfg, kind="anisotropic_vti")
    got = one[px:px + 2, px:px + 2].double().cpu().numpy()
    err = float(np.linalg.norm(got - ref_out.image) / np.linalg.norm(ref_out.image))
    k.cleanup()
    del imgs, folds, bins, tb
    torch.cuda.empty_cache()
    return {
        "value": world * pairs / (ms_batched / 1e3), "unit": UNIT,
        "per_bin_calls_value": world * pairs / (ms_per_bin / 1e3) if ms_per_bin else None,
        "speedup_vs_per_bin_calls": ms_per_bin / ms_batched if ms_per_bin else None,
        "ms_per_launch": ms_batched, "ms_per_bin_calls": ms_per_bin, "launches_timed": reps,
        "bins": int(len(counts)), "traces": int(counts.sum()), "traces_full_case": int(full.sum()),
        "trace_scale": "full case" if scale == 1 else f"1/{scale} of every bin's traces",
        "tile": [nx, ny, nt], "trace_dtype": "bf16", "image_dtype": "f32", "traveltime": "anisotropic_vti",
        "autotune": tune, "rel_l2_vs_fp64": err,
        "rel_l2_sample": f"2x2 pillars x {nt} samples of the smallest bin ({int(counts[i])} traces), FP64 "
                         "oracle on the same BF16-valued traces",
        "graph": "captured once, replayed per launch",
    }


def measure_scatter(args):
    """The trace-centric (scatter) schedule against the tiled gather on a
    high-overlap region: the case-2 geometry (1,048,576 FP32 traces x 1500 @2 ms
    over 3.2 km, 3-D v_rms, AA) with a 500 m aperture, the central 128 x 128
    pillars x 1500 samples.  Gather: TiledExecutor with the midpoint-ordered
    panel, 16 tiles of 32 x 32, each migrated against its selection box (tile
    + 500 m; neighbouring boxes overlap, so most traces are read by several
    tiles).  Scatter: one call over the region, every trace read once.  Both
    from the same sorted panel; CUDA-event time of the whole region; the images
    are compared."""
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.cuda_kernel import CudaKernel
    from pstm_b200.executor import TiledExecutor
    from pstm_b200.spatial import MidpointIndex, sort_panel
    N = args.traces
    sv, amps = workloads.survey_device(N, GRID, GRID, NT, DT_MS, NS, dx=DX, seed=7, dtype=torch.float32)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    mx, my = (sv.s[:, 0] + sv.r[:, 0]) / 2.0, (sv.s[:, 1] + sv.r[:, 1]) / 2.0
    tb = TraceBlock(amplitudes=amps, source_x=dev(sv.s[:, 0]), source_y=dev(sv.s[:, 1]), receiver_x=dev(sv.r[:, 0]),
                    receiver_y=dev(sv.r[:, 1]), offset=dev(np.hypot(*(sv.r - sv.s).T)), midpoint_x=dev(mx),
                    midpoint_y=dev(my), sample_rate_ms=DT_MS, start_time_ms=0.0)
    index = MidpointIndex(mx, my, 50.0)
    panel = sort_panel(tb, index)
    del tb, amps
    torch.cuda.empty_cache()
    cfg = workloads.survey_config(kernel_type="straight_ray", aa=True, dx=DX)
    cfg.max_aperture_m = 500.0
    r0, R = 64, 128
    xa, ya = sv.x_axis[r0:r0 + R], sv.y_axis[r0:r0 + R]
    vfull = dev(sv.velocity(r0, r0 + R, r0, r0 + R))
    k = CudaKernel()
    k.initialize(cfg)

    ex = TiledExecutor(k, panel, xa, ya, sv.t_axis_ms,
                       lambda x0, x1, y0, y1: VelocitySlice(vrms=vfull[x0:x1, y0:y1].contiguous(), is_1d=False),
                       cfg, tile=32)
    ex.index = MidpointIndex(index.mx_sorted, index.my_sorted, 50.0)   # identity order: the panel is sorted
    img_g = torch.zeros((R, R, NT), dtype=torch.float64, device="cuda")
    fold_g = torch.zeros((R, R, NT), dtype=torch.int32, device="cuda")
    ex.run(img_g, fold_g, ex.tiles()[:1])   # warm-up (one tile), then the timed region
    img_g.zero_()
    fold_g.zero_()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    res_g = ex.run(img_g, fold_g)
    e1.record()
    torch.cuda.synchronize()
    ms_g = e0.elapsed_time(e1)
    out = OutputTile(image=torch.zeros((R, R, NT), dtype=torch.float64, device="cuda"),
                     fold=torch.zeros((R, R, NT), dtype=torch.int32, device="cuda"), x_axis=dev(xa), y_axis=dev(ya),
                     t_axis_ms=dev(sv.t_axis_ms))
    vel = VelocitySlice(vrms=vfull, is_1d=False)
    m = k.migrate_scatter(panel, out, vel, cfg, count_items=True)   # warm-up, item count
    out.image.zero_()
    out.fold.zero_()
    torch.cuda.synchronize()
    e0.record()
    k.migrate_scatter(panel, out, vel, cfg)
    e1.record()
    torch.cuda.synchronize()
    k.synchronize()
    ms_s = e0.elapsed_time(e1)
    rel = float((out.image - img_g).norm() / img_g.norm())
    fold_eq = bool(torch.equal(out.fold, fold_g))
    read_by_tiles = sum(r.processed_traces for r in res_g)
    k.cleanup()
    del panel
    torch.cuda.empty_cache()
    return {"scatter_ms": ms_s, "gather_tiles_ms": ms_g, "speedup_scatter_vs_gather": ms_g / ms_s,
            "region": [R, R, NT], "tiles": len(res_g), "tile": 32, "max_aperture_m": 500.0, "traces": N,
            "trace_rows_read_by_tiles": int(read_by_tiles), "traces_read_by_scatter": N,
            "scatter_items": int(getattr(m, "n_items", 0)), "image_rel_l2_scatter_vs_gather": rel,
            "fold_equal": fold_eq,
            "workload": "case-2 geometry, central 128x128 pillars, 500 m aperture, straight exact, AA, 3-D v"}


def measure_learned(args, sv, amps, world, dist):
    """The learned form on the curved/VTI case (case-2 geometry and velocity,
    eta(t0) = 0.15 t0 / 3 s): train the surrogate with the package's own
    kernels on seeded exact targets, report its traveltime error in ms on
    held-out samples, then migrate a sample tile (24 x 24 pillars x 1500
    samples x 65,536 traces, FP32 traces) three ways: exact VTI kernel, the
    learned entry point with the 0.1 ms probe (which falls back to the exact
    kernel when the probe fails) and the surrogate forced on every pair."""
    import dataclasses
    import torch
    from pstm_b200 import replicas, workloads
    from pstm_b200 import surrogate as S
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.cuda_kernel import CudaKernel
    tr = S.Trainer(int(os.environ.get("LOCAL_RANK", "0")))
    dom = S.survey_domain("anisotropic_vti", t0_max_s=(NT - 1) * DT_MS / 1000.0, h_max_m=GRID * DX)
    t0 = time.perf_counter()
    net = tr.train(dom, n_train=50_000_000, steps=args.learned_steps, batch=65536, lr=2e-3,
                   log_every=max(1, args.learned_steps // 4))
    train_s = time.perf_counter() - t0
    err = tr.error_ms(net, n=1 << 20)
    tr.close()

    n_tr, P = 1 << 16, 24
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    tb = TraceBlock(amplitudes=amps[:n_tr].float().contiguous(), source_x=dev(sv.s[:n_tr, 0]),
                    source_y=dev(sv.s[:n_tr, 1]), receiver_x=dev(sv.r[:n_tr, 0]), receiver_y=dev(sv.r[:n_tr, 1]),
                    offset=dev(np.hypot(*(sv.r[:n_tr] - sv.s[:n_tr]).T)),
                    midpoint_x=dev((sv.s[:n_tr, 0] + sv.r[:n_tr, 0]) / 2), midpoint_y=dev((sv.s[:n_tr, 1] + sv.r[:n_tr, 1]) / 2),
                    sample_rate_ms=DT_MS, start_time_ms=0.0)
    ix0 = iy0 = 120
    out, vel = sv.tile(ix0, ix0 + P, iy0, iy0 + P)
    eta = workloads.survey_eta(sv.t_axis_ms)
    cfg = workloads.survey_config(kernel_type="anisotropic_vti", aa=True, dx=DX, eta=eta)
    cfg.vti_eta_array = dev(eta)
    dvel = VelocitySlice(vrms=dev(vel.vrms), is_1d=False)

    def fresh():
        return OutputTile(image=torch.zeros(out.image.shape, dtype=torch.float64, device="cuda"),
                          fold=torch.zeros(out.fold.shape, dtype=torch.int32, device="cuda"),
                          x_axis=dev(out.x_axis), y_axis=dev(out.y_axis), t_axis_ms=dev(out.t_axis_ms))
    k = CudaKernel(precision="fp32")   # the forms' FP32 arithmetic (1e-3 bar)
    k.initialize(cfg)
    pairs = P * P * NT * n_tr

    def timed(fn):
        o = fresh()
        fn(o)
        torch.cuda.synchronize()
        o = fresh()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn(o)
        e1.record()
        torch.cuda.synchronize()
        return replicas.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda"), o, r

    ms_exact, o_exact, _ = timed(lambda o: k.migrate_tile_vti(tb, o, dvel, cfg))
    ms_probe, o_probe, r_probe = timed(lambda o: k.migrate_tile_learned(tb, o, dvel, net, cfg, max_residual_ms=0.1)[1])
    ms_forced, o_forced, r_forced = timed(lambda o: k.migrate_tile_learned(tb, o, dvel, net, cfg,
                                                                           max_residual_ms=-1.0)[1])
    k.cleanup()
    ref = o_exact.image.cpu().numpy()
    rel = lambda a: float(np.linalg.norm(a.image.cpu().numpy() - ref) / np.linalg.norm(ref))
    return {
        "value": world * pairs / (ms_probe / 1e3), "unit": UNIT,
        "traveltime": "anisotropic_vti", "trace_dtype": "f32",
        "sample": f"{P}x{P} pillars x {NT} samples x {n_tr} traces of the case-2 tile (eta(t0) = 0.15 t0/3 s)",
        "exact_value": world * pairs / (ms_exact / 1e3),
        "learned_with_probe": {"value": world * pairs / (ms_probe / 1e3), **r_probe,
                               "rel_l2_vs_exact_kernel": rel(o_probe)},
        "learned_forced": {"value": world * pairs / (ms_forced / 1e3), **r_forced,
                           "rel_l2_vs_exact_kernel": rel(o_forced)},
        "surrogate": {"layers": "7-64-64-64-1 SiLU, BF16 weights, FP32 accumulate (mma.sync m16n8k16)",
                      "target": "T_exact - T_DSR(v_rms), exact FP64 targets", "train_samples": 50_000_000,
                      "steps": args.learned_steps, "batch": 65536, "train_seconds": train_s,
                      "loss_history": net.history, "heldout_error": err},
        "threshold_ms": 0.1,
    }


# ------------------------------------------------------------------ our arm
def main_ours(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from pstm_b200 import build, workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.cuda_kernel import CudaKernel
    build.build()

    tdtype = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[args.dtype]
    N = args.traces
    sv, amps = workloads.survey_device(N, GRID, GRID, NT, DT_MS, NS, dx=DX, seed=7, dtype=tdtype)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    geo = {k: dev(v) for k, v in (("source_x", sv.s[:, 0]), ("source_y", sv.s[:, 1]),
                                  ("receiver_x", sv.r[:, 0]), ("receiver_y", sv.r[:, 1]),
                                  ("midpoint_x", (sv.s[:, 0] + sv.r[:, 0]) / 2.0),
                                  ("midpoint_y", (sv.s[:, 1] + sv.r[:, 1]) / 2.0))}
    offset = dev(np.hypot(sv.r[:, 0] - sv.s[:, 0], sv.r[:, 1] - sv.s[:, 1]))
    tb = TraceBlock(amplitudes=amps, offset=offset, sample_rate_ms=DT_MS, start_time_ms=0.0, **geo)
    cfg = config()
    from pstm_b200 import replicas
    tiles = tiles_of(args.tile)
    my_tiles = replicas.rank_schedule(tiles, rank, world, args.warmup + args.steps)
    T = args.tile
    img = torch.zeros((T, T, NT), dtype=torch.float64, device="cuda")
    fold = torch.zeros((T, T, NT), dtype=torch.int32, device="cuda")
    t_axis = dev(sv.t_axis_ms)
    tile_args = {}
    for tl in set(my_tiles):
        ix0, ix1, iy0, iy1 = tl
        tile_args[tl] = (OutputTile(image=img, fold=fold, x_axis=dev(sv.x_axis[ix0:ix1]),
                                    y_axis=dev(sv.y_axis[iy0:iy1]), t_axis_ms=t_axis),
                         VelocitySlice(vrms=dev(sv.velocity(ix0, ix1, iy0, iy1)), is_1d=False))
    k = CudaKernel(precision=args.precision)
    k.initialize(cfg)
    pairs_per_step = T * T * NT * N

    def step(j):
        out, vel = tile_args[my_tiles[j]]
        k.migrate_tile(tb, out, vel)

    for j in range(args.warmup):
        step(j)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for j in range(args.warmup, args.warmup + args.steps):
            step(j)
        e1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda")
    value = world * args.steps * pairs_per_step / (ms / 1e3)
    clocks = clk.summary()

    # ---- roofline of the migration kernel (one launch per step; the table and
    # geometry-packing kernels of a step take ~1e-4 of it)
    per_launch_s = ms / 1e3 / args.steps
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    mufu_derived = 148 * 16 * sm_mhz * 1e6       # MUFU ops/s: 148 SMs x 16/clk x median SM clock
    mufu_peak, mufu_src = measured_sfu_peak(local), "measured: MUFU-throughput kernel on this GPU " \
        "(sqrt.approx/rcp.approx chains, full occupancy, CUDA events, best of 3), same run"
    if not mufu_peak:
        mufu_peak, mufu_src = mufu_derived, "derived: 148 SMs x 16 MUFU/clk x median SM clock under load"
    achieved_mufu = pairs_per_step * MUFU_PER_PAIR / per_launch_s
    elem = amps.element_size()
    alg_bytes = N * NS * elem + N * 6 * 8 + T * T * NT * (8 + 8 + 4 + 4) + T * T * NT * 8
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else \
        "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"
    roofline = {
        "bound": "sfu", "unit": "Gop/s", "achieved": achieved_mufu / 1e9, "peak": mufu_peak / 1e9,
        "frac": achieved_mufu / mufu_peak,
        "peak_source": mufu_src, "peak_derived": mufu_derived / 1e9,
        "per_pair": f"{FLOP_PER_PAIR} FP32 FLOP + {MUFU_PER_PAIR} MUFU (straight-ray DSR + AA + weights)",
        "fp32": {"achieved_tflops": pairs_per_step * FLOP_PER_PAIR / per_launch_s / 1e12,
                 "peak_tflops": 148 * 128 * 2 * sm_mhz * 1e6 / 1e12},
        "hbm": {"achieved_gbs": alg_bytes / per_launch_s / 1e9, "peak_gbs": hbm_peak,
                "frac": alg_bytes / per_launch_s / 1e9 / hbm_peak, "algorithmic_bytes_per_launch": alg_bytes,
                "peak_source": hbm_src},
        "traffic": (DRAM_BYTES_PER_TRACE_TILE64 * N / 1e9) if T == 64 else None,
        "traffic_unit": "GB per launch (ncu dram__bytes read+write of a 262,144-trace launch, scaled by traces)",
    }

    # ---- end to end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        h_amps = torch.empty(amps.shape, dtype=amps.dtype, pin_memory=True)
        h_amps.copy_(amps)
        amps_np = h_amps.view(torch.int16).numpy().view(np.uint16) if tdtype == torch.bfloat16 else h_amps.numpy()

        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()
        htb = TraceBlock(amplitudes=amps_np, offset=pinned(offset.cpu().numpy()), sample_rate_ms=DT_MS,
                         start_time_ms=0.0, **{kk: pinned(v.cpu().numpy()) for kk, v in geo.items()})
        h_img = torch.zeros((T, T, NT), dtype=torch.float64, pin_memory=True).numpy()
        h_fold = torch.zeros((T, T, NT), dtype=torch.int32, pin_memory=True).numpy()
        h_tiles = {}
        for tl in set(my_tiles):
            ix0, ix1, iy0, iy1 = tl
            h_tiles[tl] = (OutputTile(image=h_img, fold=h_fold, x_axis=sv.x_axis[ix0:ix1], y_axis=sv.y_axis[iy0:iy1],
                                      t_axis_ms=sv.t_axis_ms),
                           VelocitySlice(vrms=pinned(sv.velocity(ix0, ix1, iy0, iy1)), is_1d=False))
        ke = CudaKernel(trace_dtype="auto", precision=args.precision)
        ke.initialize(cfg)
        ke.migrate_tile(htb, *h_tiles[my_tiles[0]])   # warm the staging buffers
        if dist:
            dist.barrier()
        e2e_steps = args.e2e_steps or min(args.steps, 4)
        t0 = time.perf_counter()
        for j in range(e2e_steps):   # the tiles of the timed device steps, in order
            ke.migrate_tile(htb, *h_tiles[my_tiles[args.warmup + j % args.steps]])
        e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, dist, device="cuda")
        h2d = amps_np.nbytes + sum(htb.__dict__[kk].nbytes for kk in geo) + T * T * NT * (8 + 8 + 4) + \
            3 * T * 8 + NT * 8
        d2h = T * T * NT * (8 + 4)
        e2e = {"value": world * e2e_steps * pairs_per_step / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "steps": e2e_steps, "timer": "perf_counter around synchronous migrate_tile calls"}
        ke.cleanup()

    forms = None
    # the forms are single-GPU measurements: every rank skips them alike when N > 1
    single = world == 1
    if not args.no_forms and single:
        forms = measure_forms(args, k, tb, amps, tile_args, my_tiles, pairs_per_step, world, dist, sv, cfg)
        forms["case1_tile"] = measure_case1()
        forms["case1_tile_sinc8"] = measure_case1_interp("sinc8")
        forms["case1_tile_sinc8_fast"] = measure_case1_interp("sinc8", "fast")
    if not args.no_batched and single:
        forms = forms or {}
        forms["batched_offset_bins_bf16_vti"] = measure_batched(args, world, dist, scale=args.batch_scale,
                                                                per_bin_compare=args.batch_scale > 1)
        if args.batch_scale == 1:   # the per-bin comparison on a reduced copy of the case
            forms["batched_offset_bins_bf16_vti_1_16"] = measure_batched(args, world, dist, scale=16)
    if not args.no_learned and single:
        forms = forms or {}
        forms["learned_vti"] = measure_learned(args, sv, amps, world, dist)

    if not args.no_scatter and single:
        forms = forms or {}
        forms["scatter_vs_gather_high_overlap"] = measure_scatter(args)
    if not args.no_case5 and single:
        forms = forms or {}
        forms["case5_large_survey"] = measure_case5(args)

    numba_line = None
    if single and not args.no_numba:
        import tempfile
        with tempfile.TemporaryDirectory(prefix="pstm_numba_") as td:
            numba_line = numba_comparison(td)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle
        oracle.build()
        n_tr = 1 << 18
        amps_host = amps[:n_tr].float().cpu().numpy()
        rate, pairs, dt = cpu_sample(sv, cfg, tiles[0], n_tr, 4, 4, amps_host)
        cpu = {"value": rate, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"4x4 pillars x {NT} samples x {n_tr} traces ({pairs:.3g} pairs, {dt:.1f} s), "
                         "FP64 C port of the reference semantics, OpenMP on all host threads"}

    k.cleanup()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
            "config": {"workload": "case-2 production tile: 1,048,576 traces x 1500 samples @2 ms, "
                                   "3.2 km patch, 3-D v_rms, AA on, 5 km aperture; one step = "
                                   f"{T}x{T}x{NT} output tile (pillars x samples)",
                       "traces": N, "tile": [T, T, NT], "grid": [GRID, GRID, NT], "traveltime": "straight_ray",
                       "trace_dtype": args.dtype, "precision": args.precision,
                       "accumulate": "fp32 per trace chunk -> f64 image",
                       "l2": "inputs larger than L2 (trace panel > 126 MB), no flush",
                       "parallelism": f"replicas x{world} (disjoint tiles)"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "forms": forms,
            "reference_numba": numba_line,
            "gpu_launches": 3 * args.steps, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ case 5
def main_case5(args):
    """``--case5``: the large-survey case alone, one JSON line (see :func:`measure_case5`)."""
    print(json.dumps(measure_case5(args)), flush=True)


def _mem_available_bytes() -> int:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def measure_case5(args):
    """The large-survey case: 512 x 512 bins at 12.5 m x 2000 samples at 2 ms
    (2.1 GB FP32 image), 8,388,608 FP16 traces of 2000 samples (33.6 GB, all
    resident in HBM) with offsets up to 5 km over a 6.4 km patch, curved-ray +
    VTI traveltime (learned surrogate with the exact fallback), triangle AA and
    weights on.  The tiled executor migrates --case5-tiles 64 x 64 tiles; the
    aperture is capped at --case5-aperture m so that the FP64 oracle check of
    64 random output traces stays feasible.  Then the streaming executor
    migrates one of those tiles again from a host copy of the panel through a
    small device pool (panels larger than HBM), reporting how much of its
    host->device copy time ran under the kernels, when the host has the memory
    for the copy.  Returns the result line."""
    import torch
    from oracle import oracle
    from pstm_b200 import build, replicas, workloads
    from pstm_b200 import surrogate as S
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.cuda_kernel import CudaKernel
    from pstm_b200.executor import TiledExecutor, tile_ranges
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    build.build()
    G5, NT5, NS5, N5 = 512, 2000, 2000, args.traces if args.traces != (1 << 20) else 8_388_608
    t_gen = time.perf_counter()
    sv, amps = workloads.survey_device(N5, G5, G5, NT5, DT_MS, NS5, dx=DX, max_offset=5000.0, seed=55,
                                       dtype=torch.float16)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    mx, my = (sv.s[:, 0] + sv.r[:, 0]) / 2.0, (sv.s[:, 1] + sv.r[:, 1]) / 2.0
    tb = TraceBlock(amplitudes=amps, source_x=dev(sv.s[:, 0]), source_y=dev(sv.s[:, 1]), receiver_x=dev(sv.r[:, 0]),
                    receiver_y=dev(sv.r[:, 1]), offset=dev(np.hypot(*(sv.r - sv.s).T)), midpoint_x=dev(mx),
                    midpoint_y=dev(my), sample_rate_ms=DT_MS, start_time_ms=0.0)
    vfull = dev(sv.velocity())
    gen_s = time.perf_counter() - t_gen
    eta = workloads.survey_eta(sv.t_axis_ms)
    cfg = workloads.survey_config(kernel_type="curved_vti", aa=True, dx=DX, eta=eta, v0=1500.0, k=0.5)
    cfg.max_aperture_m = args.case5_aperture
    cfg.vti_eta_array = dev(eta)
    tr = S.Trainer(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    dom = S.survey_domain("curved_vti", t0_max_s=(NT5 - 1) * DT_MS / 1000.0,
                          h_max_m=64 * DX + args.case5_aperture + 2500.0, v0=1500.0, k=0.5)
    net = tr.train(dom, n_train=50_000_000, steps=args.learned_steps, batch=65536, lr=2e-3,
                   log_every=max(1, args.learned_steps // 4))
    train_s = time.perf_counter() - t0
    heldout = tr.error_ms(net, n=1 << 20)
    tr.close()

    k = CudaKernel(precision="fp32")   # the forms' FP32 arithmetic (1e-3 bar)
    k.initialize(cfg)
    ex = TiledExecutor(k, tb, sv.x_axis, sv.y_axis, sv.t_axis_ms,
                       lambda x0, x1, y0, y1: VelocitySlice(vrms=vfull[x0:x1, y0:y1].contiguous(), is_1d=False),
                       cfg, kernel_type="curved_vti", tile=64, surrogate=net, max_residual_ms=0.1)
    tiles_all = tile_ranges(G5, G5, 64)
    centre = sorted(tiles_all, key=lambda t: abs(t[0] + 32 - G5 / 2) + abs(t[2] + 32 - G5 / 2))
    tiles = centre[:max(1, args.case5_tiles)]
    image = torch.zeros((G5, G5, NT5), dtype=torch.float32, device="cuda")
    fold = torch.zeros((G5, G5), dtype=torch.int32, device="cuda")
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        results = ex.run(image, fold, tiles)
    clocks = clk.summary()
    pairs = sum(r.pairs for r in results)
    kernel_s = sum(r.kernel_ms for r in results) / 1e3
    value = pairs / kernel_s

    # FP64 oracle on 64 random output traces of the first tile, each against a
    # seeded 1/32 sample of that tile's selected traces (the same sample on the GPU)
    rng = np.random.default_rng(5)
    ix0, ix1, iy0, iy1 = tiles[0]
    pix = rng.integers(ix0, ix1, 64)
    piy = rng.integers(iy0, iy1, 64)
    idx = ex.select(tiles[0])[::32]
    sub = ex._gather(idx)
    xg, yg = sv.x_axis[pix].reshape(64, 1), sv.y_axis[piy].reshape(64, 1)
    v64 = vfull[dev(pix), dev(piy)].cpu().numpy().reshape(64, 1, NT5)
    g_out = OutputTile(image=torch.zeros((64, 1, NT5), dtype=torch.float64, device="cuda"),
                       fold=torch.zeros((64, 1), dtype=torch.int32, device="cuda"),
                       x_axis=dev(np.arange(64.0)), y_axis=dev(np.zeros(1)), t_axis_ms=dev(sv.t_axis_ms),
                       x_grid=dev(xg), y_grid=dev(yg))
    _, rep = k.migrate_tile_learned(sub, g_out, VelocitySlice(vrms=dev(v64), is_1d=False), net, cfg,
                                    kernel_type="curved_vti", max_residual_ms=0.1)
    torch.cuda.synchronize()
    k.cleanup()
    from pstm_b200.base import create_trace_block
    ii = idx.cpu().numpy()
    htb = create_trace_block(sub.amplitudes.float().cpu().numpy(), sv.s[ii, 0], sv.s[ii, 1], sv.r[ii, 0],
                             sv.r[ii, 1], sample_rate_ms=DT_MS)
    o_out = OutputTile(image=np.zeros((64, 1, NT5)), fold=np.zeros((64, 1), np.int32), x_axis=np.arange(64.0),
                       y_axis=np.zeros(1), t_axis_ms=sv.t_axis_ms, x_grid=xg, y_grid=yg)
    ocfg = workloads.survey_config(kernel_type="curved_vti", aa=True, dx=DX, eta=eta, v0=1500.0, k=0.5)
    ocfg.max_aperture_m = args.case5_aperture
    t_or = time.perf_counter()
    oracle.build()
    oracle.migrate(htb, o_out, VelocitySlice(vrms=v64, is_1d=False), ocfg, kind="curved_vti")
    oracle_s = time.perf_counter() - t_or
    got = g_out.image.cpu().numpy()
    err = float(np.linalg.norm(got - o_out.image) / np.linalg.norm(o_out.image))
    fold_ok = bool((g_out.fold.cpu().numpy() == o_out.fold).all())

    # ---- the streaming executor on one tile, from a host copy of the panel
    streaming = None
    panel_bytes = N5 * NS5 * 2 + N5 * 7 * 8
    avail = _mem_available_bytes()
    if args.no_streaming:
        streaming = {"skipped": "--no-streaming"}
    elif avail < 2 * panel_bytes + (16 << 30):
        streaming = {"skipped": f"host MemAvailable {avail / 1e9:.1f} GB < 2 x the {panel_bytes / 1e9:.1f} GB panel "
                                "+ 16 GB"}
    else:
        from pstm_b200.streaming import StreamingExecutor
        st_tile = tiles[-1]
        h_amps = amps.cpu().numpy()
        htb5 = create_trace_block(h_amps, sv.s[:, 0], sv.s[:, 1], sv.r[:, 0], sv.r[:, 1], sample_rate_ms=DT_MS)
        del amps, tb, sub
        ex.tb = None
        torch.cuda.empty_cache()
        ks = CudaKernel(precision="fp32")
        ks.initialize(cfg)
        sx = StreamingExecutor(ks, htb5, sv.x_axis, sv.y_axis, sv.t_axis_ms,
                               lambda x0, x1, y0, y1: VelocitySlice(vrms=vfull[x0:x1, y0:y1].contiguous(),
                                                                    is_1d=False),
                               cfg, kernel_type="curved_vti", tile=64, block_traces=65536, pool_blocks=16)
        simg = torch.zeros((G5, G5, NT5), dtype=torch.float32, device="cuda")
        rep_s = sx.run(simg, None, [st_tile])
        a0, a1, b0, b1 = st_tile
        ref_t, got_t = image[a0:a1, b0:b1].double(), simg[a0:a1, b0:b1].double()
        ks.cleanup()
        streaming = {
            "tile": list(st_tile), "passes": len(rep_s.passes), "pool_blocks": sx.S, "block_traces": sx.B,
            "pool_gb": sx.S * sx.B * (NS5 * 2 + 56) / 1e9, "blocks_loaded": rep_s.misses, "block_hits": rep_s.hits,
            "h2d_gb": rep_s.h2d_bytes / 1e9, "copy_ms": rep_s.copy_ms, "kernel_ms": rep_s.kernel_ms,
            "wall_ms": rep_s.wall_s * 1e3, "exposed_ms": rep_s.exposed_ms,
            "first_load_ms": rep_s.first_load_ms, "copy_overlap_ms": rep_s.copy_overlap_ms,
            "overlapped_copy_fraction": rep_s.overlapped_copy_fraction,
            "h2d_gbs": rep_s.h2d_bytes / max(rep_s.copy_ms, 1e-9) / 1e6,
            "value": sum(r.pairs for r in results if r.tile == st_tile) / (rep_s.wall_s or 1e-9),
            "unit": UNIT, "rel_l2_vs_resident_tile": float((got_t - ref_t).norm() / ref_t.norm()),
            "note": "exact curved+VTI kernel (the resident run's surrogate fell back to it); host panel "
                    f"{panel_bytes / 1e9:.1f} GB, device pool only",
        }

    sm_mhz = clocks.get("sm_mhz") or 1965.0
    mufu_peak, peak_src = measured_sfu_peak(int(os.environ.get("LOCAL_RANK", "0"))), "measured (MUFU-throughput kernel)"
    if not mufu_peak:
        mufu_peak, peak_src = 148 * 16 * sm_mhz * 1e6, "derived: 148 SMs x 16 MUFU/clk x median SM clock"
    mufu_per_pair = 8   # straight DSR 3 + AA 1 + curved legs 2 + VTI 2
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": len(results), "warmup": 0,
        "ms_per_step": 1e3 * kernel_s / len(results), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16", "data": "synthetic",
        "config": {"workload": "case-5 large survey: 512x512 bins @12.5 m x 2000 samples @2 ms, 8,388,608 FP16 "
                               "traces x 2000 (offsets <= 5 km, 6.4 km patch), curved-ray + VTI, AA + weights, "
                               "tiled executor (one step = one 64x64 tile against its selected traces)",
                   "traces": N5, "traces_resident_gb": N5 * NS5 * 2 / 1e9, "tiles_run": [list(t) for t in tiles],
                   "max_aperture_m": args.case5_aperture, "image": "FP32 (512, 512, 2000) on the device"},
        "tiles": [{"tile": list(r.tile), "selected_traces": r.n_traces, "pairs": r.pairs, "ms": r.kernel_ms,
                   "used_surrogate": r.used_surrogate, "probe_max_ms": r.probe_max_ms} for r in results],
        "roofline": {"bound": "sfu", "unit": "Gop/s", "achieved": value * mufu_per_pair / 1e9,
                     "peak": mufu_peak / 1e9, "frac": value * mufu_per_pair / mufu_peak,
                     "per_pair": f"{mufu_per_pair} MUFU (DSR 3 + AA 1 + curved 2 + VTI 2)",
                     "peak_source": peak_src},
        "oracle_check": {"rel_l2_vs_fp64": err, "fold_bit_exact": fold_ok, "pillars": 64,
                         "sample": f"64 random output traces of tile {list(tiles[0])} x {NT5} samples against "
                                   f"every 32nd of its {int(ex.select(tiles[0]).numel())} selected traces "
                                   f"({int(idx.numel())} traces)", "oracle_seconds": oracle_s,
                         "used_surrogate": rep["used_surrogate"]},
        "surrogate": {"train_seconds": train_s, "steps": args.learned_steps, "heldout_error": heldout},
        "generation_seconds": gen_s, "wall_seconds_tiles": ex.wall_s, "clocks": clocks,
        "gpu_launches": 3 * len(results), "streaming_executor": streaming,
    }
    return line


def main():
    args = parse()
    if args.numba_leg:
        numba_leg_child(args.numba_leg)
        return
    if args.case5:
        main_case5(args)
        return
    if args.impl == "reference":
        reference_arm(args)
    else:
        main_ours(args)


if __name__ == "__main__":
    main()
