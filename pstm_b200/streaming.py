"""Tiled migration of a survey whose trace panel stays in host memory.

The reference executor keeps the survey on disk and, tile by tile, loads the
traces a tile needs through an LRU cache of trace chunks
(``LRUTraceCache``, ``pstm/data/trace_cache.py:20``) fed by a prefetch thread
that reads the next tile's traces while the current one migrates
(``pstm/pipeline/executor.py:1203-1243``).  This is the same pipeline with
the GPU as the cache:

* the panel (amplitudes and geometry, NumPy, any size) stays on the host;
  a ``MidpointIndex`` over its midpoints cuts the midpoint order into blocks
  of ``block_traces`` traces;
* a fixed pool of device slots, one block each, is the cache (least recently
  used blocks are replaced); a tile's traces are the row ranges of its
  selection box, which touch a few blocks, and the tile migrates against
  those ranges where the blocks lie in the pool
  (``CudaKernel.migrate_tile_runs``): the pool is one device panel;
* while the kernel migrates one pass (a tile, or the part of a tile whose
  blocks fit in half the pool), host threads gather the next pass's missing
  blocks into a ring of pinned staging buffers, several blocks at a time, and
  the main thread copies each gathered block to its slot on a second stream,
  so host->device traffic overlaps the kernel.  A copy into a slot waits for
  the last kernel that read that slot.

So panels larger than HBM run, and HBM holds only the pool.  The result is
the resident executor's up to the order of floating-point additions (a tile
split over several passes adds each pass into its image and fold).
"""
from __future__ import annotations

import time
import weakref
from collections import OrderedDict, deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from .executor import selection_box, tile_ranges


def plan_passes(index, block_traces: int, pool_slots: int, boxes) -> list[tuple[int, list, np.ndarray]]:
    """Passes (tile number, blocks, runs in midpoint-order positions) for the
    tiles' selection boxes: each tile's blocks in groups of at most half the
    pool, so that one pass migrates while the next one's blocks load.  The
    groups are consecutive slices of the tile's sorted blocks, so clipping the
    tile's runs to a group's span keeps exactly the group's positions."""
    B, G = int(block_traces), max(1, int(pool_slots) // 2)
    out = []
    for ti, box in enumerate(boxes):
        runs = index.runs(*box)
        if not len(runs):
            continue
        blocks = sorted({j for a, b in runs for j in range(int(a) // B, (int(b) - 1) // B + 1)})
        for g0 in range(0, len(blocks), G):
            grp = blocks[g0:g0 + G]
            lo, hi = grp[0] * B, (grp[-1] + 1) * B
            clipped = [(max(int(a), lo), min(int(b), hi)) for a, b in runs if int(b) > lo and int(a) < hi]
            out.append((ti, grp, np.array(clipped, np.int64).reshape(-1, 2)))
    return out


def pool_runs(runs: np.ndarray, block_traces: int, slot_of) -> np.ndarray:
    """Runs in midpoint-order positions -> ascending, merged runs in pool rows
    (block j lives in rows slot_of[j] * block_traces + [0, block_traces))."""
    segs = []
    B = int(block_traces)
    for a, b in runs:
        a, b = int(a), int(b)
        while a < b:
            j = a // B
            e = min(b, (j + 1) * B)
            s = slot_of[j] * B
            segs.append((s + a - j * B, s + e - j * B))
            a = e
    segs.sort()
    merged: list[list[int]] = []
    for a, b in segs:
        if merged and merged[-1][1] == a:
            merged[-1][1] = b
        else:
            merged.append([a, b])
    return np.array(merged, np.int64).reshape(-1, 2)


@dataclass
class PassResult:
    tile: tuple
    blocks: list
    loaded: int            # blocks copied to the device for this pass (cache misses)
    h2d_bytes: int
    kernel_ms: float = 0.0


@dataclass
class StreamReport:
    passes: list = field(default_factory=list)
    wall_s: float = 0.0
    kernel_ms: float = 0.0         # sum of the migration calls' CUDA-event times
    copy_ms: float = 0.0           # sum of the block copies' CUDA-event times (copy stream)
    copy_overlap_ms: float = 0.0   # the part of copy_ms during which a migration kernel ran
    first_load_ms: float = 0.0     # run start -> first kernel start: the first pass's gather and copies
    h2d_bytes: int = 0
    hits: int = 0
    misses: int = 0

    @property
    def exposed_ms(self) -> float:
        """Wall time not covered by migration kernels (first loads, host work)."""
        return max(0.0, self.wall_s * 1e3 - self.kernel_ms)

    @property
    def overlapped_copy_fraction(self) -> float:
        """Share of the copy time that ran while a migration kernel ran, from the
        CUDA events of both streams (timestamps on one device clock)."""
        if self.copy_ms <= 0:
            return 1.0
        return float(min(1.0, self.copy_overlap_ms / self.copy_ms))


def overlap_ms(intervals, cover) -> float:
    """Total length of the parts of ``intervals`` (start, end) that lie inside
    the union of ``cover`` (start, end)."""
    merged: list[list[float]] = []
    for a, b in sorted(cover):
        if merged and a <= merged[-1][1]:
            merged[-1][1] = max(merged[-1][1], b)
        else:
            merged.append([a, b])
    tot = 0.0
    for a, b in intervals:
        for c, d in merged:
            lo, hi = max(a, c), min(b, d)
            if hi > lo:
                tot += hi - lo
    return tot


class StreamingExecutor:
    """Migrate a survey grid tile by tile from a host-resident trace panel.

    ``traces`` is a TraceBlock of NumPy arrays (amplitudes float32, float16, or
    uint16 BF16 bit patterns); ``velocity(ix0, ix1, iy0, iy1)`` returns a tile's
    v_rms as a CUDA tensor; axes are the full grid's (NumPy).  The pool holds
    ``pool_blocks`` blocks of ``block_traces`` traces (default: as many as
    ``pool_bytes`` allow, itself half the free device memory by default).
    """

    def __init__(self, kernel, traces, x_axis, y_axis, t_axis_ms, velocity, config,
                 kernel_type: str = "straight_ray", tile: int = 64, block_traces: int = 65536,
                 pool_blocks: int | None = None, pool_bytes: int | None = None,
                 column_width_m: float | None = None, gather_threads: int = 4):
        import torch
        from .spatial import MidpointIndex
        self.torch = torch
        self.k = kernel
        self.tb = traces
        self.x_axis, self.y_axis = np.asarray(x_axis, np.float64), np.asarray(y_axis, np.float64)
        self.t_axis_ms = np.asarray(t_axis_ms, np.float64)
        self.velocity = velocity
        self.cfg = config
        self.kind = kernel_type
        self.tile = int(tile)
        amps = np.asarray(traces.amplitudes)
        if amps.ndim != 2:
            raise ValueError("amplitudes must be (n_traces, n_samples)")
        self.n, self.ns = amps.shape
        self.B = int(block_traces)
        if self.B < 1:
            raise ValueError("block_traces must be >= 1")
        tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.float16): torch.float16,
               np.dtype(np.uint16): torch.bfloat16}.get(amps.dtype)
        if tdt is None:
            raise ValueError(f"unsupported host amplitude dtype {amps.dtype}")
        self._host_amps = amps.view(np.int16) if amps.dtype == np.uint16 else amps
        self._host_geo = [np.asarray(getattr(traces, f), np.float64) for f in
                          ("source_x", "source_y", "receiver_x", "receiver_y", "midpoint_x", "midpoint_y")]
        w = getattr(traces, "weights", None)
        self._host_geo.append(np.ones(self.n) if w is None else np.asarray(w, np.float64))
        if column_width_m is None:
            dx = abs(float(self.x_axis[1] - self.x_axis[0])) if len(self.x_axis) > 1 else 1.0
            column_width_m = max(self.tile * dx / 8.0, 1e-3)
        self.index = MidpointIndex(self._host_geo[4], self._host_geo[5], column_width_m)
        self.n_blocks = (self.n + self.B - 1) // self.B

        row_bytes = self.ns * amps.itemsize + 7 * 8
        if pool_blocks is None:
            if pool_bytes is None:
                pool_bytes = torch.cuda.mem_get_info()[0] // 2
            pool_blocks = max(2, int(pool_bytes // (row_bytes * self.B)))
        self.S = int(min(max(2, pool_blocks), max(2, self.n_blocks)))
        rows = self.S * self.B
        self._pool_amps = torch.empty((rows, self.ns), dtype=tdt, device="cuda")
        self._pool_geo = torch.zeros((7, rows), dtype=torch.float64, device="cuda")
        # a ring of pinned staging buffers, one host gather thread each
        self.n_stage = max(2, int(gather_threads))
        self._stage_amps = [torch.empty((self.B, self.ns), dtype=tdt, pin_memory=True) for _ in range(self.n_stage)]
        self._stage_geo = [torch.empty((7, self.B), dtype=torch.float64, pin_memory=True)
                           for _ in range(self.n_stage)]
        self._stage_done = [None] * self.n_stage   # copy-stream events of the staging buffers' last copies
        self._stage_next = 0
        self._gather_pool = ThreadPoolExecutor(max_workers=self.n_stage)
        weakref.finalize(self, self._gather_pool.shutdown, wait=False)
        self._copy = torch.cuda.Stream()
        self._slot_of: "OrderedDict[int, int]" = OrderedDict()   # block -> slot, least recent first
        self._free = list(range(self.S))
        self._slot_reader = [None] * self.S    # compute event of the last pass that read the slot
        self._loaded_ev = {}                   # block -> copy-stream event of its load
        self._copy_events = []                 # (start, end) per block copy
        from .base import TraceBlock
        g = self._pool_geo
        self.pool_traces = TraceBlock(amplitudes=self._pool_amps, source_x=g[0], source_y=g[1], receiver_x=g[2],
                                      receiver_y=g[3], offset=None, midpoint_x=g[4], midpoint_y=g[5], weights=g[6],
                                      sample_rate_ms=traces.sample_rate_ms, start_time_ms=traces.start_time_ms)
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
        self._x, self._y, self._t = dev(self.x_axis), dev(self.y_axis), dev(self.t_axis_ms)

    # ------------------------------------------------------------- planning
    def tiles(self):
        return tile_ranges(len(self.x_axis), len(self.y_axis), self.tile)

    def plan(self, tiles=None) -> list[tuple[tuple, list, np.ndarray]]:
        """Passes (tile, blocks, runs in midpoint-order positions); see :func:`plan_passes`."""
        tiles = list(tiles if tiles is not None else self.tiles())
        boxes = [selection_box(self.x_axis, self.y_axis, t, self.cfg.max_aperture_m) for t in tiles]
        return [(tiles[ti], grp, runs) for ti, grp, runs in plan_passes(self.index, self.B, self.S, boxes)]

    # ------------------------------------------------------------- the cache
    def _victim(self, keep: set) -> int:
        for blk in self._slot_of:   # least recently used first
            if blk not in keep:
                slot = self._slot_of.pop(blk)
                self._loaded_ev.pop(blk, None)
                return slot
        raise RuntimeError("the device pool cannot hold two passes' blocks; give it more slots")

    def _gather(self, blk: int, k: int) -> int:
        """Host side of a block load: its traces (midpoint order) into staging
        buffer k (runs in a gather thread; NumPy releases the GIL here)."""
        torch = self.torch
        idx = self.index.order[blk * self.B:(blk + 1) * self.B]
        n = len(idx)
        sa = self._stage_amps[k]
        sa_np = (sa.view(torch.int16) if sa.dtype == torch.bfloat16 else sa).numpy()
        np.take(self._host_amps, idx, axis=0, out=sa_np[:n])
        sg = self._stage_geo[k].numpy()
        for i, a in enumerate(self._host_geo):
            np.take(a, idx, out=sg[i, :n])
        return n

    def _copy_in(self, blk: int, slot: int, k: int, n: int) -> int:
        """Device side of a block load: staging buffer k -> the block's slot on
        the copy stream, after the last kernel that read the slot."""
        torch = self.torch
        sa = self._stage_amps[k]
        r0 = slot * self.B
        with torch.cuda.stream(self._copy):
            if self._slot_reader[slot] is not None:
                self._copy.wait_event(self._slot_reader[slot])   # the last kernel that read this slot
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self._copy)
            # contiguous copies only: a strided destination would make torch run a
            # copy kernel, which waits for SMs the migration kernel holds
            self._pool_amps[r0:r0 + n].copy_(sa[:n], non_blocking=True)
            for f in range(7):
                self._pool_geo[f, r0:r0 + n].copy_(self._stage_geo[k][f, :n], non_blocking=True)
            e1.record(self._copy)
        self._stage_done[k] = e1
        self._copy_events.append((e0, e1))
        self._loaded_ev[blk] = e1
        self._slot_of[blk] = slot
        return n * (self.ns * self._host_amps.itemsize + 7 * 8)

    def _ensure(self, blocks, keep: set) -> tuple[int, int]:
        """Loads the blocks missing from the pool: slots are chosen in order
        (least recently used first), gathers run n_stage at a time in host
        threads, and each gathered block is copied as soon as it is ready."""
        loaded = nbytes = 0
        inflight: deque = deque()

        def finish():
            nonlocal nbytes
            fut, blk, slot, k = inflight.popleft()
            nbytes += self._copy_in(blk, slot, k, fut.result())

        for blk in blocks:
            if blk in self._slot_of:
                self._slot_of.move_to_end(blk)
                continue
            slot = self._free.pop() if self._free else self._victim(keep)
            if len(inflight) == self.n_stage:
                finish()
            k = self._stage_next
            self._stage_next = (k + 1) % self.n_stage
            if self._stage_done[k] is not None:
                self._stage_done[k].synchronize()      # the staging buffer's previous copy has left it
            inflight.append((self._gather_pool.submit(self._gather, blk, k), blk, slot, k))
            loaded += 1
        while inflight:
            finish()
        return loaded, nbytes

    # ------------------------------------------------------------- running
    def run(self, image, fold=None, tiles=None) -> StreamReport:
        """Migrate the tiles into ``image`` (and ``fold``), CUDA tensors shaped
        like the full grid; returns the per-pass record and the totals."""
        torch = self.torch
        from .base import OutputTile
        passes = self.plan(tiles)
        rep = StreamReport()
        self._copy_events = []
        t0 = time.perf_counter()
        compute = torch.cuda.current_stream()
        origin = torch.cuda.Event(enable_timing=True)   # the common time origin of both streams' events
        origin.record(compute)
        self._copy.wait_event(origin)
        nt = len(self.t_axis_ms)
        cur_tile, timg, tfold, out, vel = None, None, None, None, None
        pending = []
        if passes:
            loaded, nb = self._ensure(passes[0][1], set(passes[0][1]))
            rep.passes.append(PassResult(passes[0][0], passes[0][1], loaded, nb))
        for i, (tile, blocks, runs) in enumerate(passes):
            pr = rep.passes[i]
            ix0, ix1, iy0, iy1 = tile
            if tile != cur_tile:
                cur_tile = tile
                timg = torch.zeros((ix1 - ix0, iy1 - iy0, nt), dtype=image.dtype, device="cuda")
                tfold = None if fold is None else \
                    torch.zeros((ix1 - ix0, iy1 - iy0) + tuple(fold.shape[2:]), dtype=torch.int32, device="cuda")
                out = OutputTile(image=timg, fold=tfold, x_axis=self._x[ix0:ix1].contiguous(),
                                 y_axis=self._y[iy0:iy1].contiguous(), t_axis_ms=self._t)
                vel = self.velocity(ix0, ix1, iy0, iy1)
            for blk in blocks:
                compute.wait_event(self._loaded_ev[blk])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(compute)
            self.k.migrate_tile_runs(self.pool_traces, pool_runs(runs, self.B, self._slot_of), out, vel, self.cfg,
                                     kernel_type=self.kind)
            e1.record(compute)
            for blk in blocks:
                self._slot_reader[self._slot_of[blk]] = e1
            pending.append((pr, e0, e1))
            last_of_tile = i + 1 == len(passes) or passes[i + 1][0] != tile
            if last_of_tile:
                image[ix0:ix1, iy0:iy1] += timg
                if fold is not None:
                    fold[ix0:ix1, iy0:iy1] += tfold
            if i + 1 < len(passes):   # the next pass's blocks load while this one migrates
                nxt = passes[i + 1][1]
                loaded, nb = self._ensure(nxt, set(blocks) | set(nxt))
                rep.passes.append(PassResult(passes[i + 1][0], nxt, loaded, nb))
        torch.cuda.synchronize()
        rep.wall_s = time.perf_counter() - t0
        for pr, e0, e1 in pending:
            pr.kernel_ms = e0.elapsed_time(e1)
        rep.kernel_ms = sum(p.kernel_ms for p in rep.passes)
        rep.copy_ms = sum(a.elapsed_time(b) for a, b in self._copy_events)
        rel = lambda e: origin.elapsed_time(e)
        kern = [(rel(e0), rel(e1)) for _, e0, e1 in pending]
        rep.copy_overlap_ms = overlap_ms([(rel(a), rel(b)) for a, b in self._copy_events], kern)
        rep.first_load_ms = kern[0][0] if kern else 0.0
        rep.h2d_bytes = sum(p.h2d_bytes for p in rep.passes)
        rep.misses = sum(p.loaded for p in rep.passes)
        rep.hits = sum(len(p.blocks) for p in rep.passes) - rep.misses
        return rep
