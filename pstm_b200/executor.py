"""Device-resident tiled migration of a survey grid.

The reference executor walks the output grid tile by tile; for every tile it
asks its spatial index for the traces whose midpoints can reach the tile
(``SpatialIndex.query_traces_for_tile``, ``pstm/data/spatial_index.py:423-460``),
loads them, calls the backend's ``migrate_tile`` and adds the tile into the
output volume (``pstm/pipeline/executor.py:1397-1858``, accumulation at
:1776-1777).  This driver does the same with everything on the GPU: the whole
trace panel stays resident in HBM, the traces of a tile are those whose
midpoint lies in the tile's bounding box grown by the maximum aperture (every
other trace is outside the aperture of every pillar of the tile, so it adds
nothing to the image or the fold), they are gathered into a contiguous tile
panel, migrated by ``CudaKernel`` and the tile is added into the full image.

With ``spatial`` the executor first puts the panel in midpoint order
(``pstm_b200.spatial``): a tile's selection box is then a few contiguous row
ranges found by binary search, and the tile is migrated against them in place
(``CudaKernel.migrate_tile_runs``), with no per-tile gather.  The learned form
keeps the gather (its probe and fallback decide per gathered tile).

Torch holds the buffers and does the remaining selection/gather plumbing.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np


def tile_ranges(nx: int, ny: int, tile: int) -> list[tuple[int, int, int, int]]:
    """(ix0, ix1, iy0, iy1) of the tiles covering an nx x ny grid, row-major."""
    return [(x0, min(nx, x0 + tile), y0, min(ny, y0 + tile))
            for x0 in range(0, nx, tile) for y0 in range(0, ny, tile)]


def selection_box(x_axis, y_axis, tile, max_aperture_m: float) -> tuple[float, float, float, float]:
    """Midpoint box (x_lo, x_hi, y_lo, y_hi) of the traces that can reach a tile."""
    ix0, ix1, iy0, iy1 = tile
    xs, ys = np.asarray(x_axis[ix0:ix1]), np.asarray(y_axis[iy0:iy1])
    a = float(max_aperture_m)
    return float(xs.min()) - a, float(xs.max()) + a, float(ys.min()) - a, float(ys.max()) + a


@dataclass
class TileResult:
    tile: tuple
    n_traces: int
    pairs: int          # pillars x samples x selected traces
    kernel_ms: float    # CUDA-event time of the migration call
    processed_traces: int | None = None   # rows the kernel read (spatial mode: whole runs)
    used_surrogate: bool | None = None
    probe_max_ms: float | None = None


class TiledExecutor:
    """Migrate a survey grid tile by tile with one ``CudaKernel``.

    ``traces`` is a TraceBlock of CUDA tensors holding the whole survey;
    ``velocity(ix0, ix1, iy0, iy1)`` returns the tile's v_rms as a CUDA tensor
    (nt,) or (tile_nx, tile_ny, nt); ``x_axis``/``y_axis``/``t_axis_ms`` are the
    full grid's axes (NumPy).  ``spatial`` (True, or a column width in m;
    True takes an eighth of a tile's width) sorts the panel into midpoint order
    once -- a second copy of the panel while the caller holds the first -- and
    migrates each tile against its row ranges in place.  Without it, a
    midpoint index on the host selects each tile's traces (no per-tile scan of
    the panel) and they are gathered into a tile panel.  Panels larger than
    HBM: ``pstm_b200.streaming.StreamingExecutor``.
    """

    def __init__(self, kernel, traces, x_axis, y_axis, t_axis_ms, velocity, config,
                 kernel_type: str = "straight_ray", tile: int = 64, surrogate=None,
                 max_residual_ms: float = 0.1, spatial: bool | float = False):
        import torch
        self.torch = torch
        self.k = kernel
        self.tb = traces
        self.x_axis, self.y_axis = np.asarray(x_axis, np.float64), np.asarray(y_axis, np.float64)
        self.t_axis_ms = np.asarray(t_axis_ms, np.float64)
        self.velocity = velocity
        self.cfg = config
        self.kind = kernel_type
        self.tile = int(tile)
        self.surrogate = surrogate
        self.max_residual_ms = max_residual_ms
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
        self._x, self._y, self._t = dev(self.x_axis), dev(self.y_axis), dev(self.t_axis_ms)
        from .spatial import MidpointIndex, sort_panel
        if spatial is True or spatial is False or spatial is None:
            dx = abs(float(self.x_axis[1] - self.x_axis[0])) if len(self.x_axis) > 1 else 1.0
            width = max(self.tile * dx / 8.0, 1e-3)
        else:
            width = float(spatial)
        host = lambda a: a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
        # The midpoint index finds a tile's traces in O(log n + selected) on the
        # host instead of a mask over the whole panel per tile.  Only the
        # spatial mode reorders the panel itself (one copy of it).
        midx = MidpointIndex(host(traces.midpoint_x), host(traces.midpoint_y), width)
        self.index = None
        if spatial is not False and spatial is not None:
            self.index = midx
            self.tb = sort_panel(traces, self.index)
        else:
            self._lookup = midx

    def tiles(self):
        return tile_ranges(len(self.x_axis), len(self.y_axis), self.tile)

    def select(self, tile):
        """Indices (CUDA int64, ascending) of the traces that can reach the tile."""
        x_lo, x_hi, y_lo, y_hi = selection_box(self.x_axis, self.y_axis, tile, self.cfg.max_aperture_m)
        if self.index is not None:   # positions in the sorted panel
            return self.torch.as_tensor(self.index.select(x_lo, x_hi, y_lo, y_hi), device="cuda")
        pos = self._lookup.select(x_lo, x_hi, y_lo, y_hi)   # positions in midpoint order
        return self.torch.as_tensor(np.sort(self._lookup.order[pos]), device="cuda")

    def _gather(self, idx):
        from .base import TraceBlock
        t = self.tb
        take = lambda a: None if a is None else a.index_select(0, idx)
        return TraceBlock(amplitudes=t.amplitudes.index_select(0, idx), source_x=take(t.source_x),
                          source_y=take(t.source_y), receiver_x=take(t.receiver_x), receiver_y=take(t.receiver_y),
                          offset=take(t.offset), midpoint_x=take(t.midpoint_x), midpoint_y=take(t.midpoint_y),
                          weights=take(getattr(t, "weights", None)), sample_rate_ms=t.sample_rate_ms,
                          start_time_ms=t.start_time_ms)

    def run_tile(self, tile, image, fold=None) -> TileResult:
        """Migrate one tile and add it into ``image`` (and ``fold``), CUDA tensors
        shaped like the full grid (fold (nx, ny, nt) or (nx, ny))."""
        torch = self.torch
        from .base import OutputTile
        ix0, ix1, iy0, iy1 = tile
        nt = len(self.t_axis_ms)
        runs = None
        if self.index is not None and self.surrogate is None:
            runs, n = self.index.runs(*selection_box(self.x_axis, self.y_axis, tile, self.cfg.max_aperture_m),
                                      with_count=True)
            processed = int((runs[:, 1] - runs[:, 0]).sum()) if len(runs) else 0
        else:
            idx = self.select(tile)
            n = processed = int(idx.numel())
        res = TileResult(tile, n, (ix1 - ix0) * (iy1 - iy0) * nt * n, 0.0, processed_traces=processed)
        if processed == 0:
            return res
        sub = self._gather(idx) if runs is None else None
        timg = torch.zeros((ix1 - ix0, iy1 - iy0, nt), dtype=image.dtype, device="cuda")
        tfold = None
        if fold is not None:
            tfold = torch.zeros((ix1 - ix0, iy1 - iy0) + tuple(fold.shape[2:]), dtype=torch.int32, device="cuda")
        out = OutputTile(image=timg, fold=tfold, x_axis=self._x[ix0:ix1].contiguous(),
                         y_axis=self._y[iy0:iy1].contiguous(), t_axis_ms=self._t)
        vel = self.velocity(ix0, ix1, iy0, iy1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if self.surrogate is not None:
            _, rep = self.k.migrate_tile_learned(sub, out, vel, self.surrogate, self.cfg, kernel_type=self.kind,
                                                 max_residual_ms=self.max_residual_ms)
            res.used_surrogate, res.probe_max_ms = rep["used_surrogate"], rep["probe_max_ms"]
        elif runs is not None:
            self.k.migrate_tile_runs(self.tb, runs, out, vel, self.cfg, kernel_type=self.kind)
        else:
            method = {"straight_ray": self.k.migrate_tile, "curved_ray": self.k.migrate_tile_curved_ray,
                      "anisotropic_vti": self.k.migrate_tile_vti,
                      "curved_vti": self.k.migrate_tile_curved_vti}[self.kind]
            method(sub, out, vel, self.cfg)
        e1.record()
        image[ix0:ix1, iy0:iy1] += timg
        if fold is not None:
            fold[ix0:ix1, iy0:iy1] += tfold
        torch.cuda.synchronize()
        res.kernel_ms = e0.elapsed_time(e1)
        return res

    def run(self, image, fold=None, tiles=None) -> list[TileResult]:
        t0 = time.perf_counter()
        out = [self.run_tile(t, image, fold) for t in (tiles if tiles is not None else self.tiles())]
        self.wall_s = time.perf_counter() - t0
        return out
