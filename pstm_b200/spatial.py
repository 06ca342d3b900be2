"""Midpoint-ordered trace panels: the GPU form of the reference's spatial query.

The reference finds the traces of an output tile with a KD-tree over trace
midpoints (``SpatialIndex.query_rectangle``, ``pstm/data/spatial_index.py:178-231``;
``query_traces_for_tile``, ``:423-460``) and then loads those traces into a
fresh array for the backend.  Here the panel is put in midpoint order once --
by column ``floor((mx - x0) / column_width)``, then by ``my`` within a column
(ties in trace order) -- so the traces whose midpoints fall in a rectangle
are, column by column, contiguous row ranges found by binary search.  A tile
is then migrated against those ranges where they lie in HBM
(``CudaKernel.migrate_tile_runs``, the C entry point
``pstm_cuda_migrate_tile_runs_dev``): there is no per-tile gather.

The ranges of the rectangle's two edge columns also hold traces whose ``mx``
lies outside the rectangle.  For a tile's selection box (the tile's bounding
box grown by the maximum aperture) such traces are farther than the maximum
aperture from every pillar of the tile, so they add nothing to the image or
the fold; they only cost the kernel its per-(pillar, trace) distance test.
"""
from __future__ import annotations

import math

import numpy as np


class MidpointIndex:
    """Column-major midpoint order of a trace panel.

    ``order`` is the permutation that sorts the panel (``sorted = panel[order]``);
    ``runs`` works in positions of the sorted panel.
    """

    def __init__(self, midpoint_x, midpoint_y, column_width_m: float, x0: float | None = None):
        mx = np.ascontiguousarray(midpoint_x, dtype=np.float64)
        my = np.ascontiguousarray(midpoint_y, dtype=np.float64)
        if mx.ndim != 1 or mx.shape != my.shape:
            raise ValueError("midpoint_x and midpoint_y must be 1-D arrays of one length")
        if not (np.isfinite(mx).all() and np.isfinite(my).all()):
            raise ValueError("midpoints must be finite")
        if not (column_width_m > 0 and math.isfinite(column_width_m)):
            raise ValueError("column_width_m must be a positive number")
        self.width = float(column_width_m)
        self.x0 = float(x0) if x0 is not None else (float(mx.min()) if mx.size else 0.0)
        col = np.floor((mx - self.x0) / self.width).astype(np.int64)
        if col.size and col.min() < 0:
            raise ValueError("x0 must not exceed the smallest midpoint x")
        self.order = np.lexsort((my, col))
        self.n_columns = int(col.max()) + 1 if col.size else 0
        self.col_start = np.searchsorted(col[self.order], np.arange(self.n_columns + 1), side="left")
        self.mx_sorted = mx[self.order]
        self.my_sorted = my[self.order]

    @property
    def n_traces(self) -> int:
        return int(self.order.size)

    def _column_range(self, x_lo: float, x_hi: float) -> tuple[int, int]:
        if self.n_columns == 0 or not (x_hi >= x_lo):
            return 0, -1
        c_lo = max(0, math.floor((x_lo - self.x0) / self.width))
        c_hi = min(self.n_columns - 1, math.floor((x_hi - self.x0) / self.width))
        return c_lo, c_hi

    def runs(self, x_lo: float, x_hi: float, y_lo: float, y_hi: float, with_count: bool = False):
        """Ascending, disjoint [begin, end) ranges of the sorted panel holding
        every trace with x_lo <= mx <= x_hi and y_lo <= my <= y_hi (and the
        edge columns' traces with y in range but x outside).  With
        ``with_count``, also the number of traces inside the rectangle."""
        c_lo, c_hi = self._column_range(x_lo, x_hi)
        out: list[list[int]] = []
        count = 0
        if y_hi >= y_lo:
            for c in range(c_lo, c_hi + 1):
                s, e = int(self.col_start[c]), int(self.col_start[c + 1])
                ys = self.my_sorted[s:e]
                a = s + int(np.searchsorted(ys, y_lo, side="left"))
                b = s + int(np.searchsorted(ys, y_hi, side="right"))
                if b <= a:
                    continue
                if with_count:
                    if c in (c_lo, c_hi):
                        xs = self.mx_sorted[a:b]
                        count += int(np.count_nonzero((xs >= x_lo) & (xs <= x_hi)))
                    else:
                        count += b - a
                if out and out[-1][1] == a:
                    out[-1][1] = b
                else:
                    out.append([a, b])
        r = np.array(out, dtype=np.int64).reshape(-1, 2)
        return (r, count) if with_count else r

    def select(self, x_lo: float, x_hi: float, y_lo: float, y_hi: float) -> np.ndarray:
        """Positions (ascending) in the sorted panel of the traces inside the rectangle."""
        r = self.runs(x_lo, x_hi, y_lo, y_hi)
        if not len(r):
            return np.zeros(0, np.int64)
        pos = np.concatenate([np.arange(a, b, dtype=np.int64) for a, b in r])
        xs, ys = self.mx_sorted[pos], self.my_sorted[pos]
        return pos[(xs >= x_lo) & (xs <= x_hi) & (ys >= y_lo) & (ys <= y_hi)]


def sort_panel(traces, index: MidpointIndex):
    """The TraceBlock in the index's midpoint order (one copy of the panel;
    CUDA tensors stay on their device, NumPy arrays stay NumPy)."""
    from .base import TraceBlock
    order = index.order
    if hasattr(traces.amplitudes, "is_cuda"):
        import torch
        o = torch.as_tensor(order, device=traces.amplitudes.device)
        take = lambda a: None if a is None else a.index_select(0, o)
    else:
        take = lambda a: None if a is None else np.ascontiguousarray(np.asarray(a)[order])
    return TraceBlock(amplitudes=take(traces.amplitudes), source_x=take(traces.source_x),
                      source_y=take(traces.source_y), receiver_x=take(traces.receiver_x),
                      receiver_y=take(traces.receiver_y), offset=take(traces.offset),
                      midpoint_x=take(traces.midpoint_x), midpoint_y=take(traces.midpoint_y),
                      weights=take(getattr(traces, "weights", None)), sample_rate_ms=traces.sample_rate_ms,
                      start_time_ms=traces.start_time_ms)
