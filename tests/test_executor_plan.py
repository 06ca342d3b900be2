"""Tile enumeration and trace-selection boxes of the tiled executor (CPU)."""
from __future__ import annotations

import numpy as np

from pstm_b200.executor import selection_box, tile_ranges


def test_tiles_cover_the_grid_once():
    tiles = tile_ranges(10, 7, 4)
    cover = np.zeros((10, 7), int)
    for x0, x1, y0, y1 in tiles:
        cover[x0:x1, y0:y1] += 1
    assert (cover == 1).all() and len(tiles) == 3 * 2


def test_selection_box_keeps_every_trace_inside_the_aperture():
    """A midpoint outside the box is farther than max_aperture from every pillar."""
    rng = np.random.default_rng(1)
    x, y = np.arange(20) * 12.5, np.arange(16) * 12.5
    tile = (4, 12, 3, 9)
    ap = 60.0
    box = selection_box(x, y, tile, ap)
    m = rng.uniform(-200, 500, (20000, 2))
    out = ~((m[:, 0] >= box[0]) & (m[:, 0] <= box[1]) & (m[:, 1] >= box[2]) & (m[:, 1] <= box[3]))
    X, Y = np.meshgrid(x[4:12], y[3:9], indexing="ij")
    d = np.sqrt((X.ravel()[None, :] - m[out, 0:1]) ** 2 + (Y.ravel()[None, :] - m[out, 1:2]) ** 2)
    assert (d.min(axis=1) > ap).all()
