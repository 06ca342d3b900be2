"""Replica plan for several GPUs: disjoint output tiles, no data collective.

Output tiles of a migration are independent and the trace panel is read-only
(the reference executor migrates tiles one after another, pstm/pipeline/
executor.py:1208-1301), so N processes, one per GPU, each take a disjoint
subset of the tiles.  The only cross-rank communication is timing: a barrier
around the timed region and the maximum of the per-rank times.
"""
from __future__ import annotations

from typing import Sequence


def grid_tiles(grid_nx: int, grid_ny: int, tile: int) -> list[tuple[int, int, int, int]]:
    """(ix0, ix1, iy0, iy1) of the tiles covering the grid, row-major."""
    out = []
    for ix0 in range(0, grid_nx, tile):
        for iy0 in range(0, grid_ny, tile):
            out.append((ix0, min(grid_nx, ix0 + tile), iy0, min(grid_ny, iy0 + tile)))
    return out


def rank_schedule(tiles: Sequence, rank: int, world: int, n_steps: int) -> list:
    """Tiles of one rank for n_steps steps: tile (rank + j * world) mod n_tiles.

    Within any window of len(tiles) // world consecutive steps the ranks'
    tiles are disjoint; with more steps than that the walk wraps around.
    """
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    n = len(tiles)
    return [tiles[(rank + j * world) % n] for j in range(n_steps)]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank float over the process group (identity without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
