"""Multi-process replica logic on CPU: 2 gloo ranks, disjoint tiles, max timing."""
from __future__ import annotations

import os

import pytest


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from pstm_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tiles = replicas.grid_tiles(256, 256, 64)
        mine = replicas.rank_schedule(tiles, rank, world, 8)
        t = replicas.max_over_ranks(10.0 * (rank + 1), dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        q.put((rank, t, gathered))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_take_disjoint_tiles_and_max_time():
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, gathered in res:
        assert t == 20.0                      # max over ranks, on every rank
        a, b = gathered
        assert not set(a) & set(b)            # 8 steps x 2 ranks = all 16 tiles, disjoint
        assert len(set(a) | set(b)) == 16


def test_single_process_schedule():
    from pstm_b200 import replicas
    tiles = replicas.grid_tiles(256, 200, 64)
    assert len(tiles) == 16 and tiles[-1] == (192, 256, 192, 200)
    assert replicas.rank_schedule(tiles, 0, 1, 3) == tiles[:3]
    assert replicas.max_over_ranks(3.5) == 3.5
    with pytest.raises(ValueError):
        replicas.rank_schedule(tiles, 2, 2, 1)
