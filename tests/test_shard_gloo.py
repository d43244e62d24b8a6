"""Ensemble sharding over ranks: partition properties, and a world_size-2 gloo run
in which every rank derives the same partition and the gathered shards cover the
ensemble exactly once (CPU only; no data-path collective)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from qasmhd_b200 import problems as P
from qasmhd_b200 import shard


def test_partition_covers_and_balances():
    cells = [p.interior_cells for p in P.ensemble(512)]
    for world in (1, 2, 4, 8):
        parts = shard.partition(cells, world)
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(len(cells)))
        assert shard.imbalance(cells, parts) < 1.01


def test_partition_deterministic_ties():
    assert shard.partition([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.partition([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cells = [p.interior_cells for p in P.ensemble(64, lo=16, hi=64)]
        mine = shard.partition(cells, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        q.put((rank, gathered, sum(cells[i] for i in mine)))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_agree():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g0, g1 = res[0][1], res[1][1]
    assert g0 == g1
    flat = sorted(i for part in g0 for i in part)
    assert flat == list(range(64))
    loads = [r[2] for r in res]
    assert max(loads) / (sum(loads) / 2) < 1.1
