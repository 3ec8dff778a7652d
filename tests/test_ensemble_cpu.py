"""Host logic of the ensemble across ranks (no GPU): round-robin box sharding, and the gather of
per-box results over a world-size-2 gloo group."""
import os

import pytest
import torch.multiprocessing as mp

from lucky_droplets_b200.ensemble import box_counts, gather_per_box, shard


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_shard_covers_every_box_once(world):
    ids = [b for r in range(world) for b in shard(64, r, world)]
    assert sorted(ids) == list(range(64))
    counts = box_counts(64, 0)
    assert counts.min() >= 5000 and counts.max() <= 50000


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ids = shard(10, rank, world)
    got = gather_per_box([100 + b for b in ids], ids, 10, world)
    q.put((rank, got))
    dist.destroy_process_group()


def test_gather_per_box_two_ranks():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res[0] == res[1] == [100 + b for b in range(10)]
