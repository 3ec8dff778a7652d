"""bench.py host logic without a GPU: argument defaults of the contract, the reference arm's
sizing, and the max-over-ranks timing of the multi-rank path over a world-size-2 gloo group."""
import os
import socket

import torch.multiprocessing as mp

import bench


def test_defaults():
    a = bench.parse_args([])
    assert a.gpus == 1 and a.warmup >= 3 and a.steps > 0
    assert a.interp == "learned" and a.N == 256 and a.nd == 1_000_000
    assert a.run_steps == 500 and a.judge_every == 500


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    q.put((rank, bench.allreduce_max(10.0 + rank, world)))
    dist.destroy_process_group()


def test_max_over_ranks_two_ranks():
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
    assert res == {0: 11.0, 1: 11.0}
