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


def test_reference_arm_line(capsys, monkeypatch):
    """The reference arm (CPU restatement, no GPU) at 32^3 with 2000 droplets prints one JSON line
    with the contract's keys: impl, metric, value, cpu_baseline (kind, cores, sample) and a
    host-only e2e."""
    import json
    monkeypatch.delenv("RANK", raising=False)
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    bench.main(["--impl", "reference", "--N", "32", "--nd", "2000", "--steps", "2", "--warmup", "3"])
    lines = [l for l in capsys.readouterr().out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["config"]["N"] == 32 and d["config"]["n_droplets"] == 2000 and d["config"]["interp"] == "tricubic"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing(capsys, monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    bench.main(["--impl", "reference", "--N", "32", "--nd", "100", "--steps", "1"])
    assert capsys.readouterr().out == ""


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
