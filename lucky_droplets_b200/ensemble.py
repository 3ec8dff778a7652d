"""Ensembles of independent small boxes, advanced by CUDA-graph replays (no counterpart in the
reference, which runs one box; lucky-droplet statistics need many rare-event samples).

The ensemble configuration: 64 independent 64^3 boxes (flow seeds 0..63, the 64^3 parameters:
nu = 0.01, dt = 2e-3, RK2 + integrating factor, eps = 0.1 on shells 1..2, trilinear droplets with
log-uniform Stokes times and settling), droplet counts uniform in [5e3, 5e4] per box, collision
counts per box.

Each box is a ForcedDNS with its droplets and collider.  The boxes' steps are spread over
`streams` CUDA streams and captured, `steps_per_graph` steps at a time, into one CUDA graph: one
graph launch advances every box by that many steps, the boxes running concurrently on the GPU,
with no host work between the kernels.  `autotune()` picks the stream count and the steps per
graph by timing short replays.  With several ranks the boxes are dealt out round-robin by box
index; there is no exchange between boxes, per-box results are gathered on the host.

    python -m lucky_droplets_b200.ensemble [--boxes 64] [--N 64] [--steps 2000]
"""
import argparse
import json
import os
import time

import numpy as np

from . import _lib
from .dns import ForcedDNS, Droplets
from .init import init_flow, init_droplets


def _torch():
    import torch
    return torch


def box_counts(n_boxes, seed=0, lo=5000, hi=50000):
    """Droplet count of every box: uniform integers in [lo, hi] from a seeded generator."""
    rng = np.random.default_rng(seed + 4242)
    return rng.integers(lo, hi + 1, n_boxes)


def shard(n_boxes, rank, world):
    """Box indices of one rank: round-robin, so uneven droplet counts spread over the ranks."""
    return list(range(rank, n_boxes, world))


def gather_per_box(local, ids, n_boxes, world):
    """Per-box values held by each rank (in the order of its `ids`) -> the list over all boxes, in
    box order, on every rank (host gather; there is no device exchange)."""
    out = [None] * n_boxes
    if world == 1:
        for b, v in zip(ids, local):
            out[b] = v
        return out
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, list(zip(ids, local)))
    for part in parts:
        for b, v in part:
            out[b] = v
    return out


class Ensemble:
    def __init__(self, n_boxes=64, N=64, nu=0.01, dt=2e-3, eps=0.1, kf=2, precision="f32", nd=(5000, 50000),
                 seed=0, interp="trilinear", g=0.1, collide=True, sort_every=20, rank=0, world=1, device=None):
        from .collide import Collider
        self.n_boxes = n_boxes
        self.N = N
        self.counts = box_counts(n_boxes, seed, *nd)
        self.ids = shard(n_boxes, rank, world)
        self.world = world
        self.boxes = []
        for b in self.ids:
            dns = ForcedDNS.config(N, nu, dt, eps=eps, kf=kf, precision=precision, device=device)
            init_flow(dns, seed + b)
            pos, tau, radius = init_droplets(int(self.counts[b]), seed + b, "uniform_tau")
            d = Droplets(dns.plan, pos, np.zeros((tau.shape[0], 3)), tau, method=interp, g=g, radius=radius)
            u = dns.velocity()
            d.vel.copy_(d.gather(u))
            del u
            # cells of at least 2 r_max (the search is exact for any larger cell); with few droplets
            # per box, cells of about one droplet each keep the cell-sized work (starts, column
            # blocks) proportional to the droplets
            cell = max(2.0 * float(radius.max()), 2.0 * np.pi / max(1.0, d.n ** (1.0 / 3.0)))
            col = Collider(d.n, cell, device=dns.plan.device) if collide else None
            dns.attach(d, collider=col, sort_every=sort_every)
            self.boxes.append(dns)
        # FFT launch variants: timed on the first box, applied to all (same N and precision)
        self.fft_tuning = self.boxes[0].plan.autotune() if self.boxes else None
        for b in self.boxes[1:]:
            b.plan.set_tuning(self.fft_tuning["choice"])
        self.graph = None
        self.streams = []
        self.steps_per_graph = 0
        self.tuning = []

    @property
    def n_droplets(self):
        return int(sum(int(self.counts[b]) for b in self.ids))

    # ---- eager stepping (reference for the graph path) -------------------------------------------
    def step_eager(self, nsteps, n_streams=1):
        torch = _torch()
        streams = self._streams(n_streams)
        cur = torch.cuda.current_stream()
        for s in streams:
            s.wait_stream(cur)
        for _ in range(nsteps):
            for j, box in enumerate(self.boxes):
                s = streams[j % len(streams)]
                with torch.cuda.stream(s):
                    box.step(1, stream=s)
        for s in streams:
            cur.wait_stream(s)

    def _streams(self, n):
        torch = _torch()
        while len(self.streams) < n:
            self.streams.append(torch.cuda.Stream(device=self.boxes[0].plan.device))
        return self.streams[:n]

    # ---- CUDA graph ------------------------------------------------------------------------------
    def capture(self, steps_per_graph, n_streams):
        """Capture `steps_per_graph` steps of every box, spread over `n_streams` streams, as one
        CUDA graph.  Every box must have stepped once eagerly before (its tables are built on the
        first step)."""
        torch = _torch()
        self.graph = None
        streams = self._streams(n_streams)
        saved = [(b.t, b.nstep) for b in self.boxes]
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(device=self.boxes[0].plan.device)
        cap.wait_stream(torch.cuda.current_stream())
        with torch.cuda.graph(g, stream=cap, capture_error_mode="thread_local"):
            for s in streams:
                s.wait_stream(cap)
            for _ in range(steps_per_graph):
                for j, box in enumerate(self.boxes):
                    s = streams[j % n_streams]
                    with torch.cuda.stream(s):
                        box.step(1, stream=s)
            for s in streams:
                cap.wait_stream(s)
        for b, (t, n) in zip(self.boxes, saved):  # capturing ran nothing
            b.t, b.nstep = t, n
        self.graph = g
        self.steps_per_graph = steps_per_graph
        self.n_graph_streams = n_streams
        return g

    def replay(self, n_graphs=1):
        """Advance every box by n_graphs * steps_per_graph steps (graph launches on the current
        stream)."""
        for _ in range(n_graphs):
            self.graph.replay()
        k = n_graphs * self.steps_per_graph
        for b in self.boxes:
            b.t += k * b.dt
            b.nstep += k

    def run(self, nsteps):
        """nsteps steps of every box: whole graphs, then eager steps for the remainder."""
        full = nsteps // self.steps_per_graph if self.graph is not None else 0
        if full:
            self.replay(full)
        rest = nsteps - full * self.steps_per_graph
        if rest:
            self.step_eager(rest, max(1, getattr(self, "n_graph_streams", 1)))

    def autotune(self, streams=(4, 8, 16), steps_per_graph=(5, 10, 20), trial_graphs=2):
        """Time `trial_graphs` replays of every (streams, steps per graph) candidate and keep the
        fastest per step; the trial steps advance the boxes like any other steps.  Returns the
        table of candidates (ms per step)."""
        torch = _torch()
        best = None
        self.tuning = []
        for S in streams:
            for K in steps_per_graph:
                self.capture(K, S)
                self.replay(1)  # first replay uploads the graph
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                self.replay(trial_graphs)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / (trial_graphs * K)
                self.tuning.append({"streams": S, "steps_per_graph": K, "ms_per_step": ms})
                if best is None or ms < best[0]:
                    best = (ms, S, K)
        self.capture(best[2], best[1])
        return self.tuning

    # ---- results ---------------------------------------------------------------------------------
    def collision_counts(self):
        """Colliding pairs of the last step, per local box (host)."""
        return [int(b.collider.count.item()) if b.collider is not None else 0 for b in self.boxes]

    def check(self):
        return [b.check() for b in self.boxes]


def main(argv=None):
    torch = _torch()
    ap = argparse.ArgumentParser()
    ap.add_argument("--boxes", type=int, default=64)
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--precision", default="f32")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--streams", type=int, default=0, help="0: autotune")
    ap.add_argument("--steps-per-graph", type=int, default=10)
    a = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    t0 = time.perf_counter()
    ens = Ensemble(a.boxes, a.N, precision=a.precision, seed=a.seed, rank=rank, world=world)
    ens.step_eager(1)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    if a.streams:
        ens.capture(a.steps_per_graph, a.streams)
        tuning = None
    else:
        tuning = ens.autotune()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.run(a.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    flags = ens.check()
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    coll = gather_per_box(ens.collision_counts(), ens.ids, a.boxes, world)
    nd = [int(c) for c in ens.counts]
    out = {"workload": f"{a.boxes} boxes x {a.N}^3 RK2+IF (nu=0.01, dt=2e-3), droplets per box uniform in "
                       f"[5e3, 5e4] (trilinear, settling), collisions every step",
           "n_gpus": world, "steps": a.steps, "ms_per_step": ms / a.steps,
           "box_steps_per_s": a.boxes * a.steps / (ms / 1e3),
           "droplet_steps_per_s": sum(nd) * a.steps / (ms / 1e3),
           "graph": {"streams": ens.n_graph_streams, "steps_per_graph": ens.steps_per_graph},
           "autotune": tuning, "fft_autotune": ens.fft_tuning, "setup_s": setup_s, "status_flags_max": max(flags) if flags else 0,
           "droplets_per_box": nd, "collision_pairs_last_step_per_box": coll}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
