"""Ensembles of independent small boxes advanced together (no counterpart in the reference, which
runs one box; lucky-droplet statistics need many rare-event samples).

The ensemble configuration: 64 independent 64^3 boxes (flow seeds 0..63, the 64^3 parameters:
nu = 0.01, dt = 2e-3, RK2 + integrating factor, eps = 0.1 on shells 1..2, trilinear droplets with
log-uniform Stokes times and settling), droplet counts uniform in [5e3, 5e4] per box, collision
counts per box.

The boxes are a batch dimension of one multi-box plan (ld_plan_create_boxes): every pass of the
flow step - transforms, fused z pass, k-space update, epilogue - is one launch over all boxes, with
per-box forcing.  The droplets of all boxes live in one set of arrays, each droplet carrying its
box; one droplet launch per stage samples each droplet's own box, and one multi-box collider
(cells keyed box-major) sorts, searches and counts the pairs of every box.  `steps_per_graph`
steps are captured into one CUDA graph, so one graph launch advances every box by that many
steps with no host work between the kernels.  `autotune()` picks the launch variants of the
strided transform passes on the multi-box plan (one-shot tiles or pipelined CTAs, 1..3 per SM) and
the steps per graph.  With several ranks the boxes are dealt out round-robin by box index; there
is no exchange between boxes, per-box results are gathered on the host.

    python -m lucky_droplets_b200.ensemble [--boxes 64] [--N 64] [--steps 2000]
"""
import argparse
import ctypes
import json
import os
import time

import numpy as np

from . import _lib
from ._lib import check, ptr, stream_ptr
from .collide import Collider
from .dns import ForcedDNS, Droplets
from .init import init_flow, init_droplets
from .spectral import Plan, flow_params, TWO_PI


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


def box_cell_size(radius_max, droplets_per_box):
    """Collision cells of at least 2 r_max (the search is exact for any larger cell); with few
    droplets per box, cells of about one droplet each keep the per-cell work proportional to the
    droplets."""
    return max(2.0 * float(radius_max), TWO_PI / max(1.0, float(droplets_per_box) ** (1.0 / 3.0)))


class Ensemble:
    """The boxes of one rank, advanced as one batch."""

    def __init__(self, n_boxes=64, N=64, nu=0.01, dt=2e-3, eps=0.1, kf=2, precision="f32", nd=(5000, 50000),
                 seed=0, interp="trilinear", g=0.1, collide=True, sort_every=20, rank=0, world=1, device=None):
        torch = _torch()
        self.n_boxes = n_boxes
        self.N = N
        self.counts = box_counts(n_boxes, seed, *nd)
        self.ids = shard(n_boxes, rank, world)
        self.world = world
        B = len(self.ids)
        self.nb = B
        self.dt, self.nu = float(dt), float(nu)
        self.g = float(g)
        self.method = _lib.LD_INTERP[interp]
        self.sort_every = int(sort_every)
        self.prm = flow_params(dt, nu, eps * TWO_PI ** 3 / kf, tuple(range(1, kf + 1)))
        p = self.plan = Plan(N, precision, device, nbox=B)
        check(_lib.lib().ld_plan_prepare(p.handle, ctypes.byref(self.prm), stream_ptr()))
        shape = (B, 3, p.Mx, p.My, p.Mzp)
        self.uk = torch.zeros(shape, dtype=p.cdtype, device=p.device)
        self.aux = torch.zeros_like(self.uk)
        self.acc = torch.zeros_like(self.uk)
        self.u4 = torch.empty((B, N, N, N, 4), dtype=p.rdtype, device=p.device)
        # initial state of every box: the single-box construction (flow seed + b, droplets at the
        # interpolated fluid velocity), copied into the batch
        one = ForcedDNS.config(N, nu, dt, eps=eps, kf=kf, precision=precision, device=p.device)
        pos_l, vel_l, tau_l, rad_l, box_l, id_l = [], [], [], [], [], []
        for j, b in enumerate(self.ids):
            init_flow(one, seed + b)
            self.uk[j].copy_(one.uk)
            pos, tau, radius = init_droplets(int(self.counts[b]), seed + b, "uniform_tau")
            d = Droplets(one.plan, pos, np.zeros((tau.shape[0], 3)), tau, method=interp, g=g, radius=radius)
            u = one.velocity()
            vel_l.append(d.gather(u))
            del u
            pos_l.append(d.pos)
            tau_l.append(d.tau)
            rad_l.append(d.radius)
            box_l.append(torch.full((d.n,), j, dtype=torch.int32, device=p.device))
            id_l.append(torch.arange(d.n, dtype=torch.int64, device=p.device) + int(b) * (1 << 32))
        del one
        self.pos = torch.cat(pos_l).contiguous()
        self.vel = torch.cat(vel_l).contiguous()
        self.tau = torch.cat(tau_l).contiguous()
        self.radius = torch.cat(rad_l).contiguous()
        self.box = torch.cat(box_l).contiguous()
        self.dids = torch.cat(id_l).contiguous()  # droplet id: box << 32 | index within the box
        self.a1 = torch.zeros_like(self.vel)
        self.n = int(self.pos.shape[0])
        self.collider = None
        self.pairs = None
        cell = box_cell_size(float(self.radius.max()), self.n / max(1, B))
        self.collider = Collider(self.n, cell, device=p.device, nbox=B)
        if collide:
            self.pairs = torch.empty((max(1024, 4 * self.n), 2), dtype=torch.int32, device=p.device)
        self._order = torch.empty(self.n, dtype=torch.int32, device=p.device)
        self._scratch = {}
        self.sort()
        self.collide = collide
        self.fft_tuning = p.autotune()
        self.t = 0.0
        self.nstep = 0
        self.graph = None
        self.graphs = {}
        self.steps_per_graph = 0
        self.tuning = []
        torch.cuda.synchronize(p.device)

    @property
    def n_droplets(self):
        return self.n

    # ---- one step of every box ---------------------------------------------------------------------
    def arrays(self):
        return [("pos", self.pos), ("vel", self.vel), ("tau", self.tau), ("a1", self.a1), ("radius", self.radius),
                ("box", self.box), ("dids", self.dids)]

    def sort(self, stream=None):
        """Every per-droplet array into (box, cell) order, in place (addresses kept for graphs)."""
        torch = _torch()
        L = _lib.lib()
        st = stream_ptr(stream)
        self.collider.cell_order_boxes(self.pos, self.box, self._order, stream)
        for name, t in self.arrays():
            row = t.element_size() * (t.shape[1] if t.dim() > 1 else 1)
            tmp = self._scratch.get(name)
            if tmp is None:
                tmp = self._scratch[name] = torch.empty_like(t)
            check(L.ld_permute_rows(ptr(t), ptr(tmp), ptr(self._order), self.n, row, st))
            check(L.ld_copy_async(ptr(t), ptr(tmp), t.numel() * t.element_size(), st))

    def _step_one(self, stream=None):
        L = _lib.lib()
        h = self.plan.handle
        st = stream_ptr(stream)
        prm = ctypes.byref(self.prm)
        args = (ptr(self.u4), ptr(self.box), ptr(self.pos), ptr(self.vel), ptr(self.tau), ptr(self.a1), self.n,
                self.method, self.dt, self.g, st)
        check(L.ld_rk2if_stage(h, 1, ptr(self.uk), ptr(self.aux), ptr(self.acc), ptr(self.u4), prm, st))
        check(L.ld_droplet_stage_boxes(h, 1, *args))
        check(L.ld_rk2if_stage(h, 2, ptr(self.uk), ptr(self.aux), ptr(self.acc), ptr(self.u4), prm, st))
        check(L.ld_step_epilogue_plane0(h, ptr(self.uk), st))
        check(L.ld_droplet_stage_boxes(h, 2, *args))
        self.t += self.dt
        self.nstep += 1
        if self.sort_every > 0 and self.nstep % self.sort_every == 0:
            self.sort(stream)
        if self.collide:
            self.collider.collide_boxes(self.pos, self.radius, self.box, self.pairs, stream)

    def step_eager(self, nsteps, stream=None):
        for _ in range(nsteps):
            self._step_one(stream)

    # ---- CUDA graph ------------------------------------------------------------------------------
    def _phase(self):
        return self.nstep % self.sort_every if self.sort_every > 0 else 0

    def _capture_one(self):
        torch = _torch()
        saved = (self.t, self.nstep)
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(device=self.plan.device)
        cap.wait_stream(torch.cuda.current_stream())
        try:
            with torch.cuda.graph(g, stream=cap, capture_error_mode="thread_local"):
                self.step_eager(self.steps_per_graph, stream=cap)
        finally:
            self.t, self.nstep = saved
        self.graphs[self._phase()] = g
        return g

    def capture(self, steps_per_graph):
        """Capture `steps_per_graph` steps of every box as one CUDA graph (nothing runs during the
        capture; the step counters are restored).  The re-sorting every sort_every steps sits in a
        graph at the positions its starting step gives: replays from another phase of the
        re-sorting period get a graph of their own, captured on first use."""
        self.graphs = {}
        self.steps_per_graph = int(steps_per_graph)
        self.graph = self._capture_one()
        return self.graph

    def replay(self, n_graphs=1):
        """Advance every box by n_graphs * steps_per_graph steps (graph launches on the current
        stream)."""
        for _ in range(n_graphs):
            g = self.graphs.get(self._phase())
            if g is None:
                g = self._capture_one()
            g.replay()
            for _ in range(self.steps_per_graph):
                self.t += self.dt
            self.nstep += self.steps_per_graph

    def run(self, nsteps):
        """nsteps steps of every box: whole graphs, then eager steps for the rest."""
        full = nsteps // self.steps_per_graph if self.graph is not None else 0
        self.replay(full)
        if nsteps - full * self.steps_per_graph:
            self.step_eager(nsteps - full * self.steps_per_graph)

    def autotune(self, steps_per_graph=(5, 10, 20), trial_graphs=2):
        """The launch variants of the strided transform passes are timed on the multi-box plan at
        construction (ld_plan_autotune: one-shot tiles, or pipelined with 1, 2, 3 CTAs per SM);
        here the steps per graph are picked by timing `trial_graphs` rounds of replays of each
        candidate (a round visits every phase of the re-sorting period once, after a first round
        that captures and uploads the graphs; the trial steps advance the boxes like any other
        steps).  Returns the table (ms per step)."""
        import math
        torch = _torch()
        best = None
        self.tuning = []
        for K in steps_per_graph:
            self.capture(K)
            rounds = self.sort_every // math.gcd(self.sort_every, K) if self.sort_every > 0 else 1
            self.replay(rounds)  # captures and uploads the graph of every phase
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.replay(trial_graphs * rounds)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / (trial_graphs * rounds * K)
            self.tuning.append({"steps_per_graph": K, "ms_per_step": ms})
            if best is None or ms < best[0]:
                best = (ms, K)
        self.capture(best[1])
        return self.tuning

    # ---- results ---------------------------------------------------------------------------------
    def collision_counts(self):
        """Colliding pairs of the last step, per local box (host)."""
        if not self.collide:
            return [0] * self.nb
        return [int(c) for c in self.collider.box_counts.cpu().tolist()]

    def box_state(self, j):
        """Local box j: its spectrum (cube layout) and its droplets' positions and velocities in
        droplet-index order (host numpy)."""
        torch = _torch()
        sel = torch.nonzero(self.box == j).flatten()
        order = torch.argsort(self.dids[sel])
        idx = sel[order]
        return self.uk[j], self.pos[idx].cpu().numpy(), self.vel[idx].cpu().numpy()

    def check(self):
        """Host check of the device status word of the batch (NaN / blow-up of any box)."""
        return self.plan.status(clear=True)


def main(argv=None):
    torch = _torch()
    ap = argparse.ArgumentParser()
    ap.add_argument("--boxes", type=int, default=64)
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--precision", default="f32")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--steps-per-graph", type=int, default=0, help="0: autotune")
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
    if a.steps_per_graph:
        ens.capture(a.steps_per_graph)
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
           "launch": "multi-box plan: one launch per pass over all boxes, steps captured in a CUDA graph",
           "steps_per_graph": ens.steps_per_graph, "autotune": tuning, "fft_autotune": ens.fft_tuning,
           "setup_s": setup_s, "status_flags": flags, "droplets_per_box": nd,
           "collision_pairs_last_step_per_box": coll}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
