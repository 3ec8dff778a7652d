#!/usr/bin/env python
"""Throughput of the forced pseudospectral DNS step with droplets on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): the 256^3 configuration - FP32 fields and transforms, nu = 2.5e-3, dt = 1e-3,
constant power eps = 0.1 on shells 1..2, RK2 + viscous integrating factor, end-of-step
projection; 1e6 droplets with lognormal radii (median 0.002*2pi, sigma 0.3), tau ~ r^2 with median
St = 0.5, Stokes drag + settling g = 0.1, FP64 positions, cell-list collisions every step, and the
learned interpolation (tricubic + MLP correction).  Inputs are seeded synthetic data of those
shapes (the reference publishes no dataset); the working set (~1.3 GB per step) is far larger
than L2, so no flush is needed between steps.

Learned interpolation protocol (--interp learned, the default):
  1. calibration run: the same configuration with flow seed + 1 for 500 steps; snapshots every 100
     steps give 2e7 exact-target training pairs; the network is trained on them (untimed);
  2. production run (flow seed): droplets on the learned interpolation from step 0; untimed steps
     up to 500 - warmup - steps, then the warm-up and the timed steps, so that the run ends at
     step 500 (the configuration's length) when it fits;
  3. the judge at the end: exact spectral sum at a random 1% of the droplets, against the learned
     and the tricubic values.  Its device time is charged to the step time once per output
     interval (500 steps: the reference saves every 0.5 time units).
The plain comparators run the same seed and droplets in FP64 with tricubic interpolation for 500
steps, timed over their last ``steps`` steps, with their own errors at the end: ``plain_fp64`` on
the same grid, and ``plain_fp64_same_error`` on the smallest grid the library has (powers of two
and the mixed-radix sizes 360, 384) on which plain tricubic meets the error tolerance (its error
falls about as dx^4), from the same physical initial field embedded in the finer grid.

A "step" is one full time step (two flow stages, two droplet stages, epilogue, collisions).
``value`` is steps/s of the whole job (N replicas, one per GPU: the single-box step does not
shard), timed on the device with CUDA events between barriers, max over ranks.  ``e2e`` is the
same metric through ForcedDNS.step_host() with the state in pinned host memory, copied in and out
every step, the spectrum in the reference's own layout (3, N, N, N/2+1) (``e2e_cube_layout``: the
same with the dealiased cube the device keeps).  ``--impl reference`` times the CPU restatement of the same step (FP64 NumPy/SciPy,
all host cores) on rank 0.
"""
import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "steps/s at 256^3+1M droplets: FP32+learned interp vs plain FP64, same error"
# grids the library has kernels for (powers of two and the mixed-radix sizes)
GRID_SIZES = (16, 32, 64, 96, 128, 192, 256, 360, 384, 512)
FALLBACK_HBM_GBS = 6650.0


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--nd", type=int, default=1_000_000)
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--interp", choices=["trilinear", "tricubic", "cosine", "learned"], default="learned")
    ap.add_argument("--run-steps", type=int, default=500, help="length of the production run")
    ap.add_argument("--graph-steps", type=int, default=20,
                    help="timed steps as replays of a CUDA graph of this many steps (0: launched one by one)")
    ap.add_argument("--judge-every", type=int, default=500, help="output interval of the judge (steps)")
    ap.add_argument("--judge-frac", type=float, default=0.01)
    ap.add_argument("--train-pairs", type=int, default=20_000_000)
    ap.add_argument("--train-epochs", type=int, default=16)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 tricubic comparators")
    ap.add_argument("--no-plain-fine", action="store_true", help="skip the plain FP64 run on the finer grid")
    ap.add_argument("--no-plain-512", action="store_true", help="skip the plain FP64 512^3 scale point")
    ap.add_argument("--tolerance", type=float, default=1e-4, help="droplet-velocity error tolerance")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--sort-every", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-budget-s", type=float, default=150.0)
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------------------------
def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x, world):
    """The maximum of x over the ranks (device tensors under NCCL, host tensors under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clock, max clock, power and clock-event reasons every 20 ms through NVML while
    the timed region runs (read-only queries)."""
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}

    def __init__(self, device_index, period=0.02):
        import threading
        self.rows, self.err = [], None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            pr = torch.cuda.get_device_properties(device_index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            self.h = nv.nvmlDeviceGetHandleByPciBusId(bus)
            self.nv = nv
            self.smax = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)

            def loop():
                while not self._stop.is_set():
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                        pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                        self.rows.append((sm, pw, rs))
                    except Exception as e:  # keep sampling; report the first error
                        self.err = self.err or str(e)
                    self._stop.wait(period)

            self._t = threading.Thread(target=loop, daemon=True)
            self._t.start()
        except Exception as e:
            self.err = str(e)

    def stop(self):
        if self._t is None:
            return {"error": self.err or "NVML unavailable"}
        self._stop.set()
        self._t.join(timeout=2)
        if not self.rows:
            return {"error": self.err or "no samples"}
        sm = [r[0] for r in self.rows]
        reasons = sorted({name for r in self.rows for bit, name in self.REASONS.items() if r[2] & bit})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.smax, "reasons": reasons,
                "power_w_max": max(r[1] for r in self.rows), "samples": len(self.rows)}


def measured_tensor_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["bf16_tflops"]), "measured"
        except Exception:
            pass
    return 1590.0, "fallback"


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------------------------
# algorithmic bytes per launch of each kernel of the step
# ---------------------------------------------------------------------------------------------
def algorithmic_bytes(plan, nd, learned=False):
    """Compulsory HBM bytes per launch: every input read once, every output written once.  With
    the learned interpolation the droplet stages take the fluid velocity at the droplets (n, 3)
    from the MLP instead of gathering it from the field."""
    N, My, Mzp, kc = plan.N, plan.My, plan.Mzp, plan.kc
    r = 4 if plan.precision == "f32" else 8
    c = 2 * r
    cube = plan.Mx * My * Mzp * c
    xrows = N * My * Mzp * c      # (N, My, Mzp): after/before the x pass
    yrows = N * N * Mzp * c       # (N, N, Mzp): after/before the y pass
    zin = N * N * (kc + 1) * c    # kz <= kc of one (N, N) set of rows
    phys = N ** 3 * r
    drop = 24 + 3 * r + r         # pos, vel, tau
    plane0 = 3 * plan.Mx * My * c  # the kz = 0 plane of a cube 3-vector
    if learned:
        # k_droplet_given: stage 1 reads up, vel, tau and writes a1; stage 2 reads up, vel, tau,
        # a1 and pos, writes pos and vel
        d1 = nd * (3 * r + 3 * r + r + 3 * r)
        d2 = nd * (3 * r + 3 * r + r + 3 * r + 24 + 24 + 3 * r)
    else:
        d1 = nd * (drop + 3 * r) + 3 * phys  # + a1 written; field read once
        d2 = nd * (drop + 3 * r + 24 + 3 * r) + 3 * phys
    return {
        "xinv": 3 * cube + 6 * xrows,
        "yinv": 6 * xrows + 6 * yrows,
        "zcross": 6 * zin + 3 * yrows + 3 * phys,
        "yfwd": 3 * yrows + 3 * xrows,
        "xfwd_update": 3 * xrows + 7.5 * cube,       # mean of the two RK2 stages (9 and 6 cube fields)
        "epilogue": 2 * plane0,  # the plane-only epilogue: read and write the kz = 0 plane
        "droplet1": d1,
        "droplet2": d2,
        "forcing": 0,
        # collisions: keys (read pos, write key+id) + 3 radix passes (read+write key+id);
        # ranges, sorted copy (read pos+radius+id, write 32 B), count and emit (read 32 B each)
        "collide_sort": nd * (24 + 8 + 3 * 16),
        "collide_pairs": nd * (4 + 36 + 32 + 32 + 32 + 8),
        "cell_order": nd * (24 + 8 + 3 * 16 + 4),
        # learned interpolation: features read the field once (3 components) and the positions,
        # write bf16 rows (208) and aux (8 floats); the MLP reads rows + aux, writes (n,3)
        "mlp_features": 3 * phys + nd * (24 + 2 * 208 + 32),
        "mlp_infer": nd * (2 * 208 + 32 + 3 * r),
    }


def load_traffic(kernel, N, precision):
    """dram bytes per launch from the committed ncu summary (profiles/traffic.json), if any."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d.get(f"{kernel}/{N}/{precision}")
    except Exception:
        return None


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------
def flow_params_for(N):
    return (2.5e-3, 1e-3) if N == 256 else ((1e-3, 5e-4) if N == 512 else (0.01, 2e-3))


def embed_spectrum(uk_full, N2):
    """A reference-layout spectrum (3, N, N, N/2+1) of an N^3 field as the same physical field on an
    N2^3 grid (N2 > N): the modes keep their wavenumbers, times (N2/N)^3 for the unnormalised
    forward transform."""
    import torch
    N = uk_full.shape[1]
    src = torch.as_tensor(uk_full).cuda()
    out = torch.zeros((3, N2, N2, N2 // 2 + 1), dtype=torch.complex128, device="cuda")
    h = N // 2
    si = torch.cat([torch.arange(0, h), torch.arange(h + 1, N)]).cuda()          # Nyquist dropped
    di = torch.cat([torch.arange(0, h), torch.arange(N2 - h + 1, N2)]).cuda()
    blk = src[:, si][:, :, si][..., : h + 1].to(torch.complex128) * (N2 / N) ** 3
    out[:, di[:, None], di[None, :], : h + 1] = blk
    return out


def build_workload(a, seed, precision=None, interp=None, droplets=True, N=None):
    """DNS (+ droplets at the interpolated fluid velocity, + collider) from seeded inputs.  With N
    larger than the configuration's grid, the configuration's initial field is embedded in the
    finer grid (same physics, same field, finer resolution)."""
    import torch
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200.init import init_flow, init_droplets
    precision = precision or a.precision
    interp = interp or a.interp
    nu, dt = flow_params_for(a.N)
    Ng = N or a.N
    dns = ForcedDNS.config(Ng, nu, dt, eps=0.1, kf=2, precision=precision)
    dns.tuning = dns.plan.autotune()  # launch variants of the y passes, timed on this plan
    if Ng == a.N:
        init_flow(dns, seed)
    else:
        base = ForcedDNS.config(a.N, nu, dt, eps=0.1, kf=2, precision="f64")
        init_flow(base, seed)
        dns.set_uk_full(embed_spectrum(base.uk_full(), Ng))
        del base
    d = None
    if droplets and a.nd > 0:
        from lucky_droplets_b200.collide import Collider
        pos, tau, radius = init_droplets(a.nd, seed, "lognormal_r", nu=nu)
        method = "tricubic" if interp == "learned" else interp
        d = Droplets(dns.plan, pos, np.zeros((a.nd, 3)), tau, method=method, g=0.1, radius=radius)
        u = dns.velocity()
        d.vel.copy_(d.gather(u))  # droplets start at the interpolated fluid velocity
        del u
        # collision cells of twice the 0.9999 radius quantile (the few wider droplets search the
        # cells within their diameter); colliding pairs found after every step; droplets
        # re-sorted into cell order every sort_every steps
        from lucky_droplets_b200.collide import cell_size_for
        col = Collider(a.nd, cell_size_for(radius), device=dns.plan.device)
        dns.attach(d, collider=col, sort_every=a.sort_every)
    torch.cuda.synchronize()
    return dns, d


def train_learned(a, seed):
    """Calibration run (flow seed + 1): snapshots every 100 steps of the configuration's run,
    then the network is fitted on 2e7 exact-target pairs from them."""
    import torch
    from lucky_droplets_b200.mlp import LearnedInterp
    t0 = time.perf_counter()
    cal, _ = build_workload(a, seed + 1, droplets=False)
    snaps = []
    every = 100
    for _ in range(max(1, a.run_steps // every)):
        cal.step(every)
        snaps.append(cal.uk.clone())
    cal.check()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    li = LearnedInterp(cal.plan, seed=seed)
    info = li.fit(snaps, n_pairs=a.train_pairs, epochs=a.train_epochs)
    torch.cuda.synchronize()
    info.update({"calibration_seed": seed + 1, "snapshot_steps": [every * (i + 1) for i in range(len(snaps))],
                 "calibration_run_s": t1 - t0, "fit_s": time.perf_counter() - t1,
                 "final_loss": info["losses"][-1]})
    del info["losses"]
    del snaps, cal
    return li, info


def judge_learned(dns, d, li, frac, seed):
    """The judge: exact spectral sum at a random fraction of the droplets against the learned and
    the tricubic velocities of the current state.  The errors (and the network's enabled flag)
    come from LearnedInterp.judge; its device time is taken on a second, identical pass of the
    device work alone (interleaved field, exact sum, inference, tricubic gather), so that neither
    first-use allocations nor the host reductions fall between the events."""
    import torch
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, ptr, stream_ptr
    n = max(1, int(round(frac * d.n)))
    g = torch.Generator(device="cpu").manual_seed(seed)
    sel = torch.randperm(d.n, generator=g)[:n].to(d.pos.device)
    pos = d.pos[sel].contiguous()
    e_l, e_t = li.judge(dns.uk, li.interleaved(dns.uk), pos)
    p = dns.plan
    tric = torch.empty((n, 3), dtype=p.rdtype, device=p.device)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    u4 = li.interleaved(dns.uk)
    p.exact_sum(dns.uk, pos)
    li.infer(u4, pos)
    check(_lib.lib().ld_gather4(p.handle, ptr(u4), ptr(pos), n, _lib.LD_INTERP["tricubic"], ptr(tric), stream_ptr()))
    e1.record(s)
    torch.cuda.synchronize()
    return {"learned": e_l, "tricubic": e_t, "n_sample": n, "enabled": li.enabled, "judge_ms": e0.elapsed_time(e1)}


def error_plain(dns, d, frac, seed):
    """Tricubic (the droplets' own method) against the exact spectral sum, same sampling."""
    import torch
    n = max(1, int(round(frac * d.n)))
    g = torch.Generator(device="cpu").manual_seed(seed)
    sel = torch.randperm(d.n, generator=g)[:n].to(d.pos.device)
    pos = d.pos[sel].contiguous()
    exact = dns.plan.exact_sum(dns.uk, pos)
    u = dns.velocity()
    got = d.gather(u, pos).to(torch.float64)
    return float(torch.linalg.norm(got - exact) / torch.linalg.norm(exact))


def advance_to_window(dns, a):
    """Untimed production steps so that warm-up + timed steps end at step run_steps.  With
    --graph-steps G > 0 (and G dividing the timed steps) the timed steps are replays of a CUDA
    graph of G steps, captured here at the step phase (modulo the droplet re-sorting period) of the
    timed window and replayed over the untimed steps already, so that the graph is uploaded before
    the timed region.  Returns (untimed steps, graph or None)."""
    pre = max(0, a.run_steps - a.warmup - a.steps)
    G = getattr(a, "graph_steps", 0)
    if G <= 0 or a.steps % G != 0:
        dns.step(pre)
        return pre, None
    period = dns.sort_every if (dns.droplets is not None and dns.sort_every > 0) else 0
    timed_start = dns.nstep + pre + a.warmup
    k0 = min(pre, (timed_start - dns.nstep) % period) if period else 0
    dns.step(k0)
    g = dns.capture(G)
    reps = (pre - k0) // G
    if reps:
        g.replay(reps)
    dns.step(pre - k0 - reps * G)
    return pre, g


def time_steps(dns, K, W, world, graph=None):
    import torch
    s = torch.cuda.current_stream()
    dns.step(W)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    if graph is not None:
        graph.replay(K // graph.nsteps)
    else:
        dns.step(K)
    e1.record(s)
    torch.cuda.synchronize()
    barrier(world)
    return e0.elapsed_time(e1)


def time_e2e(dns, d, K, W, world, layout="full"):
    """K steps through ForcedDNS.step_host with the state in pinned host memory, copied in and out
    every step: the spectrum in the reference's layout (3, N, N, N/2+1) ("full", what the
    reference's time loop holds, F:158) or in the dealiased cube ("cube")."""
    import torch
    if layout == "full":
        uk_h = torch.empty((3, dns.N, dns.N, dns.N // 2 + 1), dtype=dns.uk.dtype).pin_memory()
        uk_h.copy_(dns.plan.from_cube(dns.uk))
    else:
        uk_h = torch.empty_like(dns.uk, device="cpu").pin_memory()
        uk_h.copy_(dns.uk)
    pos_h = vel_h = None
    if d is not None:
        pos_h = torch.empty_like(d.pos, device="cpu").pin_memory()
        vel_h = torch.empty_like(d.vel, device="cpu").pin_memory()
        pos_h.copy_(d.pos)
        vel_h.copy_(d.vel)
    for _ in range(W):
        dns.step_host(uk_h, pos_h, vel_h, layout=layout)
    barrier(world)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(K):
        dns.step_host(uk_h, pos_h, vel_h, layout=layout)
    e1.record(s)
    torch.cuda.synchronize()
    barrier(world)
    if layout == "full":  # after the first call only the rows of the dealiased cube move
        p = dns.plan
        nbytes = 3 * p.My * p.My * (p.kc + 1) * uk_h.element_size()
    else:
        nbytes = uk_h.numel() * uk_h.element_size()
    if d is not None:
        nbytes += pos_h.numel() * pos_h.element_size() + vel_h.numel() * vel_h.element_size()
    return e0.elapsed_time(e1), nbytes


def count_launches(dns, steps=20):
    """Kernels (and memset/memcpy operations) the step launches, counted from a CUDA-graph
    capture of `steps` steps (capture runs nothing; the step counters are restored): per step."""
    import torch
    from cuda.bindings import runtime as rt
    saved = (dns.t, dns.nstep)
    try:
        g = torch.cuda.CUDAGraph(keep_graph=True)
        cap = torch.cuda.Stream()
        cap.wait_stream(torch.cuda.current_stream())
        with torch.cuda.graph(g, stream=cap, capture_error_mode="thread_local"):
            dns.step(steps, stream=cap)
        graph = rt.cudaGraph_t(init_value=g.raw_cuda_graph())
        err, _, n = rt.cudaGraphGetNodes(graph, 0)
        err, nodes, n = rt.cudaGraphGetNodes(graph, n)
        kinds = {}
        for nd in nodes:
            e, t = rt.cudaGraphNodeGetType(nd)
            kinds[t] = kinds.get(t, 0) + 1
        k = kinds.get(rt.cudaGraphNodeType.cudaGraphNodeTypeKernel, 0)
        other = sum(v for t, v in kinds.items() if t != rt.cudaGraphNodeType.cudaGraphNodeTypeKernel)
        del g
        return {"kernels_per_step": k / steps, "memset_memcpy_per_step": other / steps,
                "method": f"CUDA-graph capture of {steps} steps"}
    finally:
        dns.t, dns.nstep = saved


def profile_kernels(dns, d, P):
    """Per-kernel device time over P steps with launch-bracketing events on the launch stream.
    The steps run inside the NVTX range "profile_steps", so that an ncu capture can be limited to
    production launches (`--nvtx --nvtx-include "profile_steps/"`)."""
    import torch
    p = dns.plan
    p.profile_read(reset=True)
    p.profile(True)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("profile_steps")
    dns.step(P)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    prof = p.profile_read(reset=True)
    p.profile(False)
    return prof


def cpu_baseline(dns, d, a, budget_s=30.0, min_steps=2, max_steps=5):
    """The FP64 CPU restatement of the same step (oracle/config_np) on this host's cores, from the
    same state: consecutive steps until `budget_s` of CPU work (at least min_steps, at most
    max_steps), a bounded sample of the workload; the rate is steps / summed step time."""
    import torch
    from oracle import config_np as C
    N = dns.N
    grid = C.ConfigGrid(N)
    prm = C.ConfigParams(N=N, nu=dns.nu, dt=dns.dt, eps=0.1, kf=2, g=0.1)
    uk = dns.uk_full()
    pos = d.pos.cpu().numpy() if d is not None else None
    vel = d.vel.cpu().numpy().astype(np.float64) if d is not None else None
    tau = d.tau.cpu().numpy().astype(np.float64) if d is not None else None
    radius = d.radius.cpu().numpy() if d is not None else None
    del torch
    from oracle import collide_np as K
    method = "tricubic" if a.interp == "learned" else a.interp  # the CPU path has no learned part
    times = []
    while len(times) < max_steps and (len(times) < min_steps or sum(times) < budget_s):
        t0 = time.perf_counter()
        uk, pos, vel = C.step(grid, prm, uk, pos, vel, tau, method)
        uk = grid.project(np.stack([grid.rfft(grid.irfft(uk[c])) for c in range(3)]))  # step epilogue
        if pos is not None:
            K.collide(pos, radius, 2.0 * radius.max())
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    return {"value": len(times) / tot, "unit": "steps/s", "cores": C._WORKERS, "kind": "port",
            "steps_timed": len(times), "s_per_step": [round(t, 3) for t in times],
            "sample": f"{len(times)} consecutive full steps of the same workload from the GPU run's state "
                      f"({N}^3 FP64 RK2+IF flow with the end-of-step projection, {a.nd} droplets {method}, "
                      f"cell-list collisions), {tot:.1f} s in all; NumPy/SciPy/numba FP64 restatement, "
                      f"scipy.fft workers={C._WORKERS}"}


def run_plain(a, seed, world, N=None):
    """The plain comparator: the same seed and droplets, FP64 fields and transforms, tricubic
    (on the configuration's grid, or on a finer one N with the same initial field)."""
    import torch
    dns, d = build_workload(a, seed, precision="f64", interp="tricubic", N=N)
    _, graph = advance_to_window(dns, a)
    ms = time_steps(dns, a.steps, a.warmup, world, graph)
    del graph
    ms = allreduce_max(ms, world)
    dns.check()
    err = error_plain(dns, d, a.judge_frac, seed + 99) if d is not None else None
    out = {"value": world * a.steps / (ms / 1e3), "unit": "steps/s", "ms_per_step": ms / a.steps,
           "N": dns.N, "precision": "f64", "interp": "tricubic", "droplet_velocity_rel_l2": err,
           "at_step": dns.nstep}
    del dns, d
    torch.cuda.empty_cache()
    return out


def run_ours(a):
    import torch
    world, rank, local = dist_setup()
    from lucky_droplets_b200 import _lib
    seed = a.seed + 1000 * rank
    li = fit_info = None
    if a.interp == "learned":
        li, fit_info = train_learned(a, seed)
    dns, d = build_workload(a, seed)
    judge0 = None
    if li is not None:
        li.plan = dns.plan  # same N and precision as the calibration run
        d.use_learned(li)
        # the first output interval (F:575, i % st == 0 at i = 0): the judge decides, in the time
        # loop, whether the network steps the droplets (ForcedDNS.evolve runs the same call)
        judge0 = dns.judge(a.judge_frac, seed + 98)
    pre, graph = advance_to_window(dns, a)
    clocks = ClockSampler(local)
    ms = time_steps(dns, a.steps, a.warmup, world, graph)
    clk = clocks.stop()
    del graph
    flags = dns.check()
    pairs = int(dns.collider.count.item()) if getattr(dns, "collider", None) is not None else None
    ms = allreduce_max(ms, world)
    judge = None
    judge_ms_per_step = 0.0
    if li is not None:
        judge = judge_learned(dns, d, li, a.judge_frac, seed + 99)
        judge["at_step"] = dns.nstep
        judge["every_steps"] = a.judge_every
        judge_ms = allreduce_max(judge["judge_ms"], world)
        judge_ms_per_step = judge_ms / a.judge_every
    ms_per_step = ms / a.steps + judge_ms_per_step
    value = world / (ms_per_step / 1e3)
    # per-kernel timing and the roofline of the dominant kernel
    P = max(1, a.profile_steps)
    prof = profile_kernels(dns, d, P)
    launches_per_step = sum(c for c, _ in prof.values()) / P
    algo = algorithmic_bytes(dns.plan, a.nd, learned=(li is not None and li.enabled))
    flops = {"mlp_infer": 2.0 * (195 * 128 + 128 * 128 + 128 * 3) * a.nd}
    kernels = {}
    tot = sum(t for _, t in prof.values())
    for name, (cnt, tms) in prof.items():
        avg = tms / cnt
        b = algo.get(name)
        kernels[name] = {"launches_per_step": cnt / P, "avg_ms": avg, "share": tms / tot,
                         "algo_bytes": b, "gbs": (b / (avg * 1e-3) / 1e9) if b else None}
        if name in flops:
            kernels[name]["algo_flops"] = flops[name]
            kernels[name]["tflops"] = flops[name] / (avg * 1e-3) / 1e12
    dom = max((k for k in kernels if algo.get(k) or k in flops), key=lambda k: kernels[k]["share"])
    kd = kernels[dom]
    if dom in flops:
        peak, peak_kind = measured_tensor_peak()
        roof = {"bound": "tensor", "kernel": dom, "achieved": kd["tflops"], "peak": peak, "unit": "TFLOP/s",
                "frac": kd["tflops"] / peak, "peak_source": peak_kind, "traffic": load_traffic(dom, a.N, a.precision),
                "algo_flops_per_launch": kd["algo_flops"], "avg_launch_ms": kd["avg_ms"]}
    else:
        peak, peak_kind = measured_peaks()
        roof = {"bound": "hbm", "kernel": dom, "achieved": kd["gbs"], "peak": peak, "unit": "GB/s",
                "frac": kd["gbs"] / peak, "peak_source": peak_kind,
                "traffic": load_traffic(dom, a.N, a.precision),
                "algo_bytes_per_launch": kd["algo_bytes"], "avg_launch_ms": kd["avg_ms"]}
    step_bytes = sum((algo.get(k) or 0) * v["launches_per_step"] for k, v in kernels.items())
    interp_desc = "learned (tricubic + MLP correction)" if a.interp == "learned" else a.interp
    out = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32" if a.precision == "f32" else "f64", "data": "synthetic",
           "config": {"workload": f"{a.N}^3 DNS RK2+IF (nu={flow_params_for(a.N)[0]}, dt={flow_params_for(a.N)[1]}, "
                                  f"eps=0.1 on shells 1-2) + {a.nd} droplets {interp_desc}, Heun, settling g=0.1, "
                                  f"cell-list collisions every step",
                      "N": a.N, "n_droplets": a.nd, "interp": a.interp, "precision": a.precision,
                      "run": f"steps {pre}..{dns.nstep} of a {a.run_steps}-step run (timed: the last {a.steps})",
                      "parallelism": f"replicas x{world}", "l2": "working set > 1 GB per step (> L2); no flush",
                      "launch": (f"timed steps replayed from a CUDA graph of {a.graph_steps} steps (also for the FP64 comparators)"
                                 if a.graph_steps > 0 and a.steps % a.graph_steps == 0 else "kernels launched one by one")},
           "droplet_steps_per_s": value * a.nd,
           "step_algo_gbs": step_bytes / (ms / a.steps * 1e-3) / 1e9,
           "roofline": roof,
           "kernels": kernels,
           "gpu_launches": int(round(launches_per_step * a.steps)),
           "gpu_launches_detail": {"method": "profile scopes", "scopes_per_step": launches_per_step},
           "status_flags": flags,
           "collision_pairs_last_step": pairs,
           "fft_autotune": getattr(dns, "tuning", None),
           "clocks": clk}
    try:
        lc = count_launches(dns)
        out["gpu_launches"] = int(round(lc["kernels_per_step"] * a.steps))
        out["gpu_launches_detail"] = dict(lc, scopes_per_step=launches_per_step)
    except Exception as e:  # keep the scope count, say why
        out["gpu_launches_detail"]["capture_error"] = str(e)[:200]
    if judge is not None:
        out["judge"] = judge
        out["judge_at_first_output"] = judge0
        out["judge_ms_per_step_amortised"] = judge_ms_per_step
        out["training"] = fit_info
        train_s = fit_info["calibration_run_s"] + fit_info["fit_s"]
        out["training_cost"] = {
            "seconds": train_s, "production_steps_equivalent": train_s / (ms_per_step * 1e-3),
            "note": f"calibration run + sample generation + {fit_info['epochs']} epochs of Adam, once per "
                    "configuration; not in value. It equals this many production steps of the timed step; a run "
                    "of that many steps doubles its wall time, longer runs amortise it"}
    if not a.no_e2e:
        Ke = max(3, min(a.steps, 10))
        for layout, key in (("full", "e2e"), ("cube", "e2e_cube_layout")):
            ems, nbytes = time_e2e(dns, d, Ke, 1, world, layout=layout)
            ems = allreduce_max(ems, world)
            e_ms = ems / Ke + judge_ms_per_step
            out[key] = {"value": world / (e_ms / 1e3), "unit": "steps/s", "h2d_bytes_per_step": nbytes,
                        "d2h_bytes_per_step": nbytes,
                        "api": f"ForcedDNS.step_host(layout='{layout}') (pinned host state in/out every step)",
                        "host_layout": ("reference (3, N, N, N/2+1) complex, what the reference's loop holds; "
                                        "the rows of the dealiased cube move by strided copies"
                                        if layout == "full" else "dealiased cube (3, Mx, My, Mzp) complex")}
    cpu_state = (dns, d) if (rank == 0 and world == 1 and not a.no_cpu_baseline) else None
    if li is not None and not a.no_plain:
        if cpu_state is not None:
            out["cpu_baseline"] = cpu_baseline(dns, d, a)
            cpu_state = None
        del dns, d
        torch.cuda.empty_cache()
        plain = run_plain(a, seed, world)
        out["plain_fp64"] = plain
        out["speedup_vs_plain_fp64_same_grid"] = value / plain["value"]
        e_plain = plain["droplet_velocity_rel_l2"]
        out["error"] = {"learned_f32": judge["learned"], "tricubic_f32": judge["tricubic"],
                        "plain_fp64_tricubic": e_plain, "tolerance": a.tolerance,
                        "learned_within_tolerance": judge["learned"] <= a.tolerance,
                        "learned_over_plain": judge["learned"] / e_plain if e_plain else None}
        # plain FP64 at equal error: the smallest grid (powers of two and the mixed-radix sizes
        # the library has) on which plain tricubic meets the tolerance, from the same physical
        # initial field and droplets.  Its error falls about as dx^4: grids predicted to miss are
        # skipped, the others run in increasing order until one meets the tolerance.  The 512^3
        # run is kept beside it as a scale point for the mixed-radix timing.
        if e_plain is not None and e_plain > a.tolerance and not a.no_plain_fine:
            tried = []
            fine = None
            for N2 in sorted(n for n in GRID_SIZES if n > a.N):
                if e_plain * (a.N / N2) ** 4 > a.tolerance:
                    continue
                r = run_plain(a, seed, world, N=N2)
                tried.append(r)
                if r["droplet_velocity_rel_l2"] <= a.tolerance:
                    fine = r
                    break
            if fine is not None:
                out["plain_fp64_same_error"] = fine
                out["speedup_vs_plain_fp64_same_error"] = value / fine["value"]
                out["error"]["plain_fp64_same_error_tricubic"] = fine["droplet_velocity_rel_l2"]
            out["plain_fp64_grids_tried"] = [{k: r[k] for k in ("N", "ms_per_step", "droplet_velocity_rel_l2")}
                                             for r in tried]
            r512 = next((r for r in tried if r["N"] == 512), None)
            if r512 is None and not a.no_plain_512 and 512 > a.N:
                r512 = run_plain(a, seed, world, N=512)
            if r512 is not None:
                out["plain_fp64_512"] = {k: r512[k] for k in ("N", "ms_per_step", "value", "droplet_velocity_rel_l2")}
            # the mixed-radix transforms run at a lower fraction of HBM than the power-of-two ones:
            # the same-error comparator is also stated at power-of-two efficiency, from the fit
            # T(N) = c N^3 log2 N + d through the two power-of-two FP64 runs of this bench
            if fine is not None and r512 is not None and fine["N"] not in (a.N, 512):
                def w(n):
                    return n ** 3 * np.log2(n)
                c = (r512["ms_per_step"] - plain["ms_per_step"]) / (w(512) - w(a.N))
                d = plain["ms_per_step"] - c * w(a.N)
                t_fit = c * w(fine["N"]) + d
                out["plain_fp64_same_error_pow2_fit"] = {
                    "N": fine["N"], "ms_per_step": t_fit, "value": world / (t_fit / 1e3),
                    "fit": f"T(N) = {c:.4g} N^3 log2 N + {d:.4g} ms through the FP64 runs at {a.N}^3 and 512^3"}
                out["speedup_vs_plain_fp64_same_error_pow2_fit"] = value / (world / (t_fit / 1e3))
    if cpu_state is not None:
        out["cpu_baseline"] = cpu_baseline(*cpu_state, a)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# reference arm: the CPU restatement of the same step on this host
# ---------------------------------------------------------------------------------------------
def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import config_np as C
    nu, dt = flow_params_for(a.N)
    method = "tricubic" if a.interp == "learned" else a.interp  # the CPU path has no learned part
    prm = C.ConfigParams(N=a.N, nu=nu, dt=dt, eps=0.1, kf=2, g=0.1)
    grid = C.ConfigGrid(a.N)
    uk, u = C.init_flow(grid, prm, a.seed)
    pos = tau = vel = radius = None
    if a.nd > 0:
        pos, tau, radius = C.init_droplets(prm, a.seed, "lognormal_r", nd=a.nd)
        vel = C.gather(u, pos, method)
    del u
    t_first = None
    done, total = 0, 0.0
    for i in range(max(0, min(a.warmup, 1))):
        t0 = time.perf_counter()
        uk, pos, vel = C.step(grid, prm, uk, pos, vel, tau, method)
        t_first = time.perf_counter() - t0
    from oracle import collide_np as K
    for i in range(a.steps):
        t0 = time.perf_counter()
        uk, pos, vel = C.step(grid, prm, uk, pos, vel, tau, method)
        if pos is not None:
            K.collide(pos, radius, 2.0 * radius.max())
        total += time.perf_counter() - t0
        done += 1
        if total > a.cpu_budget_s:
            break
    value = done / total
    sample = (f"{done} of {a.steps} requested steps timed (bounded to ~{a.cpu_budget_s:.0f} s), "
              f"warm-up {min(a.warmup, 1)}; FP64 NumPy/SciPy restatement of the step, scipy.fft workers={C._WORKERS}")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
           "steps": done, "warmup": min(a.warmup, 1), "ms_per_step": 1e3 * total / done, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"{a.N}^3 DNS RK2+IF (nu={nu}, dt={dt}, eps=0.1 on shells 1-2) + "
                                  f"{a.nd} droplets {method}, Heun, settling g=0.1",
                      "N": a.N, "n_droplets": a.nd, "interp": method},
           "cpu_baseline": {"value": value, "unit": "steps/s", "cores": C._WORKERS, "kind": "port",
                            "sample": sample},
           "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main(argv=None):
    a = parse_args(argv)
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
