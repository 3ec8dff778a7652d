"""The time loop of forced-dns-sm.py (F:556-627) on one GPU, with inertial droplets.

``ForcedDNS`` keeps the reference's driver parameters (N, nu, dt, f0, shell_no) and advances
the dealiased spectral velocity with either
  * ``integrator="rk4"``   - the reference's classical RK4 with explicit viscosity (F:335-362),
  * ``integrator="rk2if"`` - Heun with the viscous integrating factor exp(-nu k^2 h);
and after every step applies the reference's end-of-step epilogue (F:596-620: reality round
trip, div-free projection, blow-up test).  ``Droplets`` advances one-way-coupled droplets
(x' = v, v' = (u(x) - v)/tau - g z) by Heun on the two RK2 stages.

All device work goes through liblucky_droplets.so; there is no CPU path.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ptr, stream_ptr
from .spectral import Plan, flow_params, TWO_PI


def _torch():
    import torch
    return torch


class BlowUpError(FloatingPointError):
    """The state met the abort test of forced-dns-sm.py:618-620 or became non-finite."""


class ForcedDNS:
    """Forced, triply periodic pseudospectral DNS in [0, 2 pi)^3 on one GPU."""

    def __init__(self, N, nu, dt, f0, shell_no=(1,), integrator="rk2if", precision="f32", device=None,
                 epilogue=True, overlap=False):
        if integrator not in ("rk2if", "rk4"):
            raise ValueError("integrator must be 'rk2if' or 'rk4'")
        self.plan = Plan(N, precision, device)
        self.N, self.nu, self.dt, self.f0 = N, float(nu), float(dt), float(f0)
        self.shell_no = tuple(shell_no)
        self.integrator = integrator
        self.epilogue = epilogue
        self.overlap = bool(overlap)  # droplet work on a second stream (see _dstream)
        self.prm = flow_params(dt, nu, f0, shell_no)
        p = self.plan
        if integrator == "rk2if":  # the integrating-factor table, built before any capture
            check(_lib.lib().ld_plan_prepare(p.handle, ctypes.byref(self.prm), stream_ptr()))
        self.uk = p.empty_cube(3)
        self.aux = p.empty_cube(3)   # ustar (rk2if) or the stage input y (rk4)
        self.acc = p.empty_cube(3)
        self.u_phys = None
        self.droplets = None
        self.collider = None
        self.sort_every = 0
        self.t = 0.0
        self.nstep = 0

    # ---- constructors with the reference's and the configurations' parameters --------------------
    @classmethod
    def reference(cls, N, precision="f64", nshells=1, nu0=0.8, m=1.5, **kw):
        """Parameters of forced-dns-sm.py as functions of N: dt = 0.256/N (F:29),
        nu = nu0 (3m/N)^(4/3) (F:83), f0 = nu0^3 (2pi)^3 / nshells (F:97), RK4 (F:21)."""
        dt = 0.256 / N
        nu = nu0 * (3 * m / N) ** (2 * (1 - 1 / 3))
        f0 = nu0 ** 3 * TWO_PI ** 3 / nshells
        kw.setdefault("integrator", "rk4")
        return cls(N, nu, dt, f0, shell_no=tuple(range(1, nshells + 1)), precision=precision, **kw)

    @classmethod
    def config(cls, N, nu, dt, eps=0.1, kf=2, precision="f32", **kw):
        """Configuration semantics: constant power eps on shells 1..kf, RK2 + integrating factor."""
        f0 = eps * TWO_PI ** 3 / kf
        return cls(N, nu, dt, f0, shell_no=tuple(range(1, kf + 1)), precision=precision, **kw)

    # ---- state -----------------------------------------------------------------------------------
    def set_velocity(self, u):
        """uk = dealias * rfft(u) from a physical (3, N, N, N) velocity (F:567-569)."""
        torch = _torch()
        p = self.plan
        ut = torch.as_tensor(u).to(device=p.device, dtype=p.rdtype).contiguous()
        p.rfft_cube(ut, self.uk)
        self.t = 0.0
        return self

    def set_uk_full(self, uk_full):
        """Load a reference-layout spectrum (3, N, N, N/2+1); modes outside the mask are dropped."""
        torch = _torch()
        p = self.plan
        ft = torch.as_tensor(uk_full).to(device=p.device, dtype=p.cdtype).contiguous()
        p.to_cube(ft, self.uk)
        return self

    def uk_full(self):
        """The state in the reference's layout (3, N, N, N/2+1), complex128 numpy."""
        return self.plan.from_cube(self.uk).cpu().numpy().astype(np.complex128)

    def velocity(self, out=None):
        """Physical velocity (3, N, N, N) on the device."""
        return self.plan.irfft_cube(self.uk, out)

    def energy_spectrum(self):
        """Shell spectrum ek_arr of F:423, F:431 (FP64 numpy)."""
        return self.plan.e3d_to_e1d(self.uk).cpu().numpy()

    def flux_spectrum(self):
        """Pik_arr of save() (F:424-428): shell sums of Re(conj(uk) . N(uk)) with N the inviscid,
        unforced RHS, then the reversed cumulative sum (FP64 numpy)."""
        from .outputs import flux_from_transfer
        p = self.plan
        ku = p.velocity_rhs(self.uk, self.nu, 0.0, self.shell_no, visc=0.0)
        return flux_from_transfer(p.shell_cross(self.uk, ku).cpu().numpy())

    def diagnostics(self):
        """What save() prints (F:464-484): energy from the physical field and from the shell
        spectrum, and the maximum divergence."""
        torch = _torch()
        p = self.plan
        u = self.velocity()
        dx = TWO_PI / self.N
        eng1 = float(0.5 * (u.double() ** 2).sum() * dx ** 3)
        eng2 = float(self.energy_spectrum().sum())
        divmax = float(p.divergence(self.uk).abs().max())
        del u
        return {"t": self.t, "energy": eng1, "energy_spectral": eng2, "divergence_max": divmax}

    def save(self, dirpath, droplets=None, state_dir=None):
        """Write the reference's output files (Fields_k_0, Energy_spectrum, Flux_spectrum and, with
        droplets, state_0 with pos, vel, prtclid and the fluid velocity at the droplets, umat) into
        dirpath; returns (paths, diagnostics)."""
        from .outputs import write_outputs
        state = None
        d = droplets if droplets is not None else self.droplets
        if d is not None:
            u = self.velocity()
            umat = d.gather(u).double()
            order = _torch().argsort(d.ids)
            state = {"pos": d.pos[order].cpu().numpy(), "vel": d.vel[order].double().cpu().numpy(),
                     "prtclid": d.ids[order].cpu().numpy(), "umat": umat[order].cpu().numpy()}
            if getattr(d, "mass", None) is not None:
                state["mass"] = d.mass[order].double().cpu().numpy()
            if state_dir is not None:
                state["dir"] = state_dir
            del u
        paths = write_outputs(dirpath, self.uk_full(), self.energy_spectrum(), self.flux_spectrum(), state=state)
        return paths, self.diagnostics()

    def load(self, dirpath):
        """Restart from the Fields_k_{slab}.npz files of a checkpoint written by any number of
        ranks (the spectral velocity in the reference's layout, re-slabbed as load_npz does,
        F:374-407).  Raises outputs.CheckpointError for a missing, truncated or mis-shaped
        checkpoint, or one of another grid size."""
        from .outputs import CheckpointError, read_fields
        uk = read_fields(dirpath)
        if uk.shape[1] != self.N:
            raise CheckpointError(f"checkpoint grid N = {uk.shape[1]}, this run N = {self.N}")
        return self.set_uk_full(uk)

    def attach(self, droplets, collider=None, sort_every=0, pair_capacity=None):
        """Advance ``droplets`` with the flow.

        Allocates the interleaved (N, N, N, 4) physical-velocity buffer the droplet stages read.
        With a ``collider`` the colliding pairs are found after every step (``self.pairs`` /
        ``collider.count`` on the device); with ``sort_every`` > 0 the droplets are re-sorted into
        cell order every that many steps, which keeps their stencil loads local in memory."""
        torch = _torch()
        self.droplets = droplets
        if self.u_phys is None:
            p = self.plan
            self.u_phys = torch.empty((p.N, p.N, p.N, 4), dtype=p.rdtype, device=p.device)
            # the second stage's velocity, so that it may be written while stage 1's is still read
            self.u_phys2 = torch.empty_like(self.u_phys) if self.overlap else self.u_phys
        self.collider = collider
        self.sort_every = int(sort_every)
        if collider is not None:
            check(_lib.lib().ld_collider_trace(collider._h, self.plan.handle))
        if collider is not None:
            cap = pair_capacity or max(1024, 4 * droplets.n)
            self.pairs = torch.empty((cap, 2), dtype=torch.int32, device=self.plan.device)
        if self.sort_every > 0:
            self._sorter = collider
            if self._sorter is None:
                from .collide import Collider
                self._sorter = Collider(droplets.n, 4 * self.plan.dx, device=self.plan.device)
                check(_lib.lib().ld_collider_trace(self._sorter._h, self.plan.handle))
            droplets.sort(self._sorter)
        return self

    # ---- stepping ---------------------------------------------------------------------------------
    def step(self, nsteps=1, stream=None):
        torch = _torch()
        s = torch.cuda.current_stream(self.plan.device) if stream is None else stream
        for k in range(nsteps):
            self._step_one(s)
        self._join(s)

    # ---- overlap of the droplet work with the flow ----------------------------------------------
    # With droplets attached and `overlap` on, a step's droplet work runs on a second stream: the
    # droplet stage of the first flow stage runs while the second flow stage transforms, and the
    # re-sort and the collision search run while the next step's first flow stage transforms.  The
    # two flow stages write their physical velocity into two buffers (u_phys, u_phys2) so that the
    # second stage does not overwrite what the first droplet stage reads, and the next step's
    # first stage waits for the first droplet stage.  The kernels and their inputs are the same as
    # with everything on one stream, so the results are identical.  Off by default: at 256^3 with
    # 1e6 learned droplets the step already keeps the GPU busy (2.04 -> 2.03 ms per step measured),
    # and concurrent kernels blur the per-kernel timings.
    def _dstream(self, s):
        torch = _torch()
        if not (self.overlap and self.droplets is not None and self.integrator == "rk2if"):
            return s
        if getattr(self, "_ds", None) is None:
            self._ds = torch.cuda.Stream(device=self.plan.device)
        return self._ds

    def _join(self, s):
        """Make `s` wait for the droplet stream (the state is complete on `s` afterwards)."""
        ds = self._dstream(s)
        if ds is not s:
            s.wait_stream(ds)

    def interp_state(self):
        """The droplet interpolation the next step will enqueue (what a captured graph freezes)."""
        d = self.droplets
        return None if d is None else d.interp_state()

    def judge(self, frac=0.01, seed=0, stream=None):
        """The judge of the learned interpolation on the current state: the exact spectral sum at a
        random fraction of the droplets against the learned and the tricubic velocities; the
        LearnedInterp's rule then switches the network off (tricubic fallback) or on.  Returns
        {"step", "learned", "tricubic", "n_sample", "enabled"} or None without a network."""
        torch = _torch()
        d = self.droplets
        li = getattr(d, "learned", None) if d is not None else None
        if li is None:
            return None
        n = max(1, int(round(frac * d.n)))
        g = torch.Generator(device="cpu").manual_seed(int(seed) * 1000003 + self.nstep)
        sel = torch.randperm(d.n, generator=g)[:n].to(d.pos.device)
        pos = d.pos[sel].contiguous()
        e_l, e_t = li.judge(self.uk, li.interleaved(self.uk), pos)
        return {"step": self.nstep, "learned": e_l, "tricubic": e_t, "n_sample": n, "enabled": li.enabled}

    def evolve(self, nsteps, st=0, on_output=None, judge_frac=0.01, judge_seed=0, graph_steps=0):
        """The time loop of evolve_and_save (F:556-627): `nsteps` steps; at every output interval -
        a step count divisible by `st` (F:575 `i % st == 0`), and once more after the last step
        (F:624) - the judge of the learned interpolation runs (when the droplets have one) and then
        `on_output(self)` (e.g. ``self.save(...)``).  The blow-up test of F:618-620 is read from the
        device status word at every output (and raises BlowUpError); the kernels raise the flag at
        the step it happens.  With graph_steps > 0 the steps between outputs run as replays of
        CUDA graphs of that many steps (one graph per re-sorting phase, re-captured when the
        judge switches the interpolation).  Returns the list of judgements."""
        verdicts = []

        def output():
            self.check()
            v = self.judge(judge_frac, judge_seed)
            if v is not None:
                verdicts.append(v)
            if on_output is not None:
                on_output(self)

        graphs = {}
        end = self.nstep + int(nsteps)
        while self.nstep < end:
            if st and self.nstep % st == 0:
                output()
            nxt = end if not st else min(end, (self.nstep // st + 1) * st)
            while graph_steps > 0 and nxt - self.nstep >= graph_steps:
                period = self.sort_every if (self.droplets is not None and self.sort_every > 0) else 0
                key = self.nstep % period if period else 0
                g = graphs.get(key)
                if g is None:
                    g = graphs[key] = self.capture(graph_steps)
                g.replay()
            self.step(nxt - self.nstep)
        output()
        return verdicts

    def capture(self, nsteps):
        """Capture `nsteps` steps from the current step count into a CUDA graph (nothing runs
        during the capture; the step counters are left as they were).  Returns a StepGraph whose
        replay() advances the state by nsteps steps with one graph launch.  The re-sorting of the
        droplets every sort_every steps is part of the graph, at the positions the current step
        count gives, so a replay must start at the same step count modulo sort_every."""
        return StepGraph(self, nsteps)

    def _step_one(self, stream, before_droplets=None, before_collide=None, after_flow=None):
        """One time step on `stream`.  `before_droplets()` is called just before the first droplet
        stage is enqueued, `after_flow()` once the flow state is final (last stage and epilogue
        enqueued; the last droplet stage follows), `before_collide()` after the droplet state is
        final (update and any re-sorting enqueued) and before the collision search: the hooks of
        `step_host` that overlap host copies with the flow transforms, the last droplet stage and
        the collision search.  The epilogue touches only the spectrum and the last droplet stage
        only the droplets, so running the epilogue first changes no result."""
        torch = _torch()
        L = _lib.lib()
        h = self.plan.handle
        if stream is None:
            stream = torch.cuda.current_stream(self.plan.device)
        st = stream_ptr(stream)
        prm = ctypes.byref(self.prm)
        d = self.droplets
        ds = self._dstream(stream)  # the droplet work's stream (the step's stream without overlap)
        ovl = ds is not stream
        u1 = self.u_phys if d is not None else None
        u2 = (self.u_phys2 if ovl else self.u_phys) if d is not None else None
        hooks = [before_droplets]
        e_d1 = None

        def droplets_ready():
            if hooks[0] is not None:
                hooks[0](ds)
                hooks[0] = None

        def fork():
            if ovl:
                ev = torch.cuda.Event()
                ev.record(stream)
                ds.wait_event(ev)

        if self.integrator == "rk2if":
            check(L.ld_rk2if_stage(h, 1, ptr(self.uk), ptr(self.aux), ptr(self.acc), ptr(u1), prm, st))
            if d is not None:
                fork()
                droplets_ready()
                d.stage(1, u1, self.dt, ds)
                if ovl:
                    e_d1 = torch.cuda.Event()
                    e_d1.record(ds)
            check(L.ld_rk2if_stage(h, 2, ptr(self.uk), ptr(self.aux), ptr(self.acc), ptr(u2), prm, st))
            if self.epilogue:
                check(L.ld_step_epilogue_plane0(h, ptr(self.uk), st))
            if after_flow is not None:
                after_flow()
            if d is not None:
                fork()
                d.stage(2, u2, self.dt, ds)
        else:
            for s in (1, 2, 3, 4):
                check(L.ld_rk4_stage(h, s, ptr(self.uk), ptr(self.aux), ptr(self.acc), None, prm, st))
            if self.epilogue:
                check(L.ld_step_epilogue_plane0(h, ptr(self.uk), st))
            if after_flow is not None:
                after_flow()
        self.t += self.dt
        self.nstep += 1
        droplets_ready()
        if d is not None and self.sort_every > 0 and self.nstep % self.sort_every == 0:
            d.sort(self._sorter, ds)
        if before_collide is not None:
            before_collide(ds)
        if d is not None and self.collider is not None:
            d.collide(self.collider, self.pairs, ds)
        if e_d1 is not None:
            stream.wait_event(e_d1)  # the next first stage rewrites what droplet stage 1 read

    def step_host(self, uk_host, pos_host=None, vel_host=None, nsteps=1, stream=None, layout="cube"):
        """Drop-in for one call of the reference's time-loop body with host state (F:582-610):
        copies the spectrum (and droplet positions/velocities) from host memory, advances
        ``nsteps`` steps and copies the new state back into the same host arrays.  ``layout``:
        "cube" - the dealiased cube (3, Mx, My, Mzp) the step keeps on the device; "full" - the
        reference's own layout (3, N, N, N/2+1) (F:158): only the rows of the dealiased cube move
        (strided copies), the modes outside the mask are dropped on the way in (the dealias of
        F:567-569); on the way out the first call for a host array writes all of it (zeros outside
        the mask), later calls only the cube rows (the rest stays zero unless the caller writes
        there).  Host tensors should be pinned for asynchronous copies.  Returns the host tensors.

        The spectrum is needed by the first kernel, so its copy precedes the step; the droplet
        copies run on a side stream under the first stage's flow transforms (the droplets are
        first read by the droplet stage).  The copies back run on a side stream: the spectrum's
        as soon as the flow state is final, under the last droplet stage and the collision
        search; the droplets' after their last update, under the collision search, which reads
        the positions but writes no state."""
        torch = _torch()
        if layout not in ("cube", "full"):
            raise ValueError("layout must be 'cube' or 'full'")
        s = torch.cuda.current_stream() if stream is None else stream
        d = self.droplets if pos_host is not None else None
        side = self._copy_streams()
        full = layout == "full"
        first_out = False
        if full:
            clean = getattr(self, "_clean_hosts", None)
            if clean is None:
                clean = self._clean_hosts = set()
            key = (uk_host.data_ptr(), tuple(uk_host.shape))
            first_out = key not in clean
            clean.add(key)
        with torch.cuda.stream(s):
            if not full:
                self.uk.copy_(uk_host, non_blocking=True)
            else:
                self.plan.copy_region_in(uk_host, self.uk, stream=s)
        if d is not None:
            side[0].wait_stream(s)  # earlier users of pos/vel are done before they are overwritten
            with torch.cuda.stream(side[0]):
                d.pos.copy_(pos_host, non_blocking=True)
                d.vel.copy_(vel_host, non_blocking=True)

        def droplets_in(ds):
            ds.wait_stream(side[0])

        def flow_out():
            if full and first_out:
                dev = self.plan.from_cube(self.uk, stream=s)
                side[1].wait_stream(s)
                with torch.cuda.stream(side[1]):
                    uk_host.copy_(dev, non_blocking=True)
                dev.record_stream(side[1])
                return
            side[1].wait_stream(s)
            with torch.cuda.stream(side[1]):
                if full:
                    self.plan.copy_region_out(self.uk, uk_host, stream=side[1])
                else:
                    uk_host.copy_(self.uk, non_blocking=True)

        def droplets_out(ds):
            if d is not None:
                side[1].wait_stream(ds)
                with torch.cuda.stream(side[1]):
                    pos_host.copy_(d.pos, non_blocking=True)
                    vel_host.copy_(d.vel, non_blocking=True)

        with torch.cuda.stream(s):
            for k in range(nsteps):
                last = k == nsteps - 1
                self._step_one(s, droplets_in if (k == 0 and d is not None) else None,
                               droplets_out if last else None, flow_out if last else None)
            if nsteps == 0:
                droplets_in(s)
                flow_out()
                droplets_out(s)
            self._join(s)
        s.wait_stream(side[1])
        s.synchronize()
        return uk_host, pos_host, vel_host

    def _copy_streams(self):
        torch = _torch()
        if getattr(self, "_side", None) is None:
            self._side = (torch.cuda.Stream(device=self.plan.device), torch.cuda.Stream(device=self.plan.device))
        return self._side

    def check(self, stream=None):
        """Host check of the device status word (the blow-up abort of F:618-620)."""
        flags = self.plan.status(clear=True, stream=stream)
        if flags & (_lib.STATUS_BLOWUP | _lib.STATUS_NONFINITE):
            raise BlowUpError(f"threshold exceeded or non-finite state at t={self.t:.6g} (flags={flags})")
        return flags


class StepGraph:
    """`nsteps` steps of a ForcedDNS captured as one CUDA graph (see ForcedDNS.capture).  The
    buffers the steps use must stay where they are (they do: every operation works in place)."""

    def __init__(self, dns, nsteps):
        self.dns = dns
        self.nsteps = int(nsteps)
        self.period = dns.sort_every if (dns.droplets is not None and dns.sort_every > 0) else 0
        self.phase = dns.nstep % self.period if self.period else 0
        self.recaptures = 0
        self._capture()

    def _capture(self):
        torch = _torch()
        dns = self.dns
        self.interp = dns.interp_state()
        saved = (dns.t, dns.nstep)
        self.graph = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(device=dns.plan.device)
        cap.wait_stream(torch.cuda.current_stream())
        try:
            with torch.cuda.graph(self.graph, stream=cap, capture_error_mode="thread_local"):
                dns.step(self.nsteps, stream=cap)
        finally:
            dns.t, dns.nstep = saved

    def replay(self, n=1):
        """Advance the state by n * nsteps steps (graph launches on the current stream).  A graph
        whose droplet interpolation is no longer the droplets' current one (the judge switched the
        learned interpolation off or on since the capture) is captured again first."""
        dns = self.dns
        for _ in range(n):
            if self.period and dns.nstep % self.period != self.phase:
                raise RuntimeError(f"step graph captured at step phase {self.phase} (mod {self.period}), "
                                   f"replayed at step {dns.nstep}")
            if dns.interp_state() != self.interp:
                self.graph = None
                self._capture()
                self.recaptures += 1
            self.graph.replay()
            for _ in range(self.nsteps):  # the same sum as stepping one by one
                dns.t += dns.dt
            dns.nstep += self.nsteps


class Droplets:
    """One-way-coupled inertial droplets: pos (n,3) FP64, vel (n,3), tau (n) on the device.

    ``ids`` (int64) follows every droplet through re-sorting, like the reference's prtclid
    (particles.py:92-93); ``radius`` (FP64, optional) is used by the collision search."""

    def __init__(self, plan, pos, vel, tau, method="tricubic", g=0.0, radius=None, ids=None):
        torch = _torch()
        self.plan = plan
        dev = plan.device
        self.pos = torch.as_tensor(pos).to(device=dev, dtype=torch.float64).contiguous()
        self.vel = torch.as_tensor(vel).to(device=dev, dtype=plan.rdtype).contiguous()
        self.tau = torch.as_tensor(tau).to(device=dev, dtype=plan.rdtype).contiguous()
        self.a1 = torch.zeros_like(self.vel)
        self.n = int(self.pos.shape[0])
        self.ids = (torch.arange(self.n, dtype=torch.int64, device=dev) if ids is None
                    else torch.as_tensor(ids).to(device=dev, dtype=torch.int64).contiguous())
        self.radius = (None if radius is None
                       else torch.as_tensor(radius).to(device=dev, dtype=torch.float64).contiguous())
        self._order = torch.empty(self.n, dtype=torch.int32, device=dev)
        if self.pos.shape != (self.n, 3) or self.vel.shape != (self.n, 3) or self.tau.shape != (self.n,):
            raise ValueError("pos (n,3), vel (n,3), tau (n,) expected")
        self.method = method
        self.m = _lib.LD_INTERP[method]
        self.g = float(g)

    def gather(self, field, pos=None, out=None, stream=None):
        """Interpolate the (C, N, N, N) field at pos (default: the droplet positions)."""
        torch = _torch()
        pos = self.pos if pos is None else pos
        C = int(field.shape[0])
        if out is None:
            out = torch.empty((pos.shape[0], C), dtype=self.plan.rdtype, device=self.plan.device)
        check(_lib.lib().ld_gather(self.plan.handle, ptr(field), C, ptr(pos), int(pos.shape[0]), self.m,
                                   ptr(out), stream_ptr(stream)))
        return out

    def arrays(self):
        """Every per-droplet array, in the order they are permuted together."""
        out = [("pos", self.pos), ("vel", self.vel), ("tau", self.tau), ("a1", self.a1), ("ids", self.ids)]
        if self.radius is not None:
            out.append(("radius", self.radius))
        return out

    def sort(self, collider, stream=None):
        """Re-order every per-droplet array into the collider's cell order, in place: each array
        is permuted into a persistent scratch buffer and copied back, so the arrays keep their
        device addresses (a captured CUDA graph replays against the same buffers)."""
        torch = _torch()
        L = _lib.lib()
        st = stream_ptr(stream)
        check(L.ld_cell_order(collider._h, ptr(self.pos), self.n, collider.L, ptr(self._order), st))
        if not hasattr(self, "_scratch"):
            self._scratch = {}
        for name, t in self.arrays():
            row = t.element_size() * (t.shape[1] if t.dim() > 1 else 1)
            tmp = self._scratch.get(name)
            if tmp is None or tmp.dtype != t.dtype or tmp.shape != t.shape:
                tmp = torch.empty_like(t)
                self._scratch[name] = tmp
            check(L.ld_permute_rows(ptr(t), ptr(tmp), ptr(self._order), self.n, row, st))
            check(L.ld_copy_async(ptr(t), ptr(tmp), t.numel() * t.element_size(), st))

    def collide(self, collider, pairs, stream=None):
        """Colliding pairs (array indices, i < j) into ``pairs``; the count stays on the device."""
        if self.radius is None:
            raise ValueError("droplet radii are needed for the collision search")
        check(_lib.lib().ld_collide(collider._h, ptr(self.pos), ptr(self.radius), self.n, collider.L, ptr(pairs),
                                    int(pairs.shape[0]), ptr(collider.count), stream_ptr(stream)))

    def by_id(self, t):
        """Rows of a per-droplet tensor in droplet-id order (host numpy)."""
        order = _torch().argsort(self.ids)
        return t[order].cpu().numpy()

    def interp_state(self):
        """"learned" while an attached network is enabled, else the droplets' own method."""
        li = getattr(self, "learned", None)
        return "learned" if (li is not None and li.enabled) else self.method

    def use_learned(self, learned):
        """Interpolate with a trained LearnedInterp (tricubic + learned correction); the judge of
        the LearnedInterp switches back to tricubic when it fails."""
        torch = _torch()
        self.learned = learned
        self._up = torch.empty((self.n, 3), dtype=self.plan.rdtype, device=self.plan.device)
        self._xs = torch.empty((self.n, 3), dtype=torch.float64, device=self.plan.device)
        # feature tiles of their own: the droplet stage may overlap the plan's transforms
        self._mlp_work = learned.workspace(self.n)

    def stage(self, s, u_phys, h, stream=None):
        li = getattr(self, "learned", None)
        if li is not None and li.enabled:
            L = _lib.lib()
            st = stream_ptr(stream)
            if s == 1:
                li.infer(u_phys, self.pos, out=self._up, stream=stream, work=self._mlp_work)
            else:
                check(L.ld_droplet_predict(self.plan.handle, ptr(self.pos), ptr(self.vel), self.n, float(h),
                                           ptr(self._xs), st))
                li.infer(u_phys, self._xs, out=self._up, stream=stream, work=self._mlp_work)
            check(L.ld_droplet_update(self.plan.handle, int(s), ptr(self._up), ptr(self.pos), ptr(self.vel),
                                      ptr(self.tau), ptr(self.a1), self.n, float(h), self.g, st))
            return
        check(_lib.lib().ld_droplet_stage(self.plan.handle, int(s), ptr(u_phys), ptr(self.pos), ptr(self.vel),
                                          ptr(self.tau), ptr(self.a1), self.n, self.m, float(h), self.g,
                                          stream_ptr(stream)))
