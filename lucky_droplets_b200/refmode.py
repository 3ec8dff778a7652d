"""The reference's own physics on the GPU: forced-dns-sm.py's time loop with its droplets and the
number-density field of small droplets (F:278-362, F:556-627; particles.py P:52-96, P:191-195,
P:514-577, P:817-837).

State (FP64, as the reference):
  uk     the spectral velocity (dealiased cube), RK4 with explicit viscosity (F:335-362)
  n      the number density of small droplets on the grid (N, N, N), advected with the
         slow-manifold velocity v = u - tps Du/Dt - tps g z and fed by the mass the big droplets
         take up (F:319-330), kept non-negative with the reference's clip_zero (F:278-285)
  coord  the big droplets (n, 7): position, velocity, mass, moved by pRHS (P:817-837) with
         cosine interpolation; their mass uptake is deposited back with the same kernel

`ReferenceRun.step()` is `rk4_step` of the oracle (F:582-620) step for step: the same stage
inputs, the in-place clipping of n at the first stage, the same weights.  Droplets keep their
index order (`ids` = prtclid); positions are not wrapped (every interpolation wraps them).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ptr, stream_ptr
from .dns import ForcedDNS
from .spectral import TWO_PI


def _torch():
    import torch
    return torch


class ReferenceDroplets:
    """MPI_particles state on one GPU (P:52-111): coord (n, 7) and the intrinsic constants."""

    def __init__(self, plan, coord, st_s, g, nu, tau_eta, rho_p, M0):
        torch = _torch()
        dev = plan.device
        self.plan = plan
        self.coord = torch.as_tensor(np.asarray(coord, np.float64)).to(dev).contiguous()
        self.n = int(self.coord.shape[0])
        self.factor = (nu * tau_eta / (2 * rho_p)) ** 3 / 2 * (36 * np.pi * rho_p) / M0  # P:74, as written
        self.growthfactor = 9 * np.pi * nu / (2 * rho_p)                                    # P:75
        self.st_s, self.g, self.tau_eta = float(st_s), float(g), float(tau_eta)
        self.ids = torch.arange(self.n, dtype=torch.int64, device=dev)
        n = max(1, self.n)
        f64 = dict(dtype=torch.float64, device=dev)
        self.pos = torch.empty((n, 3), **f64)
        self.iu = torch.empty((n, 3), **f64)
        self.iv = torch.empty((n, 3), **f64)
        self.ic = torch.empty((n,), **f64)
        self.mdot = torch.empty((n,), **f64)
        self.w = torch.empty((n, 12), **f64)
        self.key = torch.empty((n,), dtype=torch.int32, device=dev)
        self.val = torch.empty((n,), dtype=torch.int32, device=dev)
        N = plan.N
        self.cs = torch.empty((N ** 3 + 1,), dtype=torch.int32, device=dev)
        self.bits = int(np.ceil(np.log2(max(2, N ** 3))))
        from .collide import Collider
        self._sorter = Collider(n, TWO_PI, device=dev)  # radix-sort workspace only

    @property
    def st(self):
        """St = (m / factor)^(2/3) (P:191-195)."""
        return (self.coord[:, 6] / self.factor) ** (2.0 / 3.0)

    def rhs(self, coord, u4, v, n_field, kp, fc, stream=None):
        """pRHS (P:817-837) at coord with the fluid velocity u4 (interleaved (N,N,N,4)), the
        slow-manifold velocity v (3, N, N, N) and the number density n_field (N, N, N): kp (n, 7),
        and the deposited mass sink fc (N, N, N)."""
        L = _lib.lib()
        p = self.plan
        st = stream_ptr(stream)
        n = self.n
        if n == 0:
            fc.zero_()
            return kp, fc
        check(L.ld_extract_pos(ptr(coord), n, ptr(self.pos), st))
        check(L.ld_gather4(p.handle, ptr(u4), ptr(self.pos), n, _lib.LD_INTERP["cosine"], ptr(self.iu), st))
        check(L.ld_gather(p.handle, ptr(v), 3, ptr(self.pos), n, _lib.LD_INTERP["cosine"], ptr(self.iv), st))
        check(L.ld_gather(p.handle, ptr(n_field), 1, ptr(self.pos), n, _lib.LD_INTERP["cosine"], ptr(self.ic), st))
        check(L.ld_prhs_ref(ptr(coord), ptr(self.iu), ptr(self.iv), ptr(self.ic), n, self.factor, self.growthfactor,
                            self.st_s, self.tau_eta, self.g, ptr(kp), ptr(self.mdot), st))
        # deposition (exterp_cosine_scalar, P:514-577), deterministic pull in the reference's order
        check(L.ld_cell_weights(ptr(coord), n, p.N, TWO_PI, ptr(self.key), ptr(self.val), ptr(self.w), st))
        check(L.ld_radix_sort_u32(self._sorter._h, ptr(self.key), ptr(self.val), n, self.bits, st))
        check(L.ld_cell_starts(ptr(self.key), n, p.N ** 3, ptr(self.cs), st))
        check(L.ld_deposit_pull(ptr(self.val), ptr(self.cs), ptr(self.w), ptr(self.mdot), p.N, TWO_PI, ptr(fc), st))
        return kp, fc


class ReferenceRun:
    """forced-dns-sm.py's time loop (RK4, F:556-627) with the n field and the big droplets."""

    def __init__(self, dns, n0, droplets, tps, g):
        torch = _torch()
        if dns.plan.precision != "f64":
            raise ValueError("the reference mode runs in FP64")
        self.dns = dns
        self.drops = droplets
        self.tps, self.g = float(tps), float(g)
        p = dns.plan
        N = p.N
        dev = p.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.n = torch.as_tensor(np.asarray(n0, np.float64)).to(dev).reshape(N, N, N).contiguous()
        self.u4 = torch.empty((N, N, N, 4), **f64)
        self.u = p.empty_phys(3)
        self.vk = p.empty_cube(3)
        self.v = p.empty_phys(3)
        self.n_stage = torch.empty((N, N, N), **f64)
        self.n_tmp = torch.empty((N, N, N), **f64)
        self.n_new = torch.empty((N, N, N), **f64)
        self.kn = torch.empty((1, N, N, N), **f64)
        self.fc = torch.empty((N, N, N), **f64)
        self.nv = p.empty_phys(3)
        self.nvk = p.empty_cube(3)
        self.fck = p.empty_cube(1)
        self.knk = p.empty_cube(1)
        nd = max(1, droplets.n if droplets is not None else 1)
        self.kp = torch.empty((nd, 7), **f64)
        self.sump = torch.empty((nd, 7), **f64)
        self.c_stage = torch.empty((nd, 7), **f64)
        self.work = torch.empty((int(_lib.lib().ld_ref_workspace_doubles()),), **f64)

    def load(self, dirpath, n_dir=None):
        """Restart the flow and the number density from a checkpoint of the reference written by
        any number of ranks (load_npz, F:374-407): Fields_k_{slab}.npz in dirpath, n_{slab}.npz
        in n_dir (the reference keeps them in its droplet directory, F:449-450; default dirpath)."""
        from .outputs import CheckpointError, read_n
        self.dns.load(dirpath)
        n = read_n(dirpath if n_dir is None else n_dir)
        N = self.dns.N
        if n.shape != (N, N, N):
            raise CheckpointError(f"n of shape {n.shape} in a run of N = {N}")
        self.n.copy_(_torch().as_tensor(np.asarray(n, np.float64)))
        return self

    # ---- pieces -----------------------------------------------------------------------------------
    def n_rhs(self, n_field, fc, out, stream=None):
        """kn = irfft((-i k . (n v)^ - fc^) dealias) (F:325-330), with v = self.v."""
        L = _lib.lib()
        p = self.dns.plan
        st = stream_ptr(stream)
        check(L.ld_n_products(p.handle, ptr(n_field), ptr(self.v), ptr(self.nv), st))
        p.rfft_cube(self.nv, self.nvk, stream=stream)
        p.rfft_cube(fc.reshape(1, p.N, p.N, p.N), self.fck, stream=stream)
        check(L.ld_n_combine(p.handle, ptr(self.nvk), ptr(self.fck), ptr(self.knk), st))
        return p.irfft_cube(self.knk, out, stream=stream)

    def clip_zero(self, x, out, clip_src, stream=None):
        check(_lib.lib().ld_clip_zero(ptr(x), ptr(out), x.numel(), int(clip_src), ptr(self.work),
                                      stream_ptr(stream)))
        return out

    def full_rhs(self, n_field=None, coord=None, stream=None):
        """full_RHS (F:287-332) at the current uk, n_field (used as given) and coord: returns
        (ku, kn (N,N,N), kp (n,7), fc (N,N,N))."""
        L = _lib.lib()
        p = self.dns.plan
        n_field = self.n if n_field is None else n_field
        ku = p.empty_cube(3)
        check(L.ld_slow_manifold(p.handle, ptr(self.vk), self.tps, self.g))
        try:
            check(L.ld_velocity_rhs(p.handle, ptr(self.dns.uk), ptr(ku), ptr(self.u), ctypes.byref(self.dns.prm), 1.0,
                                    stream_ptr(stream)))
        finally:
            check(L.ld_slow_manifold(p.handle, None, 0.0, 0.0))
        p.irfft_cube(self.vk, self.v, stream=stream)
        check(L.ld_interleave3(p.handle, ptr(self.u), ptr(self.u4), stream_ptr(stream)))
        if self.drops is not None and self.drops.n > 0:
            coord = self.drops.coord if coord is None else coord
            self.drops.rhs(coord, self.u4, self.v, n_field, self.kp, self.fc, stream)
        else:
            self.fc.zero_()
        self.n_rhs(n_field, self.fc, self.kn, stream)
        return ku, self.kn[0], self.kp[: (self.drops.n if self.drops else 0)], self.fc

    # ---- the RK4 step (F:582-620) -----------------------------------------------------------------
    def step(self, nsteps=1, stream=None):
        L = _lib.lib()
        dns = self.dns
        p = dns.plan
        st = stream_ptr(stream)
        h = dns.dt
        m = p.N ** 3
        d = self.drops
        nd = d.n if d is not None else 0
        for _ in range(nsteps):
            if nd:
                check(L.ld_copy_async(ptr(self.sump), ptr(d.coord), nd * 7 * 8, st))       # sump = coord
            check(L.ld_copy_async(ptr(self.n_new), ptr(self.n), m * 8, st))                  # nnew = n
            self.clip_zero(self.n, self.n_stage, True, stream)                                # n clipped in place
            coord_stage = d.coord if nd else None
            weights = (h / 6.0, h / 3.0, h / 3.0, h / 6.0)
            alphas = (h / 2.0, h / 2.0, h)
            check(L.ld_slow_manifold(p.handle, ptr(self.vk), self.tps, self.g))
            try:
                for s in (1, 2, 3, 4):
                    # flow stage at the stage input (updates the RK4 state, writes u and v of the input)
                    check(L.ld_rk4_stage(p.handle, s, ptr(dns.uk), ptr(dns.aux), ptr(dns.acc), ptr(self.u4),
                                         ctypes.byref(dns.prm), st))
                    p.irfft_cube(self.vk, self.v, stream=stream)
                    if nd:
                        d.rhs(coord_stage, self.u4, self.v, self.n_stage, self.kp, self.fc, stream)
                    else:
                        self.fc.zero_()
                    self.n_rhs(self.n_stage, self.fc, self.kn, stream)
                    if nd:
                        check(L.ld_axpy(ptr(self.sump), weights[s - 1], ptr(self.kp), nd * 7, st))
                    check(L.ld_axpy(ptr(self.n_new), weights[s - 1], ptr(self.kn), m, st))
                    if s < 4:
                        a = alphas[s - 1]
                        if nd:
                            check(L.ld_waxpy(ptr(self.c_stage), ptr(d.coord), a, ptr(self.kp), nd * 7, st))
                            coord_stage = self.c_stage
                        check(L.ld_waxpy(ptr(self.n_tmp), ptr(self.n), a, ptr(self.kn), m, st))
                        self.clip_zero(self.n_tmp, self.n_stage, False, stream)
            finally:
                check(L.ld_slow_manifold(p.handle, None, 0.0, 0.0))
            if nd:
                check(L.ld_copy_async(ptr(d.coord), ptr(self.sump), nd * 7 * 8, st))          # F:582
            self.clip_zero(self.n_new, self.n, False, stream)                                 # F:584
            check(L.ld_step_epilogue_plane0(p.handle, ptr(dns.uk), st))                       # F:596-620
            dns.t += h
            dns.nstep += 1
