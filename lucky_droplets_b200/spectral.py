"""Grid, transforms and spectral operators on one GPU (forced-dns-sm.py:49-233).

``Plan`` wraps one ``ld_plan`` of the C ABI.  Its buffers are torch tensors on the plan's
device; the methods keep the reference's names and argument meaning where one exists:

    rfft_mpi(u, fu)  -> fu        forced-dns-sm.py:201-206  (one GPU: no slab all-to-all)
    irfft_mpi(fu, u) -> u         forced-dns-sm.py:208-213
    e3d_to_e1d(uk)   -> ek_arr    forced-dns-sm.py:232-233, 243-245  (shell spectrum, FP64)

plus the dealiased "cube" layout every transform of the DNS step uses internally.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ptr, stream_ptr

TWO_PI = 2.0 * np.pi


def _torch():
    import torch
    return torch


class Plan:
    """One N^3 grid in FP32 ("f32") or FP64 ("f64") on a CUDA device."""

    def __init__(self, N, precision="f32", device=None, nbox=1):
        """nbox > 1: a plan for nbox independent boxes; its stage calls advance states laid out
        (nbox, 3, Mx, My, Mzp) in one launch per pass (ld_plan_create_boxes)."""
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("lucky_droplets_b200 needs a CUDA device (no CPU fallback)")
        dev = torch.device(device if device is not None else "cuda")
        if dev.type != "cuda":
            raise ValueError("a Plan lives on a CUDA device")
        self.device = torch.device("cuda", dev.index if dev.index is not None else torch.cuda.current_device())
        self.precision = precision
        prec = {"f32": _lib.LD_F32, "f64": _lib.LD_F64}[precision]
        self.rdtype = torch.float32 if precision == "f32" else torch.float64
        self.cdtype = torch.complex64 if precision == "f32" else torch.complex128
        L = _lib.lib()
        h = ctypes.c_void_p()
        self.nbox = int(nbox)
        with torch.cuda.device(self.device):
            check(L.ld_plan_create_boxes(ctypes.byref(h), int(N), prec, self.nbox))
        self._h = h
        dims = (ctypes.c_int32 * 8)()
        wb = ctypes.c_size_t()
        check(L.ld_plan_dims(h, dims, ctypes.byref(wb)))
        self.N, self.kc, self.Mx, self.My, self.Mz, self.Mzp, self.Nf = list(dims)[:7]
        self.work_bytes = wb.value
        self.L = TWO_PI
        self.dx = TWO_PI / self.N

    # ---- lifetime -----------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().ld_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ---- buffers ---------------------------------------------------------------------------------
    def empty_cube(self, ncomp=3):
        return _torch().zeros((ncomp, self.Mx, self.My, self.Mzp), dtype=self.cdtype, device=self.device)

    def empty_phys(self, ncomp=3):
        return _torch().empty((ncomp, self.N, self.N, self.N), dtype=self.rdtype, device=self.device)

    def empty_full(self, ncomp=3):
        return _torch().empty((ncomp, self.N, self.N, self.Nf), dtype=self.cdtype, device=self.device)

    def _chk(self, t, dtype, tail):
        if t.device != self.device or t.dtype != dtype or not t.is_contiguous():
            raise ValueError(f"expected a contiguous {dtype} tensor on {self.device}")
        if tuple(t.shape[-len(tail):]) != tuple(tail):
            raise ValueError(f"expected trailing shape {tail}, got {tuple(t.shape)}")
        return int(np.prod(t.shape[:-len(tail)])) if t.dim() > len(tail) else 1

    # ---- transforms --------------------------------------------------------------------------------
    def rfft_mpi(self, u, fu=None, stream=None):
        """Forward R2C of (..., N, N, N) real fields into the reference layout (..., N, N, N/2+1)."""
        N = self.N
        nc = self._chk(u, self.rdtype, (N, N, N))
        if fu is None:
            fu = _torch().empty(tuple(u.shape[:-3]) + (N, N, self.Nf), dtype=self.cdtype, device=self.device)
        self._chk(fu, self.cdtype, (N, N, self.Nf))
        check(_lib.lib().ld_rfft_mpi(self._h, ptr(u), ptr(fu), nc, stream_ptr(stream)))
        return fu

    def irfft_mpi(self, fu, u=None, stream=None):
        """Inverse C2R of reference-layout spectra (1/N^3 normalisation, scipy convention)."""
        N = self.N
        nc = self._chk(fu, self.cdtype, (N, N, self.Nf))
        if u is None:
            u = _torch().empty(tuple(fu.shape[:-3]) + (N, N, N), dtype=self.rdtype, device=self.device)
        self._chk(u, self.rdtype, (N, N, N))
        check(_lib.lib().ld_irfft_mpi(self._h, ptr(fu), ptr(u), nc, stream_ptr(stream)))
        return u

    def rfft_cube(self, u, uk=None, stream=None):
        """Forward transform keeping only the dealiased cube (modes outside it are dropped)."""
        N = self.N
        nc = self._chk(u, self.rdtype, (N, N, N))
        if uk is None:
            uk = _torch().empty(tuple(u.shape[:-3]) + (self.Mx, self.My, self.Mzp), dtype=self.cdtype,
                                device=self.device)
        self._chk(uk, self.cdtype, (self.Mx, self.My, self.Mzp))
        check(_lib.lib().ld_rfft_cube(self._h, ptr(u), ptr(uk), nc, stream_ptr(stream)))
        return uk

    def irfft_cube(self, uk, u=None, stream=None):
        """Inverse transform of cube-layout spectra (zero outside the cube)."""
        N = self.N
        nc = self._chk(uk, self.cdtype, (self.Mx, self.My, self.Mzp))
        if u is None:
            u = _torch().empty(tuple(uk.shape[:-3]) + (N, N, N), dtype=self.rdtype, device=self.device)
        self._chk(u, self.rdtype, (N, N, N))
        check(_lib.lib().ld_irfft_cube(self._h, ptr(uk), ptr(u), nc, stream_ptr(stream)))
        return u

    def to_cube(self, full, cube=None, stream=None):
        """dealias * full, restricted to the cube (the dealias of F:567-569)."""
        nc = self._chk(full, self.cdtype, (self.N, self.N, self.Nf))
        if cube is None:
            cube = _torch().empty(tuple(full.shape[:-3]) + (self.Mx, self.My, self.Mzp), dtype=self.cdtype,
                                  device=self.device)
        check(_lib.lib().ld_spec_to_cube(self._h, ptr(full), ptr(cube), nc, stream_ptr(stream)))
        return cube

    def from_cube(self, cube, full=None, stream=None):
        """Cube layout -> reference layout (zeros outside the cube)."""
        nc = self._chk(cube, self.cdtype, (self.Mx, self.My, self.Mzp))
        if full is None:
            full = _torch().empty(tuple(cube.shape[:-3]) + (self.N, self.N, self.Nf), dtype=self.cdtype,
                                  device=self.device)
        check(_lib.lib().ld_spec_from_cube(self._h, ptr(cube), ptr(full), nc, stream_ptr(stream)))
        return full

    def copy_region_in(self, full, cube, stream=None):
        """Cube-layout spectra from reference-layout ones (host pinned or device): only the rows of
        the dealiased cube are copied, then masked - the result of to_cube."""
        nc = self._chk(cube, self.cdtype, (self.Mx, self.My, self.Mzp))
        if full.dtype != self.cdtype or not full.is_contiguous() or tuple(full.shape[-3:]) != (self.N, self.N, self.Nf):
            raise ValueError(f"expected a contiguous {self.cdtype} (..., N, N, N/2+1) tensor")
        check(_lib.lib().ld_spec_copy_region(self._h, ptr(full), ptr(cube), nc, 0, stream_ptr(stream)))
        return cube

    def copy_region_out(self, cube, full, stream=None):
        """Write the dealiased cube rows of reference-layout spectra (host pinned or device) from
        cube-layout ones; no other element of `full` is written."""
        nc = self._chk(cube, self.cdtype, (self.Mx, self.My, self.Mzp))
        if full.dtype != self.cdtype or not full.is_contiguous() or tuple(full.shape[-3:]) != (self.N, self.N, self.Nf):
            raise ValueError(f"expected a contiguous {self.cdtype} (..., N, N, N/2+1) tensor")
        check(_lib.lib().ld_spec_copy_region(self._h, ptr(cube), ptr(full), nc, 1, stream_ptr(stream)))
        return full

    # ---- spectra and RHS ---------------------------------------------------------------------------
    def e3d_to_e1d(self, uk, out=None, stream=None):
        """Shell energy spectrum of a cube-layout 3-vector (FP64, length N/2+1)."""
        self._chk(uk, self.cdtype, (3, self.Mx, self.My, self.Mzp))
        if out is None:
            out = _torch().zeros(self.Nf, dtype=_torch().float64, device=self.device)
        check(_lib.lib().ld_shell_spectrum(self._h, ptr(uk), ptr(out), stream_ptr(stream)))
        return out

    def autotune(self, stream=None):
        """Time every launch variant of the y passes on this plan and keep the fastest; returns
        {"ms": {pass: [one-shot, pipelined 1..3 CTAs/SM]}, "choice": [inverse, forward]}."""
        ms = (ctypes.c_double * 8)()
        ch = (ctypes.c_int32 * 2)()
        check(_lib.lib().ld_plan_autotune(self._h, ms, ch, stream_ptr(stream)))
        return {"ms": {"inverse_y": [round(x, 5) for x in ms[:4]], "forward_y": [round(x, 5) for x in ms[4:]]},
                "choice": [int(ch[0]), int(ch[1])]}

    def set_wait_limit(self, limit=0, stall=False):
        """Polls before a bounded device wait of this plan's kernels gives up (0: the default);
        stall=True makes the first waits run out on purpose (a test of the time-out path)."""
        check(_lib.lib().ld_plan_set_wait_limit(self._h, int(limit), int(bool(stall))))

    def set_tuning(self, choice):
        ch = (ctypes.c_int32 * 2)(*[int(c) for c in choice])
        check(_lib.lib().ld_plan_set_tuning(self._h, ch))

    def shell_cross(self, a, b, out=None, stream=None):
        """Shell sums of Re(conj(a) . b) * normalize (FP64, length N/2+1) of cube-layout 3-vectors."""
        self._chk(a, self.cdtype, (3, self.Mx, self.My, self.Mzp))
        self._chk(b, self.cdtype, (3, self.Mx, self.My, self.Mzp))
        if out is None:
            out = _torch().zeros(self.Nf, dtype=_torch().float64, device=self.device)
        check(_lib.lib().ld_shell_cross(self._h, ptr(a), ptr(b), ptr(out), stream_ptr(stream)))
        return out

    def divergence(self, uk, stream=None):
        """Physical divergence (N, N, N) of a cube-layout 3-vector (spectral derivatives)."""
        self._chk(uk, self.cdtype, (3, self.Mx, self.My, self.Mzp))
        dk = self.empty_cube(1)
        check(_lib.lib().ld_divergence_spec(self._h, ptr(uk), ptr(dk), stream_ptr(stream)))
        return self.irfft_cube(dk, stream=stream)[0]

    def velocity_rhs(self, uk, nu, f0=0.0, shell_no=(1,), visc=1.0, ku=None, u_out=None, stream=None):
        """ku = P[(u x w)^ + f] dealias - visc nu k^2 uk  (full_RHS velocity part, F:287-316)."""
        self._chk(uk, self.cdtype, (3, self.Mx, self.My, self.Mzp))
        if ku is None:
            ku = self.empty_cube(3)
        prm = flow_params(0.0, nu, f0, shell_no)
        check(_lib.lib().ld_velocity_rhs(self._h, ptr(uk), ptr(ku), ptr(u_out), ctypes.byref(prm), float(visc),
                                         stream_ptr(stream)))
        return ku

    def exact_sum(self, uk, pos, out=None, stream=None):
        """Direct Fourier-sum velocity (FP64) of a cube-layout 3-vector at pos (n, 3) double."""
        torch = _torch()
        self._chk(uk, self.cdtype, (3, self.Mx, self.My, self.Mzp))
        n = int(pos.shape[0])
        if out is None:
            out = torch.empty((n, 3), dtype=torch.float64, device=self.device)
        check(_lib.lib().ld_exact_sum(self._h, ptr(uk), ptr(pos), n, ptr(out), stream_ptr(stream)))
        return out

    def profile(self, enable=True):
        """Start/stop bracketing every kernel launch of this plan with CUDA events."""
        check(_lib.lib().ld_profile(self._h, int(bool(enable))))

    def profile_read(self, reset=True):
        """{kernel name: (launches, total device ms)} since the last reset (synchronises)."""
        cap = 64
        kid = (ctypes.c_int32 * cap)()
        cnt = (ctypes.c_int64 * cap)()
        ms = (ctypes.c_double * cap)()
        n = ctypes.c_int32()
        check(_lib.lib().ld_profile_read(self._h, kid, cnt, ms, cap, ctypes.byref(n), int(bool(reset))))
        L = _lib.lib()
        return {(L.ld_kernel_name(kid[i]) or b"k%d" % kid[i]).decode(): (int(cnt[i]), float(ms[i]))
                for i in range(min(n.value, cap))}

    def status(self, clear=True, stream=None):
        v = ctypes.c_uint32()
        check(_lib.lib().ld_status(self._h, ctypes.byref(v), int(bool(clear)), stream_ptr(stream)))
        return v.value


def flow_params(dt, nu, f0, shell_no):
    shells = list(shell_no) if shell_no is not None else []
    lo, hi = (min(shells), max(shells)) if shells else (1, 0)
    if shells and shells != list(range(lo, hi + 1)):
        raise ValueError("forced shells must be consecutive (shell_no = 1..nshells, F:89-90)")
    return _lib.FlowParams(float(dt), float(nu), float(f0) if shells else 0.0, int(lo), int(hi))
