"""Seeded initial conditions (forced-dns-sm.py:691-736, particles.py:91-96).

Flow: the reference's random-phase construction - per-mode amplitude sqrt(E(kint)/kint^2/normalize)
with uniform phases, masked to 0 < kint < 31 and the dealias sphere (F:699-707) - is built on the
host (elementwise NumPy, RNG draws in the same order as the reference: uk, vk, wk phases), then on
the GPU: the irfft -> rfft round trip (which for a field inside the dealiased cube is the
symmetrisation of the kz = 0 plane), the div-free projection (F:717-720) and the scaling to the
target energy (F:722-728) with the FP64 shell spectrum.

Droplets: positions uniform in [0, 2pi)^3 and Stokes times either log-uniform in [0.05, 2] or from
lognormal radii (tau ~ r^2, median St = 0.5); velocities are set by the caller (the
configurations start droplets at the interpolated fluid velocity).
"""
import numpy as np

from .spectral import TWO_PI


def _torch():
    import torch
    return torch


def reference_profile(kint):
    """E(k) ~ k^2 exp(-k^2/2) (F:700)."""
    return kint.astype(np.float64) ** 2 * np.exp(-kint.astype(np.float64) ** 2 / 2)


def config_profile(kint):
    """E(k) ~ k^4 exp(-2 (k/4)^2)."""
    return kint.astype(np.float64) ** 4 * np.exp(-2.0 * (kint / 4.0) ** 2)


def mode_tables(N):
    """kint (F:127), dealias (F:129) and normalize (F:136) in the reference layout."""
    Kx = np.fft.fftfreq(N, 1.0 / N)
    Kz = np.abs(Kx[: N // 2 + 1])
    kx, ky, kz = np.meshgrid(Kx, Kx, Kz, indexing="ij", sparse=True)
    k2 = kx ** 2 + ky ** 2 + kz ** 2
    kint = np.clip(np.round(np.sqrt(k2)).astype(np.int64), None, N // 2)
    dealias = kint <= N / 3
    normalize = np.where((kz == 0) | (kz == N // 2), 1.0, 2.0) / (N ** 6 / TWO_PI ** 3)
    return kint, dealias, normalize


def random_phase_spectrum(N, phases, profile, kinit=31):
    """uk_c = amp exp(i th_c) (kint^2 < kinit^2) (kint > 0) dealias  (F:699-707), host complex128."""
    kint, dealias, normalize = mode_tables(N)
    eprofile = profile(kint) / normalize
    amp = np.sqrt(eprofile / np.where(kint == 0, np.inf, kint.astype(np.float64) ** 2))
    mask = (kint ** 2 < kinit ** 2) & (kint > 0) & dealias
    amp = np.where(mask, amp, 0.0)
    return np.stack([amp * np.exp(1j * th) for th in phases])


def init_flow(dns, seed, E0=0.5, profile=config_profile, kinit=31, phases=None):
    """Set ``dns.uk`` to the seeded random-phase solenoidal field with energy E0 (2pi)^3.

    ``phases`` (three (N, N, N/2+1) arrays) overrides the draws from np.random.default_rng(seed)."""
    torch = _torch()
    N = dns.N
    if phases is None:
        rng = np.random.default_rng(seed)
        phases = [rng.uniform(0, TWO_PI, (N, N, N // 2 + 1)) for _ in range(3)]
    uk = random_phase_spectrum(N, phases, profile, kinit)
    p = dns.plan
    full = torch.as_tensor(uk).to(device=p.device, dtype=p.cdtype)
    p.to_cube(full, dns.uk)
    del full
    _project(dns)
    ek = p.e3d_to_e1d(dns.uk)
    e0 = float(ek.sum().item())
    dns.uk.mul_((E0 * TWO_PI ** 3 / e0) ** 0.5)
    dns.t = 0.0
    return dns


def _project(dns):
    from . import _lib
    from ._lib import check, ptr, stream_ptr
    check(_lib.lib().ld_step_epilogue(dns.plan.handle, ptr(dns.uk), stream_ptr()))


def init_droplets(n, seed, kind, nu=None, eps=0.1):
    """Seeded droplets: returns (pos (n,3) f64, tau (n,) f64, radius (n,) f64).

    kind "uniform_tau": tau log-uniform in [0.05, 2];
    kind "lognormal_r": r = 0.002*2pi exp(0.3 Z), tau = 0.5 sqrt(nu/eps) (r / r_med)^2."""
    rng = np.random.default_rng(seed + 7919)
    pos = rng.uniform(0, TWO_PI, (n, 3))
    if kind == "uniform_tau":
        tau = np.exp(rng.uniform(np.log(0.05), np.log(2.0), n))
        radius = np.full(n, 0.002 * TWO_PI) * np.sqrt(tau / np.median(tau))
    elif kind == "lognormal_r":
        r_med = 0.002 * TWO_PI
        radius = r_med * np.exp(0.3 * rng.standard_normal(n))
        tau = 0.5 * (nu / eps) ** 0.5 * (radius / r_med) ** 2
    else:
        raise ValueError(kind)
    return pos, tau, radius
