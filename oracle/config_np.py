"""FP64 CPU oracle for the benchmark-configuration semantics (not present in the reference).

TEST INFRASTRUCTURE ONLY: used by tests, smoke() and bench.py's CPU legs, never by the product.

What it restates and where each part comes from:
  * the flow RHS is the reference's velocity part of full_RHS (forced-dns-sm.py:287-316) with the
    viscous term removed from the RHS and put into an integrating factor;
  * the forcing is the reference's constant-power forcing (forced-dns-sm.py:239-275) with
    f0 = eps (2 pi)^3 / nshells on shells 1..kf (kf = 2 for |k| <= 2);
  * time integration is Heun (RK2) with the integrating factor E = exp(-nu k^2 h):
        u*      = E (u_n + h N(u_n))
        u_{n+1} = E (u_n + h/2 N(u_n)) + h/2 N(u*)
  * droplets follow x' = v, v' = (u(x) - v)/tau - g z (the reference's form, particles.py:831-834,
    with tau given directly), advanced by Heun on the same two stages, u* supplying stage 2;
  * gathers: trilinear (2^3), tricubic = tensor-product 4-point Lagrange on offsets -1..2
    (exact for cubics), and the reference's cosine kernel (particles.py:6-20, 435-511).
"""
import os

import numpy as np
import scipy.fft as sfft

from . import reference_np as R

TWO_PI = 2.0 * np.pi
_WORKERS = os.cpu_count() or 1


class ConfigGrid(R.Grid):
    """The reference grid with multi-threaded transforms (same arithmetic as R.Grid)."""

    def rfft(self, u):
        return sfft.rfftn(u, workers=_WORKERS)

    def irfft(self, fu):
        return sfft.irfftn(fu, s=(self.N,) * 3, workers=_WORKERS)


class ConfigParams:
    """Parameters of one benchmark configuration."""

    PRESETS = {
        # name: N, nu, dt, n_droplets, interpolation
        "config1": dict(N=64, nu=0.01, dt=2e-3, n_droplets=10_000, interp="trilinear"),
        "config2": dict(N=256, nu=2.5e-3, dt=1e-3, n_droplets=1_000_000, interp="tricubic"),
        "config3": dict(N=512, nu=1e-3, dt=5e-4, n_droplets=4_000_000, interp="tricubic"),
    }

    def __init__(self, N, nu, dt, eps=0.1, kf=2, E0=0.5, g=0.1, n_droplets=0, interp="trilinear"):
        self.N, self.nu, self.dt, self.eps, self.kf = N, nu, dt, eps, kf
        self.shell_no = np.arange(1, kf + 1)
        self.f0 = eps * TWO_PI ** 3 / len(self.shell_no)
        self.einit = E0 * TWO_PI ** 3
        self.g = g
        self.n_droplets = n_droplets
        self.interp = interp
        self.tau_eta = (nu / eps) ** 0.5

    @classmethod
    def preset(cls, name, **over):
        kw = dict(cls.PRESETS[name])
        kw.update(over)
        return cls(**kw)


def config_profile(kint):
    """Shell energy E(k) ~ k^4 exp(-2 (k/4)^2)."""
    return kint.astype(np.float64) ** 4 * np.exp(-2.0 * (kint / 4.0) ** 2)


def init_flow(grid, prm, seed):
    """Random-phase solenoidal field (the reference's construction, F:691-736, with the
    configuration's spectrum and energy), phases from ``np.random.default_rng(seed)``.
    Returns (uk, u) where uk is the dealiased spectrum the loop starts from (F:567-569)."""
    rng = np.random.default_rng(seed)
    th = [rng.uniform(0, TWO_PI, grid.k.shape) for _ in range(3)]
    _, u = R.init_field(grid, th, prm.einit, profile=config_profile)
    return R.start_spectrum(grid, u), u


def init_droplets(prm, seed, kind, nd=None):
    """Seeded droplet positions and Stokes times.

    kind "uniform_tau": tau log-uniform in [0.05, 2]           (configuration 1)
    kind "lognormal_r": r lognormal(median 0.002*2pi, sigma 0.3), tau = tau_med (r/r_med)^2
                        with tau_med = 0.5 tau_eta, tau_eta = sqrt(nu/eps)  (configuration 2)
    Returns (pos (nd,3) f64, tau (nd,) f64, radius (nd,) f64).
    """
    nd = prm.n_droplets if nd is None else nd
    rng = np.random.default_rng(seed + 7919)
    pos = rng.uniform(0, TWO_PI, (nd, 3))
    if kind == "uniform_tau":
        tau = np.exp(rng.uniform(np.log(0.05), np.log(2.0), nd))
        radius = np.full(nd, 0.002 * TWO_PI) * np.sqrt(tau / np.median(tau))
    elif kind == "lognormal_r":
        r_med = 0.002 * TWO_PI
        radius = r_med * np.exp(0.3 * rng.standard_normal(nd))
        tau = 0.5 * prm.tau_eta * (radius / r_med) ** 2
    else:
        raise ValueError(kind)
    return pos, tau, radius


# ---- flow ------------------------------------------------------------------------------------
def nonlinear(grid, prm, uk):
    """N(u) = P[(u x omega)^ + f] * dealias (the reference's RHS with nu = 0).  Returns (N, u)."""
    fk, _ = R.forcing(grid, uk, prm.f0, prm.shell_no)
    ku, u, _ = R.velocity_rhs(grid, uk, 0.0, fk, visc=0.0)
    return ku, u


def if_factor(grid, nu, h):
    """Integrating factor exp(-nu k^2 h)."""
    return np.exp(nu * grid.lap * h)


def rk2if_step(grid, prm, uk, h=None):
    """One Heun step with integrating factor.  Returns (uk_new, u_n, u_star): the physical
    velocity at the two stages, which is what the droplet stages sample."""
    h = prm.dt if h is None else h
    E = if_factor(grid, prm.nu, h)
    N1, u_n = nonlinear(grid, prm, uk)
    ustar_k = E * (uk + h * N1)
    acc = E * (uk + 0.5 * h * N1)
    N2, u_star = nonlinear(grid, prm, ustar_k)
    return acc + 0.5 * h * N2, u_n, u_star


# ---- droplet gathers -------------------------------------------------------------------------
def _axis_cells(p, N, L, taps):
    """Base cell, fractional offset and periodic stencil indices along one axis."""
    s = np.mod(p, L) * (N / L)
    i0 = np.floor(s).astype(np.int64)
    t = s - i0
    i0 = np.mod(i0, N)
    if taps == 2:
        offs = np.arange(0, 2)
    else:
        offs = np.arange(-1, 3)
    return np.mod(i0[:, None] + offs[None, :], N), t


def weights_trilinear(t):
    return np.stack([1.0 - t, t], axis=1)


def weights_tricubic(t):
    """4-point Lagrange weights on offsets -1, 0, 1, 2."""
    return np.stack([-t * (t - 1) * (t - 2) / 6.0,
                     (t + 1) * (t - 1) * (t - 2) / 2.0,
                     -(t + 1) * t * (t - 2) / 2.0,
                     (t + 1) * t * (t - 1) / 6.0], axis=1)


def _numba_gather():
    """numba-parallel version of ``gather`` (the reference's own gather is numba, P:6-20), used
    for large droplet counts so the CPU baseline uses every host core."""
    global _NB
    if _NB is not None:
        return _NB
    import numba as nb

    @nb.njit(parallel=True, cache=False)
    def run(field, pos, method, L, out):
        C, N = field.shape[0], field.shape[-1]
        dx = L / N
        for i in nb.prange(pos.shape[0]):
            w = np.zeros((3, 4))
            j = np.zeros((3, 4), dtype=np.int64)
            T = 2 if method == 0 else 4
            for a in range(3):
                p = pos[i, a] - L * np.floor(pos[i, a] / L)
                if method == 2:
                    i0 = np.int64(np.floor(p / dx)) % N
                    for q in range(4):
                        jj = (i0 - 1 + q) % N
                        j[a, q] = jj
                        w[a, q] = (1 + np.cos((p - jj * dx) * (np.pi / (2 * dx)))) / 4.0
                else:
                    s_ = p * (N / L)
                    fl = np.floor(s_)
                    t = s_ - fl
                    i0 = np.int64(fl) % N
                    if method == 0:
                        j[a, 0] = i0
                        j[a, 1] = (i0 + 1) % N
                        w[a, 0] = 1.0 - t
                        w[a, 1] = t
                    else:
                        for q in range(4):
                            j[a, q] = (i0 - 1 + q) % N
                        w[a, 0] = -t * (t - 1) * (t - 2) / 6.0
                        w[a, 1] = (t + 1) * (t - 1) * (t - 2) / 2.0
                        w[a, 2] = -(t + 1) * t * (t - 2) / 2.0
                        w[a, 3] = (t + 1) * t * (t - 1) / 6.0
            for c in range(C):
                acc = 0.0
                for qa in range(T):
                    for qb in range(T):
                        wab = w[0, qa] * w[1, qb]
                        for qc in range(T):
                            acc += field[c, j[0, qa], j[1, qb], j[2, qc]] * wab * w[2, qc]
                out[i, c] = acc
        return out

    _NB = run
    return run


_NB = None
_METHOD_ID = {"trilinear": 0, "tricubic": 1, "cosine": 2}


def gather(field, pos, method, L=TWO_PI):
    """Interpolate every component of ``field`` (C, N, N, N) at ``pos`` (n, 3)."""
    if pos.shape[0] >= 50_000:
        out = np.zeros((pos.shape[0], field.shape[0]))
        return _numba_gather()(np.ascontiguousarray(field, dtype=np.float64), np.ascontiguousarray(pos),
                               _METHOD_ID[method], float(L), out)
    N = field.shape[-1]
    if method == "cosine":
        X = np.linspace(0, L, N, endpoint=False)
        dx = X[1] - X[0]
        p = np.mod(pos, L)
        jw = [R.cosine_weights(p[:, a], X, dx, N) for a in range(3)]
    else:
        taps = 2 if method == "trilinear" else 4
        wf = weights_trilinear if taps == 2 else weights_tricubic
        jw = []
        for a in range(3):
            j, t = _axis_cells(pos[:, a], N, L, taps)
            jw.append((j, wf(t)))
    (jx, wx), (jy, wy), (jz, wz) = jw
    T = jx.shape[1]
    out = np.zeros((pos.shape[0], field.shape[0]))
    for a in range(T):
        for b in range(T):
            wab = wx[:, a] * wy[:, b]
            for c in range(T):
                out += field[:, jx[:, a], jy[:, b], jz[:, c]].T * (wab * wz[:, c])[:, None]
    return out


def stencil_4x4x4(field, pos, L=TWO_PI):
    """The 4x4x4 stencil of every component around each point (n, C, 4, 4, 4) and the
    fractional cell offsets (n, 3): the learned-interpolation input."""
    N = field.shape[-1]
    js, ts = [], []
    for a in range(3):
        j, t = _axis_cells(pos[:, a], N, L, 4)
        js.append(j)
        ts.append(t)
    jx, jy, jz = js
    st = field[:, jx[:, :, None, None], jy[:, None, :, None], jz[:, None, None, :]]
    return np.moveaxis(st, 0, 1), np.stack(ts, axis=1)


# ---- droplet dynamics ------------------------------------------------------------------------
def droplet_rhs(vel, u_p, tau, g):
    """(x', v') = (v, (u - v)/tau - g z)."""
    acc = (u_p - vel) / tau[:, None]
    acc[:, 2] -= g
    return vel, acc


def droplet_heun(pos, vel, tau, u_n, u_star, prm, method, h=None):
    """Heun step of the droplets on the two flow stages.  Returns (pos, vel, up_n) with up_n the
    fluid velocity sampled at the start positions."""
    h = prm.dt if h is None else h
    up1 = gather(u_n, pos, method)
    k1x, k1v = droplet_rhs(vel, up1, tau, prm.g)
    pos_s, vel_s = pos + h * k1x, vel + h * k1v
    up2 = gather(u_star, pos_s, method)
    k2x, k2v = droplet_rhs(vel_s, up2, tau, prm.g)
    return pos + 0.5 * h * (k1x + k2x), vel + 0.5 * h * (k1v + k2v), up1


def step(grid, prm, uk, pos, vel, tau, method):
    """One coupled step (one-way): flow RK2+IF and droplets Heun."""
    uk_new, u_n, u_star = rk2if_step(grid, prm, uk)
    if pos is not None and pos.shape[0] > 0:
        pos, vel, _ = droplet_heun(pos, vel, tau, u_n, u_star, prm, method)
    return uk_new, pos, vel
