"""Restatement, in FP64 NumPy on one rank, of the reference algorithm of lucky-droplets.

TEST INFRASTRUCTURE ONLY (the oracle): imported by tests, smoke() and bench.py's CPU legs, never
by the product package.

Every function names the reference lines it follows (F = forced-dns-sm.py, P = particles.py).
With one MPI rank the reference's slab machinery collapses:
  * rfft_mpi / irfft_mpi (F:201-213) are rfft2 over (y, z) then fft over x, and the inverse;
  * the halo exchanges of interp_cosine / exterp_cosine_scalar (P:435-577) become periodic
    indexing;
  * ``send`` (P:233-275) only moves droplets whose x left [0, L) to the end of the arrays and
    wraps the stage position; this restatement keeps droplets in ``prtclid`` order instead and
    wraps the stage position, so results are compared by ``prtclid`` and positions modulo L.
Pinned against tests/golden/ref_*.npz, which were produced by running the reference itself.
"""
import numpy as np
from scipy.fft import fft, ifft, rfft2, irfft2, fftfreq

TWO_PI = 2.0 * np.pi


class Grid:
    """Grid and spectral operators, F:49-141 with one rank (Np = N)."""

    def __init__(self, N, L=TWO_PI, lp=1):
        self.N, self.L, self.lp = N, L, lp
        self.Nf = N // 2 + 1
        self.X = np.linspace(0, L, N, endpoint=False)                      # F:55
        self.dx = self.X[1] - self.X[0]
        Kx = fftfreq(N, 1.0 / N) * TWO_PI / L                              # F:59
        Kz = np.abs(Kx[: self.Nf])                                         # F:60
        self.kx, self.ky, self.kz = np.meshgrid(Kx, Kx, Kz, indexing="ij")  # F:62
        self.lap = -(self.kx ** 2 + self.ky ** 2 + self.kz ** 2)            # F:125
        self.k = (-self.lap) ** 0.5                                         # F:126
        self.kint = np.clip(np.round(self.k, 0).astype(int), None, N // 2)  # F:127
        self.dealias = self.kint <= N / 3                                   # F:129 spherical
        self.invlap = self.dealias / np.where(self.lap == 0, np.inf, self.lap)  # F:131
        self.normalize = np.where((self.kz == 0) + (self.kz == N // 2),
                                  1 / (N ** 6 / TWO_PI ** 3), 2 / (N ** 6 / TWO_PI ** 3))  # F:136
        self.shells = np.arange(-0.5, self.Nf, 1.0)                         # F:137
        self.shells[0] = 0.0                                                # F:138

    # ---- transforms, F:201-213 -------------------------------------------------------------
    def rfft(self, u):
        """rfft_mpi on one rank: rfft2 over (y, z), then fft over x."""
        return fft(rfft2(u, axes=(1, 2)), axis=0)

    def irfft(self, fu):
        """irfft_mpi on one rank: ifft over x, then irfft2 over (y, z) (scipy: 1/N^3 overall)."""
        return irfft2(ifft(fu, axis=0), (self.N, self.N), axes=(1, 2))

    def shell_sum(self, x):
        """e3d_to_e1d, F:232-233: histogram of |k| into shells [0,.5),[.5,1.5),...,[Nf-1.5,Nf-.5]."""
        return np.histogram(self.k.ravel(), bins=self.shells, weights=x.ravel())[0]

    def energy3d(self, uk):
        """Per-mode energy, F:243."""
        return 0.5 * (np.abs(uk[0]) ** 2 + np.abs(uk[1]) ** 2 + np.abs(uk[2]) ** 2) * self.normalize

    def project(self, uk):
        """Div-free projection of F:607-610: uk + k * invlap (k . uk)."""
        pk = self.invlap * (self.kx * uk[0] + self.ky * uk[1] + self.kz * uk[2])
        return np.stack([uk[0] + self.kx * pk, uk[1] + self.ky * pk, uk[2] + self.kz * pk])


class ReferenceParams:
    """Driver parameters of F:11-38, F:78-97 as functions of N (forcestart run, one rank)."""

    def __init__(self, N, nshells=1, nu0=0.8, m=1.5, lp=1, gravity=False, sts=0.001, stb0=0.05,
                 M0=4e-6, rhop=1000.0, einit=None):
        self.N = N
        self.dt = 0.256 / N                                  # F:29
        self.nu0, self.m, self.lp = nu0, m, lp
        self.nu = nu0 * (3 * m / N) ** (2 * (lp - 1 / 3))    # F:83
        self.einit = TWO_PI ** 3 if einit is None else einit  # F:86
        self.nshells = nshells                               # F:89
        self.shell_no = np.arange(1, 1 + nshells)            # F:90
        self.tf = (9 * (m / N) ** (2 / 3)) / nu0             # F:92
        self.sts, self.stb0 = sts, stb0                      # F:33-34
        self.tps = sts * self.tf                             # F:93
        self.g = 9.81 * 0.1 / self.tf if gravity else 0.0    # F:94
        self.f0 = nu0 ** 3 * TWO_PI ** 3 / nshells           # F:97
        self.M0, self.rhop = M0, rhop                        # F:37-38


# ---- flow RHS ------------------------------------------------------------------------------
def forcing(grid, uk, f0, shell_no):
    """Constant-power forcing, F:239-275.  Returns (fk, ek_arr)."""
    ek_arr = grid.shell_sum(grid.energy3d(uk))                          # F:243-245
    ek_arr = np.where(np.abs(ek_arr) < 1e-10, np.inf, ek_arr)           # F:250
    factor = np.zeros(grid.Nf)
    factor[shell_no] = f0 / (2 * ek_arr[shell_no])                       # F:253-254
    factor3d = factor[grid.kint]                                         # F:255
    fk = np.stack([factor3d * uk[c] * grid.dealias for c in range(3)])   # F:262-264
    pk = grid.invlap * (grid.kx * fk[0] + grid.ky * fk[1] + grid.kz * fk[2]) * grid.dealias  # F:268
    fk = np.stack([fk[0] + grid.kx * pk, fk[1] + grid.ky * pk, fk[2] + grid.kz * pk])       # F:270-272
    return fk * grid.dealias, ek_arr                                     # F:275 (isforcing=True)


def clip_zero(x):
    """F:278-285 (note: clips its argument in place, as the reference does)."""
    N3 = x.size
    oldmean = np.sum(x) / N3
    x[:] = np.clip(x, 0, None)
    newmean = np.sum(x) / N3
    return x * oldmean / newmean


def velocity_rhs(grid, uk, nu, fk, visc=1.0):
    """Velocity part of full_RHS, F:287-316.  Returns (ku, u, pk) with u the physical velocity."""
    kx, ky, kz = grid.kx, grid.ky, grid.kz
    u = np.stack([grid.irfft(uk[c]) for c in range(3)])                  # F:291-293
    omg = np.stack([grid.irfft(1j * (ky * uk[2] - kz * uk[1])),          # F:295-297
                    grid.irfft(1j * (kz * uk[0] - kx * uk[2])),
                    grid.irfft(1j * (kx * uk[1] - ky * uk[0]))])
    rhs = np.stack([omg[2] * u[1] - omg[1] * u[2],                       # F:299-301
                    omg[0] * u[2] - omg[2] * u[0],
                    omg[1] * u[0] - omg[0] * u[1]])
    rhsk = np.stack([(grid.rfft(rhs[c]) + fk[c]) * grid.dealias for c in range(3)])  # F:304-306
    pk = 1j * grid.invlap * (kx * rhsk[0] + ky * rhsk[1] + kz * rhsk[2])  # F:309
    lapp = nu * ((-grid.lap) ** grid.lp)
    ku = np.stack([rhsk[0] - 1j * kx * pk - lapp * uk[0] * visc,          # F:314-316
                   rhsk[1] - 1j * ky * pk - lapp * uk[1] * visc,
                   rhsk[2] - 1j * kz * pk - lapp * uk[2] * visc])
    return ku, u, pk


def slow_manifold_velocity(grid, uk, pk, nu, tps, g, visc=1.0):
    """Small-droplet velocity v = u - tps Du/Dt - tps g z, F:319-321."""
    kk = (grid.kx, grid.ky, grid.kz)
    lapp = nu * ((-grid.lap) ** grid.lp)
    v = np.stack([grid.irfft((uk[c] - tps * (-1j * kk[c] * pk - lapp * uk[c] * visc)) * grid.dealias)
                  for c in range(3)])
    v[2] = v[2] - tps * g
    return v


def n_rhs(grid, n, v, fc):
    """Number-density RHS, F:325-330 (physical-space result)."""
    fck = grid.rfft(fc) * grid.dealias
    vnk = [grid.rfft(n * v[c]) * grid.dealias for c in range(3)]
    return grid.irfft((-1j * (grid.kx * vnk[0] + grid.ky * vnk[1] + grid.kz * vnk[2]) - fck) * grid.dealias)


# ---- droplets (MPI_particles on one rank) ---------------------------------------------------
def cosine_weights(pos, X, dx, N):
    """Cell index and 4 cosine weights per axis, P:441, P:454-456, P:9-16.

    Stencil offsets -1..2 around idx = pos // dx; weight (1 + cos((pos - X_j) pi / (2 dx))) / 4
    with X_j taken at the periodic index, as the reference does (X[slx % N], Y[(yidx+i) % N]).
    """
    idx = (pos // dx).astype(np.int64)
    offs = np.arange(-1, 3)
    j = np.mod(idx[:, None] + offs[None, :], N)
    w = (1 + np.cos((pos[:, None] - X[j]) * (np.pi / (2 * dx)))) / 4.0
    return j, w


class Droplets:
    """State and RHS of MPI_particles (P:52-111, P:191-195, P:817-837) on one rank."""

    def __init__(self, N, L, Nprtcl, st_s, st, g, nu, tau_eta, rho_p, M0, d=3, coord=None):
        self.N, self.L, self.d, self.g, self.tau_eta = N, L, d, g, tau_eta
        self.X = np.linspace(0, L, N, endpoint=False)
        self.dx = self.X[1] - self.X[0]
        self.factor = (nu * tau_eta / (2 * rho_p)) ** 3 / 2 * (36 * np.pi * rho_p) / M0  # P:74 (as written)
        self.growthfactor = 9 * np.pi * nu / (2 * rho_p)                  # P:75
        self.st_s = st_s                                                  # P:95
        if coord is None:
            coord = np.random.uniform(0, L, (Nprtcl, 2 * d + 1))          # P:91
            coord[:, -1] = st ** 1.5 * self.factor                        # P:94
        self.coord = np.array(coord, dtype=np.float64)
        self.prtclid = np.arange(self.coord.shape[0]).reshape((-1, 1))    # P:92-93
        self.update_intrinsic()

    def update_intrinsic(self):
        """P:191-195."""
        self.st = (self.coord[:, -1] / self.factor) ** (2 / 3.0)

    def interp_cosine(self, coord, fields):
        """4x4x4 cosine-kernel gather of every component of ``fields`` (C, N, N, N), P:435-511."""
        pos = np.mod(coord[:, : self.d], self.L)
        jx, wx = cosine_weights(pos[:, 0], self.X, self.dx, self.N)
        jy, wy = cosine_weights(pos[:, 1], self.X, self.dx, self.N)
        jz, wz = cosine_weights(pos[:, 2], self.X, self.dx, self.N)
        out = np.zeros((pos.shape[0], fields.shape[0]))
        for a in range(4):
            for b in range(4):
                for c in range(4):
                    w = wx[:, a] * wy[:, b] * wz[:, c]
                    out += fields[:, jx[:, a], jy[:, b], jz[:, c]].T * w[:, None]
        return out

    def exterp_cosine_scalar(self, coord, mdot):
        """Deposit mdot with the same kernel, divided by the cell volume, P:514-577."""
        pos = np.mod(coord[:, : self.d], self.L)
        jx, wx = cosine_weights(pos[:, 0], self.X, self.dx, self.N)
        jy, wy = cosine_weights(pos[:, 1], self.X, self.dx, self.N)
        jz, wz = cosine_weights(pos[:, 2], self.X, self.dx, self.N)
        c = np.zeros((self.N, self.N, self.N))
        for a in range(4):
            for b in range(4):
                for cc in range(4):
                    w = mdot * wx[:, a] * wy[:, b] * wz[:, cc] / (self.dx ** 3)
                    np.add.at(c, (jx[:, a], jy[:, b], jz[:, cc]), w)
        return c

    def pRHS(self, coord, u, us, c):
        """Droplet RHS and deposited mass sink, P:817-837.  Returns (rhs, fc, interpmat).

        The drag is (u - v) / (St tau_eta) only: the deceleration term of P:833 starts a new
        statement and is discarded by the reference.
        """
        d = self.d
        st = (coord[:, -1] / self.factor) ** (2 / 3.0)                       # P:823
        interp = self.interp_cosine(coord, np.concatenate((u, us, c[None]), axis=0))  # P:826
        rel = np.linalg.norm(coord[:, d: 2 * d] - interp[:, d: 2 * d], axis=1)
        mdot = self.growthfactor * (1 + (self.st_s / st) ** 0.5) ** 2 * interp[:, -1] * rel  # P:828
        fc = self.exterp_cosine_scalar(coord, mdot)                           # P:829
        rhs = np.zeros_like(coord)
        rhs[:, :d] = coord[:, d: 2 * d]                                       # P:831
        rhs[:, d: 2 * d] = (interp[:, :d] - coord[:, d: 2 * d]) / (st[:, None] * self.tau_eta)  # P:832
        rhs[:, 2 * d - 1] -= self.g                                           # P:834
        rhs[:, -1] = mdot                                                     # P:835
        return rhs, fc, interp


# ---- full RHS and the RK4 time loop ----------------------------------------------------------
def full_rhs(grid, prm, uk, n, coord, drops, visc=1.0, forc=1.0):
    """full_RHS, F:287-332.  Returns (ku, kn, kp)."""
    fk, _ = forcing(grid, uk, prm.f0, prm.shell_no)
    fk = fk * forc                                                          # F:289
    ku, u, pk = velocity_rhs(grid, uk, prm.nu, fk, visc)
    v = slow_manifold_velocity(grid, uk, pk, prm.nu, prm.tps, prm.g, visc)  # F:319-321
    if drops is not None and coord.shape[0] > 0:
        kp, fc, _ = drops.pRHS(coord, u, v, n)                              # F:324
    else:
        kp, fc = np.zeros_like(coord), np.zeros_like(n)
    kn = n_rhs(grid, n, v, fc)                                              # F:325-330
    return ku, kn, kp


def rk4_step(grid, prm, uk, n, drops, h):
    """One pass of the time loop body, F:582-620 (RK4 of F:335-362, explicit viscosity).

    Returns (uk, n, coord); raises FloatingPointError on the blow-up test of F:618.
    """
    coord = drops.coord if drops is not None else np.zeros((0, 7))
    sump, uknew, nnew = coord.copy(), uk.copy(), n.copy()
    ku, kn, kp = full_rhs(grid, prm, uk, clip_zero(n), coord, drops)
    sump += h / 6.0 * kp; uknew += h / 6.0 * ku; nnew += h / 6.0 * kn
    ku, kn, kp = full_rhs(grid, prm, uk + ku * h / 2, clip_zero(n + kn * h / 2), coord + h / 2 * kp, drops)
    sump += h / 3.0 * kp; uknew += h / 3.0 * ku; nnew += h / 3.0 * kn
    ku, kn, kp = full_rhs(grid, prm, uk + ku * h / 2, clip_zero(n + kn * h / 2), coord + h / 2 * kp, drops)
    sump += h / 3.0 * kp; uknew += h / 3.0 * ku; nnew += h / 3.0 * kn
    ku, kn, kp = full_rhs(grid, prm, uk + ku * h, clip_zero(n + kn * h), coord + h * kp, drops)
    sump += h / 6.0 * kp; uknew += h / 6.0 * ku; nnew += h / 6.0 * kn
    if drops is not None:
        drops.coord = sump                                                   # F:582
        drops.update_intrinsic()                                             # F:583
    n_out = clip_zero(nnew)                                                  # F:584
    u = np.stack([grid.irfft(uknew[c]) for c in range(3)])                   # F:597-599
    uk = np.stack([grid.rfft(u[c]) for c in range(3)])                       # F:601-603
    uk = grid.project(uk)                                                    # F:607-610
    if uk.max() > 100 * grid.N ** 3:                                         # F:618
        raise FloatingPointError("threshold exceeded")
    return uk, n_out, sump


# ---- initial condition ------------------------------------------------------------------------
def draw_reference_randoms(grid, nprtcl, d=3, seed=None):
    """The reference's draws from the global RNG in order: droplets (P:91), then the three phase
    arrays (F:695-697).  ``seed`` mirrors an ``np.random.seed`` placed after the numpy import."""
    if seed is not None:
        np.random.seed(seed)
    coord = np.random.uniform(0, grid.L, (nprtcl, 2 * d + 1))
    th = [np.random.uniform(0, TWO_PI, grid.k.shape) for _ in range(3)]
    return coord, th


def init_field(grid, thetas, einit, kinit=31, profile=None):
    """Random-phase solenoidal field of F:691-736.  Returns (uk, u).

    ``profile(kint)`` is the shell-energy shape E(k); the reference uses k^2 exp(-k^2/2) (F:700).
    """
    kint = grid.kint
    prof = kint ** 2 * np.exp(-kint ** 2 / 2) if profile is None else profile(kint)
    eprofile = prof / grid.normalize                                          # F:700
    amp = (eprofile / np.where(kint == 0, np.inf, kint ** 2)) ** 0.5         # F:703
    mask = (kint ** 2 < kinit ** 2) * (kint > 0) * grid.dealias
    uk = np.stack([amp * np.exp(1j * th) * mask for th in thetas])           # F:705-707
    u = np.stack([grid.irfft(uk[c]) for c in range(3)])                      # F:709-711
    uk = np.stack([grid.rfft(u[c]) for c in range(3)])                       # F:713-715
    trm = grid.kx * uk[0] + grid.ky * uk[1] + grid.kz * uk[2]                # F:717-720
    uk = np.stack([uk[0] + grid.invlap * grid.kx * trm, uk[1] + grid.invlap * grid.ky * trm,
                   uk[2] + grid.invlap * grid.kz * trm])
    e0 = np.sum(grid.shell_sum(grid.energy3d(uk)))                           # F:722-725
    uk = uk * (einit / e0) ** 0.5                                            # F:726-728
    u = np.stack([grid.irfft(uk[c]) for c in range(3)])                      # F:731-733
    return uk, u


def start_spectrum(grid, u):
    """The spectral state the time loop starts from, F:567-569."""
    return np.stack([grid.rfft(u[c]) * grid.dealias for c in range(3)])
