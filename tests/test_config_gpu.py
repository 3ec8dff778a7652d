"""Whole configurations over the horizons the correctness statement names.

Configuration 1 end to end: 64^3, nu = 0.01, dt = 2e-3, RK2 + integrating factor, eps = 0.1 on
shells 1..2, 1e4 droplets (log-uniform Stokes times, settling 0.1 along -z, trilinear), 200
steps from seeded inputs - the GPU step in FP64 and in FP32 against the FP64 oracle
(oracle/config_np: the reference's RHS, forcing and epilogue, F:239-316, F:596-620, restated for
the configuration), with the errors stated below:

    quantity (after 200 steps)                         FP64 GPU    FP32 GPU
    velocity spectrum, relative L2                     1e-11       1e-4
    shell spectrum, max relative error (E_s > 1e-12 E) 1e-10       2e-4
    droplet positions by id, max |dx| (mod 2 pi)       1e-11       1e-5
    droplet velocities by id, relative L2              1e-10       1e-4
    collision pairs of the last step                   bit-exact against the FP64 rule on the
                                                       GPU's own positions (radii x5 so that
                                                       pairs exist)

The FP32-against-FP64 statement on the GPU (both runs on the device, same seed, 128^3, 1e5
tricubic droplets, 100 steps): velocity relative L2, shell spectrum and position drift, with the
tolerances in test_fp32_against_fp64_128.
"""
import numpy as np
import pytest

from oracle import config_np as C
from oracle import collide_np as K

pytestmark = pytest.mark.gpu

STEPS = 200
TOL = {"f64": dict(u=1e-11, ek=1e-10, x=1e-11, v=1e-10), "f32": dict(u=1e-4, ek=2e-4, x=1e-5, v=1e-4)}


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


def wrap_diff(a, b):
    return np.abs((a - b + np.pi) % (2 * np.pi) - np.pi)


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def config1():
    """The configuration's inputs and the FP64 oracle run over STEPS steps (shared by both
    precisions)."""
    prm = C.ConfigParams.preset("config1", g=0.1)
    grid = C.ConfigGrid(prm.N)
    uk0, u0 = C.init_flow(grid, prm, seed=101)
    pos, tau, rad = C.init_droplets(prm, 101, "uniform_tau")
    rad = rad * 5.0
    vel = C.gather(u0, pos, "trilinear")
    uk, p_, v_ = uk0.copy(), pos.copy(), vel.copy()
    for _ in range(STEPS):
        uk, p_, v_ = C.step(grid, prm, uk, p_, v_, tau, "trilinear")
        uk = grid.project(np.stack([grid.rfft(grid.irfft(uk[c])) for c in range(3)]))
    return dict(prm=prm, grid=grid, uk0=uk0, pos=pos, tau=tau, rad=rad, vel=vel, uk=uk * grid.dealias,
                p=p_, v=v_)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_config1_end_to_end(torch, config1, prec):
    from lucky_droplets_b200.collide import Collider
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    c = config1
    prm, grid = c["prm"], c["grid"]
    dns = ForcedDNS.config(prm.N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision=prec)
    dns.set_uk_full(c["uk0"])
    d = Droplets(dns.plan, c["pos"], c["vel"], c["tau"], method="trilinear", g=prm.g, radius=c["rad"])
    col = Collider(d.n, 2 * c["rad"].max())
    dns.attach(d, collider=col, sort_every=20)
    dns.step(STEPS)
    assert dns.check() == 0
    tol = TOL[prec]
    e_u = rel(dns.uk_full(), c["uk"])
    ek_ref = grid.shell_sum(grid.energy3d(c["uk"]))
    ek = dns.energy_spectrum()
    live = ek_ref > 1e-12 * ek_ref.sum()
    e_ek = np.max(np.abs(ek[live] - ek_ref[live]) / ek_ref[live])
    e_x = wrap_diff(d.by_id(d.pos), c["p"]).max()
    e_v = rel(d.by_id(d.vel).astype(np.float64), c["v"])
    print(f"config 1 {prec}: u {e_u:.2e}  ek {e_ek:.2e}  x {e_x:.2e}  v {e_v:.2e}")
    assert e_u < tol["u"] and e_ek < tol["ek"] and e_x < tol["x"] and e_v < tol["v"]
    # the last step's pairs, bit-exact against the FP64 rule on the GPU's positions
    m = int(col.count.item())
    ids = d.ids.cpu().numpy()
    got = ids[dns.pairs[:m].cpu().numpy().astype(np.int64)]
    got = np.stack([got.min(axis=1), got.max(axis=1)], axis=1)
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    ref = K.collide(d.by_id(d.pos), c["rad"], 2 * c["rad"].max())
    assert m > 0 and np.array_equal(got, ref)


def test_fp32_against_fp64_128(torch):
    """The precision statement at 128^3 over 100 steps: FP32 fields and transforms (FP64 positions
    and energy reductions) against an FP64 run of the same seed on the GPU."""
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200.init import init_flow, init_droplets
    N, nu, dt, nd = 128, 5e-3, 1e-3, 100_000
    runs = {}
    for prec in ("f64", "f32"):
        dns = ForcedDNS.config(N, nu, dt, precision=prec)
        init_flow(dns, 31)
        pos, tau, rad = init_droplets(nd, 31, "lognormal_r", nu=nu)
        d = Droplets(dns.plan, pos, np.zeros((nd, 3)), tau, method="tricubic", g=0.1, radius=rad)
        d.vel.copy_(d.gather(dns.velocity()))
        dns.attach(d, sort_every=20)
        dns.step(100)
        assert dns.check() == 0
        runs[prec] = (dns, d)
    (a, da), (b, db) = runs["f64"], runs["f32"]
    e_u = rel(b.uk_full(), a.uk_full())
    ek_a, ek_b = a.energy_spectrum(), b.energy_spectrum()
    live = ek_a > 1e-10 * ek_a.sum()
    e_ek = np.max(np.abs(ek_b[live] - ek_a[live]) / ek_a[live])
    e_x = wrap_diff(db.by_id(db.pos), da.by_id(da.pos)).max()
    print(f"128^3 FP32 vs FP64, 100 steps: u {e_u:.2e}  ek {e_ek:.2e}  x {e_x:.2e}")
    assert e_u < 2e-5 and e_ek < 1e-4 and e_x < 1e-5
