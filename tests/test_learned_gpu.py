"""Droplet steps with the learned interpolation: the split path (MLP inference, then the droplet
update with the given fluid velocity) against the fused tricubic stage and against the FP64 oracle
with the same network."""
import numpy as np
import pytest

from oracle import config_np as C
from oracle import mlp_np as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def _setup(N, prec, seed, nd):
    from lucky_droplets_b200.dns import ForcedDNS
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    grid = C.ConfigGrid(N)
    uk0, u0 = C.init_flow(grid, prm, seed=seed)
    pos, tau, _ = C.init_droplets(prm, seed, "uniform_tau", nd=nd)
    vel = C.gather(u0, pos, "tricubic")
    dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision=prec)
    dns.set_uk_full(uk0)
    return prm, grid, uk0, pos, tau, vel, dns


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_zero_correction_equals_tricubic(torch, prec):
    """A network whose last layer is zero predicts tricubic: the split path reproduces the fused
    tricubic droplet stage.  The learned path evaluates its tricubic base in FP32 (the network's
    precision) on FP64 plans too, so both precisions agree to FP32 rounding."""
    from lucky_droplets_b200.dns import Droplets
    from lucky_droplets_b200 import mlp as G
    prm, grid, uk0, pos, tau, vel, dns_a = _setup(32, prec, 3, 3000)
    _, _, _, _, _, _, dns_b = _setup(32, prec, 3, 3000)
    a = Droplets(dns_a.plan, pos, vel, tau, method="tricubic", g=prm.g)
    b = Droplets(dns_b.plan, pos, vel, tau, method="tricubic", g=prm.g)
    p = M.init_params(1)
    p["W3"][:] = 0.0
    li = G.LearnedInterp(dns_b.plan, params=G.flat_from_mats(**p))
    b.use_learned(li)
    dns_a.attach(a)
    dns_b.attach(b)
    dns_a.step(3)
    dns_b.step(3)
    tol = 2e-6
    assert rel(b.vel.cpu().numpy(), a.vel.cpu().numpy()) < tol
    assert np.abs(b.pos.cpu().numpy() - a.pos.cpu().numpy()).max() < tol


def _oracle_learned(u, pos, p, fs, os):
    st, t = C.stencil_4x4x4(u, pos)
    X, scale, perm, refl = M.features(st.reshape(pos.shape[0], 192), t, fs)
    y, _ = M.forward(p, X)
    return C.gather(u, pos, "tricubic") + scale[:, None] * os * M.from_canonical(y, perm, refl)


def test_learned_step_matches_oracle(torch):
    """Two coupled steps (flow RK2+IF, droplet Heun with the learned velocity at x and at x + h v)
    against the oracle with the same network."""
    from lucky_droplets_b200.dns import Droplets
    from lucky_droplets_b200 import mlp as G
    prm, grid, uk0, pos, tau, vel, dns = _setup(32, "f32", 4, 2000)
    p = M.init_params(2)
    fs = np.random.default_rng(5).uniform(0.5, 3.0, 64).astype(np.float32)
    os = 0.05
    d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g)
    d.use_learned(G.LearnedInterp(dns.plan, params=G.flat_from_mats(**p, fs=fs, os=os)))
    dns.attach(d)
    uk, x, v = uk0.copy(), pos.copy(), vel.copy()
    h = prm.dt
    for _ in range(2):
        uk_new, u_n, u_s = C.rk2if_step(grid, prm, uk)
        up1 = _oracle_learned(u_n, x, p, fs, os)
        k1x, k1v = C.droplet_rhs(v, up1, tau, prm.g)
        xs, vs = x + h * k1x, v + h * k1v
        up2 = _oracle_learned(u_s, xs, p, fs, os)
        k2x, k2v = C.droplet_rhs(vs, up2, tau, prm.g)
        x, v = x + 0.5 * h * (k1x + k2x), v + 0.5 * h * (k1v + k2v)
        uk = grid.project(np.stack([grid.rfft(grid.irfft(uk_new[c])) for c in range(3)]))
    dns.step(2)
    assert rel(d.vel.cpu().numpy(), v) < 1e-4
    assert np.abs(d.pos.cpu().numpy() - x).max() < 1e-7


def test_predict_positions(torch):
    """xs = x + h v in FP64."""
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, ptr, stream_ptr
    plan = Plan(16, "f32")
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 7, (1001, 3))
    v = rng.standard_normal((1001, 3)).astype(np.float32)
    xs = torch.empty((1001, 3), dtype=torch.float64, device="cuda")
    xg, vg = torch.as_tensor(x).cuda(), torch.as_tensor(v).cuda()
    check(_lib.lib().ld_droplet_predict(plan.handle, ptr(xg), ptr(vg), 1001, 1e-3, ptr(xs), stream_ptr()))
    assert np.abs(xs.cpu().numpy() - (x + 1e-3 * v.astype(np.float64))).max() < 1e-15
