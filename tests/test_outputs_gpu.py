"""Output step on the GPU: flux spectrum against the oracle restatement of F:424-428, Parseval and
divergence diagnostics, and a save/load round trip through the reference's files."""
import numpy as np
import pytest

from oracle import reference_np as R
from oracle import config_np as C

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _dns(prec, N=32):
    from lucky_droplets_b200.dns import ForcedDNS
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3)
    grid = C.ConfigGrid(N)
    uk0, _ = C.init_flow(grid, prm, seed=4)
    dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision=prec)
    dns.set_uk_full(uk0)
    return dns, uk0


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_flux_spectrum_matches_oracle(torch, prec):
    dns, uk0 = _dns(prec)
    grid = R.Grid(dns.N)
    uk = uk0 * grid.dealias
    ku, _, _ = R.velocity_rhs(grid, uk, 0.0, np.zeros_like(uk), 0.0)
    T = grid.shell_sum(np.real(np.conj(uk[0]) * ku[0] + np.conj(uk[1]) * ku[1] + np.conj(uk[2]) * ku[2])
                       * grid.dealias * grid.normalize)
    ref = np.cumsum(T[::-1])[::-1]
    got = dns.flux_spectrum()
    tol = 1e-10 if prec == "f64" else 2e-4
    assert np.abs(got - ref).max() < tol * np.abs(ref).max()


def test_diagnostics_and_round_trip(torch, tmp_path):
    from lucky_droplets_b200.dns import Droplets
    dns, _ = _dns("f64")
    prm = C.ConfigParams(N=dns.N, nu=0.01, dt=2e-3)
    pos, tau, rad = C.init_droplets(prm, 4, "uniform_tau", nd=500)
    d = Droplets(dns.plan, pos, np.zeros((500, 3)), tau, method="trilinear", radius=rad)
    dns.attach(d)
    dns.step(2)
    paths, diag = dns.save(tmp_path)
    assert abs(diag["energy"] - diag["energy_spectral"]) < 1e-10 * diag["energy"]  # Parseval
    assert diag["divergence_max"] < 1e-10
    from lucky_droplets_b200.dns import ForcedDNS
    other = ForcedDNS.config(dns.N, dns.nu, dns.dt, eps=0.1, kf=2, precision="f64")
    other.load(tmp_path)
    assert torch.equal(other.uk, dns.uk)
    s = np.load(tmp_path / "state_0.npz")
    assert np.array_equal(s["prtclid"], np.arange(500))
    assert np.array_equal(s["pos"], d.by_id(d.pos))
    u = dns.velocity().cpu().numpy()
    ref = C.gather(u, s["pos"], "trilinear")
    assert np.abs(s["umat"] - ref).max() < 1e-12


def test_restart_from_multi_rank_checkpoint(torch, tmp_path):
    """ForcedDNS.load and ReferenceRun.load take a 4-slab checkpoint (as a 4-rank reference run
    writes it, F:446-450) and restore uk and n exactly; a truncated slab raises CheckpointError."""
    from lucky_droplets_b200.dns import ForcedDNS
    from lucky_droplets_b200.outputs import CheckpointError, write_outputs
    from lucky_droplets_b200.refmode import ReferenceRun
    dns, _ = _dns("f64", N=16)
    dns.step(2)
    rng = np.random.default_rng(11)
    n = rng.random((16, 16, 16))
    write_outputs(tmp_path, dns.uk_full(), dns.energy_spectrum(), dns.flux_spectrum(), n=n, slabs=4)
    other = ForcedDNS.reference(16, precision="f64")
    run = ReferenceRun(other, np.ones((16, 16, 16)), None, tps=0.0, g=0.0)
    run.load(tmp_path)
    assert torch.equal(other.uk, dns.uk)
    assert np.array_equal(run.n.cpu().numpy(), n)
    raw = (tmp_path / "Fields_k_3.npz").read_bytes()
    (tmp_path / "Fields_k_3.npz").write_bytes(raw[:100])
    with pytest.raises(CheckpointError):
        other.load(tmp_path)
    big = ForcedDNS.config(32, 0.01, 2e-3, precision="f64")
    write_outputs(tmp_path, dns.uk_full(), dns.energy_spectrum(), dns.flux_spectrum(), slabs=2)
    for r in (2, 3):
        (tmp_path / f"Fields_k_{r}.npz").unlink()
    with pytest.raises(CheckpointError, match="N = 16"):
        big.load(tmp_path)
