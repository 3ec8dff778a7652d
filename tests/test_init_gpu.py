"""The product's flow initialisation (lucky_droplets_b200/init.py, F:691-736) against the oracle's
restatement and against the reference's own initial field (golden vectors from its run)."""
import numpy as np
import pytest

from oracle import config_np as C
from oracle import reference_np as R

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 2e-6}


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("N", [32, 64])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_init_flow_matches_oracle(torch, N, prec):
    """Same seed: the same phases, projection and energy scaling as oracle/config_np.init_flow, and
    the resulting start spectrum (dealiased, F:567-569) agrees to the precision's tolerance."""
    from lucky_droplets_b200.dns import ForcedDNS
    from lucky_droplets_b200.init import init_flow
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3)
    grid = C.ConfigGrid(N)
    uk0, u0 = C.init_flow(grid, prm, seed=21)
    dns = ForcedDNS.config(N, prm.nu, prm.dt, precision=prec)
    init_flow(dns, 21)
    assert rel(dns.uk_full(), uk0) < TOL[prec]
    assert rel(dns.velocity().cpu().numpy(), u0) < TOL[prec]
    ek = dns.energy_spectrum()
    assert abs(ek.sum() - prm.einit) < (1e-12 if prec == "f64" else 1e-6) * prm.einit
    assert float(dns.plan.divergence(dns.uk).abs().max()) < (1e-12 if prec == "f64" else 1e-5)


@pytest.mark.parametrize("name,seed", [("N16", 7), ("N32", 11)])
def test_init_flow_matches_reference_run(torch, golden, name, seed):
    """The reference's own initial state: phases drawn from the reference's global RNG order
    (droplets first, P:91, then the three phase arrays, F:695-697), the reference's profile
    E(k) ~ k^2 exp(-k^2/2) and energy (2 pi)^3 (F:86, F:700) - against uk0 and init_u of its run."""
    from lucky_droplets_b200.dns import ForcedDNS
    from lucky_droplets_b200.init import init_flow, reference_profile
    g = golden(name)
    N = int(g["N"])
    grid = R.Grid(N)
    _, th = R.draw_reference_randoms(grid, g["init_coord"].shape[0], seed=seed)
    dns = ForcedDNS.reference(N, precision="f64")
    init_flow(dns, None, E0=1.0, profile=reference_profile, phases=th)
    assert rel(dns.uk_full(), g["uk0"]) < 1e-12
    assert rel(dns.velocity().cpu().numpy(), g["init_u"]) < 1e-12
