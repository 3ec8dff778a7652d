"""The reference's own droplet physics on the GPU against the reference's run (golden vectors
from forced-dns-sm.py / particles.py): full_RHS with the n field and the droplets (kn, kp, the
deposited sink fc), and two RK4 steps of flow, n field and droplets together."""
import numpy as np
import pytest

from oracle import reference_np as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _run(golden, name):
    from lucky_droplets_b200.dns import ForcedDNS
    from lucky_droplets_b200.refmode import ReferenceDroplets, ReferenceRun
    g = golden(name)
    N = int(g["N"])
    prm = R.ReferenceParams(N)
    dns = ForcedDNS.reference(N, precision="f64")
    dns.set_uk_full(g["uk0"])
    d = ReferenceDroplets(dns.plan, g["init_coord"], prm.sts, prm.g, prm.nu, prm.tf, prm.rhop, prm.M0)
    assert d.factor == float(g["prt_factor"])
    run = ReferenceRun(dns, np.ones((N, N, N)), d, prm.tps, prm.g)
    return g, N, prm, dns, d, run


@pytest.mark.parametrize("name", ["N16", "N32"])
def test_full_rhs_matches_reference(torch, golden, name):
    g, N, prm, dns, d, run = _run(golden, name)
    coord = torch.as_tensor(g["rhs_coord_in"]).cuda().contiguous()
    ku, kn, kp, fc = run.full_rhs(coord=coord)
    assert np.abs(fc.cpu().numpy() - g["rhs_fc"]).max() < 1e-12 * max(1.0, np.abs(g["rhs_fc"]).max())
    assert np.abs(kn.cpu().numpy() - g["rhs_kn"]).max() < 1e-12
    ids = g["rhs_prtclid"].ravel().astype(int)  # the reference reorders droplets in send()
    assert np.abs(kp.cpu().numpy()[ids] - g["rhs_kp"]).max() < 1e-11


@pytest.mark.parametrize("name", ["N16", "N32"])
def test_rk4_with_n_field_and_droplets_matches_reference(torch, golden, name):
    g, N, prm, dns, d, run = _run(golden, name)
    run.step(int(g["nsteps"]))
    full = dns.uk_full()
    grid = R.Grid(N)
    ref = g["run_uk"] * grid.dealias
    assert np.linalg.norm(full - ref) / np.linalg.norm(ref) < 1e-13
    assert np.abs(run.n.cpu().numpy() - g["run_n"]).max() < 1e-12
    ids = g["run_prtclid"].ravel().astype(int)
    c = d.coord.cpu().numpy()[ids]
    dpos = (c[:, :3] - g["run_coord"][:, :3] + np.pi) % (2 * np.pi) - np.pi
    assert np.abs(dpos).max() < 1e-12
    assert np.abs(c[:, 3:] - g["run_coord"][:, 3:]).max() < 1e-11


def test_clip_zero_matches_oracle(torch):
    """clip_zero of F:278-285, including its in-place side effect."""
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, ptr, stream_ptr
    rng = np.random.default_rng(0)
    x = rng.standard_normal(20000) + 0.3
    ref_in = x.copy()
    ref = R.clip_zero(ref_in)
    xg = torch.as_tensor(x).cuda()
    out = torch.empty_like(xg)
    work = torch.empty(int(_lib.lib().ld_ref_workspace_doubles()), dtype=torch.float64, device="cuda")
    check(_lib.lib().ld_clip_zero(ptr(xg), ptr(out), 20000, 1, ptr(work), stream_ptr()))
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-14
    assert np.array_equal(xg.cpu().numpy(), ref_in)
