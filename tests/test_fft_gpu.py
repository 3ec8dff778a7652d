"""GPU transforms (ld_rfft_mpi / ld_irfft_mpi / cube transforms) against the reference's own
rfft_mpi / irfft_mpi outputs (golden) and the FP64 scipy oracle."""
import numpy as np
import pytest
import scipy.fft as sfft

pytestmark = pytest.mark.gpu

# relative L2 tolerances per plan precision
TOL = {"f32": 2e-6, "f64": 1e-13}


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def plan(N, prec):
    from lucky_droplets_b200.spectral import Plan
    return Plan(N, prec)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_rfft_irfft_golden_N16(torch, golden, prec):
    g = golden("N16")
    p = plan(16, prec)
    u = torch.as_tensor(g["fft_in"]).to("cuda", p.rdtype).contiguous()
    fu = p.rfft_mpi(u).cpu().numpy()
    assert rel(fu, g["fft_out"]) < TOL[prec]
    X = torch.as_tensor(g["ifft_in"]).to("cuda", p.cdtype).contiguous()
    x = p.irfft_mpi(X).cpu().numpy()
    assert rel(x, g["ifft_out"]) < TOL[prec]


# powers of two, and the mixed-radix sizes (radix-3 and radix-5 stages; the reference takes any N,
# scipy.fft being mixed-radix)
@pytest.mark.parametrize("N", [16, 32, 64, 128, 256, 96, 192, 360, 384])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_rfft_matches_scipy(torch, N, prec):
    rng = np.random.default_rng(N)
    a = rng.standard_normal((2, N, N, N))
    p = plan(N, prec)
    fu = p.rfft_mpi(torch.as_tensor(a).to("cuda", p.rdtype).contiguous()).cpu().numpy()
    ref = sfft.rfftn(a, axes=(1, 2, 3))
    assert rel(fu, ref) < TOL[prec] * (2 if N >= 128 else 1)
    # inverse of a (non-Hermitian) random spectrum: pocketfft c2r semantics
    X = rng.standard_normal((2, N, N, N // 2 + 1)) + 1j * rng.standard_normal((2, N, N, N // 2 + 1))
    x = p.irfft_mpi(torch.as_tensor(X).to("cuda", p.cdtype).contiguous()).cpu().numpy()
    assert rel(x, sfft.irfftn(X, s=(N, N, N), axes=(1, 2, 3))) < TOL[prec] * (2 if N >= 128 else 1)


@pytest.mark.parametrize("N", [16, 64, 256, 96, 360])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_cube_transforms(torch, N, prec):
    """Dealiased (cube-layout) transforms equal the full ones applied to dealiased spectra."""
    from oracle.reference_np import Grid
    grid = Grid(N)
    rng = np.random.default_rng(3 + N)
    u = rng.standard_normal((3, N, N, N))
    p = plan(N, prec)
    ut = torch.as_tensor(u).to("cuda", p.rdtype).contiguous()
    cube = p.rfft_cube(ut)
    full = p.from_cube(cube).cpu().numpy()
    ref = sfft.rfftn(u, axes=(1, 2, 3)) * grid.dealias
    assert rel(full, ref) < TOL[prec] * 2
    # to_cube agrees with rfft_cube
    cube2 = p.to_cube(torch.as_tensor(sfft.rfftn(u, axes=(1, 2, 3))).to("cuda", p.cdtype).contiguous())
    assert rel(cube2.cpu().numpy(), cube.cpu().numpy()) < TOL[prec] * 2
    # inverse of the dealiased spectrum
    back = p.irfft_cube(cube).cpu().numpy()
    assert rel(back, sfft.irfftn(ref, s=(N, N, N), axes=(1, 2, 3))) < TOL[prec] * 2


@pytest.mark.parametrize("N", [64, 256])
def test_autotuned_variants_give_identical_rhs(N):
    """Every launch variant of the y passes computes the same RHS bit for bit; the autotuner
    reports a time for each available variant and keeps one of them."""
    import torch
    from lucky_droplets_b200.spectral import Plan
    from oracle import config_np as C
    prm = C.ConfigParams(N=N, nu=2.5e-3, dt=1e-3)
    uk0, _ = C.init_flow(C.ConfigGrid(N), prm, seed=1)
    p = Plan(N, "f32")
    uk = p.to_cube(torch.as_tensor(uk0).to("cuda", p.cdtype).contiguous())
    res = p.autotune()
    assert all(c in (0, 1, 2, 3) for c in res["choice"])
    outs = []
    for choice in ([0, 0], [1, 1], [3, 3], res["choice"]):
        p.set_tuning(choice)
        outs.append(p.velocity_rhs(uk, prm.nu, prm.f0, prm.shell_no).clone())
    for o in outs[1:]:
        assert torch.equal(o, outs[0])


def test_unsupported_sizes_are_refused():
    """Sizes without kernel instances, and the learned interpolation on a mixed-radix grid, fail
    with LD_ERR_UNSUPPORTED and a message."""
    from lucky_droplets_b200._lib import LDError
    from lucky_droplets_b200.spectral import Plan
    import torch
    from lucky_droplets_b200.mlp import LearnedInterp
    for N in (100, 48, 1024):
        with pytest.raises(LDError, match="grids are"):
            Plan(N, "f32")
    p = Plan(96, "f32")
    li = LearnedInterp(p)
    u4 = torch.zeros((96, 96, 96, 4), dtype=torch.float32, device="cuda")
    pos = torch.zeros((10, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(LDError, match="power of two"):
        li.infer(u4, pos)


@pytest.mark.parametrize("N", [32, 96])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_region_copies_match_layout_conversions(torch, N, prec):
    """ld_spec_copy_region moves only the dealiased cube rows between a reference-layout spectrum
    (pinned host or device) and the cube: in, it equals ld_spec_to_cube; out, it writes exactly
    the cube rows of from_cube and leaves every other element as it was."""
    p = plan(N, prec)
    rng = np.random.default_rng(N)
    shape = (3, N, N, N // 2 + 1)
    X = torch.as_tensor(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).to(p.cdtype)
    ref = p.to_cube(X.cuda())
    for src in (X.pin_memory(), X.cuda()):
        got = p.empty_cube(3)
        got.fill_(1.0)
        p.copy_region_in(src, got)
        torch.cuda.synchronize()
        assert torch.equal(got, ref)
    full = p.from_cube(ref).cpu()
    inside = torch.zeros(shape, dtype=torch.bool)
    kc = p.kc
    rows = list(range(0, kc + 1)) + list(range(N - kc, N))
    inside[:, rows[0]:kc + 1, :, :kc + 1] = True
    inside[:, N - kc:, :, :kc + 1] = True
    cols = torch.zeros(N, dtype=torch.bool)
    cols[rows] = True
    inside &= cols[None, None, :, None]
    for dst in (torch.full(shape, 7 + 7j, dtype=p.cdtype).pin_memory(), torch.full(shape, 7 + 7j, dtype=p.cdtype).cuda()):
        p.copy_region_out(ref, dst)
        torch.cuda.synchronize()
        d = dst.cpu()
        assert torch.equal(d[inside], full[inside])
        assert bool((d[~inside] == 7 + 7j).all())
