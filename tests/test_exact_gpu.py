"""Exact spectral (direct Fourier sum) velocity on the GPU against the CPU oracle and, at grid
points, against the inverse transform."""
import numpy as np
import pytest

from oracle import config_np as C
from oracle import exact_np as X

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("N,npts", [(32, 700), (256, 48)])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_exact_sum_matches_oracle(torch, N, npts, prec):
    from lucky_droplets_b200.spectral import Plan
    prm = C.ConfigParams(N=N, nu=0.01, dt=1e-3)
    grid = C.ConfigGrid(N)
    uk, _ = C.init_flow(grid, prm, seed=N + 1)
    p = Plan(N, prec)
    cube = p.to_cube(torch.as_tensor(uk).to("cuda", p.cdtype).contiguous())
    # the oracle sees exactly the spectrum the GPU sums (rounded to the plan precision)
    ukr = p.from_cube(cube).cpu().numpy().astype(np.complex128)
    rng = np.random.default_rng(N)
    pos = rng.uniform(-1.0, 2 * np.pi + 1.0, (npts, 3))
    got = p.exact_sum(cube, torch.as_tensor(pos).cuda()).cpu().numpy()
    ref = X.exact_sum(ukr, pos)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12


def test_exact_sum_at_grid_points_equals_inverse_transform(torch):
    from lucky_droplets_b200.spectral import Plan
    N = 64
    prm = C.ConfigParams(N=N, nu=0.01, dt=1e-3)
    grid = C.ConfigGrid(N)
    uk, _ = C.init_flow(grid, prm, seed=4)
    p = Plan(N, "f64")
    cube = p.to_cube(torch.as_tensor(uk).to("cuda", p.cdtype).contiguous())
    u = p.irfft_cube(cube).cpu().numpy()
    rng = np.random.default_rng(1)
    idx = rng.integers(0, N, (500, 3))
    pos = idx * (2 * np.pi / N)
    got = p.exact_sum(cube, torch.as_tensor(pos).cuda()).cpu().numpy()
    ref = u[:, idx[:, 0], idx[:, 1], idx[:, 2]].T
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12
