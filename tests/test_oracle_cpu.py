"""CPU checks of two oracles the GPU parity tests rest on: the cell-list collision search of
oracle/collide_np.py returns exactly the pairs of its all-pairs FP64 rule (empty and single
inputs, 1, 2, 3 and many cells per axis, droplets outside [0, L), pairs across the periodic
faces, coincident droplets, cells narrower than twice the largest radius), and the direct Fourier sum of oracle/exact_np.py equals the inverse
transform at grid points and moves with a phase shift of the spectrum."""
import numpy as np
import pytest

from oracle import collide_np as K
from oracle import config_np as C
from oracle import exact_np as X

L = 2.0 * np.pi


@pytest.mark.parametrize("n, r_max", [(0, 0.1), (1, 0.1), (2, 3.0), (200, 2.5), (300, 1.2), (250, 1.0),
                                      (400, 0.05), (1500, 0.12)])
def test_cell_list_equals_all_pairs(n, r_max):
    """cell size = 2 r_max: r_max 3.0 and 2.5 give one cell per axis, 1.2 two, 1.0 three."""
    rng = np.random.default_rng(1000 + n)
    pos = rng.uniform(-L, 2 * L, (n, 3))
    rad = rng.uniform(0.5 * r_max, r_max, n)
    got = K.collide(pos, rad, 2 * r_max)
    ref = K.collide_bruteforce(pos, rad)
    assert got.dtype == np.int64 and got.shape == ref.shape and got.shape[1:] == (2,)
    assert np.array_equal(got, ref)
    if n > 1:
        assert np.all(got[:, 0] < got[:, 1])


def test_pairs_across_periodic_faces_and_coincident_droplets():
    r = 0.05
    pos = np.array([[1e-3, 1.0, 1.0], [L - 1e-3, 1.0, 1.0],       # across the x face
                    [2.0, -1e-3, 3.0], [2.0, L + 1e-3, 3.0],      # across y, both outside [0, L)
                    [4.0, 4.0, L], [4.0, 4.0, 0.0],               # z = L wraps onto z = 0
                    [5.0, 5.0, 5.0], [5.0, 5.0, 5.0],             # coincident
                    [3.0, 3.0, 3.0], [3.0, 3.0, 3.0 + 2.5 * r]])  # apart: 2.5 r > r + r
    rad = np.full(len(pos), r)
    got = K.collide(pos, rad, 2 * r)
    assert np.array_equal(got, K.collide_bruteforce(pos, rad))
    assert [tuple(p) for p in got] == [(0, 1), (2, 3), (4, 5), (6, 7)]


@pytest.mark.parametrize("case", ["lognormal", "equal_radii", "huge_droplet", "dense"])
def test_narrow_cells_equal_all_pairs(case):
    """Cells narrower than twice the largest radius (collide_wide): the neighbour-cell search plus
    the wide droplets' owner search give exactly the all-pairs list; equal radii exercise the
    owner tie rule, a droplet of radius L/3 a search over every cell."""
    rng = np.random.default_rng({"lognormal": 1, "equal_radii": 2, "huge_droplet": 3, "dense": 4}[case])
    n = 2500
    pos = rng.uniform(-1.0, L + 1.0, (n, 3))
    if case == "lognormal":
        rad = 0.05 * np.exp(0.6 * rng.standard_normal(n))
    elif case == "equal_radii":
        rad = np.full(n, 0.12)
    elif case == "huge_droplet":
        rad = 0.03 * rng.random(n) + 0.01
        rad[7] = L / 3
    else:
        pos = rng.uniform(1.0, 2.0, (n, 3))
        rad = 0.03 * np.exp(0.4 * rng.standard_normal(n))
    ref = K.collide_bruteforce(pos, rad)
    assert len(ref) > 50
    wide = 0
    for cell in (rad.max(), 2.5 * np.median(rad), 1.2 * np.median(rad)):
        nc = K.cell_count(L, cell)
        if nc < 3:
            continue
        wide += int((rad > 0.5 * L / nc).sum())
        assert np.array_equal(K.collide_wide(pos, rad, cell), ref), cell
    assert wide > 0


def _flow(N, seed):
    uk, _ = C.init_flow(C.ConfigGrid(N), C.ConfigParams(N=N, nu=0.01, dt=1e-3), seed=seed)
    return uk


def test_exact_sum_at_grid_points_equals_inverse_transform():
    N = 16
    uk = _flow(N, 4)
    u = np.fft.irfftn(uk, s=(N, N, N), axes=(1, 2, 3))
    idx = np.random.default_rng(1).integers(0, N, (300, 3))
    got = X.exact_sum(uk, idx * (L / N))
    ref = u[:, idx[:, 0], idx[:, 1], idx[:, 2]].T
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12


def test_exact_sum_moves_with_a_phase_shift():
    """sum_k w Re(c_k e^{i k.(x + s)}) = sum_k w Re((c_k e^{i k.s}) e^{i k.x}) term by term."""
    N = 16
    uk = _flow(N, 5)
    K1 = np.fft.fftfreq(N, 1.0 / N)
    kx, ky, kz = np.meshgrid(K1, K1, np.abs(K1[:N // 2 + 1]), indexing="ij")
    s = np.array([0.37, -1.21, 2.9])
    shifted = uk * np.exp(1j * (kx * s[0] + ky * s[1] + kz * s[2]))[None]
    x = np.random.default_rng(2).uniform(0, L, (200, 3))
    a = X.exact_sum(shifted, x)
    b = X.exact_sum(uk, x + s)
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-12
