"""The CPU oracle (oracle/reference_np.py) against golden vectors made by running the reference.

The fixtures tests/golden/ref_N16.npz and ref_N32.npz were written by tests/golden/make_golden.py,
which executes forced-dns-sm.py + particles.py themselves (single-rank mpi4py stand-in, seeded).
"""
import numpy as np
import pytest

from oracle import reference_np as R

CASES = {"N16": 7, "N32": 11}


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


def _setup(golden, name):
    g = golden(name)
    N = int(g["N"])
    return g, N, R.Grid(N), R.ReferenceParams(N)


def test_parameters_match(golden):
    for name in CASES:
        g, N, grid, prm = _setup(golden, name)
        assert prm.nu == pytest.approx(float(g["nu"]), rel=0, abs=0)
        assert prm.dt == float(g["dt"]) and prm.f0 == float(g["f0"]) and prm.tps == float(g["tps"])
        assert list(prm.shell_no) == list(g["shell_no"])


def test_operators_match(golden):
    g, N, grid, _ = _setup(golden, "N16")
    assert (grid.kint == g["op_kint"]).all()
    assert (grid.dealias == g["op_dealias"]).all()
    assert np.array_equal(grid.normalize, g["op_normalize"])
    assert np.array_equal(grid.invlap, g["op_invlap"])


def test_transforms_match(golden):
    g, N, grid, _ = _setup(golden, "N16")
    assert np.array_equal(grid.rfft(g["fft_in"]), g["fft_out"])
    assert np.array_equal(grid.irfft(g["ifft_in"]), g["ifft_out"])


@pytest.mark.parametrize("name", list(CASES))
def test_initial_field_and_droplets(golden, name):
    g, N, grid, prm = _setup(golden, name)
    nprt = g["init_coord"].shape[0]
    coord, th = R.draw_reference_randoms(grid, nprt, seed=CASES[name])
    # the mass column is overwritten after the draw (particles.py:94)
    assert np.array_equal(coord[:, :6], g["init_coord"][:, :6])
    _, u = R.init_field(grid, th, prm.einit)
    assert rel(u, g["init_u"]) < 1e-14
    assert rel(R.start_spectrum(grid, u), g["uk0"]) < 1e-14


def test_forcing_and_shell_spectrum(golden):
    g, N, grid, prm = _setup(golden, "N16")
    fk, ek = R.forcing(grid, g["uk0"], prm.f0, prm.shell_no)
    assert rel(fk, g["forcing_fk"]) < 1e-14
    ref = g["forcing_ek_arr"]
    finite = np.isfinite(ref)
    assert (np.isfinite(ek) == finite).all()
    assert np.allclose(ek[finite], ref[finite], rtol=1e-13, atol=0)


@pytest.mark.parametrize("name", list(CASES))
def test_cosine_interpolation(golden, name):
    g, N, grid, prm = _setup(golden, name)
    d = R.Droplets(N, grid.L, 0, prm.sts, prm.stb0, prm.g, prm.nu, prm.tf, prm.rhop, prm.M0,
                   coord=g["init_coord"].copy())
    assert d.factor == float(g["prt_factor"])
    fields = np.concatenate((g["init_u"], g["init_u"] * 0.5, g["init_n"][None]), axis=0)
    out = d.interp_cosine(g["interp_coord"], fields)
    assert np.abs(out - g["interp_out"]).max() < 1e-13


@pytest.mark.parametrize("name", list(CASES))
def test_full_rhs(golden, name):
    g, N, grid, prm = _setup(golden, name)
    d = R.Droplets(N, grid.L, 0, prm.sts, prm.stb0, prm.g, prm.nu, prm.tf, prm.rhop, prm.M0,
                   coord=g["init_coord"].copy())
    ku, kn, kp = R.full_rhs(grid, prm, g["uk0"].copy(), np.ones((N, N, N)), g["rhs_coord_in"].copy(), d)
    assert rel(ku, g["rhs_ku"]) < 1e-14
    assert np.abs(kn - g["rhs_kn"]).max() < 1e-12
    ids = g["rhs_prtclid"].ravel().astype(int)  # the reference reorders droplets in send()
    assert np.abs(kp[ids] - g["rhs_kp"]).max() < 1e-11


@pytest.mark.parametrize("name", list(CASES))
def test_rk4_time_loop(golden, name):
    g, N, grid, prm = _setup(golden, name)
    d = R.Droplets(N, grid.L, 0, prm.sts, prm.stb0, prm.g, prm.nu, prm.tf, prm.rhop, prm.M0,
                   coord=g["init_coord"].copy())
    uk, n = g["uk0"].copy(), np.ones((N, N, N))
    for _ in range(int(g["nsteps"])):
        uk, n, _ = R.rk4_step(grid, prm, uk, n, d, prm.dt)
    assert rel(uk, g["run_uk"]) < 1e-14
    assert np.abs(n - g["run_n"]).max() < 1e-12
    ids = g["run_prtclid"].ravel().astype(int)
    dpos = (d.coord[ids, :3] - g["run_coord"][:, :3] + np.pi) % (2 * np.pi) - np.pi
    assert np.abs(dpos).max() < 1e-12
    assert np.abs(d.coord[ids, 3:] - g["run_coord"][:, 3:]).max() < 1e-12
