"""Output files with the reference's names and keys (forced-dns-sm.py save(), F:419-460), and the
flux-spectrum restatement of F:424-428 on the oracle (no GPU)."""
import numpy as np

from lucky_droplets_b200.outputs import flux_from_transfer, read_fields, reference_dirs, write_outputs
from oracle import reference_np as R


def test_files_and_keys(tmp_path):
    rng = np.random.default_rng(0)
    uk = rng.standard_normal((3, 8, 8, 5)) + 1j * rng.standard_normal((3, 8, 8, 5))
    state = {"pos": rng.random((4, 3)), "vel": rng.random((4, 3)), "prtclid": np.arange(4), "umat": rng.random((4, 3))}
    paths = write_outputs(tmp_path, uk, np.arange(5.0), np.arange(5.0)[::-1], state=dict(state), n=np.ones((8, 8, 8)))
    names = sorted(p.name for p in paths)
    assert names == ["Energy_spectrum.npz", "Fields_k_0.npz", "Flux_spectrum.npz", "n_0.npz", "state_0.npz"]
    f = np.load(tmp_path / "Fields_k_0.npz")
    assert sorted(f.files) == ["uk", "vk", "wk"]
    assert np.array_equal(read_fields(tmp_path), uk)
    assert np.load(tmp_path / "Energy_spectrum.npz").files == ["ek"]
    assert np.load(tmp_path / "Flux_spectrum.npz").files == ["Pik"]
    s = np.load(tmp_path / "state_0.npz")
    assert sorted(s.files) == ["pos", "prtclid", "umat", "vel"]
    root, drop = reference_dirs(tmp_path, 1.25, "wg", 0.1, 0.5)
    assert root.name == "time_1.2" and drop.name == "wg_stb_0.500_sts_0.100"


def test_flux_is_reversed_cumulative_transfer():
    """Pik_arr = cumsum(T[::-1])[::-1] with T the shell sums of Re(conj(uk) N(uk)) dealias
    normalize (F:425-428); the inviscid nonlinear term transfers energy between shells only, so
    the total transfer (Pik_arr[0]) vanishes for a solenoidal, dealiased field."""
    N = 16
    grid = R.Grid(N)
    rng = np.random.default_rng(1)
    u = rng.standard_normal((3, N, N, N))
    uk = grid.project(np.stack([grid.rfft(u[c]) for c in range(3)])) * grid.dealias
    ku, _, _ = R.velocity_rhs(grid, uk, 0.0, np.zeros_like(uk), 0.0)
    T = grid.shell_sum(np.real(np.conj(uk[0]) * ku[0] + np.conj(uk[1]) * ku[1] + np.conj(uk[2]) * ku[2])
                       * grid.dealias * grid.normalize)
    pik = flux_from_transfer(T)
    assert np.allclose(pik, np.cumsum(T[::-1])[::-1])
    scale = np.abs(T).max()
    assert abs(pik[0]) < 1e-10 * scale * N
