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


def _slab_checkpoint(tmp_path, P, N=16, seed=3):
    """The files a P-rank run of the reference leaves (F:446-450): rank r writes the ky slab r of
    the spectra and the x slab r of n."""
    rng = np.random.default_rng(seed)
    Nf = N // 2 + 1
    uk = rng.standard_normal((3, N, N, Nf)) + 1j * rng.standard_normal((3, N, N, Nf))
    n = rng.random((N, N, N))
    Np = N // P
    for r in range(P):
        np.savez_compressed(tmp_path / f"Fields_k_{r}.npz", uk=uk[0][:, r * Np:(r + 1) * Np],
                            vk=uk[1][:, r * Np:(r + 1) * Np], wk=uk[2][:, r * Np:(r + 1) * Np])
        np.savez_compressed(tmp_path / f"n_{r}.npz", n=n[r * Np:(r + 1) * Np])
    return uk, n


def _load_npz_restated(path, N):
    """load_npz of F:374-407 on one rank (Np = N): ky plane j from slab j // (N/P), index j % (N/P)."""
    P = len([x for x in path.iterdir() if "Fields" in x.name and x.name.endswith(".npz")])
    per = N // P
    uk = np.zeros((3, N, N, N // 2 + 1), complex)
    n = np.zeros((N, N, N))
    for j in range(N):
        F = np.load(path / f"Fields_k_{j // per}.npz")
        nF = np.load(path / f"n_{j // per}.npz")
        uk[0, :, j] = F["uk"][:, j % per]
        uk[1, :, j] = F["vk"][:, j % per]
        uk[2, :, j] = F["wk"][:, j % per]
        n[j] = nF["n"][j % per]
    return uk, n


def test_multi_slab_checkpoint_reads_back_exactly(tmp_path):
    """A 4-rank checkpoint is re-slabbed onto one GPU exactly as load_npz (F:374-407) does."""
    from lucky_droplets_b200.outputs import read_n
    uk, n = _slab_checkpoint(tmp_path, 4)
    got = read_fields(tmp_path)
    assert np.array_equal(got, uk)
    assert np.array_equal(read_n(tmp_path), n)
    ref_uk, ref_n = _load_npz_restated(tmp_path, 16)
    assert np.array_equal(got, ref_uk) and np.array_equal(read_n(tmp_path), ref_n)


def test_written_slabs_round_trip(tmp_path):
    """write_outputs(slabs=P) writes what a P-rank run writes; reading it back is exact."""
    from lucky_droplets_b200.outputs import read_n
    rng = np.random.default_rng(5)
    uk = rng.standard_normal((3, 16, 16, 9)) + 1j * rng.standard_normal((3, 16, 16, 9))
    n = rng.random((16, 16, 16))
    paths = write_outputs(tmp_path, uk, np.zeros(9), np.zeros(9), n=n, slabs=8)
    assert sorted(p.name for p in paths if p.name.startswith("Fields")) == [f"Fields_k_{r}.npz" for r in range(8)]
    assert np.load(tmp_path / "Fields_k_3.npz")["uk"].shape == (16, 2, 9)
    assert np.load(tmp_path / "n_3.npz")["n"].shape == (2, 16, 16)
    assert np.array_equal(read_fields(tmp_path), uk)
    assert np.array_equal(read_n(tmp_path), n)


def test_bad_checkpoints_raise_cleanly(tmp_path):
    """Missing slabs, truncated archives, missing keys and a wrong shape raise CheckpointError."""
    import pytest
    from lucky_droplets_b200.outputs import CheckpointError
    with pytest.raises(CheckpointError):
        read_fields(tmp_path / "absent")
    with pytest.raises(CheckpointError):
        read_fields(tmp_path)  # no Fields files
    _slab_checkpoint(tmp_path, 4)
    (tmp_path / "Fields_k_2.npz").unlink()
    with pytest.raises(CheckpointError, match="slabs"):
        read_fields(tmp_path)
    _slab_checkpoint(tmp_path, 4)
    raw = (tmp_path / "Fields_k_1.npz").read_bytes()
    (tmp_path / "Fields_k_1.npz").write_bytes(raw[: len(raw) // 2])  # truncated archive
    with pytest.raises(CheckpointError, match="Fields_k_1"):
        read_fields(tmp_path)
    _slab_checkpoint(tmp_path, 4)
    np.savez_compressed(tmp_path / "Fields_k_0.npz", uk=np.zeros((16, 4, 9)), vk=np.zeros((16, 4, 9)))
    with pytest.raises(CheckpointError, match="wk"):
        read_fields(tmp_path)
    _slab_checkpoint(tmp_path, 4)
    np.savez_compressed(tmp_path / "Fields_k_0.npz", uk=np.zeros((16, 3, 9)), vk=np.zeros((16, 3, 9)),
                        wk=np.zeros((16, 3, 9)))
    with pytest.raises(CheckpointError):
        read_fields(tmp_path)
