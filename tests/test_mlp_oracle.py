"""CPU checks of the learned-interpolation oracle (oracle/mlp_np.py): the canonical-frame features
are invariant under reflections and axis permutations of field and point together, and the
frame maps of vectors invert each other."""
import numpy as np

from oracle import config_np as C
from oracle import mlp_np as M

L = 2 * np.pi


def _features(u, pos, fs):
    st, t = C.stencil_4x4x4(u, pos)
    return M.features(st.reshape(pos.shape[0], 192), t, fs)


def _setup(seed=0, N=16, n=400):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((3, N, N, N))
    pos = rng.uniform(0, L, (n, 3))
    fs = rng.uniform(0.5, 2.0, 64)
    return u, pos, fs


def test_reflection_invariance():
    u, pos, fs = _setup(1)
    N = u.shape[-1]
    X, scale, _, _ = _features(u, pos, fs)
    for ax in range(3):
        # u'(x) = R u(R x) with R the reflection of axis ax: grid index j -> -j, component ax flips
        idx = [slice(None)] * 4
        idx[1 + ax] = (-np.arange(N)) % N
        ur = u[tuple(idx)].copy()
        ur[ax] *= -1
        pr = pos.copy()
        pr[:, ax] = L - pr[:, ax]
        Xr, scale_r, _, _ = _features(ur, pr, fs)
        assert np.allclose(scale, scale_r, rtol=1e-12)
        assert np.allclose(X, Xr, rtol=1e-2, atol=1e-5)


def test_permutation_invariance():
    u, pos, fs = _setup(2)
    X, _, _, _ = _features(u, pos, fs)
    for perm in ((1, 0, 2), (0, 2, 1), (2, 0, 1)):
        # u'(x) = P u(P^T x): components and grid axes permuted together
        up = np.transpose(u[list(perm)], (0, 1 + perm[0], 1 + perm[1], 1 + perm[2])).copy()
        pp = pos[:, list(perm)]
        Xp, _, _, _ = _features(up, pp, fs)
        assert np.allclose(X, Xp, rtol=1e-2, atol=1e-5)


def test_frame_round_trip_and_range():
    rng = np.random.default_rng(3)
    t = rng.uniform(0, 1, (1000, 3))
    perm, refl, tc = M.frames(t)
    assert np.all((tc >= 0) & (tc <= 0.5))
    assert np.all(tc[:, 0] >= tc[:, 1]) and np.all(tc[:, 1] >= tc[:, 2])
    assert np.all(np.sort(perm, axis=1) == np.arange(3))
    v = rng.standard_normal((1000, 3))
    assert np.allclose(M.from_canonical(M.to_canonical(v, perm, refl), perm, refl), v)
