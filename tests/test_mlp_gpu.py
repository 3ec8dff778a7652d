"""Learned interpolation on the GPU: gradients and inference against the CPU oracle
(oracle/mlp_np.py), the exact training targets against the direct Fourier sum, and a short
training run that must beat tricubic interpolation."""
import numpy as np
import pytest

from oracle import config_np as C
from oracle import mlp_np as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def test_gradients_match_oracle(torch):
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import mlp as G
    rng = np.random.default_rng(0)
    nb = 200  # not a multiple of the 128-sample tile: padded rows must not contribute
    X = np.zeros((nb, G.K1), np.float32)
    X[:, :M.D_IN] = M.bf16(rng.standard_normal((nb, M.D_IN)).astype(np.float32))
    T = rng.standard_normal((nb, 3)).astype(np.float32) * 0.3
    p = M.init_params(3)
    p["b1"] = rng.standard_normal(128).astype(np.float32) * 0.1
    p["b2"] = rng.standard_normal(128).astype(np.float32) * 0.1
    p["b3"] = rng.standard_normal(3).astype(np.float32) * 0.1
    plan = Plan(16, "f32")
    li = G.LearnedInterp(plan, params=G.flat_from_mats(p["W1"], p["b1"], p["W2"], p["b2"], p["W3"], p["b3"]))
    w = rng.uniform(0.1, 3.0, nb).astype(np.float32)
    Xg = torch.as_tensor(X).to("cuda", torch.bfloat16)
    Tg = torch.as_tensor(T).cuda()
    loss, grad = li.loss_and_grad(Xg, Tg, torch.as_tensor(w).cuda())
    gm = G.mats_from_flat(grad.cpu().numpy())
    assert np.all(gm["fs"] == 0) and gm["os"] == 0  # the scales get no gradient
    ref_loss, ref = M.mse_loss_and_grads(p, X[:, :M.D_IN], T, w=w)
    assert abs(float(loss.item()) - ref_loss) / ref_loss < 1e-4
    # dY, dZ2 and dZ1 enter the tensor-core products as two BF16 parts (about 16 bits of the FP32
    # values): every gradient within 1e-3 of the FP64 oracle (measured: 1e-5 .. 3e-4)
    for k in ("W3", "b3", "W2", "b2", "W1", "b1"):
        assert rel(gm[k], ref[k]) < 1e-3, k


def _oracle_infer(u, pos, p, fs, os):
    st, t = C.stencil_4x4x4(u, pos)
    X, scale, perm, refl = M.features(st.reshape(pos.shape[0], 192), t, fs)
    y, _ = M.forward(p, X)
    tric = C.gather(u, pos, "tricubic")
    return tric + scale[:, None] * os * M.from_canonical(y, perm, refl), tric


def test_inference_matches_oracle(torch):
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import mlp as G
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=1e-3)
    grid = C.ConfigGrid(N)
    uk, u = C.init_flow(grid, prm, seed=8)
    plan = Plan(N, "f32")
    p = M.init_params(5)
    fs = np.random.default_rng(3).uniform(0.5, 3.0, 64).astype(np.float32)
    os = 0.01  # an untrained network: keep its correction small against the velocity, as trained ones are
    li = G.LearnedInterp(plan, params=G.flat_from_mats(**p, fs=fs, os=os))
    cube = plan.to_cube(torch.as_tensor(uk).to("cuda", plan.cdtype).contiguous())
    u4 = li.interleaved(cube)
    rng = np.random.default_rng(2)
    pos = rng.uniform(-1, 7.5, (3001, 3))
    got = li.infer(u4, torch.as_tensor(pos).cuda()).cpu().numpy()
    ref, tric = _oracle_infer(u, pos, p, fs, os)
    # the correction part agrees to FP32/BF16-input accuracy, the whole to FP32 accuracy
    assert rel(got - tric, ref - tric) < 5e-3
    assert rel(got, ref) < 1e-4


def test_training_targets_are_exact(torch):
    """T * scale + tricubic at the shifted sample points equals the direct Fourier sum."""
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import mlp as G
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=1e-3)
    grid = C.ConfigGrid(N)
    uk, _ = C.init_flow(grid, prm, seed=9)
    plan = Plan(N, "f64")
    li = G.LearnedInterp(plan)
    cube = plan.to_cube(torch.as_tensor(uk).to("cuda", plan.cdtype).contiguous())
    rng = np.random.default_rng(4)
    s = rng.uniform(0, 1, 3)
    import ctypes
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, ptr, stream_ptr
    shifted = plan.empty_cube(3)
    check(_lib.lib().ld_phase_shift(plan.handle, ptr(cube), ptr(shifted), *map(float, s), stream_ptr()))
    ue = plan.irfft_cube(shifted).cpu().numpy()
    idx = rng.integers(0, N ** 3, 200)
    j = np.stack([idx // (N * N), (idx // N) % N, idx % N], axis=1)
    pos = (j + s) * (2 * np.pi / N)
    exact = plan.exact_sum(cube, torch.as_tensor(pos).cuda()).cpu().numpy()
    assert np.abs(ue.reshape(3, -1)[:, idx].T - exact).max() / np.abs(exact).max() < 1e-12


def test_inference_streams_many_tiles_per_cta(torch):
    """At 94,797 droplets on a 128^3 plan (one batch: the workspace holds about 140k rows) every
    CTA of the tensor-core forward takes 5-6 tiles of 128 droplets, the last one ragged, so the
    feature chunks stream through the shared-memory ring with refills and both groups of warps
    alternate on it.  A row's result does not depend on its tile or CTA: the whole batch must
    equal, bit for bit, the same droplets inferred in batches of 2,000 (at most one tile per CTA,
    no refill), and a subsample must match the oracle."""
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import mlp as G
    N = 128
    prm = C.ConfigParams(N=N, nu=0.01, dt=1e-3)
    grid = C.ConfigGrid(N)
    uk, u = C.init_flow(grid, prm, seed=8)
    plan = Plan(N, "f32")
    p = M.init_params(5)
    fs = np.random.default_rng(3).uniform(0.5, 3.0, 64).astype(np.float32)
    os = 0.01
    li = G.LearnedInterp(plan, params=G.flat_from_mats(**p, fs=fs, os=os))
    cube = plan.to_cube(torch.as_tensor(uk).to("cuda", plan.cdtype).contiguous())
    u4 = li.interleaved(cube)
    n = 148 * 128 * 5 + 77
    pos = np.random.default_rng(4).uniform(-1, 7.5, (n, 3))
    pos_d = torch.as_tensor(pos).cuda()
    whole = li.infer(u4, pos_d).cpu().numpy()
    parts = np.concatenate([li.infer(u4, pos_d[b:b + 2000]).cpu().numpy() for b in range(0, n, 2000)])
    assert plan.status() == 0  # no bounded wait ran out
    assert np.array_equal(whole, parts)
    sub = slice(0, n, 7)
    ref, tric = _oracle_infer(u, pos[sub], p, fs, os)
    assert rel(whole[sub] - tric, ref - tric) < 5e-3
    assert rel(whole[sub], ref) < 1e-4


def test_training_beats_tricubic(torch):
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import mlp as G
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=1e-3)
    grid = C.ConfigGrid(N)
    uk, _ = C.init_flow(grid, prm, seed=10)
    plan = Plan(N, "f32")
    li = G.LearnedInterp(plan, seed=1, tol=1e-12, rule="tolerance_or_better")
    cube = plan.to_cube(torch.as_tensor(uk).to("cuda", plan.cdtype).contiguous())
    li.calibrate(cube)
    X, T, W, _ = li.make_samples(cube, n_shifts=400, per_shift=1024, seed=1)
    losses = li.train(X, T, W, epochs=12, batch=4096, lr=2e-3, lr_final=2e-4, seed=0)
    assert losses[-1] < 0.8 * losses[0]
    rng = np.random.default_rng(77)
    pos = torch.as_tensor(rng.uniform(0, 2 * np.pi, (4000, 3))).cuda()
    e_learned, e_tric = li.judge(cube, li.interleaved(cube), pos)
    assert e_learned < e_tric, (e_learned, e_tric)
    assert li.enabled  # misses the (impossible) tolerance but beats tricubic
    li.rule = "tolerance"
    li.judge(cube, li.interleaved(cube), pos)
    assert not li.enabled  # the default rule: off above the tolerance


def test_inference_features_equal_training_features(torch):
    """The warp-cooperative inference kernel (three lanes per droplet, one canonical component
    each, sums exchanged by shuffles) and the thread-per-sample training kernel produce the same
    feature rows, tricubic values and scales, bit for bit, at the same points."""
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import mlp as G
    N, per = 32, 3000
    prm = C.ConfigParams(N=N, nu=0.01, dt=1e-3)
    uk, _ = C.init_flow(C.ConfigGrid(N), prm, seed=11)
    plan = Plan(N, "f32")
    li = G.LearnedInterp(plan, seed=2)
    cube = plan.to_cube(torch.as_tensor(uk).to("cuda", plan.cdtype).contiguous())
    seed = 5
    X, _, _, aux = li.make_samples(cube, 1, per, seed=seed)
    rng = np.random.default_rng(seed)
    s = rng.uniform(0.0, 1.0, 3)
    idx = rng.integers(0, N ** 3, per, dtype=np.int64)
    j = np.stack([idx // (N * N), (idx // N) % N, idx % N], axis=1).astype(np.float64)
    pos = (j + s) * (2.0 * np.pi / N)
    work = li.workspace(per)
    li.infer(li.interleaved(cube), torch.as_tensor(pos).cuda(), work=work)
    torch.cuda.synchronize()
    wb = work.cpu().numpy()
    tile_bytes = 128 * G.K1 * 2
    tiles = (per + 127) // 128
    rows = np.arange(per)
    t, rr = rows // 128, rows % 128
    feat = np.empty((per, G.K1), np.uint16)
    for kc in range(G.K1 // 8):
        off = t * tile_bytes + (kc * 16 + rr // 8) * 128 + (rr % 8) * 16  # the tile layout
        chunk = wb[off[:, None] + np.arange(16)[None, :]]
        feat[:, 8 * kc:8 * kc + 8] = chunk.view(np.uint16).reshape(per, 8)
    ref = X.view(torch.int16).cpu().numpy().view(np.uint16)
    assert np.array_equal(feat, ref)
    ax = wb[tiles * tile_bytes:].view(np.float32)[:8 * per].reshape(per, 8)
    a = aux.cpu().numpy()
    assert np.array_equal(ax[:, :3], a[:, :3]) and np.array_equal(ax[:, 3], a[:, 3])


def test_epoch_call_equals_grad_then_adam(torch):
    """ld_mlp_train_epoch (rows gathered inside the tensor-core kernel, the partial sums fused with
    Adam and the BF16 re-pack) against ld_mlp_grad then ld_mlp_adam on the gathered rows, batch
    by batch: bit-identical parameters, moments, packed copy and epoch losses."""
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import mlp as G
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, ptr, stream_ptr
    rng = np.random.default_rng(4)
    n, batch, epochs, lr, lr_final = 1000, 300, 2, 1e-3, 1e-4  # 300 = 2 x 128 + 44: a partial tile
    X = np.zeros((n, G.K1), np.float32)
    X[:, :M.D_IN] = rng.standard_normal((n, M.D_IN))
    T = rng.standard_normal((n, 3)).astype(np.float32) * 0.3
    W = rng.uniform(0.1, 3.0, n).astype(np.float32)
    p = M.init_params(7)
    flat = G.flat_from_mats(p["W1"], p["b1"], p["W2"], p["b2"], p["W3"], p["b3"])
    plan = Plan(16, "f32")
    a = G.LearnedInterp(plan, params=flat.copy())
    b = G.LearnedInterp(plan, params=flat.copy())
    Xg = torch.as_tensor(X).to("cuda", torch.bfloat16)
    Tg = torch.as_tensor(T).cuda()
    Wg = torch.as_tensor(W).cuda()
    la = a.train(Xg, Tg, Wg, epochs=epochs, batch=batch, lr=lr, lr_final=lr_final, seed=5)
    L = _lib.lib()
    wn = (Wg / Wg.mean()).contiguous()
    g = torch.Generator(device="cuda").manual_seed(5)
    nbatch = n // batch
    total = epochs * nbatch
    lb = []
    for _ in range(epochs):
        perm = torch.randperm(n, generator=g, device="cuda").to(torch.int32)
        acc = torch.zeros(1, dtype=torch.float32, device="cuda")
        for k in range(nbatch):
            idx = perm[k * batch:(k + 1) * batch].long()
            loss, _ = b.loss_and_grad(Xg[idx].contiguous(), Tg[idx].contiguous(), wn[idx].contiguous())
            acc += loss
            b.step_count += 1
            s = b.step_count
            lr_k = lr * (lr_final / lr) ** (min(s, total) / total)
            check(L.ld_mlp_adam(ptr(b.params), ptr(b.grad), ptr(b.m), ptr(b.v), s, float(lr_k), ptr(b.packed),
                                stream_ptr()))
        lb.append(float(acc.item()) / nbatch)
    assert la == lb
    for name in ("params", "m", "v", "packed"):
        assert torch.equal(getattr(a, name), getattr(b, name)), name
    assert la[-1] < la[0]


def test_packed_tile_copies(torch):
    """The packed BF16 weights hold W1t, W2t and W3t twice: row-major with padded rows, and in the
    tensor-core tile layout (8x8 core matrices, K-chunk major) that the kernels bulk-copy; the two
    agree element for element and the padding is zero."""
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200 import mlp as G
    H, K1, N3, N3P, KP1, KP2 = 128, G.K1, 8, 16, 216, 136
    P_W2T = H * KP1
    P_W2N = P_W2T + H * KP2
    P_W3T = P_W2N + H * KP2
    P_W3N = P_W3T + N3 * KP2
    P_TW1 = P_W3N + H * N3
    P_TW2 = P_TW1 + H * K1
    P_TW3 = P_TW2 + H * H
    assert G.sizes()[1] == P_TW3 + N3P * H
    p = M.init_params(11)
    li = G.LearnedInterp(Plan(16, "f32"), params=G.flat_from_mats(p["W1"], p["b1"], p["W2"], p["b2"], p["W3"], p["b3"]))
    q = li.packed.float().cpu().numpy()

    def tile(start, rows, kdim):  # element (row, k) of a tile -> (rows, kdim) matrix
        t = q[start:start + rows * kdim].reshape(kdim // 8, rows // 8, 8, 8)  # [kc][row/8][row%8][k%8]
        return t.transpose(1, 2, 0, 3).reshape(rows, kdim)

    w1t = q[:P_W2T].reshape(H, KP1)
    assert np.array_equal(tile(P_TW1, H, K1), w1t[:, :K1]) and not w1t[:, K1:].any()
    w2t = q[P_W2T:P_W2N].reshape(H, KP2)
    assert np.array_equal(tile(P_TW2, H, H), w2t[:, :H])
    w3t = q[P_W3T:P_W3N].reshape(N3, KP2)
    t3 = tile(P_TW3, N3P, H)
    assert np.array_equal(t3[:N3], w3t[:, :H]) and not t3[N3:].any()
    assert np.array_equal(w1t[:, :M.D_IN], M.bf16(p["W1"]).T)  # W1t[o][k] = bf16(W1[k][o])
