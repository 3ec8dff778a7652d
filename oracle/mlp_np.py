"""CPU oracle for the learned-interpolation MLP (no counterpart in the reference).

TEST INFRASTRUCTURE ONLY.

Network: 195 inputs (the 4x4x4 stencil of (u, v, w) in tap order (c, a, b, q) -> c*64 + a*16 + b*4
+ q, transformed per component into the (orthogonal, unnormalised) discrete polynomial basis of
orders 0..3 along each axis, divided by the stencil RMS and multiplied by fixed per-coefficient scales; then the
three fractional cell offsets minus 1/2) -> 128 SiLU -> 128 SiLU -> 3, times a fixed output
scale.  The GPU kernels feed
BF16 operands to the tensor cores with FP32 accumulation; this oracle rounds the same operands to
BF16 (round to nearest even) and accumulates in FP64, so the two agree to FP32 accumulation error.
"""
import numpy as np

D_IN, D_H, D_OUT = 195, 128, 3


def bf16(x):
    """Round to bfloat16 (nearest even) and return as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    nan = np.isnan(a)
    out = rounded.astype(np.uint32).view(np.float32).copy()
    out[nan] = np.nan
    return out


# discrete polynomials on 4 points, orders 0..3 (rows; orthogonal, not normalised)
P4 = np.array([[1, 1, 1, 1], [-3, -1, 1, 3], [1, -1, -1, 1], [-1, 3, -3, 1]], np.float64)


def frames(t):
    """Canonical frame of each point: reflect every axis whose offset exceeds 1/2, then order the
    axes by decreasing reflected offset (stable).  Returns (perm (n,3): canonical axis k <- grid
    axis perm[:, k], refl (n,3) bool per grid axis, tc (n,3) canonical offsets)."""
    t = np.asarray(t, np.float32)
    refl = t > np.float32(0.5)
    r = np.where(refl, np.float32(1) - t, t)
    n = t.shape[0]
    perm = np.tile(np.arange(3), (n, 1))
    for a, b in ((0, 1), (1, 2), (0, 1)):   # the same compare-exchange network as the kernels
        ra = r[np.arange(n), perm[:, a]]
        rb = r[np.arange(n), perm[:, b]]
        sw = rb > ra
        pa = perm[:, a].copy()
        perm[sw, a] = perm[sw, b]
        perm[sw, b] = pa[sw]
    tc = np.take_along_axis(r, perm, axis=1)
    return perm, refl, tc


def to_canonical(v, perm, refl):
    """Grid-frame vectors (n,3) -> canonical frame."""
    sg = np.where(refl, -1.0, 1.0)
    return np.take_along_axis(v * sg, perm, axis=1)


def from_canonical(y, perm, refl):
    """Canonical-frame vectors (n,3) -> grid frame."""
    out = np.empty_like(y)
    np.put_along_axis(out, perm, y, axis=1)
    return out * np.where(refl, -1.0, 1.0)


_ORDER = (np.arange(64) >> 4) + ((np.arange(64) >> 2) & 3) + (np.arange(64) & 3)


def features(st, t, fs, scale_mode=1):
    """Network inputs (n, 195) from stencils st (n, 192), offsets t (n, 3) and feature scales fs
    (64): returns (X rounded to BF16, scale, perm, refl).  scale: RMS of all coefficients (mode 0)
    or of those of total order >= 3 (mode 1), in the polynomial basis."""
    n = st.shape[0]
    v = st.reshape(n, 3, 4, 4, 4)
    d = np.einsum("ia,jb,kq,ncabq->ncijk", P4, P4, P4, v, optimize=True)
    d64 = d.reshape(n, 3, 64)
    if scale_mode:
        scale = np.sqrt((d64[:, :, _ORDER >= 3] ** 2).sum(axis=(1, 2)) / 162.0) + 1e-30
    else:
        scale = np.sqrt((d64 ** 2).sum(axis=(1, 2)) / 192.0) + 1e-30
    perm, refl, tc = frames(t)
    out = np.empty((n, 3, 4, 4, 4))
    # reflection of grid axis g multiplies order-j coefficients along g by (-1)^j
    par = np.array([1.0, -1.0, 1.0, -1.0])
    for i in range(n):
        p, rf = perm[i], refl[i]
        di = d[i]
        for g in range(3):
            if rf[g]:
                shp = [1, 1, 1, 1]
                shp[1 + g] = 4
                di = di * par.reshape(shp)
        di = di * np.where(rf, -1.0, 1.0)[:, None, None, None]      # velocity components
        di = di[p]                                                  # components to canonical order
        out[i] = np.transpose(di, (0, 1 + p[0], 1 + p[1], 1 + p[2]))  # coefficient axes
    dd = out.reshape(n, 3, 64) / scale[:, None, None] * np.asarray(fs, np.float64)[None, None, :]
    X = np.concatenate([dd.reshape(n, 192), tc - 0.5], axis=1)
    return bf16(X.astype(np.float32)), scale, perm, refl


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def init_params(seed=0):
    """He-style uniform initialisation, FP32 master weights."""
    rng = np.random.default_rng(seed)

    def lin(i, o):
        lim = np.sqrt(6.0 / i)
        return rng.uniform(-lim, lim, (i, o)).astype(np.float32), np.zeros(o, np.float32)

    W1, b1 = lin(D_IN, D_H)
    W2, b2 = lin(D_H, D_H)
    W3, b3 = lin(D_H, D_OUT)
    W3 *= 0.1
    return dict(W1=W1, b1=b1, W2=W2, b2=b2, W3=W3, b3=b3)


def forward(p, X, emulate_bf16=True):
    """X (B, 195) -> Y (B, 3) and the cache for backward."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float32))
    x = r(X).astype(np.float64)
    z1 = x @ r(p["W1"]).astype(np.float64) + p["b1"]
    h1 = silu(z1)
    z2 = r(h1).astype(np.float64) @ r(p["W2"]).astype(np.float64) + p["b2"]
    h2 = silu(z2)
    y = r(h2).astype(np.float64) @ r(p["W3"]).astype(np.float64) + p["b3"]
    return y, dict(x=x, z1=z1, h1=r(h1).astype(np.float64), z2=z2, h2=r(h2).astype(np.float64))


def backward(p, cache, dy, emulate_bf16=True):
    """Gradients of sum(dy * Y) with respect to every parameter."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float32))
    g = {}
    g["W3"] = cache["h2"].T @ dy
    g["b3"] = dy.sum(0)
    dh2 = dy @ r(p["W3"]).astype(np.float64).T
    dz2 = dh2 * dsilu(cache["z2"])
    g["W2"] = cache["h1"].T @ dz2
    g["b2"] = dz2.sum(0)
    dh1 = dz2 @ r(p["W2"]).astype(np.float64).T
    dz1 = dh1 * dsilu(cache["z1"])
    g["W1"] = cache["x"].T @ dz1
    g["b1"] = dz1.sum(0)
    return g


def mse_loss_and_grads(p, X, T, emulate_bf16=True, w=None):
    """sum over the batch of w |Y - T|^2 / B (w = 1 by default) and its gradients."""
    y, cache = forward(p, X, emulate_bf16)
    d = y - T
    B = X.shape[0]
    w = np.ones(B) if w is None else np.asarray(w, np.float64)
    loss = float((w[:, None] * d ** 2).sum() / B)
    g = backward(p, cache, 2.0 * w[:, None] * d / B, emulate_bf16)
    return loss, g


def adam_step(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """In-place Adam update of FP32 master weights."""
    for k in p:
        m[k] = b1 * m[k] + (1 - b1) * g[k]
        v[k] = b2 * v[k] + (1 - b2) * g[k] ** 2
        mh = m[k] / (1 - b1 ** t)
        vh = v[k] / (1 - b2 ** t)
        p[k] = (p[k] - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
