"""CPU oracle for the learned-interpolation MLP (no counterpart in the reference).

TEST INFRASTRUCTURE ONLY.

Network: 195 inputs (the 4x4x4 stencil of (u, v, w) in tap order (c, a, b, q) -> c*64 + a*16 + b*4
+ q, then the three fractional cell offsets) -> 128 SiLU -> 128 SiLU -> 3.  The GPU kernels feed
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


def mse_loss_and_grads(p, X, T, emulate_bf16=True):
    """mean over the batch of |Y - T|^2 and its gradients."""
    y, cache = forward(p, X, emulate_bf16)
    d = y - T
    B = X.shape[0]
    loss = float((d ** 2).sum() / B)
    g = backward(p, cache, 2.0 * d / B, emulate_bf16)
    return loss, g


def adam_step(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """In-place Adam update of FP32 master weights."""
    for k in p:
        m[k] = b1 * m[k] + (1 - b1) * g[k]
        v[k] = b2 * v[k] + (1 - b2) * g[k] ** 2
        mh = m[k] / (1 - b1 ** t)
        vh = v[k] / (1 - b2 ** t)
        p[k] = (p[k] - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
