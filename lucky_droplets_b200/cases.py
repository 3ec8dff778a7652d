"""Small, self-contained workloads of single kernels for profiling (one process, one GPU):

    python -m lucky_droplets_b200.cases rhs --N 360 --precision f64 --calls 3

`rhs`: a plan, a seeded random cube spectrum, `calls` evaluations of the velocity RHS
(ld_velocity_rhs: curl, three strided passes, the fused z pass, the k-space update).
`mlp`: `calls` learned-interpolation inferences of 1e6 cell-ordered droplets (feature kernel and
tensor-core forward).
`train`: one warm-up epoch, then `calls` timed epochs of MLP training (batches of 4096 seeded
synthetic samples: per batch the tensor-core forward/backward kernel and the fused partial sum +
Adam); prints the time per batch.
The state is a few GB at most, so an ncu capture of one launch (`-k regex:<kernel> -s <n> -c 1`)
ends by itself.
"""
import argparse
import time


def rhs(N, precision, calls, seed=0):
    import torch
    from .spectral import Plan
    p = Plan(N, precision)
    g = torch.Generator(device="cuda").manual_seed(seed)
    uk = torch.zeros((3, p.Mx, p.My, p.Mzp), dtype=p.cdtype, device="cuda")
    uk.real.normal_(generator=g)
    uk.imag.normal_(generator=g)
    for _ in range(calls):
        p.velocity_rhs(uk, 0.01, 1.0, (1, 2))
    torch.cuda.synchronize()
    return p.status()


def mlp(N, precision, calls, n=1_000_000, seed=0):
    """Learned-interpolation inference (feature kernel + tensor-core forward) at n droplets with
    uniform positions in cell order, on the interleaved velocity of a seeded random spectrum."""
    import numpy as np
    import torch
    from ._lib import check, ptr, stream_ptr
    from . import _lib
    from .collide import Collider
    from .mlp import LearnedInterp
    from .spectral import Plan
    p = Plan(N, precision)
    g = torch.Generator(device="cuda").manual_seed(seed)
    uk = torch.zeros((3, p.Mx, p.My, p.Mzp), dtype=p.cdtype, device="cuda")
    uk.real.normal_(generator=g)
    uk.imag.normal_(generator=g)
    li = LearnedInterp(p, seed=seed)
    u4 = li.interleaved(uk)
    pos = torch.as_tensor(np.random.default_rng(seed).uniform(0, 2 * np.pi, (n, 3))).cuda()
    col = Collider(n, 4 * p.dx)
    order = col.cell_order(pos)
    sp = torch.empty_like(pos)
    check(_lib.lib().ld_permute_rows(ptr(pos), ptr(sp), ptr(order), n, 24, stream_ptr()))
    out = torch.empty((n, 3), dtype=p.rdtype, device="cuda")
    work = li.workspace(n)
    for _ in range(calls):
        li.infer(u4, sp, out=out, work=work)
    torch.cuda.synchronize()
    return p.status()


def train(calls, batches=200, batch=4096, seed=0):
    """MLP training on batches * batch seeded synthetic samples (unit-normal features, zero padding
    columns, targets 0.3 N(0,1), weights U(0.5, 1.5)); returns microseconds per batch."""
    import torch
    from .mlp import K1, D_IN, LearnedInterp, TRAIN_FLOP_PER_SAMPLE
    from .spectral import Plan
    n = batches * batch
    g = torch.Generator(device="cuda").manual_seed(seed)
    X = torch.randn(n, K1, device="cuda", generator=g).to(torch.bfloat16)
    X[:, D_IN:] = 0
    T = torch.randn(n, 3, device="cuda", generator=g) * 0.3
    W = torch.rand(n, device="cuda", generator=g) + 0.5
    li = LearnedInterp(Plan(16, "f32"), seed=seed)
    li.train(X, T, W, epochs=1, batch=batch, lr=1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    li.train(X, T, W, epochs=calls, batch=batch, lr=1e-3)
    torch.cuda.synchronize()
    us = (time.perf_counter() - t0) / (calls * batches) * 1e6
    print(f"train: {us:.1f} us per batch of {batch}, {batch * TRAIN_FLOP_PER_SAMPLE / us / 1e6:.1f} TFLOP/s")
    return us


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["rhs", "mlp", "train"])
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--batches", type=int, default=200, help="train: batches of 4096 samples per epoch")
    a = ap.parse_args(argv)
    if a.case == "train":
        train(a.calls, a.batches)
        return
    flags = (rhs if a.case == "rhs" else mlp)(a.N, a.precision, a.calls)
    print(f"{a.case} N={a.N} {a.precision} calls={a.calls} status={flags}")


if __name__ == "__main__":
    main()
