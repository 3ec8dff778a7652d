"""Small, self-contained workloads of single kernels for profiling (one process, one GPU):

    python -m lucky_droplets_b200.cases rhs --N 360 --precision f64 --calls 3

`rhs`: a plan, a seeded random cube spectrum, `calls` evaluations of the velocity RHS
(ld_velocity_rhs: curl, three strided passes, the fused z pass, the k-space update).
`mlp`: `calls` learned-interpolation inferences of 1e6 cell-ordered droplets (feature kernel and
tensor-core forward).  The state is a few GB at most, so an ncu capture of one launch
(`-k regex:<kernel> -s <calls - 1> -c 1`) ends by itself.
"""
import argparse


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


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["rhs", "mlp"])
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--calls", type=int, default=3)
    a = ap.parse_args(argv)
    flags = (rhs if a.case == "rhs" else mlp)(a.N, a.precision, a.calls)
    print(f"{a.case} N={a.N} {a.precision} calls={a.calls} status={flags}")


if __name__ == "__main__":
    main()
