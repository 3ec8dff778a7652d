"""Small, self-contained workloads of single kernels for profiling (one process, one GPU):

    python -m lucky_droplets_b200.cases rhs --N 360 --precision f64 --calls 3

`rhs`: a plan, a seeded random cube spectrum, `calls` evaluations of the velocity RHS
(ld_velocity_rhs: curl, three strided passes, the fused z pass, the k-space update).  The state
is a few GB at most, so an ncu capture of one launch (`-k regex:<kernel> -s <calls - 1> -c 1`)
ends by itself.
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


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["rhs"])
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--calls", type=int, default=3)
    a = ap.parse_args(argv)
    flags = rhs(a.N, a.precision, a.calls)
    print(f"{a.case} N={a.N} {a.precision} calls={a.calls} status={flags}")


if __name__ == "__main__":
    main()
