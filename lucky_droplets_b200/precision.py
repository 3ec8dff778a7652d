"""Precision check: FP32 fields and transforms (FP64 droplet positions, FP64 forcing and energy
reductions) against an FP64 run of the same seed on the GPU.

Default: 512^3 (nu = 1e-3, dt = 5e-4), 4e6 droplets with lognormal radii and tricubic
interpolation, 1000 steps, a report every 50 steps:
  velocity relative L2 error  ||u32 - u64|| / ||u64||  (spectral, equal to the physical one)
  shell spectrum              max over shells with E64 > 1e-12 E_total of |E32 / E64 - 1|
  droplet position drift      max and RMS |x32 - x64| (minimum image), droplets matched by id

    python -m lucky_droplets_b200.precision [--N 512] [--nd 4000000] [--steps 1000] [--every 50]
"""
import argparse
import json
import time

import numpy as np

from .dns import ForcedDNS, Droplets
from .init import init_flow, init_droplets
from .spectral import TWO_PI


def _torch():
    import torch
    return torch


def build(N, nu, dt, precision, nd, seed, interp):
    dns = ForcedDNS.config(N, nu, dt, eps=0.1, kf=2, precision=precision)
    init_flow(dns, seed)
    d = None
    if nd > 0:
        pos, tau, radius = init_droplets(nd, seed, "lognormal_r", nu=nu)
        d = Droplets(dns.plan, pos, np.zeros((nd, 3)), tau, method=interp, g=0.1, radius=radius)
        u = dns.velocity()
        d.vel.copy_(d.gather(u))
        del u
        dns.attach(d)
    return dns, d


def compare(a, b, da, db):
    """Errors of the FP32 run a against the FP64 run b (device reductions, host scalars)."""
    torch = _torch()
    ua = a.uk.to(torch.complex128)
    err = float(torch.linalg.norm(ua - b.uk) / torch.linalg.norm(b.uk))
    ea, eb = a.energy_spectrum(), b.energy_spectrum()
    sel = eb > 1e-12 * eb.sum()
    spec = float(np.abs(ea[sel] / eb[sel] - 1.0).max())
    out = {"step": a.nstep, "t": a.t, "velocity_rel_l2": err, "spectrum_max_rel": spec,
           "energy32": float(ea.sum()), "energy64": float(eb.sum())}
    if da is not None:
        dx = da.pos - db.pos  # both keep droplets in id order (no re-sorting here)
        dx = torch.remainder(dx + np.pi, TWO_PI) - np.pi
        r = torch.linalg.norm(dx, dim=1)
        out["position_drift_max"] = float(r.max())
        out["position_drift_rms"] = float(torch.sqrt((r * r).mean()))
        out["velocity_rel_l2_droplets"] = float(torch.linalg.norm(da.vel.double() - db.vel) / torch.linalg.norm(db.vel))
    return out


def main(argv=None):
    torch = _torch()
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=512)
    ap.add_argument("--nu", type=float, default=1e-3)
    ap.add_argument("--dt", type=float, default=5e-4)
    ap.add_argument("--nd", type=int, default=4_000_000)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--interp", default="tricubic")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    r32, d32 = build(a.N, a.nu, a.dt, "f32", a.nd, a.seed, a.interp)
    r64, d64 = build(a.N, a.nu, a.dt, "f64", a.nd, a.seed, a.interp)
    rows = [compare(r32, r64, d32, d64)]
    for k in range(a.steps // a.every):
        r32.step(a.every)
        r64.step(a.every)
        r32.check()
        r64.check()
        rows.append(compare(r32, r64, d32, d64))
        print(json.dumps(rows[-1]), flush=True)
    summary = {"N": a.N, "nu": a.nu, "dt": a.dt, "n_droplets": a.nd, "steps": a.steps, "every": a.every,
               "interp": a.interp, "wall_s": time.perf_counter() - t0,
               "final": rows[-1], "max_velocity_rel_l2": max(r["velocity_rel_l2"] for r in rows),
               "max_spectrum_rel": max(r["spectrum_max_rel"] for r in rows)}
    if a.nd:
        summary["max_position_drift"] = max(r["position_drift_max"] for r in rows)
    print(json.dumps({"summary": summary}), flush=True)


if __name__ == "__main__":
    main()
