"""Cell-list collision detection of droplets (no counterpart in the reference, whose droplets
never collide).  The pair rule is bit-exact FP64 - see ld_collide in include/ld.h."""
import ctypes
import math

from . import _lib
from ._lib import check, ptr, stream_ptr

TWO_PI = 2.0 * math.pi


def _torch():
    import torch
    return torch


def cell_size_for(radius, n=None, L=TWO_PI, wide_fraction=1e-4):
    """A cell size for radii spread like ``radius`` (array): twice the radius below which all but
    ``wide_fraction`` of the droplets lie, so that few droplets are wide, kept to at least 3 and
    at most about (4 n)^(1/3) cells per side."""
    import numpy as np
    r = np.asarray(radius, dtype=np.float64)
    n = int(n if n is not None else r.size)
    cell = 2.0 * float(np.quantile(r, 1.0 - wide_fraction)) if r.size else L / 3
    nc_max = max(3, int(round((4.0 * max(n, 1)) ** (1.0 / 3.0))))
    return min(max(cell, L / nc_max), L / 3)


class Collider:
    """Workspace for the collision search of up to ``nmax`` droplets with cells >= cell_size.
    Any cell size gives the same pairs; cells near the typical diameter (rather than the largest)
    test far fewer candidates when the radii spread widely, the few droplets wider than a cell
    searching further out."""

    def __init__(self, nmax, cell_size, L=TWO_PI, device=None, nbox=1):
        """nbox > 1: one collider for the droplets of nbox independent boxes of side L (cells keyed
        box-major; collide_boxes / cell_order_boxes take each droplet's box)."""
        torch = _torch()
        self.L = float(L)
        self.nc = max(1, int(math.floor(self.L / float(cell_size))))
        self.nmax = int(nmax)
        self.nbox = int(nbox)
        self.device = torch.device(device if device is not None else "cuda")
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(_lib.lib().ld_collider_create_boxes(ctypes.byref(h), self.nmax, self.nc, self.nbox))
        self._h = h
        self.count = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.box_counts = torch.zeros(self.nbox, dtype=torch.int64, device=self.device)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().ld_collider_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def collide(self, pos, radius, pairs=None, cap=None, stream=None):
        """Pairs (i, j), i < j, sorted, as an int32 (M, 2) tensor view; the device count is in
        ``self.count`` (reading it synchronises)."""
        torch = _torch()
        n = int(pos.shape[0])
        if pairs is None:
            cap = cap or max(1024, 4 * n)
            pairs = torch.empty((cap, 2), dtype=torch.int32, device=self.device)
        cap = int(pairs.shape[0])
        check(_lib.lib().ld_collide(self._h, ptr(pos), ptr(radius), n, self.L, ptr(pairs), cap, ptr(self.count),
                                    stream_ptr(stream)))
        m = int(self.count.item())
        if m > cap:
            raise RuntimeError(f"pair capacity {cap} exceeded ({m} colliding pairs)")
        return pairs[:m]

    def cell_order(self, pos, order=None, stream=None):
        """Permutation (int32) into cell order of the wrapped positions."""
        torch = _torch()
        n = int(pos.shape[0])
        if order is None:
            order = torch.empty(n, dtype=torch.int32, device=self.device)
        check(_lib.lib().ld_cell_order(self._h, ptr(pos), n, self.L, ptr(order), stream_ptr(stream)))
        return order

    def collide_boxes(self, pos, radius, box, pairs, stream=None):
        """Pairs of the droplets of every box (array indices, i < j, box order) into ``pairs``;
        the total in ``self.count``, the pairs per box in ``self.box_counts`` (on the device)."""
        n = int(pos.shape[0])
        check(_lib.lib().ld_collide_boxes(self._h, ptr(pos), ptr(radius), ptr(box), n, self.L, ptr(pairs),
                                          int(pairs.shape[0]), ptr(self.count), ptr(self.box_counts),
                                          stream_ptr(stream)))

    def cell_order_boxes(self, pos, box, order, stream=None):
        """Permutation (int32) into (box, cell) order."""
        check(_lib.lib().ld_cell_order_boxes(self._h, ptr(pos), ptr(box), int(pos.shape[0]), self.L, ptr(order),
                                             stream_ptr(stream)))
        return order

    def status(self, clear=True, stream=None):
        v = ctypes.c_uint32()
        check(_lib.lib().ld_collider_status(self._h, ctypes.byref(v), int(bool(clear)), stream_ptr(stream)))
        return v.value


def main(argv=None):
    """Time the collision search alone on seeded droplets (uniform positions, lognormal radii
    r = 0.002 2pi exp(0.3 Z); cells of 2 r_max by default: about 5 droplets per cell at 1e6
    droplets; --cell sets the cell size).

        python -m lucky_droplets_b200.collide [--n 1000000] [--calls 20] [--cell C]
    """
    import argparse
    import json
    import numpy as np
    torch = _torch()
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--calls", type=int, default=20)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cell", type=float, default=None)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    pos = torch.as_tensor(rng.uniform(0, TWO_PI, (a.n, 3))).cuda()
    rad_np = 0.002 * TWO_PI * np.exp(0.3 * rng.standard_normal(a.n))
    rad = torch.as_tensor(rad_np).cuda()
    col = Collider(a.n, a.cell or 2 * float(rad_np.max()))
    pairs = torch.empty((max(1024, 4 * a.n), 2), dtype=torch.int32, device="cuda")
    for _ in range(3):
        col.collide(pos, rad, pairs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.calls):
        check(_lib.lib().ld_collide(col._h, ptr(pos), ptr(rad), a.n, col.L, ptr(pairs), int(pairs.shape[0]),
                                    ptr(col.count), stream_ptr(None)))
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"n": a.n, "cells_per_side": col.nc, "wide": int((rad_np > 0.5 * col.L / col.nc).sum()),
                      "pairs": int(col.count.item()), "ms_per_call": e0.elapsed_time(e1) / a.calls}), flush=True)


if __name__ == "__main__":
    main()
