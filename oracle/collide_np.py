"""CPU oracle for cell-list collision detection (no counterpart in the reference).

TEST INFRASTRUCTURE ONLY: used by tests and bench.py's CPU legs, never by the product.

Rule (the GPU kernel evaluates the same FP64 operations in the same order, without FMA, so the
pair list is bit-exact given identical positions and radii):
  * wrapped position  p = x - L * floor(x / L);
  * cell width        cw = L / nc with nc = floor(L / cell_size) (cell_size = 2 r_max; narrower
                      cells: collide_wide);
  * cell index        c = min(int(p / cw), nc - 1) per axis, key = (cx * nc + cy) * nc + cz;
  * minimum image     d = p_i - p_j; d -= L if d > L/2; d += L if d < -L/2;
  * colliding pair    (dx*dx + dy*dy) + dz*dz < (r_i + r_j) * (r_i + r_j), reported once as
                      (i, j) with i < j (droplet ids), the list sorted by (i, j).
"""
import numpy as np

TWO_PI = 2.0 * np.pi


def cell_count(L, cell_size):
    nc = int(np.floor(L / cell_size))
    return max(nc, 1)


def wrap(x, L=TWO_PI):
    return x - L * np.floor(x / L)


def cell_keys(pos, nc, L=TWO_PI):
    """Per-droplet cell index triple and flat key."""
    p = wrap(pos, L)
    cw = L / nc
    c = np.minimum((p / cw).astype(np.int64), nc - 1)
    return c, (c[:, 0] * nc + c[:, 1]) * nc + c[:, 2]


def min_image(d, L=TWO_PI):
    h = L / 2
    d = np.where(d > h, d - L, d)
    return np.where(d < -h, d + L, d)


def collide(pos, radius, cell_size, L=TWO_PI):
    """Colliding pairs (M, 2) int64 sorted by (i, j), i < j."""
    n = pos.shape[0]
    nc = cell_count(L, cell_size)
    c, key = cell_keys(pos, nc, L)
    p = wrap(pos, L)
    order = np.argsort(key, kind="stable")
    skey = key[order]
    starts = np.searchsorted(skey, np.arange(nc ** 3), side="left")
    ends = np.searchsorted(skey, np.arange(nc ** 3), side="right")
    offs = [(a, b, d) for a in (-1, 0, 1) for b in (-1, 0, 1) for d in (-1, 0, 1)]
    out = []
    for (a, b, d) in offs:
        # neighbour cell of every droplet
        nb = ((np.mod(c[:, 0] + a, nc) * nc + np.mod(c[:, 1] + b, nc)) * nc + np.mod(c[:, 2] + d, nc))
        cnt = ends[nb] - starts[nb]
        tot = int(cnt.sum())
        if tot == 0:
            continue
        ii = np.repeat(np.arange(n), cnt)
        base = np.repeat(starts[nb], cnt)
        within = np.arange(tot) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        jj = order[base + within]
        m = jj > ii
        ii, jj = ii[m], jj[m]
        dx = min_image(p[ii, 0] - p[jj, 0], L)
        dy = min_image(p[ii, 1] - p[jj, 1], L)
        dz = min_image(p[ii, 2] - p[jj, 2], L)
        d2 = (dx * dx + dy * dy) + dz * dz
        rs = radius[ii] + radius[jj]
        hit = d2 < rs * rs
        out.append(np.stack([ii[hit], jj[hit]], axis=1))
    if not out:
        return np.zeros((0, 2), np.int64)
    pairs = np.concatenate(out)
    # a pair can appear from more than one neighbour offset only when nc < 3
    pairs = np.unique(pairs, axis=0)
    return pairs


def collide_wide(pos, radius, cell_size, L=TWO_PI):
    """The same pair list with cells of any width (the GPU's search when cell_size < 2 r_max):
    the 27-cell search keeps the pairs with r_i + r_j <= cw; a pair with r_i + r_j > cw has a
    droplet with 2 r > cw ("wide"), and its owner (the larger radius; equal radii: the smaller
    cell-sorted index) finds it among the cells within R = floor(2 r / cw) + 1 of its own (all
    nc when 2 R + 1 >= nc).  Needs nc >= 3.  Returns (M, 2) int64 sorted by (i, j)."""
    n = pos.shape[0]
    nc = cell_count(L, cell_size)
    assert nc >= 3
    cw = L / nc
    c, key = cell_keys(pos, nc, L)
    p = wrap(pos, L)
    order = np.argsort(key, kind="stable")
    rank = np.empty(n, np.int64)
    rank[order] = np.arange(n)
    skey = key[order]
    starts = np.searchsorted(skey, np.arange(nc ** 3), side="left")
    ends = np.searchsorted(skey, np.arange(nc ** 3), side="right")
    near = collide(pos, radius, cell_size, L)
    if len(near):
        keep = ~(radius[near[:, 0]] + radius[near[:, 1]] > cw)
        near = near[keep]
    out = [near]
    wide = np.nonzero(radius > 0.5 * cw)[0]
    for s in wide:
        R = int(np.floor((radius[s] + radius[s]) / cw))
        R = R + 1 if R < nc else nc
        ax = nc if 2 * R + 1 >= nc else 2 * R + 1
        rng = [np.arange(nc) if ax == nc else np.mod(c[s, a] - R + np.arange(ax), nc) for a in range(3)]
        cells = ((rng[0][:, None, None] * nc + rng[1][None, :, None]) * nc + rng[2][None, None, :]).ravel()
        cand = np.concatenate([order[starts[k]:ends[k]] for k in cells])
        cand = cand[cand != s]
        rs = radius[s] + radius[cand]
        cand, rs = cand[rs > cw], rs[rs > cw]
        rt = radius[cand]
        owned_by_t = (rt > 0.5 * cw) & ((rt > radius[s]) | ((rt == radius[s]) & (rank[cand] < rank[s])))
        cand, rs = cand[~owned_by_t], rs[~owned_by_t]
        dx = min_image(p[s, 0] - p[cand, 0], L)
        dy = min_image(p[s, 1] - p[cand, 1], L)
        dz = min_image(p[s, 2] - p[cand, 2], L)
        hit = (dx * dx + dy * dy) + dz * dz < rs * rs
        t = cand[hit]
        out.append(np.stack([np.minimum(s, t), np.maximum(s, t)], axis=1))
    pairs = np.concatenate(out).astype(np.int64) if out else np.zeros((0, 2), np.int64)
    if len(pairs):
        pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]
    return pairs


def collide_bruteforce(pos, radius, L=TWO_PI):
    """All-pairs reference for small n (same FP64 rule)."""
    p = wrap(pos, L)
    n = p.shape[0]
    ii, jj = np.triu_indices(n, 1)
    dx = min_image(p[ii, 0] - p[jj, 0], L)
    dy = min_image(p[ii, 1] - p[jj, 1], L)
    dz = min_image(p[ii, 2] - p[jj, 2], L)
    d2 = (dx * dx + dy * dy) + dz * dz
    rs = radius[ii] + radius[jj]
    hit = d2 < rs * rs
    return np.stack([ii[hit], jj[hit]], axis=1).astype(np.int64)
