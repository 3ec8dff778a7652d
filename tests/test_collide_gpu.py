"""Cell-list collision detection on the GPU against the bit-exact FP64 CPU rule
(oracle/collide_np.py), and the project's radix sort against a stable argsort.  Also checks that
two calls on the same input give the identical pair list (deterministic order)."""
import ctypes

import numpy as np
import pytest

from oracle import collide_np as K

pytestmark = pytest.mark.gpu
TWO_PI = 2 * np.pi


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def gpu_pairs(torch, pos, rad, cell, cap=200000):
    from lucky_droplets_b200.collide import Collider
    c = Collider(max(1, pos.shape[0]), cell)
    p = torch.as_tensor(pos).cuda().contiguous()
    r = torch.as_tensor(rad).cuda().contiguous()
    out = c.collide(p, r, cap=cap).cpu().numpy().astype(np.int64)
    # the device order is deterministic (by cell); compare as a canonical (i, j)-sorted list
    assert (out[:, 0] < out[:, 1]).all() if len(out) else True
    out = out[np.lexsort((out[:, 1], out[:, 0]))] if len(out) else out
    return out, c


@pytest.mark.parametrize("n,scale,seed", [(20000, 1.0, 0), (50000, 0.5, 1), (5000, 3.0, 2)])
def test_pairs_bit_exact(torch, n, scale, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-2.0, TWO_PI + 2.0, (n, 3))  # unwrapped positions, as the reference keeps them
    rad = 0.01 * scale * np.exp(0.3 * rng.standard_normal(n))
    cell = 2 * rad.max()
    got, _ = gpu_pairs(torch, pos, rad, cell)
    ref = K.collide(pos, rad, cell)
    assert got.shape == ref.shape and np.array_equal(got, ref)


def test_edge_cases(torch):
    rng = np.random.default_rng(5)
    # empty and single droplet
    got, _ = gpu_pairs(torch, np.zeros((0, 3)), np.zeros(0), 0.1)
    assert got.shape == (0, 2)
    got, _ = gpu_pairs(torch, np.ones((1, 3)), np.ones(1) * 0.1, 0.2)
    assert got.shape == (0, 2)
    # everything in one cell, and fewer than three cells per side (neighbour cells repeat)
    pos = rng.uniform(0, 0.3, (400, 3))
    rad = np.full(400, 0.05)
    for cell in (2.5, 4.0, 10.0):
        got, _ = gpu_pairs(torch, pos, rad, cell)
        ref = K.collide_bruteforce(pos, rad)
        assert np.array_equal(got, ref)
    # periodic images across the box faces
    pos = np.array([[0.001, 3.0, 3.0], [TWO_PI - 0.001, 3.0, 3.0], [3.0, 3.0, TWO_PI - 1e-4], [3.0, 3.0, 1e-4]])
    rad = np.full(4, 0.01)
    got, _ = gpu_pairs(torch, pos, rad, 0.5)
    assert np.array_equal(got, K.collide_bruteforce(pos, rad))


def test_capacity_overflow_reported(torch):
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200.collide import Collider
    rng = np.random.default_rng(9)
    pos = rng.uniform(0, 0.5, (300, 3))
    rad = np.full(300, 0.05)
    ref = K.collide(pos, rad, 0.2)
    c = Collider(300, 0.2)
    with pytest.raises(RuntimeError, match="capacity"):
        c.collide(torch.as_tensor(pos).cuda(), torch.as_tensor(rad).cuda(), cap=len(ref) // 2)
    assert c.status() & _lib.STATUS_PAIR_OVERFLOW
    assert int(c.count.item()) == len(ref)


@pytest.mark.parametrize("n,bits", [(1, 8), (4095, 12), (100000, 18), (300001, 24)])
def test_radix_sort_stable(torch, n, bits):
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, ptr, stream_ptr
    from lucky_droplets_b200.collide import Collider
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint32)
    keys[: n // 3] = keys[0]  # many equal keys: stability matters
    vals = np.arange(n, dtype=np.uint32)
    c = Collider(n, 1.0)
    k = torch.as_tensor(keys.astype(np.int64)).to(torch.int32).cuda().contiguous()
    v = torch.as_tensor(vals.astype(np.int64)).to(torch.int32).cuda().contiguous()
    check(_lib.lib().ld_radix_sort_u32(c._h, ptr(k), ptr(v), n, bits, stream_ptr()))
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k.cpu().numpy().astype(np.uint32), keys[order])
    assert np.array_equal(v.cpu().numpy().astype(np.uint32), vals[order])


def test_cell_keys_match_cpu(torch):
    from lucky_droplets_b200 import _lib
    rng = np.random.default_rng(3)
    n = 30000
    pos = rng.uniform(-1, 7, (n, 3))
    rad = np.full(n, 0.02)
    _, c = gpu_pairs(torch, pos, rad, 0.04)
    kp = ctypes.c_void_p()
    ip = ctypes.c_void_p()
    assert _lib.lib().ld_collider_sorted(c._h, ctypes.byref(kp), ctypes.byref(ip)) == 0
    import torch as T
    keys = np.empty(n, np.uint32)
    ids = np.empty(n, np.uint32)
    # copy device arrays through torch (no host pointer access needed)
    kt = T.empty(n, dtype=T.int32, device="cuda")
    it = T.empty(n, dtype=T.int32, device="cuda")
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    T.cuda.synchronize()
    assert cudart.cudaMemcpy(kt.data_ptr(), kp.value, 4 * n, 3) == 0  # device to device
    assert cudart.cudaMemcpy(it.data_ptr(), ip.value, 4 * n, 3) == 0
    keys[:] = kt.cpu().numpy().astype(np.uint32)
    ids[:] = it.cpu().numpy().astype(np.uint32)
    _, ref_keys = K.cell_keys(pos, K.cell_count(TWO_PI, 0.04))
    order = np.argsort(ref_keys, kind="stable")
    assert np.array_equal(ids, order.astype(np.uint32))
    assert np.array_equal(keys, ref_keys[order].astype(np.uint32))


def test_pair_order_is_deterministic(torch):
    from lucky_droplets_b200.collide import Collider
    rng = np.random.default_rng(21)
    n = 40000
    pos = rng.uniform(0, TWO_PI, (n, 3))
    rad = 0.02 * np.exp(0.3 * rng.standard_normal(n))
    c = Collider(n, 2 * rad.max())
    p, r = torch.as_tensor(pos).cuda(), torch.as_tensor(rad).cuda()
    a = c.collide(p, r, cap=100000).cpu().numpy()
    b = c.collide(p, r, cap=100000).cpu().numpy()
    assert np.array_equal(a, b)


def _contact_pairs(rng, m, rel_gap):
    r = rng.uniform(0.005, 0.02, (m, 2))
    rs = r.sum(axis=1)
    d = rng.standard_normal((m, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    sign = np.where(np.arange(m) % 2 == 0, -1.0, 1.0)  # inside / outside by rel_gap
    sep = rs * (1.0 + sign * rel_gap)
    a = rng.uniform(0, TWO_PI, (m, 3))
    a[: m // 4, 0] = rng.uniform(-1e-3, 1e-3, m // 4)  # straddle the x = 0 face
    b = a + d * sep[:, None]
    pos = np.empty((2 * m, 3))
    pos[0::2], pos[1::2] = a, b
    rad = np.empty(2 * m)
    rad[0::2], rad[1::2] = r[:, 0], r[:, 1]
    return pos, rad


@pytest.mark.parametrize("rel_gap", [1e-7, 1e-10, 1e-13])
def test_contact_distance_boundary(torch, rel_gap):
    """Pairs placed at the contact distance (1 -/+ rel_gap) rs, a quarter across the x = 0 face:
    the FP32 pre-test keeps every pair the FP64 rule accepts (the list is bit-exact)."""
    rng = np.random.default_rng(int(-np.log10(rel_gap)))
    pos, rad = _contact_pairs(rng, 20000, rel_gap)
    cell = 2 * rad.max()
    got, _ = gpu_pairs(torch, pos, rad, cell)
    ref = K.collide(pos, rad, cell)
    assert len(ref) >= 5000  # the inside half, mostly
    assert got.shape == ref.shape and np.array_equal(got, ref)


def test_dense_cluster_many_partners(torch):
    """About 7 partners per droplet (nc >= 3): the emitted list still equals the FP64 rule's."""
    rng = np.random.default_rng(21)
    pos = rng.uniform(0.0, 1.0, (8000, 3))
    rad = np.full(8000, 0.03)
    got, _ = gpu_pairs(torch, pos, rad, 0.06, cap=400000)
    ref = K.collide(pos, rad, 0.06)
    assert len(ref) > 20000
    assert got.shape == ref.shape and np.array_equal(got, ref)


def test_crowded_cell_beside_sparse_cells(torch):
    """One cell holding 2500 droplets among sparse cells (nc >= 3): the counting sort's
    large-cell path and partner lists far longer than the recorded KEEP, against the FP64 rule;
    two calls give the identical list."""
    from lucky_droplets_b200.collide import Collider
    rng = np.random.default_rng(33)
    dense = rng.uniform(1.1, 1.4, (2500, 3))
    sparse = rng.uniform(0.0, TWO_PI, (6000, 3))
    pos = np.concatenate([sparse[:3000], dense, sparse[3000:]])
    rad = np.full(pos.shape[0], 0.006)
    cell = 0.5  # 12 cells per side
    got, _ = gpu_pairs(torch, pos, rad, cell)
    ref = K.collide(pos, rad, cell)
    assert len(ref) > 100
    assert got.shape == ref.shape and np.array_equal(got, ref)
    c = Collider(pos.shape[0], cell)
    p, r = torch.as_tensor(pos).cuda(), torch.as_tensor(rad).cuda()
    a = c.collide(p, r, cap=100000).cpu().numpy()
    b = c.collide(p, r, cap=100000).cpu().numpy()
    assert np.array_equal(a, b)


def test_partners_beyond_the_record_are_searched_again(torch):
    """About 100 partners per droplet, far beyond the sixteen the count pass records: every
    droplet's pairs come from the emit pass's second search, and the list equals the FP64
    rule's."""
    rng = np.random.default_rng(44)
    pos = rng.uniform(2.0, 2.5, (3000, 3))
    rad = np.full(3000, 0.05)
    got, _ = gpu_pairs(torch, pos, rad, 0.1, cap=400000)
    ref = K.collide(pos, rad, 0.1)
    assert len(ref) > 100000
    assert got.shape == ref.shape and np.array_equal(got, ref)


def test_multi_box_collider_matches_each_box_alone():
    """One multi-box collider over the droplets of several boxes (cells keyed box-major) finds, box
    by box, exactly the pairs the FP64 rule gives for that box alone, counts them per box, and
    never pairs droplets of different boxes; the cell order keeps the boxes contiguous."""
    import torch
    from lucky_droplets_b200.collide import Collider
    from oracle import collide_np as K
    rng = np.random.default_rng(17)
    sizes = [3000, 0, 1200, 4500]
    pos = [rng.uniform(-0.5, 2 * np.pi + 0.5, (n, 3)) for n in sizes]
    rad = [0.02 + 0.03 * rng.random(n) for n in sizes]
    box = np.concatenate([np.full(n, j, np.int32) for j, n in enumerate(sizes)])
    P = torch.as_tensor(np.concatenate(pos)).cuda()
    R = torch.as_tensor(np.concatenate(rad)).cuda()
    Bx = torch.as_tensor(box).cuda()
    n = int(P.shape[0])
    for cell in (0.11, 3.0):  # nc >= 3, and nc < 3
        col = Collider(n, cell, nbox=len(sizes))
        pairs = torch.empty((4 * n, 2), dtype=torch.int32, device="cuda")
        col.collide_boxes(P, R, Bx, pairs)
        m = int(col.count.item())
        got = pairs[:m].cpu().numpy().astype(np.int64)
        assert (box[got[:, 0]] == box[got[:, 1]]).all()
        off = np.concatenate([[0], np.cumsum(sizes)])
        bc = col.box_counts.cpu().numpy()
        for j, nj in enumerate(sizes):
            sel = got[box[got[:, 0]] == j] - off[j]
            sel = np.sort(sel, axis=1)
            sel = sel[np.lexsort((sel[:, 1], sel[:, 0]))]
            ref = K.collide(pos[j], rad[j], cell) if nj else np.zeros((0, 2), np.int64)
            assert np.array_equal(sel, ref), (cell, j)
            assert bc[j] == len(ref)
        order = torch.empty(n, dtype=torch.int32, device="cuda")
        col.cell_order_boxes(P, Bx, order)
        ob = box[order.cpu().numpy()]
        assert (np.diff(ob) >= 0).all()


@pytest.mark.parametrize("case", ["lognormal", "equal_radii", "huge_droplet"])
def test_narrow_cells_find_every_pair(torch, case):
    """Cells narrower than twice the largest radius: droplets with 2 r above the cell width search
    the cells within 2 r of them for the partners the neighbour cells leave out.  The list equals
    the FP64 rule's (computed with cells of 2 r_max), is the same from call to call, and matches
    the oracle's restatement of the narrow-cell search."""
    from lucky_droplets_b200.collide import Collider
    rng = np.random.default_rng({"lognormal": 61, "equal_radii": 62, "huge_droplet": 63}[case])
    n = 30000
    pos = rng.uniform(-1.0, TWO_PI + 1.0, (n, 3))
    if case == "lognormal":
        rad = 0.02 * np.exp(0.5 * rng.standard_normal(n))
    elif case == "equal_radii":
        rad = np.full(n, 0.03)
    else:
        rad = 0.01 + 0.01 * rng.random(n)
        rad[[5, 900, 20000]] = [1.1, 0.4, 0.4]
    # cells of 2 r_max; with the droplet of radius 1.1 (fewer than three cells per side: an
    # all-pairs search) the oracle's narrow-cell restatement, pinned to all pairs on the CPU
    ref = (K.collide(pos, rad, 2 * rad.max()) if case != "huge_droplet"
           else K.collide_wide(pos, rad, 4 * np.median(rad)))
    assert len(ref) > 500
    p, r = torch.as_tensor(pos).cuda(), torch.as_tensor(rad).cuda()
    for cell in (rad.max(), 1.5 * np.median(rad), 1.1 * np.median(rad)):
        nc = K.cell_count(TWO_PI, cell)
        assert nc >= 3 and (rad > 0.5 * TWO_PI / nc).any()
        got, c = gpu_pairs(torch, pos, rad, cell, cap=4 * len(ref))
        assert got.shape == ref.shape and np.array_equal(got, ref), cell
        a = c.collide(p, r, cap=4 * len(ref)).cpu().numpy()
        b = c.collide(p, r, cap=4 * len(ref)).cpu().numpy()
        assert np.array_equal(a, b)
    assert np.array_equal(K.collide_wide(pos[:2000], rad[:2000], 1.5 * np.median(rad)),
                          gpu_pairs(torch, pos[:2000], rad[:2000], 1.5 * np.median(rad))[0])


def test_narrow_cells_multi_box_and_overflow(torch):
    """Narrow cells in a multi-box collider: wide droplets search only their own box, the per-box
    counts include their pairs; a capacity below the total raises the overflow flag."""
    from lucky_droplets_b200.collide import Collider
    rng = np.random.default_rng(71)
    sizes = [4000, 2500, 0, 6000]
    pos = [rng.uniform(0.0, TWO_PI, (m, 3)) for m in sizes]
    rad = [0.04 * np.exp(0.6 * rng.standard_normal(m)) for m in sizes]
    box = np.concatenate([np.full(m, j, np.int32) for j, m in enumerate(sizes)])
    P = torch.as_tensor(np.concatenate(pos)).cuda()
    R = torch.as_tensor(np.concatenate(rad)).cuda()
    Bx = torch.as_tensor(box).cuda()
    n = int(P.shape[0])
    cell = 2.0 * float(np.median(np.concatenate(rad)))
    col = Collider(n, cell, nbox=len(sizes))
    pairs = torch.empty((8 * n, 2), dtype=torch.int32, device="cuda")
    col.collide_boxes(P, R, Bx, pairs)
    m = int(col.count.item())
    got = pairs[:m].cpu().numpy().astype(np.int64)
    assert (box[got[:, 0]] == box[got[:, 1]]).all()
    off = np.concatenate([[0], np.cumsum(sizes)])
    bc = col.box_counts.cpu().numpy()
    total = 0
    for j, nj in enumerate(sizes):
        sel = np.sort(got[box[got[:, 0]] == j] - off[j], axis=1)
        sel = sel[np.lexsort((sel[:, 1], sel[:, 0]))] if len(sel) else sel.reshape(0, 2)
        ref = K.collide(pos[j], rad[j], 2 * rad[j].max()) if nj else np.zeros((0, 2), np.int64)
        assert np.array_equal(sel, ref), j
        assert bc[j] == len(ref)
        total += len(ref)
    assert m == total > 100
    # overflow: the count is still the total, the flag is raised, nothing is written past cap
    small = torch.full((total // 2, 2), -7, dtype=torch.int32, device="cuda")
    guard = torch.full((64, 2), -7, dtype=torch.int32, device="cuda")
    buf = torch.cat([small, guard])
    col.status()
    col.collide_boxes(P, R, Bx, buf[: total // 2])
    assert int(col.count.item()) == total
    assert col.status() & _lib_status_overflow()
    assert (buf[total // 2:] == -7).all()


def _lib_status_overflow():
    from lucky_droplets_b200 import _lib
    return _lib.STATUS_PAIR_OVERFLOW
