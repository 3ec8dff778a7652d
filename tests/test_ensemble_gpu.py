"""Ensemble of boxes advanced by CUDA-graph replays over several streams: bit-identical to the
same boxes stepped eagerly one after another, re-sorting and collisions included."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _ens(seed):
    from lucky_droplets_b200.ensemble import Ensemble
    return Ensemble(n_boxes=4, N=32, nd=(300, 2000), seed=seed, sort_every=2)


def test_graph_replay_equals_eager(torch):
    a, b = _ens(3), _ens(3)
    a.step_eager(1)
    a.capture(3, 2)
    a.replay(2)
    b.step_eager(7)
    torch.cuda.synchronize()
    for ba, bb in zip(a.boxes, b.boxes):
        assert ba.nstep == bb.nstep == 7
        assert torch.equal(ba.uk, bb.uk)
        da, db = ba.droplets, bb.droplets
        assert np.array_equal(da.by_id(da.pos), db.by_id(db.pos))
        assert np.array_equal(da.by_id(da.vel), db.by_id(db.vel))
        assert int(ba.collider.count.item()) == int(bb.collider.count.item())
    assert a.collision_counts() == b.collision_counts()


def test_boxes_differ_and_counts_follow_the_seed(torch):
    from lucky_droplets_b200.ensemble import box_counts
    e = _ens(5)
    assert [d.droplets.n for d in e.boxes] == [int(c) for c in box_counts(4, 5, 300, 2000)]
    assert not torch.equal(e.boxes[0].uk, e.boxes[1].uk)


def test_box_equals_the_same_seed_run_alone(torch):
    """Box b of an ensemble (boxes stepped together from CUDA graphs on several streams) ends in
    exactly the state of the same seed run alone as one ForcedDNS stepped eagerly: spectrum,
    droplets by id and the collision count, bit for bit."""
    from lucky_droplets_b200.collide import Collider
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200.ensemble import box_counts
    from lucky_droplets_b200.init import init_flow, init_droplets
    seed, nb = 7, 4
    e = _ens(seed)
    e.step_eager(1)
    e.capture(3, 2)
    e.replay(2)
    counts = box_counts(nb, seed, 300, 2000)
    for b in (0, 3):
        dns = ForcedDNS.config(32, 0.01, 2e-3, eps=0.1, kf=2, precision="f32")
        dns.plan.set_tuning(e.fft_tuning["choice"])
        init_flow(dns, seed + b)
        pos, tau, radius = init_droplets(int(counts[b]), seed + b, "uniform_tau")
        d = Droplets(dns.plan, pos, np.zeros((tau.shape[0], 3)), tau, method="trilinear", g=0.1, radius=radius)
        d.vel.copy_(d.gather(dns.velocity()))
        col = Collider(d.n, 2.0 * float(radius.max()))
        dns.attach(d, collider=col, sort_every=2)
        dns.step(7)
        torch.cuda.synchronize()
        box = e.boxes[b]
        db = box.droplets
        assert box.nstep == dns.nstep == 7
        assert torch.equal(box.uk, dns.uk)
        assert np.array_equal(db.by_id(db.pos), d.by_id(d.pos))
        assert np.array_equal(db.by_id(db.vel), d.by_id(d.vel))
        assert int(box.collider.count.item()) == int(col.count.item())
