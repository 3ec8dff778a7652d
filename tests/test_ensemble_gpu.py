"""The ensemble as one multi-box batch (one launch per pass over all boxes, droplets of every box
in one set of arrays, one multi-box collider): graph replays equal eager steps, and every box
equals the same seed run alone as one ForcedDNS, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _ens(seed, **kw):
    from lucky_droplets_b200.ensemble import Ensemble
    return Ensemble(n_boxes=4, N=32, nd=(300, 2000), seed=seed, sort_every=2, **kw)


def test_graph_replay_equals_eager(torch):
    a, b = _ens(3), _ens(3)
    a.step_eager(1)
    a.capture(2)
    a.replay(3)
    b.step_eager(7)
    torch.cuda.synchronize()
    assert a.nstep == b.nstep == 7
    assert torch.equal(a.uk, b.uk)
    for j in range(a.nb):
        _, pa, va = a.box_state(j)
        _, pb, vb = b.box_state(j)
        assert np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert a.collision_counts() == b.collision_counts()
    assert int(a.collider.count.item()) == sum(a.collision_counts())
    # a replay from another phase of the re-sorting period gets a graph of its own
    a.step_eager(1)
    a.replay(2)
    b.step_eager(5)
    torch.cuda.synchronize()
    assert a.nstep == b.nstep == 12 and len(a.graphs) == 2
    assert torch.equal(a.uk, b.uk)
    for j in range(a.nb):
        assert np.array_equal(a.box_state(j)[1], b.box_state(j)[1])


def test_boxes_differ_and_counts_follow_the_seed(torch):
    from lucky_droplets_b200.ensemble import box_counts
    e = _ens(5)
    per_box = np.bincount(e.box.cpu().numpy(), minlength=4)
    assert list(per_box) == [int(c) for c in box_counts(4, 5, 300, 2000)]
    assert not torch.equal(e.uk[0], e.uk[1])


def test_box_equals_the_same_seed_run_alone(torch):
    """Box b of the batch ends in exactly the state of the same seed run alone (flow, droplets by
    index, collision count), after steps that include re-sorting and graph replays."""
    from lucky_droplets_b200.collide import Collider
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200.ensemble import box_counts
    from lucky_droplets_b200.init import init_flow, init_droplets
    seed, nb = 7, 4
    e = _ens(seed)
    e.step_eager(1)
    e.capture(2)
    e.replay(3)
    counts = box_counts(nb, seed, 300, 2000)
    coll = e.collision_counts()
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
        uk, pe, ve = e.box_state(b)
        assert torch.equal(uk, dns.uk[...])
        assert np.array_equal(pe, d.by_id(d.pos))
        assert np.array_equal(ve, d.by_id(d.vel))
        assert coll[b] == int(col.count.item())


def test_ensemble_autotune_and_status(torch):
    e = _ens(9)
    table = e.autotune(steps_per_graph=(3, 4), trial_graphs=1)
    assert [r["steps_per_graph"] for r in table] == [3, 4]
    assert e.steps_per_graph in (3, 4)
    e.run(6)
    assert e.check() == 0
    assert all(c in (0, 1, 2, 3) for c in e.fft_tuning["choice"])
