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
