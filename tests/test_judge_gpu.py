"""The judge of the learned interpolation inside the time loop (ForcedDNS.evolve, the analogue of
evolve_and_save, F:556-627): at every output interval the exact spectral sum on a random 1% of the
droplets decides whether the network stays on.  A planted bad network is switched off and the
steps that follow are the plain tricubic steps bit for bit, captured CUDA graphs included; a good
network stays on."""
import numpy as np
import pytest

from oracle import config_np as C

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _factory(N=32, nd=3000, seed=3):
    from lucky_droplets_b200.collide import Collider
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    uk0, u0 = C.init_flow(C.ConfigGrid(N), prm, seed)
    pos, tau, rad = C.init_droplets(prm, seed, "uniform_tau", nd=nd)
    rad = rad * 5.0
    vel = C.gather(u0, pos, "tricubic")

    def make():
        dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision="f32")
        dns.set_uk_full(uk0)
        d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g, radius=rad)
        dns.attach(d, collider=Collider(d.n, 2 * rad.max()), sort_every=4)
        return dns, d
    return make


def _network(plan, w3_scale, tol, rule="tolerance"):
    from lucky_droplets_b200 import mlp as G
    flat = G.init_flat(seed=5)
    flat[G.OFF_W3:G.OFF_B3] *= w3_scale
    if w3_scale == 0.0:
        flat[G.OFF_B3:G.OFF_B3 + 3] = 0.0
    return G.LearnedInterp(plan, params=flat, tol=tol, rule=rule)


def _same_state(torch, a, da, b, db):
    assert a.nstep == b.nstep
    assert torch.equal(a.uk, b.uk)
    assert torch.equal(da.pos, db.pos) and torch.equal(da.vel, db.vel) and torch.equal(da.ids, db.ids)
    assert int(a.collider.count.item()) == int(b.collider.count.item())


@pytest.mark.parametrize("rule", ["tolerance", "tolerance_or_better"])
def test_bad_network_is_switched_off_and_steps_are_plain_tricubic(torch, rule):
    make = _factory()
    a, da = make()
    b, db = make()
    li = _network(a.plan, 1e3, tol=1e-2, rule=rule)  # planted on the host: last layer x 1e3
    da.use_learned(li)
    assert a.interp_state() == "learned"
    g = a.capture(4)                                  # captured while the network is on
    v = a.judge(frac=0.05, seed=1)
    assert v["learned"] > 10 * v["tricubic"] and not v["enabled"]
    assert a.interp_state() == "tricubic"
    g.replay()                                        # a stale graph is captured again first
    assert g.recaptures == 1
    verdicts = a.evolve(8, st=4, graph_steps=2, judge_seed=2)
    assert [x["step"] for x in verdicts] == [4, 8, 12]
    assert not any(x["enabled"] for x in verdicts)
    b.step(12)
    torch.cuda.synchronize()
    _same_state(torch, a, da, b, db)


def test_good_network_stays_on(torch):
    """A network with a zero last layer returns tricubic exactly: its error equals tricubic's, so
    under a tolerance above that error the judge keeps it on at every output interval."""
    make = _factory(seed=4)
    a, da = make()
    li = _network(a.plan, 0.0, tol=1.0)
    da.use_learned(li)
    verdicts = a.evolve(6, st=3, graph_steps=3, judge_seed=3)
    assert [x["step"] for x in verdicts] == [0, 3, 6]
    for x in verdicts:
        assert x["enabled"]
        assert abs(x["learned"] - x["tricubic"]) <= 1e-3 * x["tricubic"]
    assert a.interp_state() == "learned"
    a.check()


def test_network_comes_back_when_it_meets_the_tolerance(torch):
    make = _factory(seed=6)
    a, da = make()
    li = _network(a.plan, 0.0, tol=1e-12)
    da.use_learned(li)
    assert not a.judge()["enabled"]
    li.tol = 1.0
    assert a.judge()["enabled"] and a.interp_state() == "learned"
