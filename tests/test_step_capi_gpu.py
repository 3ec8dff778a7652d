"""One-call stepping through the C ABI (ld_step, ld_ensemble_step): the same steps as the Python
steppers (ForcedDNS.step, Ensemble.step_eager), bit for bit - flow, droplets (by id), re-sorting
and collision counts."""
import ctypes

import numpy as np
import pytest

from oracle import config_np as C

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _state(torch, uk, ustar, acc, u4, pos, vel, tau, a1, radius, ids, box, method, g, sort_every, pairs, count,
           box_counts=None):
    from lucky_droplets_b200._lib import StepState
    n = int(pos.shape[0])
    keep = {"order": torch.empty(n, dtype=torch.int32, device="cuda"),
            "scratch": torch.empty(n * 24, dtype=torch.uint8, device="cuda")}
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    st = StepState(p(uk), p(ustar), p(acc), p(u4), n, p(pos), p(vel), p(tau), p(a1), p(radius), p(ids), p(box),
                   method, g, sort_every, p(keep["order"]), p(keep["scratch"]), p(pairs),
                   int(pairs.shape[0]) if pairs is not None else 0, p(count), p(box_counts), 0)
    return st, keep


def test_ld_step_equals_python_stepper(torch):
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, stream_ptr
    from lucky_droplets_b200.collide import Collider
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    uk0, u0 = C.init_flow(C.ConfigGrid(N), prm, seed=14)
    pos, tau, rad = C.init_droplets(prm, 14, "uniform_tau", nd=3000)
    rad = rad * 5.0
    vel = C.gather(u0, pos, "tricubic")
    runs = []
    for _ in range(2):
        dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision="f32")
        dns.set_uk_full(uk0)
        d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g, radius=rad)
        col = Collider(d.n, 2 * rad.max())
        dns.attach(d, collider=col, sort_every=3)
        runs.append((dns, d, col))
    (a, da, ca), (b, db, cb) = runs
    a.step(7)
    st, keep = _state(torch, b.uk, b.aux, b.acc, b.u_phys, db.pos, db.vel, db.tau, db.a1, db.radius, db.ids, None,
                      _lib.LD_INTERP["tricubic"], prm.g, 3, b.pairs, cb.count)
    check(_lib.lib().ld_step(b.plan.handle, cb._h, ctypes.byref(st), ctypes.byref(b.prm), 7, stream_ptr()))
    torch.cuda.synchronize()
    assert st.step == 7
    assert torch.equal(a.uk, b.uk)
    assert np.array_equal(da.by_id(da.pos), db.by_id(db.pos))
    assert np.array_equal(da.by_id(da.vel), db.by_id(db.vel))
    assert int(ca.count.item()) == int(cb.count.item()) > 0


def test_ld_ensemble_step_equals_ensemble(torch):
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, stream_ptr
    from lucky_droplets_b200.ensemble import Ensemble
    a = Ensemble(n_boxes=3, N=32, nd=(300, 2000), seed=4, sort_every=2)
    b = Ensemble(n_boxes=3, N=32, nd=(300, 2000), seed=4, sort_every=2)
    a.step_eager(5)
    st, keep = _state(torch, b.uk, b.aux, b.acc, b.u4, b.pos, b.vel, b.tau, b.a1, b.radius, b.dids, b.box,
                      b.method, b.g, 2, b.pairs, b.collider.count, b.collider.box_counts)
    check(_lib.lib().ld_ensemble_step(b.plan.handle, b.collider._h, ctypes.byref(st), ctypes.byref(b.prm), 5,
                                      stream_ptr()))
    torch.cuda.synchronize()
    assert torch.equal(a.uk, b.uk)
    for j in range(3):
        assert np.array_equal(a.box_state(j)[1], b.box_state(j)[1])
        assert np.array_equal(a.box_state(j)[2], b.box_state(j)[2])
    assert a.collision_counts() == b.collision_counts()


def test_one_call_steps_refuse_bad_state(torch):
    """A multi-box state through ld_step, and a missing collider for the re-sort, are refused with
    LD_ERR_ARG before anything runs."""
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200.ensemble import Ensemble
    from lucky_droplets_b200._lib import stream_ptr
    b = Ensemble(n_boxes=2, N=32, nd=(300, 600), seed=1, sort_every=2)
    st, keep = _state(torch, b.uk, b.aux, b.acc, b.u4, b.pos, b.vel, b.tau, b.a1, b.radius, b.dids, b.box,
                      b.method, b.g, 2, b.pairs, b.collider.count, b.collider.box_counts)
    L = _lib.lib()
    assert L.ld_step(b.plan.handle, b.collider._h, ctypes.byref(st), ctypes.byref(b.prm), 1, stream_ptr()) == -1
    assert L.ld_ensemble_step(b.plan.handle, None, ctypes.byref(st), ctypes.byref(b.prm), 1, stream_ptr()) == -1
    assert st.step == 0
