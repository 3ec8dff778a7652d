"""GPU DNS step against the reference (golden vectors from the reference's own run) and the
FP64 oracles: full_RHS velocity part, RK4 time loop, RK2 + integrating factor, shell spectrum."""
import numpy as np
import pytest

from oracle import reference_np as R
from oracle import config_np as C

pytestmark = pytest.mark.gpu

TOL = {"f32": 2e-5, "f64": 1e-12}


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("name", ["N16", "N32"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_velocity_rhs_matches_reference(torch, golden, name, prec):
    """ku of full_RHS (F:287-316) from the reference's own run, on its initial state."""
    from lucky_droplets_b200.spectral import Plan
    g = golden(name)
    N = int(g["N"])
    prm = R.ReferenceParams(N)
    p = Plan(N, prec)
    uk = p.to_cube(torch.as_tensor(g["uk0"]).to("cuda", p.cdtype).contiguous())
    ku = p.velocity_rhs(uk, prm.nu, prm.f0, prm.shell_no, visc=1.0)
    full = p.from_cube(ku).cpu().numpy()
    grid = R.Grid(N)
    ref = g["rhs_ku"] * grid.dealias  # the reference keeps roundoff outside the mask
    assert rel(full, ref) < TOL[prec]


@pytest.mark.parametrize("N", [64, 128, 256, 96, 360])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_velocity_rhs_matches_oracle(torch, N, prec):
    """The same RHS at larger N against the FP64 restatement, on a seeded initial field."""
    from lucky_droplets_b200.spectral import Plan
    prm = C.ConfigParams(N=N, nu=2.5e-3, dt=1e-3)
    grid = C.ConfigGrid(N)
    uk0, _ = C.init_flow(grid, prm, seed=N)
    p = Plan(N, prec)
    uk = p.to_cube(torch.as_tensor(uk0).to("cuda", p.cdtype).contiguous())
    u_out = p.empty_phys(3)
    ku = p.velocity_rhs(uk, prm.nu, prm.f0, prm.shell_no, visc=1.0, u_out=u_out)
    fk, _ = R.forcing(grid, uk0, prm.f0, prm.shell_no)
    ref, u_ref, _ = R.velocity_rhs(grid, uk0, prm.nu, fk, 1.0)
    assert rel(p.from_cube(ku).cpu().numpy(), ref * grid.dealias) < TOL[prec]
    assert rel(u_out.cpu().numpy(), u_ref) < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_shell_spectrum_matches_reference(torch, golden, prec):
    from lucky_droplets_b200.spectral import Plan
    g = golden("N16")
    p = Plan(16, prec)
    uk = p.to_cube(torch.as_tensor(g["uk0"]).to("cuda", p.cdtype).contiguous())
    ek = p.e3d_to_e1d(uk).cpu().numpy()
    grid = R.Grid(16)
    ref = grid.shell_sum(grid.energy3d(g["uk0"]))
    assert np.allclose(ek, ref, rtol=1e-6 if prec == "f32" else 1e-13, atol=1e-12 * ref.max())


@pytest.mark.parametrize("name", ["N16", "N32"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_rk4_time_loop_matches_reference(torch, golden, name, prec):
    """nsteps of the reference's own RK4 loop (F:571-623) from the same initial state."""
    from lucky_droplets_b200.dns import ForcedDNS
    g = golden(name)
    N = int(g["N"])
    dns = ForcedDNS.reference(N, precision=prec)
    dns.set_uk_full(g["uk0"])
    dns.step(int(g["nsteps"]))
    assert dns.check() == 0
    grid = R.Grid(N)
    assert rel(dns.uk_full(), g["run_uk"] * grid.dealias) < TOL[prec]


@pytest.mark.parametrize("N", [32, 64, 96])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_rk2if_matches_oracle(torch, N, prec):
    """RK2 + integrating factor against the FP64 NumPy restatement, 5 steps."""
    from lucky_droplets_b200.dns import ForcedDNS
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3)
    grid = C.ConfigGrid(N)
    uk0, _ = C.init_flow(grid, prm, seed=5)
    dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision=prec)
    dns.set_uk_full(uk0)
    uk = uk0.copy()
    for _ in range(5):
        uk, _, _ = C.rk2if_step(grid, prm, uk)
        uk = grid.project(np.stack([grid.rfft(grid.irfft(uk[c])) for c in range(3)]))
    dns.step(5)
    assert rel(dns.uk_full(), uk * grid.dealias) < TOL[prec] * 5


@pytest.mark.parametrize("method", ["trilinear", "tricubic", "cosine"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_gather_matches_oracle(torch, method, prec):
    from lucky_droplets_b200.spectral import Plan
    from lucky_droplets_b200.dns import Droplets
    N = 32
    rng = np.random.default_rng(9)
    field = rng.standard_normal((3, N, N, N))
    pos = rng.uniform(-1.0, 2 * np.pi + 1.0, (4000, 3))  # includes positions outside [0, 2pi)
    p = Plan(N, prec)
    d = Droplets(p, pos, np.zeros((4000, 3)), np.ones(4000), method=method)
    out = d.gather(torch.as_tensor(field).to("cuda", p.rdtype).contiguous()).cpu().numpy()
    ref = C.gather(field, pos, method)
    assert np.abs(out - ref).max() < (2e-5 if prec == "f32" else 1e-12)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_coupled_step_matches_oracle(torch, prec):
    """Flow RK2+IF + droplet Heun (tricubic, settling) against the FP64 oracle, 3 steps."""
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    grid = C.ConfigGrid(N)
    uk0, u0 = C.init_flow(grid, prm, seed=2)
    pos, tau, _ = C.init_droplets(prm, 2, "uniform_tau", nd=2000)
    vel = C.gather(u0, pos, "tricubic")
    dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision=prec)
    dns.set_uk_full(uk0)
    d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g)
    dns.attach(d)
    uk, p_, v_ = uk0.copy(), pos.copy(), vel.copy()
    for _ in range(3):
        uk, p_, v_ = C.step(grid, prm, uk, p_, v_, tau, "tricubic")
        uk = grid.project(np.stack([grid.rfft(grid.irfft(uk[c])) for c in range(3)]))
    dns.step(3)
    assert rel(dns.uk_full(), uk * grid.dealias) < TOL[prec] * 5
    tol_x = 1e-9 if prec == "f32" else 1e-13
    assert np.abs(d.pos.cpu().numpy() - p_).max() < tol_x * 1e3
    assert rel(d.vel.cpu().numpy(), v_) < TOL[prec] * 5


def test_sorted_droplets_with_collisions_match_oracle(torch):
    """Re-sorting droplets into cell order every step and detecting collisions does not change
    the trajectories (compared by droplet id) and the pair list matches the FP64 rule."""
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200.collide import Collider
    from oracle import collide_np as K
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    grid = C.ConfigGrid(N)
    uk0, u0 = C.init_flow(grid, prm, seed=6)
    pos, tau, rad = C.init_droplets(prm, 6, "uniform_tau", nd=3000)
    rad = rad * 5.0  # enough overlaps to test the pair list
    vel = C.gather(u0, pos, "tricubic")
    dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision="f64")
    dns.set_uk_full(uk0)
    d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g, radius=rad)
    col = Collider(d.n, 2 * rad.max())
    dns.attach(d, collider=col, sort_every=1)
    p_, v_ = pos.copy(), vel.copy()
    uk = uk0.copy()
    for _ in range(3):
        uk, p_, v_ = C.step(grid, prm, uk, p_, v_, tau, "tricubic")
        uk = grid.project(np.stack([grid.rfft(grid.irfft(uk[c])) for c in range(3)]))
    dns.step(3)
    assert np.abs(d.by_id(d.pos) - p_).max() < 1e-12
    assert rel(d.by_id(d.vel), v_) < 1e-12
    # the last step's pairs, in array indices, mapped to ids
    m = int(col.count.item())
    pairs = dns.pairs[:m].cpu().numpy().astype(np.int64)
    ids = d.ids.cpu().numpy()
    got = np.stack([ids[pairs].min(axis=1), ids[pairs].max(axis=1)], axis=1)
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    ref = K.collide(d.by_id(d.pos), rad, 2 * rad.max())
    assert np.array_equal(got, ref)


def test_step_host_matches_device_steps(torch):
    """step_host (host state in/out, droplet copies overlapped with the flow transforms and the
    copies back with the collision search) leaves exactly the state of device-resident steps,
    including a re-sort (sort_every=2) and the collision pairs of the last step."""
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200.collide import Collider
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    uk0, u0 = C.init_flow(C.ConfigGrid(N), prm, seed=8)
    pos, tau, rad = C.init_droplets(prm, 8, "uniform_tau", nd=4000)
    rad = rad * 5.0
    vel = C.gather(u0, pos, "tricubic")
    runs = []
    for _ in range(2):
        dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision="f32")
        dns.set_uk_full(uk0)
        d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g, radius=rad)
        dns.attach(d, collider=Collider(d.n, 2 * rad.max()), sort_every=2)
        runs.append((dns, d))
    (a, da), (b, db) = runs
    a.step(5)
    uk_h = b.uk.cpu().pin_memory()
    pos_h = db.pos.cpu().pin_memory()
    vel_h = db.vel.cpu().pin_memory()
    for _ in range(5):
        b.step_host(uk_h, pos_h, vel_h)
    torch.cuda.synchronize()
    assert torch.equal(uk_h, a.uk.cpu())
    assert torch.equal(pos_h, da.pos.cpu())
    assert torch.equal(vel_h, da.vel.cpu())
    assert torch.equal(db.ids, da.ids)
    assert int(b.collider.count.item()) == int(a.collider.count.item())
    m = int(a.collider.count.item())

    def pair_set(dns, d):
        ids = d.ids.cpu().numpy()
        p = ids[dns.pairs[:m].cpu().numpy().astype(np.int64)]
        p = np.stack([p.min(axis=1), p.max(axis=1)], axis=1)
        return p[np.lexsort((p[:, 1], p[:, 0]))]

    assert m > 0 and np.array_equal(pair_set(b, db), pair_set(a, da))


def test_step_graph_replay_matches_eager_steps(torch):
    """Steps replayed from a CUDA graph (ForcedDNS.capture) leave exactly the state of steps
    launched one by one, re-sorting (every 4 steps, inside the graph) and collisions included; a
    replay at another step phase of the re-sorting is refused."""
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200.collide import Collider
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    uk0, u0 = C.init_flow(C.ConfigGrid(N), prm, seed=9)
    pos, tau, rad = C.init_droplets(prm, 9, "uniform_tau", nd=3000)
    rad = rad * 5.0
    vel = C.gather(u0, pos, "tricubic")
    runs = []
    for _ in range(2):
        dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision="f32")
        dns.set_uk_full(uk0)
        d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g, radius=rad)
        dns.attach(d, collider=Collider(d.n, 2 * rad.max()), sort_every=4)
        dns.step(2)
        runs.append((dns, d))
    (a, da), (b, db) = runs
    g = b.capture(8)  # at step 2: phase 2 of the re-sorting period
    assert b.nstep == 2
    g.replay(2)
    a.step(16)
    torch.cuda.synchronize()
    assert a.nstep == b.nstep == 18 and a.t == b.t
    assert torch.equal(a.uk, b.uk)
    assert torch.equal(da.pos, db.pos) and torch.equal(da.vel, db.vel) and torch.equal(da.ids, db.ids)
    m = int(a.collider.count.item())
    assert m > 0 and m == int(b.collider.count.item())

    def pair_set(dns, d):
        ids = d.ids.cpu().numpy()
        p = ids[dns.pairs[:m].cpu().numpy().astype(np.int64)]
        p = np.stack([p.min(axis=1), p.max(axis=1)], axis=1)
        return p[np.lexsort((p[:, 1], p[:, 0]))]

    assert np.array_equal(pair_set(a, da), pair_set(b, db))
    b.step(1)
    with pytest.raises(RuntimeError):
        g.replay()


def test_step_host_reference_layout(torch):
    """step_host with the state in the reference's layout (3, N, N, N/2+1) (F:158): the same steps
    as device-resident stepping, the spectrum handed back dealiased in the reference layout."""
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200.collide import Collider
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    uk0, u0 = C.init_flow(C.ConfigGrid(N), prm, seed=18)
    pos, tau, rad = C.init_droplets(prm, 18, "uniform_tau", nd=3000)
    rad = rad * 5.0
    vel = C.gather(u0, pos, "tricubic")
    runs = []
    for _ in range(2):
        dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision="f32")
        dns.set_uk_full(uk0)
        d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g, radius=rad)
        dns.attach(d, collider=Collider(d.n, 2 * rad.max()), sort_every=2)
        runs.append((dns, d))
    (a, da), (b, db) = runs
    a.step(4)
    ukf = torch.as_tensor(uk0).to(torch.complex64).pin_memory()
    pos_h = db.pos.cpu().pin_memory()
    vel_h = db.vel.cpu().pin_memory()
    for _ in range(4):
        b.step_host(ukf, pos_h, vel_h, layout="full")
    torch.cuda.synchronize()
    assert torch.equal(b.uk, a.uk)
    assert torch.equal(ukf, a.plan.from_cube(a.uk).cpu())
    assert torch.equal(pos_h, da.pos.cpu()) and torch.equal(vel_h, da.vel.cpu())


@pytest.mark.parametrize("N", [96, 360])
def test_tricubic_droplet_step_on_mixed_radix_grid(torch, N):
    """The plain FP64 tricubic step on a mixed-radix grid (the equal-error comparator's grids):
    one coupled step against the FP64 oracle, droplets near the periodic faces included."""
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    prm = C.ConfigParams(N=N, nu=2.5e-3, dt=1e-3, g=0.1)
    grid = C.ConfigGrid(N)
    uk0, u0 = C.init_flow(grid, prm, seed=N)
    rng = np.random.default_rng(N)
    pos = rng.uniform(-0.01, 2 * np.pi + 0.01, (3000, 3))
    tau = np.exp(rng.uniform(np.log(0.05), np.log(2.0), 3000))
    vel = C.gather(u0, pos, "tricubic")
    dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision="f64")
    dns.set_uk_full(uk0)
    d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g)
    dns.attach(d)
    uk, p_, v_ = C.step(grid, prm, uk0, pos, vel, tau, "tricubic")
    uk = grid.project(np.stack([grid.rfft(grid.irfft(uk[c])) for c in range(3)]))
    dns.step(1)
    assert rel(dns.uk_full(), uk * grid.dealias) < 1e-12
    assert np.abs(d.pos.cpu().numpy() - p_).max() < 1e-13
    assert rel(d.vel.cpu().numpy(), v_) < 1e-12


@pytest.mark.parametrize("learned", [False, True])
def test_overlapped_droplet_stream_equals_one_stream(torch, learned):
    """The droplet work on a second stream (droplet stage 1 under the second flow stage, re-sort and
    collisions under the next step's first stage, two velocity buffers) gives exactly the state of
    everything on one stream - eagerly and from a captured graph."""
    from lucky_droplets_b200.collide import Collider
    from lucky_droplets_b200.dns import ForcedDNS, Droplets
    from lucky_droplets_b200 import mlp as G
    N = 32
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3, g=0.1)
    uk0, u0 = C.init_flow(C.ConfigGrid(N), prm, seed=23)
    pos, tau, rad = C.init_droplets(prm, 23, "uniform_tau", nd=3000)
    rad = rad * 5.0
    vel = C.gather(u0, pos, "tricubic")
    runs = []
    for overlap in (False, True, True):
        dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision="f32", overlap=overlap)
        dns.set_uk_full(uk0)
        d = Droplets(dns.plan, pos, vel, tau, method="tricubic", g=prm.g, radius=rad)
        dns.attach(d, collider=Collider(d.n, 2 * rad.max()), sort_every=3)
        if learned:
            d.use_learned(G.LearnedInterp(dns.plan, seed=3, tol=1.0))
        runs.append((dns, d))
    (a, da), (b, db), (c, dc) = runs
    a.step(7)
    b.step(7)
    g = c.capture(7)
    g.replay()
    torch.cuda.synchronize()
    for x, dx in ((b, db), (c, dc)):
        assert torch.equal(a.uk, x.uk)
        assert torch.equal(da.pos, dx.pos) and torch.equal(da.vel, dx.vel) and torch.equal(da.ids, dx.ids)
        assert int(a.collider.count.item()) == int(x.collider.count.item())
