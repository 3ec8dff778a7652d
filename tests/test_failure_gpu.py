"""Failure detection without a GPU fault: every failure is made on the host or by a bounded
device wait that nothing completes, and the context stays usable afterwards.

  * a NaN planted in a host spectrum before upload -> LD_STATUS_NONFINITE, BlowUpError;
  * a host-scaled field above the abort threshold 100 N^3 of F:618-620 -> LD_STATUS_BLOWUP;
  * a bounded wait that runs out (ld_plan_set_wait_limit with stall) in the fused z pass and in
    the tensor-core MLP forward -> LD_STATUS_WAIT_TIMEOUT; the copies in flight are drained, the
    tensor memory freed, and the next launches on the same plan give the right answer;
  * a truncated checkpoint -> CheckpointError (tests/test_outputs_gpu.py).
"""
import numpy as np
import pytest

from oracle import config_np as C

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _flow(N, prec, seed=12):
    from lucky_droplets_b200.dns import ForcedDNS
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3)
    uk0, _ = C.init_flow(C.ConfigGrid(N), prm, seed)
    dns = ForcedDNS.config(N, prm.nu, prm.dt, eps=prm.eps, kf=prm.kf, precision=prec)
    return dns, uk0


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_nan_in_host_state_is_flagged(torch, prec):
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200.dns import BlowUpError
    dns, uk0 = _flow(32, prec)
    bad = uk0.copy()
    bad[1, 2, 1, 1] = np.nan  # one mode inside the dealiasing sphere
    dns.set_uk_full(bad)
    dns.step(1)
    flags = dns.plan.status(clear=False)
    assert flags & _lib.STATUS_NONFINITE
    with pytest.raises(BlowUpError):
        dns.check()
    assert dns.plan.status() == 0  # cleared by check()
    dns.set_uk_full(uk0)          # the same plan carries on
    dns.step(2)
    assert dns.check() == 0


def test_blowup_threshold_of_the_reference(torch):
    """max Re(uk) > 100 N^3 (F:618-620) raises the flag in the step epilogue and BlowUpError on the
    host; a field at a fifth of the threshold raises nothing; a step from an over-threshold
    state is flagged too."""
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import check, ptr, stream_ptr
    from lucky_droplets_b200.dns import BlowUpError
    N = 32
    dns, uk0 = _flow(N, "f64")
    peak = np.abs(uk0.real).max()
    L = _lib.lib()
    dns.set_uk_full(uk0 * (20.0 * N ** 3 / peak))
    check(L.ld_step_epilogue(dns.plan.handle, ptr(dns.uk), stream_ptr()))
    assert dns.check() == 0
    dns.set_uk_full(uk0 * (200.0 * N ** 3 / peak))
    check(L.ld_step_epilogue(dns.plan.handle, ptr(dns.uk), stream_ptr()))
    assert dns.plan.status(clear=False) & _lib.STATUS_BLOWUP
    with pytest.raises(BlowUpError):
        dns.check()
    dns.set_uk_full(uk0 * (200.0 * N ** 3 / peak))
    dns.step(1)
    assert dns.plan.status(clear=False) & (_lib.STATUS_BLOWUP | _lib.STATUS_NONFINITE)
    with pytest.raises(BlowUpError):
        dns.check()


def test_wait_timeout_in_fused_z_pass(torch):
    """N = 256 runs the pipelined z pass (one warp per row, bulk-copy prefetch).  With the stall
    test on, every warp's first wait runs out: WAIT_TIMEOUT is raised, no fault; with the default
    limit the same plan then computes the RHS exactly as a fresh plan does."""
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200.spectral import Plan
    N = 256
    prm = C.ConfigParams(N=N, nu=2.5e-3, dt=1e-3)
    uk0, _ = C.init_flow(C.ConfigGrid(N), prm, seed=3)
    p = Plan(N, "f32")
    uk = p.to_cube(torch.as_tensor(uk0).to("cuda", p.cdtype).contiguous())
    p.set_wait_limit(64, stall=True)
    p.velocity_rhs(uk, prm.nu, prm.f0, prm.shell_no)
    assert p.status() & _lib.STATUS_WAIT_TIMEOUT
    p.set_wait_limit(0)
    got = p.velocity_rhs(uk, prm.nu, prm.f0, prm.shell_no)
    assert p.status() == 0
    fresh = Plan(N, "f32")
    ref = fresh.velocity_rhs(uk, prm.nu, prm.f0, prm.shell_no)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)


def test_wait_timeout_in_tensor_core_forward(torch):
    """The MLP forward (tcgen05, TMEM): with the stall test on, every group's first wait runs out
    while the CTA's first feature copy is in flight; the copy is drained, tensor memory freed,
    WAIT_TIMEOUT raised.  Afterwards the same plan infers exactly what it inferred before."""
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200.mlp import LearnedInterp
    from lucky_droplets_b200.spectral import Plan
    N = 64
    prm = C.ConfigParams(N=N, nu=0.01, dt=2e-3)
    uk0, _ = C.init_flow(C.ConfigGrid(N), prm, seed=4)
    p = Plan(N, "f32")
    cube = p.to_cube(torch.as_tensor(uk0).to("cuda", p.cdtype).contiguous())
    li = LearnedInterp(p, seed=2)
    u4 = li.interleaved(cube)
    pos = torch.as_tensor(np.random.default_rng(5).uniform(0, 2 * np.pi, (40000, 3))).cuda()
    before = li.infer(u4, pos).clone()
    assert p.status() == 0
    p.set_wait_limit(64, stall=True)
    li.infer(u4, pos)
    assert p.status() & _lib.STATUS_WAIT_TIMEOUT
    p.set_wait_limit(0)
    after = li.infer(u4, pos)
    assert p.status() == 0
    torch.cuda.synchronize()
    assert torch.equal(before, after)
