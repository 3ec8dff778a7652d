"""ld_irfft_mpi_noalloc against ld_irfft_mpi.

The no-alloc entry point serves callers that must not allocate device memory - host frameworks
that own all device memory through their own pool, and time-critical loops that may not allocate
after their set-up.  It keeps its scratch in a static device array (N <= 64), so it must give the
same result as the plan-based transform, call after call.
This file is collected last on purpose: a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2e-6  # the FP32 transform tolerance of tests/test_fft_gpu.py


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


def test_noalloc_inverse_matches_plan_transform():
    import torch
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import ptr, stream_ptr
    from lucky_droplets_b200.spectral import Plan
    assert torch.cuda.is_available()
    L = _lib.lib()
    for N in (16, 32, 64):
        rng = np.random.default_rng(100 + N)
        shape = (2, N, N, N // 2 + 1)
        X = torch.as_tensor(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).to("cuda", torch.complex64)
        p = Plan(N, "f32")
        ref = p.irfft_mpi(X).cpu().numpy()
        out = torch.empty((2, N, N, N), dtype=torch.float32, device="cuda")
        for _ in range(2):  # two calls in a row share the static scratch
            out.fill_(float("nan"))
            assert L.ld_irfft_mpi_noalloc(N, ptr(X), ptr(out), 2, stream_ptr()) == 0, L.ld_last_error()
            torch.cuda.synchronize()
            assert rel(out.cpu().numpy(), ref) < TOL
        p.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from lucky_droplets_b200 import _lib
    from lucky_droplets_b200._lib import ptr, stream_ptr
    L = _lib.lib()
    X = torch.zeros((1, 128, 128, 65), dtype=torch.complex64, device="cuda")
    u = torch.zeros((1, 128, 128, 128), dtype=torch.float32, device="cuda")
    assert L.ld_irfft_mpi_noalloc(128, ptr(X), ptr(u), 1, stream_ptr()) == -3  # LD_ERR_UNSUPPORTED
    assert b"64" in L.ld_last_error()
