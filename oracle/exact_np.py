"""CPU oracle of the exact spectral (direct Fourier sum) velocity at points (no counterpart in
the reference).  TEST INFRASTRUCTURE ONLY.

    u_c(x) = (1/N^3) sum_{kx,ky} sum_{kz} w_kz Re(uk_c(kx,ky,kz) exp(i k.x)),  w_0 = w_{N/2} = 1, else 2

over the reference layout (N, N, N/2+1) with kx, ky in FFT order (forced-dns-sm.py:59-62) and the
Hermitian weights of normalize (forced-dns-sm.py:136).  At grid points this equals scipy's irfftn,
which also drops the imaginary part of the kz = 0 and kz = N/2 coefficients.
"""
import numpy as np


def exact_sum(uk, pos, chunk=64):
    """uk (3, N, N, N/2+1) complex, pos (n, 3) -> (n, 3) float64."""
    N = uk.shape[1]
    Nf = N // 2 + 1
    K = np.fft.fftfreq(N, 1.0 / N)
    Kz = np.abs(K[:Nf])
    nz = np.nonzero(np.any(uk != 0, axis=0))
    kx, ky, kz = K[nz[0]], K[nz[1]], Kz[nz[2]]
    w = np.where((nz[2] == 0) | (nz[2] == N // 2), 1.0, 2.0)
    coef = uk[:, nz[0], nz[1], nz[2]] * w[None, :]
    out = np.zeros((pos.shape[0], 3))
    for s in range(0, pos.shape[0], chunk):
        p = pos[s:s + chunk]
        ph = np.exp(1j * (np.outer(p[:, 0], kx) + np.outer(p[:, 1], ky) + np.outer(p[:, 2], kz)))
        out[s:s + chunk] = np.real(ph @ coef.T)
    return out / N ** 3
