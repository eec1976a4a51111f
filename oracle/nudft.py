"""complex128 direct-sum operators (precision oracle).

TEST INFRASTRUCTURE.  The reference USFFT (src/cuda/radonusfft.cu:54-92)
approximates, through Gaussian gridding on a 2x oversampled grid, the
exact non-uniform DFT of the padded and masked slice at the polar points:

    g(theta, k) = (1/N) * sum_{tx,ty} fp[ty, tx] *
                  exp(-2*pi*i*(x_k (tx - N/2) + y_k (ty - N/2)))

followed by the same centred 1-D inverse FFT and crop as the gridded
operator.  (Poisson summation of the Gaussian kernel w = pi/mu *
exp(-pi^2/mu |xi|^2) gives 4N^2 * phi(t) * exp(-2 pi i xi t), and the
deapodisation divides phi and 4N^2 back out.)  The ptycho operator has no
approximation: its direct sum is a dense 2-D DFT per scan.
"""
from __future__ import annotations

import numpy as np

from .usfft import checker1, circ_mask, takexy


def radon_fwd_exact(f, theta, n, xy=None):
    """Exact NUDFT version of radonusfft::fwd, f [nz, n, n] -> [ntheta, nz, n]."""
    N = n * 3 // 2
    f = np.asarray(f).astype(np.complex128)
    nz = f.shape[0]
    c0 = N // 6
    idx = np.clip(np.arange(N), c0, 5 * N // 6 - 1) - c0
    fp = f[:, idx][:, :, idx] * circ_mask(N)
    x, y = takexy(theta, N) if xy is None else xy
    x = np.asarray(x, np.float64).ravel()
    y = np.asarray(y, np.float64).ravel()
    t = np.arange(N) - N // 2
    Ex = np.exp(-2j * np.pi * x[:, None] * t[None, :])     # [P, tx]
    Ey = np.exp(-2j * np.pi * y[:, None] * t[None, :])     # [P, ty]
    ntheta = len(np.asarray(theta))
    g = np.empty((ntheta, nz, N), np.complex128)
    for z in range(nz):
        v = np.einsum("py,yx,px->p", Ey, fp[z], Ex, optimize=True)
        g[:, z, :] = v.reshape(ntheta, N) / N
    s1 = checker1(N)
    g = np.fft.ifft(g * s1, axis=-1) * N * s1
    return g[:, :, c0:c0 + n]


def dft2_matrix(L):
    k = np.arange(L)
    return np.exp(-2j * np.pi * np.outer(k, k) / L)


def ptycho_fwd_exact(op, f):
    """Dense-DFT version of ptychofft::fwd for an oracle ``PtychoFFT`` op."""
    P, dx, dy = op.nprb, op.detx, op.dety
    Wx, Wy = dft2_matrix(dx), dft2_matrix(dy)
    f = np.asarray(f).reshape(op.ntheta, op.nz, op.n).astype(np.complex128)
    rs, cs = (dx - P) // 2, (dy - P) // 2
    g = np.zeros((op.ntheta, op.nscan, dx, dy), np.complex128)
    for t in range(op.ntheta):
        for s in range(op.nscan):
            x0, y0 = op.stx[t, s], op.sty[t, s]
            if x0 < 0 or y0 < 0:
                continue
            D = np.zeros((dx, dy), np.complex128)
            D[rs:rs + P, cs:cs + P] = op.c * op.prb * f[t, y0:y0 + P, x0:x0 + P].T
            g[t, s] = Wx @ D @ Wy.T * op.phase[t, s]
    return g
